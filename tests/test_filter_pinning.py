"""The camera-side depth filters of the oracle pinned against the reference's
own kernels (CPU): tests/golden/ref_filters.npz holds d_MedianFilter,
d_GradientFilter, d_AverageFilter and d_undistort
(Source/src/CameraSupport/CameraAbstract.cu) run on a B200 on one synthetic
640x480 frame with holes and speckles (tests/golden/make_filter_fixtures.py).

Away from the border, where the reference's unsigned wrap-around indexing
does not reach, the median, average and gradient are equal pixel for pixel
(gradient: but for pixels whose FP32 test sits on its threshold). The
undistortion is radial only (the reference's tangential terms read the
updated x) and agrees within 1 mm (truncated FP32 against FP64 bilinear
values) where the reference writes a pixel and no tap is null."""
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden" / "ref_filters.npz"
pytestmark = pytest.mark.skipif(not GOLD.exists(), reason="filter fixtures not generated")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.mark.parametrize("kind,border", [("median5", 2), ("average", 1), ("gradient", 1)])
def test_stencils_match_reference(ora, gold, kind, border):
    d = gold["depth"]
    thr = {"median5": 0.0, "average": 15.0, "gradient": 10.0}[kind]
    out, amb = ora.depth_filter(kind, d, null_value=0, thr=thr)
    ref = gold[kind]
    sl = (slice(border, -border), slice(border, -border))
    ok = np.ones(d.shape, bool) if amb is None else amb == 0
    diff = (out != ref)[sl] & ok[sl]
    assert diff.sum() == 0, (kind, int(diff.sum()))
    assert (ref[sl] != d[sl]).mean() > 0.001  # the filter changed something


def test_undistort_matches_reference(ora, gold):
    d = gold["depth"]
    prm = gold["undistort_params"]
    out, amb = ora.depth_filter("undistort", d, null_value=0, undistort=prm)
    ref = gold["undistort"]
    written = ref != 0xFFFF
    # source pixels, to leave out the reference's last-row test on the column
    # index (floor(u) == height - 1, CameraAbstract.cu:207)
    fx, fy, cx, cy, k1, k2, p1, p2 = prm
    h, w = d.shape
    y, x = np.mgrid[0:h, 0:w].astype(np.float64)
    xn, yn = (x - cx) / fx, (y - cy) / fy
    r2 = xn * xn + yn * yn
    u = fx * xn * (1 + k1 * r2 + k2 * r2 * r2) + cx
    cmp = written & (out != 0) & (amb == 0) & (np.floor(u) != h - 1)
    assert cmp.mean() > 0.8
    dd = np.abs(out[cmp].astype(np.int64) - ref[cmp].astype(np.int64))
    assert dd.max() <= 1, dd.max()
    # where the reference leaves a pixel unwritten the source is outside: null here
    assert np.all(out[~written & (amb == 0)] == 0)
