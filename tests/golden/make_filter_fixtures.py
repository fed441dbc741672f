"""Generates tests/golden/ref_filters.npz: the reference's camera-side depth
filters (d_MedianFilter, d_GradientFilter, d_AverageFilter, d_undistort of
Source/src/CameraSupport/CameraAbstract.cu, compiled from the reference
sources by oracle/ref_harness into oracle/_ref/libref_kernels.so) on one
synthetic 640x480 depth frame with holes and speckles. Runs on a GPU box:

    python tests/golden/make_filter_fixtures.py OUTDIR
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from tests.golden.make_ref_fixtures import RefCam  # noqa: E402

# radial-only distortion: the reference's tangential terms read the updated x
UNDISTORT = (525.0, 525.0, 319.5, 239.5, -0.12, 0.03, 0.0, 0.0)


def main(out: Path):
    import openfusion_b200 as of
    cfg = of.CONFIGS["c2"]
    depth = of.make_sequence(cfg, frames=1).depth[0].astype(np.uint16)
    rng = np.random.default_rng(11)
    m = rng.random(depth.shape)
    depth[m < 0.01] = 0                                    # holes
    sp = m > 0.995                                         # speckles
    depth[sp] = np.clip(depth[sp].astype(np.int64) + rng.integers(-400, 400, sp.sum()), 0, 65535)
    lib = C.CDLL(str(ROOT / "oracle" / "_ref" / "libref_kernels.so"))
    P = C.c_void_p
    lib.ref_depth_filter.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, P, P]
    lib.ref_undistort.argtypes = [P, C.c_float, C.c_float, C.c_float, C.c_float, P, P, C.c_uint16]
    h, w = depth.shape
    outs = {}
    for kind, name in ((0, "median5"), (1, "gradient"), (2, "average")):
        o = np.zeros_like(depth)
        assert lib.ref_depth_filter(kind, w, h, 0, depth.ctypes.data, o.ctypes.data) == 0
        outs[name] = o
    fx, fy, cx, cy, k1, k2, p1, p2 = UNDISTORT
    cam = RefCam(w, h, fx, fy, cx, cy, 1 / fx, 1 / fy, -cx / fx, -cy / fy, 300.0, 5000.0)
    o = np.zeros_like(depth)
    assert lib.ref_undistort(C.byref(cam), k1, k2, p1, p2, depth.ctypes.data, o.ctypes.data,
                             0xFFFF) == 0
    outs["undistort"] = o
    out.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(out / "ref_filters.npz", depth=depth, undistort_params=np.array(UNDISTORT),
                        **outs)
    print({k: int((v != 0).sum()) for k, v in outs.items()})


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else ROOT / "tests" / "golden")
