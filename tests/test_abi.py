"""The C-ABI library loads and exports every entry point of
include/openfusion_b200.h; host-side entry points answer without a GPU."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def header_functions():
    text = (ROOT / "include" / "openfusion_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(of_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = header_functions()
    assert "of_integrate" in names and "of_tracker_process" in names
    assert len(names) >= 29


def test_library_exports_every_declared_symbol(of):
    lib = of._native.lib()
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_table_matches_header(of):
    assert set(of._native.exported_symbols()) == set(header_functions())


def test_abi_version_and_status_strings(of):
    lib = of._native.lib()
    assert lib.of_abi_version() == 4
    assert lib.of_status_string(0) == b"ok"
    assert b"invalid" in lib.of_status_string(1)


def test_defaults_match_full_size_configuration(of):
    N = of._native
    f, r, i = N.FilterParams(), N.RaycastParams(), N.IcpParams()
    N.lib().of_default_params(C.byref(f), C.byref(r), C.byref(i))
    assert (f.sigma_space_px, f.sigma_range_mm, f.levels) == (4.5, 30.0, 3)
    assert list(i.iters)[:3] == [10, 5, 4] and i.dist_thresh_mm == 25.0
    assert abs(i.normal_thresh - 0.65) < 1e-7


def test_layout_and_sizes(of):
    cfg = of.CONFIGS["c2"]
    lay = of.pyramid_layout(cfg)
    assert list(lay.width)[:3] == [640, 320, 160] and list(lay.height)[:3] == [480, 240, 120]
    for l in range(3):
        assert lay.depth_offset[l] % 256 == 0 and lay.points_offset[l] % 256 == 0
    # voxels + brick flags + super-brick flags (4^3 bricks) + saturated-brick
    # bytes, each byte block padded to 256 B
    assert of.volume_bytes(cfg) == 512 ** 3 * 4 + 64 ** 3 + 16 ** 3 + (256 - 16 ** 3 % 256) % 256 + 64 ** 3
    c1 = of.level_camera(cfg, 1)
    assert (c1.fx, c1.cx, c1.cy) == (262.5, 159.5, 119.5)


def test_invalid_arguments_are_rejected(of):
    N = of._native
    lib = N.lib()
    bad = N.VolumeDesc(100, 0, 3000.0, 30.0, 128, 0)  # not a multiple of 8
    n = C.c_size_t()
    assert lib.of_volume_bytes(C.byref(bad), C.byref(n)) == 1
    cam = N.Camera(0, 480, 525, 525, 319.5, 239.5, 300, 5000)
    lay = N.PyramidLayout()
    assert lib.of_pyramid_layout(C.byref(cam), 3, C.byref(lay)) == 1
    assert lib.of_integrate(None, None, None, None, 0, None, None, None) == 1
    assert lib.of_tracker_create(None, None) == 1


def test_package_exports_resolve():
    import openfusion_b200 as of
    for name in of.__all__:
        assert getattr(of, name) is not None, name
