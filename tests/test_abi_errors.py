"""Argument checking of the C-ABI (CPU): calls with missing or out-of-range
arguments return OF_ERR_INVALID_ARGUMENT (1) before touching a device, and a
missing file returns OF_ERR_IO (6)."""
import ctypes as C

import pytest

INVALID = 1


@pytest.fixture(scope="module")
def lib(of):
    return of._native.lib()


def test_batch_and_shard_arguments(of, lib):
    N = of._native
    h = C.c_void_p()
    assert lib.of_batch_create(None, C.byref(h)) == INVALID
    d = N.BatchDesc()
    d.count = 0
    assert lib.of_batch_create(C.byref(d), C.byref(h)) == INVALID
    assert lib.of_batch_process(None, None, 0, None) == INVALID
    assert lib.of_batch_poses(None, None, None, None) == INVALID
    costs = (C.c_double * 2)(1.0, 2.0)
    out = (C.c_int32 * 2)()
    assert lib.of_batch_shard(C.cast(costs, C.c_void_p), 2, 0, C.cast(out, C.c_void_p)) == INVALID
    assert lib.of_batch_shard(None, 2, 2, C.cast(out, C.c_void_p)) == INVALID


def test_mesh_filter_and_view_arguments(of, lib):
    cfg = of.CONFIGS["c1"]
    cnt = C.c_uint32()
    assert lib.of_mesh_extract(C.byref(cfg.volume()), None, None, None, 0, C.byref(cnt), None) == INVALID
    assert lib.of_mesh_write_obj(None, None, 0) == INVALID
    p = of.depth_filter_params(["median5"])
    p.steps = 0x40  # no such filter
    assert lib.of_depth_filter(C.byref(cfg.camera()), C.byref(p), C.c_void_p(16), C.c_void_p(16),
                               None, None) == INVALID
    p = of.depth_filter_params(["median5", "average"])
    # two steps need a scratch buffer distinct from input and output
    assert lib.of_depth_filter(C.byref(cfg.camera()), C.byref(p), C.c_void_p(16), C.c_void_p(32),
                               None, None) == INVALID
    assert lib.of_depth_filter_step(C.byref(cfg.camera()), 4, C.byref(p), C.c_void_p(16),
                                    C.c_void_p(16), None) == INVALID
    assert lib.of_depth_to_rgba(C.byref(cfg.camera()), None, None, None) == INVALID
    assert lib.of_normals_to_rgba(C.byref(cfg.camera()), None, None, 1.0, None, None) == INVALID


def test_tracker_and_reader_arguments(of, lib, tmp_path):
    h = C.c_void_p()
    assert lib.of_tracker_save(None, b"x", None) == INVALID
    assert lib.of_tracker_load(None, b"x", None) == INVALID
    assert lib.of_tracker_flush(None, None) == INVALID
    assert lib.of_reader_open(None, 4, C.byref(h)) == INVALID
    assert lib.of_reader_open(str(tmp_path).encode(), 0, C.byref(h)) == INVALID
    assert lib.of_reader_open(str(tmp_path / "absent").encode(), 4, C.byref(h)) == 6
    assert lib.of_reader_next(None, None, None) == INVALID
