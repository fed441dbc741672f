"""Pins the oracle against outputs of the reference itself.

tests/golden/ref_*.npz hold the inputs and outputs of gilbs10/OpenFusion's own
CUDA kernels (d_convertDepthToWorldVertices/Normals, d_integrateVolume,
d_raycast, d_find_corresponding) and of its host routine
Cpu_buildNewTransformMatrix, compiled from the reference sources and run on a
B200 by tests/golden/make_ref_fixtures.py. Here the oracle's reference-
semantics functions consume the same inputs in FP64; they share their voxel
centre, projection, truncation, running-average, ICP-row and Euler-increment
arithmetic with the main oracle, so these checks pin that arithmetic too.
Tolerances are those of FP32 (the reference) against FP64 (the oracle);
decisions within FP32 rounding of a boundary are flagged by the oracle and
their number is bounded.
"""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def fx():
    f = np.load(GOLDEN / "ref_frames.npz")
    v = np.load(GOLDEN / "ref_volume.npz")
    return {**{k: f[k] for k in f.files}, **{"vol_" + k: v[k] for k in v.files}}


@pytest.fixture(scope="module")
def ref(ora):
    from oracle import RefSemantics
    return RefSemantics(ora)


def f32(a):
    return np.asarray(a, np.float32).astype(np.float64)


def inv_rigid(T):
    Ti = np.eye(4)
    Ti[:3, :3] = T[:3, :3].T
    Ti[:3, 3] = -T[:3, :3].T @ T[:3, 3]
    return Ti


def cam_of(ref, fx):
    w, h, fx_, fy, cx, cy, dmin, dmax = fx["cam"]
    # the inverse intrinsics as the reference received them (float)
    return ref.cam(int(w), int(h), f32(fx_), f32(fy), f32(cx), f32(cy), f32(1.0 / fx_),
                   f32(1.0 / fy), f32(-cx / fx_), f32(-cy / fy), dmin, dmax)


def vol_of(ref, fx):
    n, world, trunc, max_w = fx["volume"]
    return ref.vol(int(n), float(world), float(trunc), int(max_w), b1=1)


BAD = np.float32(np.finfo(np.float32).max)


def test_depth_to_world_maps_match_reference(ref, fx):
    cam = cam_of(ref, fx)
    for depth, T, v_ref, n_ref in ((fx["depth0"], fx["T0"], fx["vertex0"], fx["normal0"]),
                                   (fx["depth1"], fx["T1"], fx["vertex1"], fx["normal1"])):
        v, n = ref.convert(cam, depth, f32(T))
        bad_ref = v_ref[..., 0] == BAD
        bad = v[..., 0] > 1e38
        assert np.array_equal(bad, bad_ref)
        assert np.abs(v[~bad] - v_ref[~bad]).max() < 2e-3          # mm
        nz = np.abs(n_ref).sum(-1) > 0
        assert np.array_equal(nz, np.abs(n).sum(-1) > 0)
        assert np.abs(n[nz] - n_ref[nz]).max() < 2e-4


def test_integration_matches_reference_two_frames(ref, fx):
    cam, vol = cam_of(ref, fx), vol_of(ref, fx)
    n = vol.n
    idx = fx["vol_idx"].astype(np.int64)
    storage = (idx[:, 0] * n + idx[:, 1]) * n + idx[:, 2]
    T0, T1 = fx["T0"], fx["T1"]
    prev_t = np.full(len(storage), vol.trunc)
    prev_w = np.zeros(len(storage), np.int32)
    # frame 0 from the initial volume (tsdf = TRUNCATION, weight 0)
    t1, w1, amb = ref.integrate_voxels(vol, cam, f32(fx["vertex0"]), f32(inv_rigid(T0)),
                                       f32(T0[:3, 3]), storage, prev_t, prev_w)
    ok = amb == 0
    assert (~ok).mean() < 2e-3
    assert (fx["vol_w1"] > 0).sum() > 100000          # the sample covers updated voxels
    assert np.array_equal(w1[ok], fx["vol_w1"][ok].astype(np.int32))
    assert np.abs(t1[ok] - fx["vol_tsdf1"][ok]).max() < 2e-3   # mm, FP32 vs FP64
    # the storage shift of d_integrateVolume: slab 0 is never written
    assert np.all(fx["vol_w1"][idx[:, 0] == 0] == 0)
    # frame 1 on top of the reference's own state: running averages
    t2, w2, amb2 = ref.integrate_voxels(vol, cam, f32(fx["vertex1"]), f32(inv_rigid(T1)),
                                        f32(T1[:3, 3]), storage, fx["vol_tsdf1"].astype(np.float64),
                                        fx["vol_w1"].astype(np.int32))
    ok2 = (amb2 == 0) & ok
    assert np.array_equal(w2[ok2], fx["vol_w2"][ok2].astype(np.int32))
    assert (fx["vol_w2"] == 2).sum() > 50000
    assert np.abs(t2[ok2] - fx["vol_tsdf2"][ok2]).max() < 2e-3


def test_raycast_matches_reference(ref, fx):
    cam, vol = cam_of(ref, fx), vol_of(ref, fx)
    T0 = fx["T0"]
    tsdf, _ = ref.integrate_full(vol, cam, f32(fx["vertex0"]), f32(inv_rigid(T0)), f32(T0[:3, 3]),
                                 vol.trunc)
    v, n, amb = ref.raycast(vol, tsdf, cam, f32(T0), f32(T0[:3, 3]))
    v_ref, n_ref = fx["model_vertex"], fx["model_normal"]
    hit_ref = v_ref[..., 0] != BAD
    hit = v[..., 0] < 1e38
    ok = amb == 0
    assert hit_ref.mean() > 0.5
    assert (~ok).mean() < 0.01
    assert (hit != hit_ref)[ok].sum() <= 2
    both = hit & hit_ref & ok
    assert np.abs(v[both] - v_ref[both]).max() < 5e-3               # mm
    nb = both & (np.abs(n_ref).sum(-1) > 0)
    assert np.median(np.abs(n[nb] - n_ref[nb]).max(-1)) < 1e-4


def test_correspondence_sums_match_reference(ref, fx):
    cam = cam_of(ref, fx)
    T0 = fx["T0"]
    o36, o6, a36, a6 = ref.icp_system(cam, fx["depth1"], f32(fx["new_vertex"]),
                                      f32(fx["new_normal"]), f32(fx["model_vertex"]),
                                      f32(fx["model_normal"]), f32(inv_rigid(T0)))
    g36, g6 = fx["AtA"].astype(np.float64), fx["Atb"].astype(np.float64)
    upper = np.array([6 * i + j for i in range(6) for j in range(i, 6)])
    assert o36[0] > 1e6                                # many correspondences
    diag = o36[[0, 7, 14, 21, 28, 35]]
    scale36 = np.sqrt(np.outer(diag, diag)).reshape(36)
    # float block sums (reference) vs FP64 sums (oracle)
    assert np.all(np.abs(g36[upper] - o36[upper]) <= 2e-5 * scale36[upper] + a36[upper] + 1e-3)
    bb = np.sqrt(diag * max(np.abs(o6).max(), 1.0))
    assert np.all(np.abs(g6 - o6) <= 1e-4 * bb + a6 + 1e-3)


def test_transform_build_matches_reference(ref, fx):
    T0 = f32(fx["T0"])
    for x, built in zip(fx["xopt"], fx["built"]):
        T, F = ref.compose(f32(x), T0, np.eye(4))
        assert np.allclose(T.reshape(16), built[:16], rtol=0, atol=2e-4 * max(1.0, np.abs(T).max()))
        assert np.allclose(F.reshape(16), built[16:], rtol=0, atol=1e-6 * max(1.0, np.abs(F).max()) + 1e-6)


def test_transform_build_against_host_routine_directly(ref):
    """The reference's Cpu_buildNewTransformMatrix is host code: where the
    harness library was built from the reference sources, call it here."""
    import ctypes as C
    lib_path = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libref_kernels.so"
    if not lib_path.exists():
        pytest.skip("reference harness not built")
    lib = C.CDLL(str(lib_path))
    lib.ref_build_transform.argtypes = [C.c_void_p] * 3
    lib.ref_build_transform.restype = None
    rng = np.random.default_rng(3)
    for _ in range(50):
        x = np.concatenate([rng.uniform(-0.05, 0.05, 3), rng.uniform(-30, 30, 3)]).astype(np.float32)
        T = np.eye(4, dtype=np.float32)
        T[:3, 3] = rng.uniform(-500, 800, 3)
        Tf, Ff = T.reshape(16).copy(), np.eye(4, dtype=np.float32).reshape(16).copy()
        xx = x.copy()
        lib.ref_build_transform(xx.ctypes.data, Tf.ctypes.data, Ff.ctypes.data)
        To, Fo = ref.compose(x.astype(np.float64), T.astype(np.float64), np.eye(4))
        assert np.allclose(To.reshape(16), Tf, atol=5e-4)
        assert np.allclose(Fo.reshape(16), Ff, atol=1e-5)
