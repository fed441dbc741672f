"""Generates tests/golden/ref_*.npz: outputs of gilbs10/OpenFusion's own CUDA
kernels (compiled from the reference sources by oracle/ref_harness into
oracle/_ref/libref_kernels.so) on a seeded synthetic scene, with the inputs
they consumed. Runs on a GPU box:

    python tests/golden/make_ref_fixtures.py OUTDIR

The scene sits in the reference's own geometry (Constants.h: a 1024 mm cube
of 512^3 voxels, truncation 10 mm, max weight 120, camera starting 768 mm from
the centre looking along -z, MainApp.cpp:613-618). The CPU tests compare the
oracle's reference-semantics functions against these arrays.
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

W, H = 160, 128  # H a multiple of 16: d_find_corresponding returns early before its barriers otherwise (ICP.cu:129)
FX = FY = 131.25
CX, CY = 79.5, 63.5
DMIN, DMAX = 300.0, 4000.0


class RefCam(C.Structure):
    _fields_ = [("w", C.c_int32), ("h", C.c_int32), ("fx", C.c_float), ("fy", C.c_float),
                ("cx", C.c_float), ("cy", C.c_float), ("ifx", C.c_float), ("ify", C.c_float),
                ("icx", C.c_float), ("icy", C.c_float), ("dmin", C.c_float), ("dmax", C.c_float)]


def ref_cam():
    # inverse intrinsics as CameraFromFile.cpp:42-51 forms them (inverse of K)
    return RefCam(W, H, FX, FY, CX, CY, 1.0 / FX, 1.0 / FY, -CX / FX, -CY / FY, DMIN, DMAX)


def scene():
    import openfusion_b200._native as N
    sc = N.SynthScene()
    prims = [
        (0, [0, 0, 1, -420]),                       # back wall z = -420
        (0, [0, 1, 0, -380]),                       # floor y = -380
        (1, [0, 0, -120, 210]),                     # spheres: centre, radius
        (1, [260, 110, 40, 110]),
        (1, [-180, 190, 120, 80]),
        (2, [-250, -230, -150, 110, 150, 100, 0.45]),  # box: centre, half extents, yaw
        (2, [220, -260, -230, 140, 120, 90, -0.3]),
    ]
    sc.count = len(prims)
    sc.room_half_mm = 512.0
    for i, (k, p) in enumerate(prims):
        sc.prims[i].kind = k
        for j, v in enumerate(p):
            sc.prims[i].p[j] = v
    return sc


def poses():
    def rot(ax, ay, az):
        cx, sx, cy, sy, cz, sz = np.cos(ax), np.sin(ax), np.cos(ay), np.sin(ay), np.cos(az), np.sin(az)
        Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
        Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
        Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
        return Rz @ Ry @ Rx
    T0 = np.eye(4)
    T0[2, 3] = 768.0  # CAMERA_START_Z_MM (Constants.h:30-33)
    T1 = np.eye(4)
    T1[:3, :3] = rot(0.004, -0.006, 0.003)
    T1[:3, 3] = [6.0, -4.0, 765.0]
    return T0, T1


def render(sc, T, frame):
    import openfusion_b200._native as N
    d = np.zeros((H, W), np.uint16)
    P = np.ascontiguousarray(T, np.float64)
    N.synth().of_synth_render(C.byref(sc), W, H, FX, FY, CX, CY, P.ctypes.data, 77, frame, 0.5,
                              0.0, d.ctypes.data, None)
    return d


def load():
    lib = C.CDLL(str(ROOT / "oracle" / "_ref" / "libref_kernels.so"))
    P = C.c_void_p
    sigs = {
        "ref_volume_size": (C.c_int, []), "ref_max_weight": (C.c_int, []),
        "ref_world_volume": (C.c_float, []), "ref_truncation": (C.c_float, []),
        "ref_volume_init": (C.c_int, []), "ref_volume_free": (C.c_int, []),
        "ref_convert": (C.c_int, [P, P, P, P, P]),
        "ref_integrate": (C.c_int, [P, P, P, P]),
        "ref_volume_read": (C.c_int, [P, C.c_int64, P, P]),
        "ref_raycast": (C.c_int, [P, P, P, P, P, P]),
        "ref_find_corresponding": (C.c_int, [P, P, P, P, P, P, P, P, P, P]),
        "ref_build_transform": (None, [P, P, P]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def main(out: Path):
    lib = load()
    cam = ref_cam()
    n = lib.ref_volume_size()
    sc = scene()
    T0, T1 = poses()
    d0, d1 = render(sc, T0, 0), render(sc, T1, 1)
    f32 = lambda a: np.ascontiguousarray(a, np.float32)

    def convert(depth, T):
        v = np.zeros((H, W, 3), np.float32)
        nn = np.zeros((H, W, 3), np.float32)
        TT = f32(T).reshape(16)
        assert lib.ref_convert(C.byref(cam), depth.ctypes.data, TT.ctypes.data, v.ctypes.data,
                               nn.ctypes.data) == 0
        return v, nn

    def inv(T):
        Ti = np.eye(4)
        Ti[:3, :3] = T[:3, :3].T
        Ti[:3, 3] = -T[:3, :3].T @ T[:3, 3]
        return Ti

    assert lib.ref_volume_init() == 0
    # frame 0: convert, integrate, raycast (MainApp.cpp:786-810)
    v0, n0 = convert(d0, T0)
    pos0 = f32(T0[:3, 3])
    assert lib.ref_integrate(C.byref(cam), v0.ctypes.data, f32(inv(T0)).reshape(16).ctypes.data,
                             pos0.ctypes.data) == 0
    rng = np.random.default_rng(5)
    # storage indices to read back: (slab, y, z) with slab up to n (padding slab)
    m = 120000
    idx = np.stack([rng.integers(0, n + 1, m), rng.integers(0, n, m), rng.integers(0, n, m)], 1)
    # plus a dense block in front of the scene where most voxels are updated
    bx, by, bz = np.meshgrid(np.arange(200, 312), np.arange(230, 282), np.arange(300, 420),
                             indexing="ij")
    idx = np.concatenate([idx, np.stack([bx.ravel(), by.ravel(), bz.ravel()], 1)])
    flat = (idx[:, 0].astype(np.int64) * n + idx[:, 1]) * n + idx[:, 2]
    t1 = np.zeros(len(flat), np.float32)
    w1 = np.zeros(len(flat), np.uint8)
    assert lib.ref_volume_read(flat.ctypes.data, len(flat), t1.ctypes.data, w1.ctypes.data) == 0
    mv = np.zeros((H, W, 3), np.float32)
    mn = np.zeros((H, W, 3), np.float32)
    rgba = np.zeros((H, W), np.uint32)
    assert lib.ref_raycast(C.byref(cam), f32(T0).reshape(16).ctypes.data, pos0.ctypes.data,
                           mv.ctypes.data, mn.ctypes.data, rgba.ctypes.data) == 0
    # frame 1: the new depth converted at the current pose, one correspondence pass
    v1c, n1c = convert(d1, T0)
    AtA = np.zeros(36, np.float32)
    Atb = np.zeros(6, np.float32)
    nblk = C.c_int()
    assert lib.ref_find_corresponding(C.byref(cam), d1.ctypes.data, v1c.ctypes.data,
                                      n1c.ctypes.data, mv.ctypes.data, mn.ctypes.data,
                                      f32(inv(T0)).reshape(16).ctypes.data, AtA.ctypes.data,
                                      Atb.ctypes.data, C.byref(nblk)) == 0
    # second integration (frame 1 at its true pose): running averages, weight 2
    v1, n1 = convert(d1, T1)
    pos1 = f32(T1[:3, 3])
    assert lib.ref_integrate(C.byref(cam), v1.ctypes.data, f32(inv(T1)).reshape(16).ctypes.data,
                             pos1.ctypes.data) == 0
    t2 = np.zeros(len(flat), np.float32)
    w2 = np.zeros(len(flat), np.uint8)
    assert lib.ref_volume_read(flat.ctypes.data, len(flat), t2.ctypes.data, w2.ctypes.data) == 0
    # the host solve + transform build of ICP.cpp:142-172 on fixed increments
    xs = np.array([[0.004, -0.006, 0.003, 6.0, -4.0, -3.0],
                   [-0.02, 0.011, 0.007, -12.5, 3.25, 8.0]], np.float32)
    built = []
    for x in xs:
        T = f32(T0).reshape(16).copy()
        F = np.eye(4, dtype=np.float32).reshape(16).copy()
        xx = x.copy()
        lib.ref_build_transform(xx.ctypes.data, T.ctypes.data, F.ctypes.data)
        built.append(np.concatenate([T, F]))
    lib.ref_volume_free()
    out.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(out / "ref_frames.npz", depth0=d0, depth1=d1, T0=T0, T1=T1,
                        cam=np.array([W, H, FX, FY, CX, CY, DMIN, DMAX], np.float64),
                        vertex0=v0, normal0=n0, model_vertex=mv, model_normal=mn, rgba=rgba,
                        new_vertex=v1c, new_normal=n1c, AtA=AtA, Atb=Atb, blocks=nblk.value,
                        vertex1=v1, normal1=n1, xopt=xs, built=np.stack(built),
                        volume=np.array([n, lib.ref_world_volume(), lib.ref_truncation(),
                                         lib.ref_max_weight()], np.float64))
    np.savez_compressed(out / "ref_volume.npz", idx=idx.astype(np.int16), tsdf1=t1, w1=w1,
                        tsdf2=t2, w2=w2)
    print("updated voxels in the sample after frame 0:", int((w1 > 0).sum()), "of", len(w1))
    print("raycast hits:", int((mv[..., 0] < 1e30).sum()), "AtA[0]", float(AtA[0]))


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else ROOT / "tests" / "golden")
