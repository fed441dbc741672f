"""GPU tests of the boundary itself: the reference-shaped C++ classes, the
adapters to the reference's data layouts, volume export/import, the raw-depth
mode, and failure detection of the ICP grid barrier (a wait that nothing
completes must end with a status, not a hang)."""
import ctypes as C
import json
import subprocess
import sys
import time
from pathlib import Path

import numpy as np
import pytest

from conftest import pose_error

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


def dev_pose(P, device):
    import torch
    return torch.tensor(np.asarray(P, np.float64).reshape(16), dtype=torch.float64, device=device)


def c1(of, **kw):
    import dataclasses
    return dataclasses.replace(of.CONFIGS["c1"], **kw)


def test_cpp_reference_shaped_classes_track(of, cuda):
    sys.path.insert(0, str(ROOT / "tests" / "cpp"))
    import build_shim
    exe = build_shim.build()
    for args, max_mm in ((["20"], 5.0), (["8", "c2"], 5.0)):
        out = subprocess.run([str(exe), *args], capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        res = json.loads(out.stdout.strip().splitlines()[-1])
        assert res["cuda"] == "no error"
        assert res["bad_status"] == 0
        assert res["frames_per_s"] > 0
        assert res["max_trans_mm"] < max_mm and res["max_rot_rad"] < np.radians(0.5), res


def test_cpp_reference_icp_steps_equal_the_tracking_solve(of, ora, cuda):
    """The public ICP steps of the shim's C-ABI: of_icp_system then
    of_icp_solve_step (ICP::FindCorresponding + ICP::BuildNewTransformMatrix)
    equal the FP64 oracle's correspondence pass and solve on the same maps
    within the pose tolerance; a singular system leaves the pose unchanged."""
    import torch
    from test_gpu_parity import gpu_pyramid_to_oracle, icp_inputs
    cfg = c1(of)
    seq, vol, lam, model, frame = icp_inputs(of, None, cfg, cuda)
    ws = of.icp_workspace(cfg, cuda)
    lib = of._native.lib()
    stream = torch.cuda.current_stream().cuda_stream
    P0 = seq.poses[3]
    pose = dev_pose(P0, cuda)
    sys0 = of.icp_system(cfg, 0, frame, model, pose, ws)
    stats = torch.zeros(32, dtype=torch.uint8, device=cuda)
    assert lib.of_icp_solve_step(sys0.data_ptr(), pose.data_ptr(), stats.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    _, fpts = gpu_pyramid_to_oracle(of, ora, cfg, frame)
    _, mpts = gpu_pyramid_to_oracle(of, ora, cfg, model, with_depth=False)
    o, _ = ora.icp_system(cfg, 0, fpts[0], mpts[0], P0)
    st_o, Po, _ = ora.icp_step(o, P0)
    assert st_o == 0
    st = stats.cpu().numpy().view(np.int32)
    assert st[0] == 0 and st[2] == 1 and abs(st[1] - o[28]) <= 2
    rot, trans = pose_error(pose.cpu().numpy().reshape(4, 4), Po)
    assert rot < 1e-5 and trans < 1e-2, (rot, trans)
    zero = torch.zeros(32, dtype=torch.float32, device=cuda)
    before = pose.clone()
    assert lib.of_icp_solve_step(zero.data_ptr(), pose.data_ptr(), stats.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    assert torch.equal(before, pose) and stats.cpu().numpy().view(np.int32)[0] == 1


def test_icp_barrier_timeout_reports_status(of, cuda):
    import torch
    cfg = c1(of)
    seq = of.make_sequence(cfg, frames=3)
    vol, lam = of.new_volume(cfg, cuda), of.lambda_table(cfg, cuda)
    for k in range(2):
        of.integrate(cfg, vol, torch.from_numpy(seq.depth[k].astype(np.int16)).to(cuda),
                     dev_pose(seq.poses[k], cuda), lam)
    model = of.raycast(cfg, vol, dev_pose(seq.poses[1], cuda))
    frame = of.preprocess(cfg, torch.from_numpy(seq.depth[2].astype(np.int16)).to(cuda))
    ws = of.icp_workspace(cfg, cuda)
    lib = of._native.lib()
    stream = torch.cuda.current_stream().cuda_stream
    # hold every grid barrier for one arrival that never comes
    assert lib.of_icp_workspace_hold_barrier(ws.data_ptr(), 1, stream) == 0
    pose = dev_pose(seq.poses[1], cuda)
    stats = torch.zeros(32, dtype=torch.uint8, device=cuda)
    t0 = time.perf_counter()
    of.icp_track(cfg, frame, model, pose, ws, stats)
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    assert int(stats[:4].view(torch.int32).item()) == 2
    assert np.array_equal(pose.cpu().numpy().reshape(4, 4), seq.poses[1])
    assert elapsed < 5.0
    # the context is still usable and the workspace recovers
    assert lib.of_icp_workspace_hold_barrier(ws.data_ptr(), 0, stream) == 0
    of.icp_track(cfg, frame, model, pose, ws, stats)
    ws2 = of.icp_workspace(cfg, cuda)
    pose2 = dev_pose(seq.poses[1], cuda)
    of.icp_track(cfg, frame, model, pose2, ws2)
    torch.cuda.synchronize()
    assert int(stats[:4].view(torch.int32).item()) == 0
    assert np.array_equal(pose.cpu().numpy(), pose2.cpu().numpy())


def test_volume_export_import_roundtrip(of, cuda):
    import torch
    cfg = c1(of, resolution=64)
    seq = of.make_sequence(cfg, frames=2)
    vol, lam = of.new_volume(cfg, cuda), of.lambda_table(cfg, cuda)
    for k in range(2):
        of.integrate(cfg, vol, torch.from_numpy(seq.depth[k].astype(np.int16)).to(cuda),
                     dev_pose(seq.poses[k], cuda), lam)
    n = cfg.resolution
    tsdf = torch.empty(n ** 3, dtype=torch.float32, device=cuda)
    wgt = torch.empty(n ** 3, dtype=torch.int16, device=cuda)
    lib = of._native.lib()
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.of_volume_export(C.byref(cfg.volume()), vol.data_ptr(), tsdf.data_ptr(),
                                wgt.data_ptr(), stream) == 0
    q, w = of.volume_to_linear(cfg, vol.cpu().numpy())
    t = tsdf.cpu().numpy().reshape(n, n, n)
    expect = np.where(w > 0, q.view(np.int16) / 32767.0 * cfg.trunc_mm, cfg.trunc_mm)
    assert np.allclose(t, expect, atol=1e-6 * cfg.trunc_mm)
    assert np.array_equal(wgt.cpu().numpy().view(np.uint16).reshape(n, n, n), w)
    vol2 = of.new_volume(cfg, cuda)
    assert lib.of_volume_import(C.byref(cfg.volume()), vol2.data_ptr(), tsdf.data_ptr(),
                                wgt.data_ptr(), stream) == 0
    q2, w2 = of.volume_to_linear(cfg, vol2.cpu().numpy())
    assert np.array_equal(w2, w) and np.array_equal(q2[w > 0], q[w > 0])
    # imported bricks are all flagged, so the raycast cannot skip observed voxels
    flags = vol2.cpu().numpy().view(np.uint8)[4 * n ** 3:][: (n // 8) ** 3]
    assert flags.min() == 1


def test_reference_point_layout_roundtrip(of, cuda):
    import torch
    cfg = c1(of)
    seq = of.make_sequence(cfg, frames=2)
    vol, lam = of.new_volume(cfg, cuda), of.lambda_table(cfg, cuda)
    of.integrate(cfg, vol, torch.from_numpy(seq.depth[0].astype(np.int16)).to(cuda),
                 dev_pose(seq.poses[0], cuda), lam)
    model = of.raycast(cfg, vol, dev_pose(seq.poses[0], cuda))
    npx = cfg.width * cfg.height
    v3 = torch.empty(npx * 3, dtype=torch.float32, device=cuda)
    n3 = torch.empty(npx * 3, dtype=torch.float32, device=cuda)
    lib = of._native.lib()
    stream = torch.cuda.current_stream().cuda_stream
    assert lib.of_points_to_reference(C.byref(cfg.camera()), model.data_ptr(), None,
                                      v3.data_ptr(), n3.data_ptr(), stream) == 0
    vv = v3.cpu().numpy().reshape(cfg.height, cfg.width, 3)
    gv, gn = (t.cpu().numpy() for t in of.unpack_points(cfg, model, 0))
    bad = gv[..., 3] == 0
    assert np.all(vv[bad] == np.finfo(np.float32).max)       # BAD_VERTEX = FLT_MAX
    assert np.array_equal(vv[~bad], gv[..., :3][~bad])
    model2 = of.new_pyramid(cfg, cuda)
    assert lib.of_points_from_reference(C.byref(cfg.camera()), cfg.levels, v3.data_ptr(),
                                        n3.data_ptr(), model2.data_ptr(), stream) == 0
    for l in range(cfg.levels):
        a = [t.cpu().numpy() for t in of.unpack_points(cfg, model, l)]
        b = [t.cpu().numpy() for t in of.unpack_points(cfg, model2, l)]
        valid = (a[0][..., 3] > 0) & (a[1][..., 3] > 0)
        assert np.array_equal(a[0][valid], b[0][valid]) and np.array_equal(a[1][valid], b[1][valid])


def test_raw_depth_mode_matches_reference_conversion(of, ora, cuda):
    import torch
    cfg = c1(of, radius_px=-1)
    seq = of.make_sequence(cfg, frames=1)
    frame = of.preprocess(cfg, torch.from_numpy(seq.depth[0].astype(np.int16)).to(cuda))
    d0 = of.unpack_depth(cfg, frame, 0).cpu().numpy()
    raw = seq.depth[0].astype(np.float32)
    valid = (raw >= cfg.min_depth_mm) & (raw <= cfg.max_depth_mm)
    assert np.array_equal(d0, np.where(valid, raw, 0.0).astype(np.float32))
    levels, _ = ora.preprocess(cfg, seq.depth[0])
    assert np.array_equal(levels[0][0], np.where(valid, raw, 0.0))


def _pack(x, y, z, w):
    """rgbaFloatToIntCamera in float32 (saturate, scale, truncate)."""
    c = [np.clip(np.asarray(a, np.float32), 0, 1) for a in (x, y, z, w)]
    q = [(a * np.float32(255)).astype(np.uint32) for a in c]
    return (q[3] << 24) | (q[2] << 16) | (q[1] << 8) | q[0]


def test_headless_views(of, cuda):
    """Depth and normal RGBA views packed as the reference packs them."""
    import torch
    cfg = c1(of)
    seq = of.make_sequence(cfg, frames=1)
    d = torch.from_numpy(seq.depth[0].astype(np.int16)).to(cuda)
    g = of.depth_rgba(cfg, d).cpu().numpy().view(np.uint32)
    gray = seq.depth[0].astype(np.float32) * np.float32(1.0 / cfg.max_depth_mm)
    assert np.array_equal(g, _pack(gray, gray, gray, np.float32(1)))
    frame = of.preprocess(cfg, d)
    v, n = of.unpack_points(cfg, frame, 0)
    nn = n.cpu().numpy()
    ok = (v.cpu().numpy()[..., 3] != 0) & (nn[..., 3] != 0)
    nv = np.where(ok[..., None], nn[..., :3], 0).astype(np.float32)
    r = of.normals_rgba(cfg, frame, alpha=0.0).cpu().numpy().view(np.uint32)
    h = np.float32(0.5)
    exp = _pack((nv[..., 0] + 1) * h, (nv[..., 1] + 1) * h, (nv[..., 2] + 1) * h, np.float32(0))
    assert np.array_equal(r, exp)
    assert (r != _pack(h, h, h, np.float32(0))).mean() > 0.5


def test_shaded_raycast_view_matches_oracle(of, ora, cuda):
    """The raycast's shaded RGBA (Raycaster.cu:212-228, showNormal false):
    0.6 (-d . n) + 0.2 in grey, black where d . n vanishes, alpha 0, packed
    by rgbaFloatToInt. Stepwise against the FP64 restatement on the GPU's own
    normals: every channel within 1 LSB (FP32 against FP64 before the
    truncation to 8 bits), almost every pixel exact; and end to end against
    the FP64 oracle's own raycast normals on the rays both hit."""
    import torch
    from test_gpu_parity import build_state
    cfg = c1(of)
    seq, vol, lam = build_state(of, cfg, 4, cuda)
    pose = seq.poses[3]
    rgba = torch.zeros((cfg.height, cfg.width), dtype=torch.int32, device=cuda)
    model = of.raycast(cfg, vol, dev_pose(pose, cuda), rgba=rgba)
    torch.cuda.synchronize()
    g = rgba.cpu().numpy().view(np.uint32)
    v, n = (t.cpu().numpy().astype(np.float64) for t in of.unpack_points(cfg, model, 0))
    nrm = np.where(n[..., 3:4] > 0, n[..., :3], 0.0)
    exp = ora.shade_rgba(cfg, pose, nrm)
    assert np.all(g >> 24 == 0), "alpha is 0"
    ch = [(g >> s) & 0xFF for s in (0, 8, 16)]
    assert np.array_equal(ch[0], ch[1]) and np.array_equal(ch[0], ch[2]), "grey"
    diff = np.abs(ch[0].astype(np.int64) - (exp & 0xFF).astype(np.int64))
    assert diff.max() <= 1, diff.max()
    assert (diff == 0).mean() > 0.999, (diff == 0).mean()
    hit = n[..., 3] > 0
    assert hit.mean() > 0.5 and np.all(ch[0][~hit] == 0)
    lit = ch[0][hit]
    assert lit.max() > 150 and np.median(lit) > 60, "surfaces facing the camera are lit"
    # end to end: the oracle's own normals of the same volume
    host = vol.cpu().numpy()
    q, w = of.volume_to_linear(cfg, host)
    words = (q.astype(np.uint32) | (w.astype(np.uint32) << 16)).reshape(-1).copy()
    opts, amb = ora.raycast(cfg, words, pose, ambig=True)
    both = hit & (opts[..., 7] > 0) & (amb == 0)
    e2e = ora.shade_rgba(cfg, pose, np.where(opts[..., 7:8] > 0, opts[..., 4:7], 0.0))
    d2 = np.abs(ch[0][both].astype(np.int64) - (e2e[both] & 0xFF).astype(np.int64))
    assert np.quantile(d2, 0.99) <= 1 and np.median(d2) == 0, (np.quantile(d2, 0.99), d2.max())
