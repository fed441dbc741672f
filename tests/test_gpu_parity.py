"""Parity of the CUDA path against the FP64 oracle on the same seeded inputs.

Every comparison is stepwise: the oracle consumes the GPU's own input state
(volume, frame and model maps, pose) for the stage under test, so only that
stage's arithmetic is compared. Decisions that sit within FP32 rounding of a
boundary (pixel rounding at .5, a depth at the range limit, an SDF at -trunc,
a tsdf sample at 0) are flagged by the oracle and excluded; their number is
bounded. Tolerances (from the path's precision targets):
  TSDF      within 1 int16 quantisation step (trunc / 32767)
  vertices  within 1e-4 m = 0.1 mm (every ray the oracle does not flag; a
            ray whose march is chaotic must be reproduced by the oracle's
            march under a bounded position perturbation)
  pose      within 1e-5 rad and 1e-5 m = 0.01 mm
"""
import numpy as np
import pytest

from conftest import pose_error

pytestmark = pytest.mark.gpu


def small(of, name="c1", **kw):
    import dataclasses
    return dataclasses.replace(of.CONFIGS[name], **kw)


def dev_pose(P, device):
    import torch
    return torch.tensor(np.asarray(P, np.float64).reshape(16), dtype=torch.float64, device=device)


def build_state(of, cfg, frames, device):
    """Volume after fusing `frames` frames at ground-truth poses."""
    import torch
    seq = of.make_sequence(cfg, frames=frames + 1)
    vol = of.new_volume(cfg, device)
    lam = of.lambda_table(cfg, device)
    for k in range(frames):
        d = torch.from_numpy(seq.depth[k].astype(np.int16)).to(device)
        of.integrate(cfg, vol, d, dev_pose(seq.poses[k], device), lam)
    torch.cuda.synchronize()
    return seq, vol, lam


def check_rays(ora, cfg, words, flags, pose, gv, opts, amb, flagged_max=1e-2):
    """Every ray the oracle does not flag: hit and miss as the oracle, vertex
    within 0.1 mm, or, for a ray whose march is chaotic, the GPU's result
    reproduced by the oracle's march under a position perturbation of at most
    0.05 mm per update (tests/raycast_check.py); such rays are few."""
    import raycast_check
    r = raycast_check.compare(ora, cfg, words, flags, pose, gv, opts, amb)
    assert r["flagged"] <= flagged_max * r["rays"], r
    assert not r["unexplained"], r
    assert r["rounding_sensitive"] <= max(3, 1e-4 * r["rays"]), r
    assert r["max_err_mm"] < 0.1 and r["median_err_mm"] < 0.01, r
    return r


def gpu_pyramid_to_oracle(of, ora, cfg, pyr, with_depth=True):
    pts, deps = [], []
    for l in range(cfg.levels):
        v, n = of.unpack_points(cfg, pyr, l)
        pts.append(np.concatenate([v.cpu().numpy(), n.cpu().numpy()], axis=-1))
        deps.append(of.unpack_depth(cfg, pyr, l).cpu().numpy() if with_depth else None)
    return ora.pack_pyramid(cfg, pts, deps if with_depth else None), pts


# ---------------------------------------------------------------- preprocess

@pytest.mark.parametrize("name,size", [("c1", None), ("c2", None), ("c1", (161, 121))])
def test_preprocess_matches_oracle(of, ora, cuda, name, size):
    """Stepwise: the bilateral filter against the oracle on the raw depth, each
    pyramid level against the oracle's block average of the GPU's level above,
    each vertex/normal map against the oracle's maps of the GPU's depth."""
    import torch
    cfg = small(of, name) if size is None else small(
        of, name, width=size[0], height=size[1], cx=(size[0] - 1) / 2, cy=(size[1] - 1) / 2)
    seq = of.make_sequence(cfg, frames=1)
    d = torch.from_numpy(seq.depth[0].astype(np.int16)).to(cuda)
    pyr = of.preprocess(cfg, d)
    torch.cuda.synchronize()
    levels, _ = ora.preprocess(cfg, seq.depth[0])
    gdeps = [of.unpack_depth(cfg, pyr, l).cpu().numpy().astype(np.float64) for l in range(cfg.levels)]
    for l in range(cfg.levels):
        gdep = gdeps[l]
        odep = levels[0][0] if l == 0 else ora.pyr_down(cfg, gdeps[l - 1])
        valid_o, valid_g = odep > 0, gdep > 0
        assert np.array_equal(valid_o, valid_g), f"level {l} validity mismatch"
        rel = np.abs(gdep[valid_o] - odep[valid_o]) / odep[valid_o]
        # FP32 weights (ex2.approx) and sums vs FP64 exp: a few ulp relative
        assert rel.max() < 5e-6, f"level {l} filtered depth rel err {rel.max()}"
        gv, gn = (t.cpu().numpy().astype(np.float64) for t in of.unpack_points(cfg, pyr, l))
        opts = ora.vertex_normal(cfg, l, gdep)
        assert np.array_equal(gv[..., 3] > 0, opts[..., 3] > 0)
        vb = opts[..., 3] > 0
        verr = np.linalg.norm(gv[..., :3][vb] - opts[..., :3][vb], axis=-1)
        assert verr.max() < 1e-2, f"level {l} vertex err {verr.max()} mm"
        assert np.array_equal(gn[..., 3] > 0, opts[..., 7] > 0)
        nb = opts[..., 7] > 0
        nerr = np.linalg.norm(gn[..., :3][nb] - opts[..., 4:7][nb], axis=-1)
        # a few FP32 roundings, amplified where the two tangents are nearly parallel
        assert np.median(nerr) < 1e-6 and nerr.max() < 1e-4, f"level {l} normal err {nerr.max()}"
        # end to end against the FP64 oracle's own pyramid: vertices within 0.1 mm
        ov = levels[l][1]
        both = (gv[..., 3] > 0) & (ov[..., 3] > 0)
        assert (both.sum() >= 0.999 * (ov[..., 3] > 0).sum())
        e2e = np.linalg.norm(gv[..., :3][both] - ov[..., :3][both], axis=-1)
        assert e2e.max() < 0.1, f"level {l} vertex vs FP64 pipeline {e2e.max()} mm"


# ---------------------------------------------------------------- integrate

def test_visible_census_counts_the_voxels_in_view(of, cuda):
    """of_integrate_visible_census against an FP64 count of the same test:
    voxel centre inside the 2-pixel border (roundFloat pixel) with a depth in
    [min, max] (VolumeIntegrator.cu:12-16, :131)."""
    import torch
    cfg = small(of, "c1", resolution=128)
    seq = of.make_sequence(cfg, frames=3)
    vol, lam = of.new_volume(cfg, cuda), of.lambda_table(cfg, cuda)
    counts = []
    for k in (1, 2):
        d = torch.from_numpy(seq.depth[k].astype(np.int16)).to(cuda)
        n_gpu = of.integrate_visible_census(cfg, vol, d, dev_pose(seq.poses[k], cuda), lam)
        P = np.asarray(seq.poses[k], np.float64)
        n = cfg.resolution
        vs = cfg.size_mm / n
        g = -0.5 * cfg.size_mm + 0.5 * vs + vs * np.arange(n)
        X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
        pc = (np.stack([X, Y, Z], -1).reshape(-1, 3) - P[:3, 3]) @ P[:3, :3]
        with np.errstate(all="ignore"):
            u = np.floor(cfg.fx * pc[:, 0] / pc[:, 2] + cfg.cx + 0.5)
            v = np.floor(cfg.fy * pc[:, 1] / pc[:, 2] + cfg.cy + 0.5)
        z = -pc[:, 2]
        ok = ((z >= cfg.min_depth_mm) & (z <= cfg.max_depth_mm) & (u >= 2) & (u <= cfg.width - 3)
              & (v >= 2) & (v <= cfg.height - 3))
        n_np = int(ok.sum())
        counts.append(n_gpu)
        assert n_np > 0.1 * n ** 3, "the view should cover a good part of the cube"
        # FP32 pixel rounding moves only voxels within ~1e-4 px of the border
        assert abs(n_gpu - n_np) <= 20 + 1e-4 * n_np, (k, n_gpu, n_np)
    # the count does not depend on the volume's contents
    of.integrate(cfg, vol, d, dev_pose(seq.poses[2], cuda), lam)
    assert of.integrate_visible_census(cfg, vol, d, dev_pose(seq.poses[2], cuda), lam) == counts[1]


@pytest.mark.parametrize("name,res,storage,tiled", [("c1", 128, "i16", False),
                                                    ("c2", 256, "i16", False),
                                                    ("c2", 512, "i16", False),
                                                    ("c2", 512, "i16", True),
                                                    ("c1", 128, "f16", True)])
def test_integrate_matches_oracle(of, ora, cuda, name, res, storage, tiled):
    import torch
    cfg = small(of, name, resolution=res, storage=storage)
    seq, vol, lam = build_state(of, cfg, 3, cuda)
    k = 3
    q0, w0 = of.volume_to_linear(cfg, vol.cpu().numpy())
    words = ((q0.astype(np.uint32)) | (w0.astype(np.uint32) << 16)).reshape(-1).copy()
    d = seq.depth[k]
    pose = seq.poses[k]
    n_ora, amb = ora.integrate(cfg, words, d, pose, ambig=True)
    dt = torch.from_numpy(d.astype(np.int16)).to(cuda)
    pt = dev_pose(pose, cuda)
    n_gpu = of.integrate_census(cfg, vol, dt, pt, lam)
    of.integrate(cfg, vol, dt, pt, lam, of.integrate_scratch(cfg, cuda) if tiled else None)
    torch.cuda.synchronize()
    q1, w1 = of.volume_to_linear(cfg, vol.cpu().numpy())
    qo = (words & 0xFFFF).astype(np.uint16).reshape(q1.shape)
    wo = (words >> 16).astype(np.uint16).reshape(q1.shape)
    ok = amb.reshape(q1.shape) == 0
    n_amb = int((~ok).sum())
    assert abs(n_gpu - n_ora) <= n_amb, (n_gpu, n_ora, n_amb)
    assert n_amb < 5e-3 * ok.size
    assert np.array_equal(w1[ok], wo[ok]), "weights differ"
    if storage == "i16":
        dq = np.abs(q1[ok].view(np.int16).astype(np.int32) - qo[ok].view(np.int16).astype(np.int32))
        assert dq.max() <= 1, f"tsdf differs by {dq.max()} int16 steps"
    else:
        g = q1[ok].view(np.float16).astype(np.float64)
        o = qo[ok].view(np.float16).astype(np.float64)
        # fp16 of a value in [-1, 1]: one ulp is at most 2^-11
        assert np.abs(g - o).max() <= 2.0 ** -11 * 1.001


@pytest.mark.parametrize("name,res,storage,geom", [("c2", 512, "i16", None),
                                                   ("c1", 128, "f16", None),
                                                   ("c2", 512, "i16", (1024.0, 10.0, 120, 50.0))])
def test_integrate_tiled_equals_per_voxel(of, cuda, name, res, storage, geom):
    """of_integrate_tiled decides whole bricks from per-tile depth bounds (skip
    behind the surface, +1 in free space); over a run of frames the volume it
    writes, brick flags included, is bit-identical to of_integrate's."""
    import torch
    kw = dict(resolution=res, storage=storage)
    if geom:
        # the reference's cube (1 m, 10 mm truncation): the scaled room sits
        # 0.1-0.2 m from the camera
        kw.update(size_mm=geom[0], trunc_mm=geom[1], max_weight=geom[2], min_depth_mm=geom[3])
    cfg = small(of, name, **kw)
    seq = of.make_sequence(cfg, frames=8)
    lam, scratch = of.lambda_table(cfg, cuda), of.integrate_scratch(cfg, cuda)
    va, vb = of.new_volume(cfg, cuda), of.new_volume(cfg, cuda)
    for k in range(8):
        d = torch.from_numpy(seq.depth[k].astype(np.int16)).to(cuda)
        p = dev_pose(seq.poses[k], cuda)
        of.integrate(cfg, va, d, p, lam)
        of.integrate(cfg, vb, d, p, lam, scratch)
        torch.cuda.synchronize()
        assert torch.equal(va, vb), f"volumes differ after frame {k}"
    # the run touched the volume
    _, w = of.volume_to_linear(cfg, vb.cpu().numpy())
    assert (w > 0).sum() > 10000


@pytest.mark.parametrize("size", [(161, 121), (203, 157)])
def test_ragged_frame_sizes(of, ora, cuda, size):
    """Frames whose sides are not multiples of the 8x8 depth tiles or of the
    16x16 ray blocks: the tiled integration (partial tiles, the per-pixel L
    map) still writes the per-voxel path's volume bit for bit, the raycast's
    level 0 matches the oracle, and its coarser levels are the 2^l subsamples."""
    import torch
    w, h = size
    f = 262.5 * w / 320.0
    cfg = small(of, "c1", width=w, height=h, fx=f, fy=f, cx=(w - 1) / 2, cy=(h - 1) / 2)
    seq = of.make_sequence(cfg, frames=5)
    lam, scratch = of.lambda_table(cfg, cuda), of.integrate_scratch(cfg, cuda)
    va, vb = of.new_volume(cfg, cuda), of.new_volume(cfg, cuda)
    for k in range(4):
        d = torch.from_numpy(seq.depth[k].astype(np.int16)).to(cuda)
        p = dev_pose(seq.poses[k], cuda)
        of.integrate(cfg, va, d, p, lam)
        of.integrate(cfg, vb, d, p, lam, scratch)
        torch.cuda.synchronize()
        assert torch.equal(va, vb), f"volumes differ after frame {k}"
    pose = seq.poses[4]
    model = of.raycast(cfg, vb, dev_pose(pose, cuda))
    torch.cuda.synchronize()
    host = vb.cpu().numpy()
    q, wt = of.volume_to_linear(cfg, host)
    assert (wt > 0).sum() > 10000
    words = (q.astype(np.uint32) | (wt.astype(np.uint32) << 16)).reshape(-1).copy()
    nb = cfg.resolution // 8
    flags = host.view(np.uint8)[4 * cfg.resolution ** 3:][: nb ** 3].copy()
    opts, amb = ora.raycast(cfg, words, pose, ambig=True, flags=flags)
    v0, n0 = (t.cpu().numpy() for t in of.unpack_points(cfg, model, 0))
    gv = v0.astype(np.float64)
    assert (opts[..., 3] > 0).mean() > 0.3, "the scene should be mostly visible"
    check_rays(ora, cfg, words, flags, pose, gv, opts, amb)
    for l in range(1, cfg.levels):
        vl, nl = (t.cpu().numpy() for t in of.unpack_points(cfg, model, l))
        s = 1 << l
        assert vl.shape[:2] == ((h + s - 1) // s, (w + s - 1) // s)
        assert np.array_equal(vl, v0[::s, ::s]) and np.array_equal(nl, n0[::s, ::s])


def test_saturated_free_space_is_skipped_exactly(of, cuda):
    """With a maximum weight of 3, free space saturates (+1 at weight 3) after
    three frames; the tiled integration then leaves those bricks unlisted.
    Over 12 frames the volume, brick flags and saturated-brick bytes stay bit
    for bit those of the per-voxel path, and saturated bricks exist."""
    import torch
    cfg = small(of, "c2", resolution=256, max_weight=3)
    seq = of.make_sequence(cfg, frames=12)
    lam, scratch = of.lambda_table(cfg, cuda), of.integrate_scratch(cfg, cuda)
    va, vb = of.new_volume(cfg, cuda), of.new_volume(cfg, cuda)
    for k in range(12):
        d = torch.from_numpy(seq.depth[k].astype(np.int16)).to(cuda)
        p = dev_pose(seq.poses[k], cuda)
        of.integrate(cfg, va, d, p, lam)
        of.integrate(cfg, vb, d, p, lam, scratch)
        torch.cuda.synchronize()
        assert torch.equal(va, vb), f"volumes differ after frame {k}"
    host = vb.cpu().numpy().view(np.uint8)
    n, nb = cfg.resolution, cfg.resolution // 8
    ns = (nb + 3) // 4
    off = 4 * n ** 3 + (nb ** 3 + 255) // 256 * 256 + (ns ** 3 + 255) // 256 * 256
    sat = host[off:off + nb ** 3] == 0xF
    assert 100 < int(sat.sum()) < nb ** 3
    # a saturated brick holds only +1 at the maximum weight
    q, w = of.volume_to_linear(cfg, vb.cpu().numpy())
    qb = q.reshape(nb, 8, nb, 8, nb, 8).transpose(0, 2, 4, 1, 3, 5).reshape(-1, 512)
    wb = w.reshape(nb, 8, nb, 8, nb, 8).transpose(0, 2, 4, 1, 3, 5).reshape(-1, 512)
    assert np.all(qb[sat] == 0x7FFF) and np.all(wb[sat] == 3)


# ---------------------------------------------------------------- raycast

@pytest.mark.parametrize("name,res", [("c1", 128), ("c2", 512)])
def test_raycast_matches_oracle(of, ora, cuda, name, res):
    import torch
    cfg = small(of, name, resolution=res)
    seq, vol, lam = build_state(of, cfg, 4, cuda)
    pose = seq.poses[3]
    model = of.raycast(cfg, vol, dev_pose(pose, cuda))
    torch.cuda.synchronize()
    host = vol.cpu().numpy()
    q, w = of.volume_to_linear(cfg, host)
    words = (q.astype(np.uint32) | (w.astype(np.uint32) << 16)).reshape(-1).copy()
    nb = cfg.resolution // 8
    flags = host.view(np.uint8)[4 * cfg.resolution ** 3:][: nb ** 3].copy()
    # the volume keeps one super-brick flag per 4^3 bricks: the OR of theirs
    ns = (nb + 3) // 4
    soff = 4 * cfg.resolution ** 3 + (nb ** 3 + 255) // 256 * 256
    sflags = host.view(np.uint8)[soff:soff + ns ** 3].reshape(ns, ns, ns)
    pad = np.zeros((ns * 4,) * 3, np.uint8)
    pad[:nb, :nb, :nb] = flags.reshape(nb, nb, nb)
    assert np.array_equal(sflags != 0, pad.reshape(ns, 4, ns, 4, ns, 4).max(axis=(1, 3, 5)) != 0)
    opts, amb = ora.raycast(cfg, words, pose, ambig=True, flags=flags)
    # Empty-space skipping only moves where the samples after a jump fall:
    # the oracle without it finds the same surface on all but the rays whose
    # negative stretch is thinner than one step (found by one march, stepped
    # over by the other).
    plain, _ = ora.raycast(cfg, words, pose)
    hp = (plain[..., 3] > 0) & (opts[..., 3] > 0)
    assert ((plain[..., 3] > 0) != (opts[..., 3] > 0)).mean() < 5e-3
    dp = np.linalg.norm(plain[..., :3][hp] - opts[..., :3][hp], axis=-1)
    assert np.quantile(dp, 0.99) < 0.1
    # The GPU against the oracle with the same skipping, ray by ray.
    gv, gn = (t.cpu().numpy().astype(np.float64) for t in of.unpack_points(cfg, model, 0))
    ok = amb == 0
    hit_g, hit_o = gv[..., 3] > 0, opts[..., 3] > 0
    assert hit_o.mean() > 0.5, "scene should be mostly visible"
    check_rays(ora, cfg, words, flags, pose, gv, opts, amb)
    both = hit_g & hit_o & ok
    nb = both & (gn[..., 3] > 0) & (opts[..., 7] > 0)
    nerr = np.linalg.norm(gn[..., :3][nb] - opts[..., 4:7][nb], axis=-1)
    assert np.median(nerr) < 1e-3
    # the coarser model levels written by the raycast: pixel (x, y) of level l
    # is level 0's pixel (2^l x, 2^l y), exactly
    v0, n0 = (t.cpu().numpy() for t in of.unpack_points(cfg, model, 0))
    for l in range(1, cfg.levels):
        vl, nl = (t.cpu().numpy() for t in of.unpack_points(cfg, model, l))
        s = 1 << l
        assert vl.shape[:2] == ((cfg.height + s - 1) // s, (cfg.width + s - 1) // s)
        assert np.array_equal(vl, v0[::s, ::s]) and np.array_equal(nl, n0[::s, ::s])


# ---------------------------------------------------------------- ICP

def icp_inputs(of, ora, cfg, cuda):
    import torch
    seq, vol, lam = build_state(of, cfg, 4, cuda)
    model = of.raycast(cfg, vol, dev_pose(seq.poses[3], cuda))
    d = torch.from_numpy(seq.depth[4].astype(np.int16)).to(cuda)
    frame = of.preprocess(cfg, d)
    torch.cuda.synchronize()
    return seq, vol, lam, model, frame


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_icp_system_matches_oracle(of, ora, cuda, name):
    cfg = small(of, name)
    seq, vol, lam, model, frame = icp_inputs(of, ora, cfg, cuda)
    fbuf, fpts = gpu_pyramid_to_oracle(of, ora, cfg, frame)
    mbuf, mpts = gpu_pyramid_to_oracle(of, ora, cfg, model, with_depth=False)
    ws = of.icp_workspace(cfg, cuda)
    pose = seq.poses[3]  # previous pose: the usual ICP starting point
    for level in range(cfg.levels):
        g = of.icp_system(cfg, level, frame, model, dev_pose(pose, cuda), ws).cpu().numpy()
        o, amb = ora.icp_system(cfg, level, fpts[level], mpts[level], pose)
        assert o[28] > 100, "too few correspondences"
        # Cauchy-Schwarz scale of every sum: sqrt(H_ii H_jj), sqrt(H_ii sum b^2)
        diag = np.array([o[k] for k in (0, 6, 11, 15, 18, 20)])
        scale = np.zeros(29)
        k = 0
        for i in range(6):
            for j in range(i, 6):
                scale[k] = np.sqrt(diag[i] * diag[j]); k += 1
        scale[21:27] = np.sqrt(diag * o[27])
        scale[27] = o[27]
        # FP32 rows and compensated FP32 sums vs FP64 sums of the same rows,
        # plus the whole contribution of pixels at a rounding boundary
        bound = 2e-5 * scale + amb
        err = np.abs(g - o)
        assert np.all(err <= bound + 1e-6), f"level {level}: {err / (scale + 1e-30)}"


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_icp_track_matches_oracle(of, ora, cuda, name):
    import torch
    cfg = small(of, name)
    seq, vol, lam, model, frame = icp_inputs(of, ora, cfg, cuda)
    fbuf, _ = gpu_pyramid_to_oracle(of, ora, cfg, frame)
    mbuf, _ = gpu_pyramid_to_oracle(of, ora, cfg, model, with_depth=False)
    ws = of.icp_workspace(cfg, cuda)
    pose0 = seq.poses[3]
    pt = dev_pose(pose0, cuda)
    stats = torch.zeros(32, dtype=torch.uint8, device=cuda)
    of.icp_track(cfg, frame, model, pt, ws, stats)
    gpose = pt.cpu().numpy().reshape(4, 4)
    st, opose, its = ora.icp_track(cfg, fbuf, mbuf, pose0)
    assert st == 0
    status = int(stats[:4].view(torch.int32).item())
    assert status == 0
    rot, trans = pose_error(gpose, opose)
    assert rot < 1e-5 and trans < 1e-2, (rot, trans)
    # and the tracked pose is close to the ground truth of the frame
    rot_gt, trans_gt = pose_error(gpose, seq.poses[4])
    assert rot_gt < np.radians(0.5) and trans_gt < 10.0


def test_icp_singular_restores_pose(of, cuda):
    import torch
    cfg = small(of, "c1")
    seq, vol, lam = build_state(of, cfg, 2, cuda)
    model = of.raycast(cfg, vol, dev_pose(seq.poses[1], cuda))
    empty = torch.zeros((cfg.height, cfg.width), dtype=torch.int16, device=cuda)
    frame = of.preprocess(cfg, empty)
    ws = of.icp_workspace(cfg, cuda)
    pt = dev_pose(seq.poses[1], cuda)
    stats = torch.zeros(32, dtype=torch.uint8, device=cuda)
    of.icp_track(cfg, frame, model, pt, ws, stats)
    torch.cuda.synchronize()
    assert int(stats[:4].view(torch.int32).item()) == 1
    assert np.array_equal(pt.cpu().numpy().reshape(4, 4), seq.poses[1])


# ---------------------------------------------------------------- tracker

def test_tracker_graph_equals_eager(of, cuda):
    import torch
    cfg = small(of, "c1")
    seq = of.make_sequence(cfg, frames=6)
    poses = []
    for graph in (True, False):
        tr = of.Tracker(cfg, seq.poses[0], use_graph=graph)
        for k in range(6):
            tr.process(torch.from_numpy(seq.depth[k].astype(np.int16)).to(cuda))
        poses.append(tr.pose_history(6))
        tr.close()
    assert np.array_equal(poses[0], poses[1])


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_tracker_online_tuning_changes_no_result(of, cuda, name):
    """A tracker that tunes the raycast block shape online (step 2 times
    every shape, then the step graphs are captured) tracks bit for bit like
    one with the default shape, and every shape gives the same model."""
    import dataclasses
    import torch
    cfg = small(of, name)
    seq = of.make_sequence(cfg, frames=6)
    depth = [torch.from_numpy(seq.depth[k].astype(np.int16)).to(cuda) for k in range(6)]
    runs = []
    for tune in (0, 2):
        tr = of.Tracker(cfg, seq.poses[0], use_graph=True, tune=tune)
        for d in depth:
            tr.process(d)
        runs.append((tr.pose_history(6), tr.tuning()))
        tr.close()
    assert runs[0][1] == (0, False)
    assert runs[1][1][1] and 0 <= runs[1][1][0] < 7, runs[1][1]
    assert np.array_equal(runs[0][0], runs[1][0])
    vol, lam = of.new_volume(cfg, cuda), of.lambda_table(cfg, cuda)
    for k in range(3):
        of.integrate(cfg, vol, depth[k], dev_pose(seq.poses[k], cuda), lam)
    models = [of.raycast(dataclasses.replace(cfg, ray_tile=t), vol, dev_pose(seq.poses[2], cuda))
              for t in range(7)]
    torch.cuda.synchronize()
    for m in models[1:]:
        assert torch.equal(m, models[0])


def test_tracker_equals_stagewise_pipeline(of, cuda):
    """The tracker's step (fuse k-1 and raycast beside pre-process k, then
    ICP k) gives bit for bit the poses of the stage-by-stage sequence
    integrate(k-1) -> raycast(k-1) -> preprocess(k) -> ICP(k) through the
    public per-stage calls."""
    import torch
    cfg = small(of, "c1")
    n = 6
    seq = of.make_sequence(cfg, frames=n)
    depth = [torch.from_numpy(seq.depth[k].astype(np.int16)).to(cuda) for k in range(n)]
    tr = of.Tracker(cfg, seq.poses[0], use_graph=True)
    for k in range(n):
        tr.process(depth[k])
    hist = tr.pose_history(n)
    tr.close()
    vol, lam = of.new_volume(cfg, cuda), of.lambda_table(cfg, cuda)
    scratch = of.integrate_scratch(cfg, cuda)
    frame, model = of.new_pyramid(cfg, cuda), of.new_pyramid(cfg, cuda)
    ws = of.icp_workspace(cfg, cuda)
    pose = dev_pose(seq.poses[0], cuda)
    ref = [seq.poses[0]]
    for k in range(1, n):
        of.integrate(cfg, vol, depth[k - 1], pose, lam, scratch)
        of.raycast(cfg, vol, pose, model)
        of.preprocess(cfg, depth[k], frame)
        of.icp_track(cfg, frame, model, pose, ws)
        ref.append(pose.cpu().numpy().reshape(4, 4).copy())
    assert np.array_equal(hist, np.array(ref))


def test_tracker_flush_fuses_the_last_frame_once(of, cuda):
    """of_tracker_flush fuses the last frame early; later steps skip that
    fusion, so poses and the final volume equal those of a tracker that never
    flushed (and then flushes once)."""
    import ctypes as C
    import torch
    cfg = small(of, "c1", resolution=64)
    n = 8
    seq = of.make_sequence(cfg, frames=n)
    depth = [torch.from_numpy(seq.depth[k].astype(np.int16)).to(cuda) for k in range(n)]
    lib, stream = of._native.lib(), torch.cuda.current_stream().cuda_stream
    out = []
    for flush_at in ((), (2, 3, 5)):
        tr = of.Tracker(cfg, seq.poses[0], use_graph=True)
        for k in range(n):
            tr.process(depth[k])
            if k in flush_at:
                tr.flush()
                tr.flush()  # a second flush has no effect
        tr.flush()
        hist = tr.pose_history(n)
        m = cfg.resolution ** 3
        tsdf = torch.empty(m, dtype=torch.float32, device=cuda)
        wgt = torch.empty(m, dtype=torch.int16, device=cuda)
        assert lib.of_volume_export(C.byref(cfg.volume()), C.c_void_p(tr.buffers().volume),
                                    tsdf.data_ptr(), wgt.data_ptr(), stream) == 0
        torch.cuda.synchronize()
        out.append((hist, tsdf.cpu().numpy(), wgt.cpu().numpy()))
        tr.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])
    assert out[0][2].view(np.uint16).max() == n  # every frame fused exactly once


def test_tracker_follows_ground_truth(of, cuda):
    import torch
    cfg = small(of, "c1")
    seq = of.make_sequence(cfg, frames=30)
    tr = of.Tracker(cfg, seq.poses[0])
    pinned = torch.from_numpy(seq.depth.astype(np.int16)).pin_memory()
    for k in range(30):
        tr.process(pinned[k])
    hist = tr.pose_history(30)
    tr.close()
    errs = [pose_error(hist[k], seq.poses[k]) for k in range(30)]
    assert max(e[1] for e in errs) < 5.0, errs
    assert max(e[0] for e in errs) < np.radians(0.5)


def test_tracker_checkpoint_resume(of, cuda, tmp_path):
    """A tracker saved after 5 frames and loaded into a fresh tracker (graph
    or eager) continues bit for bit as the saved one: poses of frames 5..9,
    the pose history, and the final volume."""
    import ctypes as C
    import torch
    cfg = small(of, "c1", resolution=64)
    seq = of.make_sequence(cfg, frames=10)
    depth = [torch.from_numpy(seq.depth[k].astype(np.int16)).to(cuda) for k in range(10)]
    a = of.Tracker(cfg, seq.poses[0])
    for k in range(5):
        a.process(depth[k])
    a.save(tmp_path / "t.ofck")
    b = of.Tracker(cfg, np.eye(4), use_graph=False)
    b.load(tmp_path / "t.ofck")
    assert b.frames == 5
    for k in range(5, 10):
        a.process(depth[k])
        b.process(depth[k])
    assert np.array_equal(a.pose_history(10), b.pose_history(10))
    a.flush()
    b.flush()
    torch.cuda.synchronize()
    lib, st = of._native.lib(), torch.cuda.current_stream().cuda_stream
    m = cfg.resolution ** 3
    outs = []
    for tr in (a, b):
        t_ = torch.empty(m, dtype=torch.float32, device=cuda)
        w_ = torch.empty(m, dtype=torch.int16, device=cuda)
        assert lib.of_volume_export(C.byref(cfg.volume()), C.c_void_p(tr.buffers().volume),
                                    t_.data_ptr(), w_.data_ptr(), st) == 0
        torch.cuda.synchronize()
        outs.append((t_.cpu().numpy(), w_.cpu().numpy()))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    # a checkpoint of another volume is refused
    other = of.Tracker(small(of, "c1", resolution=32), seq.poses[0])
    from openfusion_b200._native import OpenFusionError
    with pytest.raises(OpenFusionError) as e:
        other.load(tmp_path / "t.ofck")
    assert e.value.status == 1
    for tr in (a, b, other):
        tr.close()


def test_tracker_survives_corrupt_frames(of, cuda):
    """Faults injected on the host: an empty frame (no depth at all) makes ICP
    singular, so the pose of the frame before stays and the status says so; a
    frame of uniform noise is tracked without error and the pose stays finite;
    good frames after them are processed as usual."""
    import torch
    cfg = small(of, "c1")
    seq = of.make_sequence(cfg, frames=8)
    tr = of.Tracker(cfg, seq.poses[0])
    for k in range(4):
        tr.process(torch.from_numpy(seq.depth[k].astype(np.int16)).to(cuda))
    tr.process(torch.zeros((cfg.height, cfg.width), dtype=torch.int16, device=cuda))
    _, st4 = tr.pose()
    assert st4.status == 1  # singular system: no correspondences
    rng = np.random.default_rng(3)
    noise = rng.integers(0, 65536, (cfg.height, cfg.width)).astype(np.uint16).view(np.int16)
    tr.process(torch.from_numpy(noise).to(cuda))
    _, st5 = tr.pose()
    assert st5.status in (0, 1)
    for k in range(6, 8):
        tr.process(torch.from_numpy(seq.depth[k].astype(np.int16)).to(cuda))
    hist = tr.pose_history(8)
    tr.close()
    assert np.array_equal(hist[4], hist[3])  # singular: the pose stays
    assert np.all(np.isfinite(hist))


@pytest.mark.parametrize("warm", [False, True])
def test_tracker_uploads_pinned_frames_inside_the_step(of, cuda, warm):
    """A pinned host frame is copied by the step graph itself, at the head of
    the pre-processing branch (beside the fusion of the previous frame, with
    the camera-side filters after it and the CNN branch waiting for both):
    the poses equal, bit for bit, those of the same tracker fed device frames
    and fed pageable host frames (copied before the step)."""
    import torch
    from openfusion_b200 import learned
    cfg = small(of, "c1")
    n = 7
    seq = of.make_sequence(cfg, frames=n)
    frames = [torch.from_numpy(seq.depth[k].astype(np.int16)) for k in range(n)]
    pinned = [f.pin_memory() for f in frames]
    device = [f.to(cuda) for f in frames]
    w = learned.load_weights() if warm else None
    p = of.depth_filter_params(["median5", "average"])
    hist = []
    for src in (device, pinned, frames):
        tr = of.Tracker(cfg, seq.poses[0], warm_start_weights=w, depth_filter=p)
        for f in src:
            tr.process(f)
        torch.cuda.synchronize()
        hist.append(tr.pose_history(n))
        tr.close()
    assert np.array_equal(hist[0], hist[1])
    assert np.array_equal(hist[0], hist[2])
