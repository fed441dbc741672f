"""Warm-started ICP (of_icp_track_warm): the judge, the early exit and the
tracker-level gain of the learned warm start, against the FP64 oracle.

No reference counterpart: the reference always starts ICP from the previous
pose and runs every iteration (Source/src/ICP.cpp:84-182). Two bars apply,
both at the pose tolerance of the parity tests (1e-5 rad, 0.01 mm):
  - parity: the GPU result equals the FP64 oracle running the same method
    (warm-started pass, judge, early exit; ora_icp_track_ex) on the same maps
    from the same starting poses;
  - equal error: plain and warm-started tracking with the early exit both land
    within the tolerance of the FP64 oracle's plain ICP with every iteration
    on the same maps.
A rejected warm start is replaced by exactly the plain result.
"""
import dataclasses

import numpy as np
import pytest

from conftest import pose_error
from test_gpu_parity import dev_pose, icp_inputs, small

pytestmark = pytest.mark.gpu


def stats_of(stats):
    import torch
    s = stats[:16].view(torch.int32).cpu().numpy()
    return {"status": int(s[0]), "inliers": int(s[1]), "iterations": int(s[2]), "warm": int(s[3])}


def perturbed(P, rot_rad, trans_mm):
    """P with its rotation turned by rot_rad about a fixed oblique axis and its
    translation moved by trans_mm along another."""
    a = np.array([0.48, -0.6, 0.64])
    a /= np.linalg.norm(a)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    R = np.eye(3) + np.sin(rot_rad) * K + (1 - np.cos(rot_rad)) * K @ K
    Q = np.array(P, np.float64).copy()
    Q[:3, :3] = R @ Q[:3, :3]
    Q[:3, 3] += trans_mm * np.array([0.6, 0.0, -0.8])
    return Q


def oracle_buffers(of, ora, cfg, frame, model):
    from test_gpu_parity import gpu_pyramid_to_oracle
    fbuf, _ = gpu_pyramid_to_oracle(of, ora, cfg, frame)
    mbuf, _ = gpu_pyramid_to_oracle(of, ora, cfg, model, with_depth=False)
    return fbuf, mbuf


def run_plain_and_warm(of, cfg, cuda, warm_of_truth):
    import torch
    seq, vol, lam, model, frame = icp_inputs(of, None, cfg, cuda)
    ws = of.icp_workspace(cfg, cuda)
    plain = dev_pose(seq.poses[3], cuda)
    st_plain = torch.zeros(32, dtype=torch.uint8, device=cuda)
    of.icp_track(cfg, frame, model, plain, ws, st_plain)
    warm = dev_pose(seq.poses[3], cuda)
    W = warm_of_truth(seq.poses[4])
    st_warm = torch.zeros(32, dtype=torch.uint8, device=cuda)
    of.icp_track_warm(cfg, frame, model, warm, dev_pose(W, cuda), ws, st_warm)
    torch.cuda.synchronize()
    return (seq, plain.cpu().numpy().reshape(4, 4), stats_of(st_plain),
            warm.cpu().numpy().reshape(4, 4), stats_of(st_warm), W, frame, model)


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_kept_warm_start_lands_on_the_plain_result(of, ora, cuda, name):
    """A warm start near the truth is kept; the result equals the FP64
    oracle's warm-started ICP from the same warm start, and plain ICP's pose,
    within 1e-5 rad / 0.01 mm."""
    cfg = small(of, name)
    seq, plain, sp, warm, sw, W, frame, model = run_plain_and_warm(
        of, cfg, cuda, lambda G: perturbed(G, np.radians(0.3), 5.0))
    assert sp["status"] == 0 and sp["warm"] == 0
    assert sw["status"] == 0 and sw["warm"] == 1, sw
    fbuf, mbuf = oracle_buffers(of, ora, cfg, frame, model)
    opose, r = ora.icp_track_ex(cfg, fbuf, mbuf, seq.poses[3], warm=W)
    assert r.status == 0 and r.warm == 1 and r.iterations == sw["iterations"], (r.warm, r.iterations)
    rot, trans = pose_error(warm, opose)
    assert rot < 1e-5 and trans < 1e-2, ("vs oracle", rot, trans)
    rot, trans = pose_error(warm, plain)
    assert rot < 1e-5 and trans < 1e-2, ("vs plain", rot, trans)
    rot_gt, trans_gt = pose_error(warm, seq.poses[4])
    assert rot_gt < np.radians(0.5) and trans_gt < 10.0


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_rejected_warm_start_is_replaced_by_plain_icp(of, ora, cuda, name):
    """A warm start 200 mm / 6 deg off is rejected (disagreement beyond the
    judge's 50 mm / 0.05 rad), as the oracle's judge rejects it, and the
    result is plain ICP's from the previous pose, bit for bit, and the
    oracle's within 1e-5 rad / 0.01 mm."""
    cfg = small(of, name)
    seq, plain, sp, warm, sw, W, frame, model = run_plain_and_warm(
        of, cfg, cuda, lambda G: perturbed(G, np.radians(6.0), 200.0))
    assert sw["status"] == 0 and sw["warm"] == 2, sw
    assert sw["iterations"] > sp["iterations"]  # both passes are counted
    assert np.array_equal(warm, plain)
    fbuf, mbuf = oracle_buffers(of, ora, cfg, frame, model)
    opose, r = ora.icp_track_ex(cfg, fbuf, mbuf, seq.poses[3], warm=W)
    assert r.warm == 2 and r.iterations == sw["iterations"], (r.warm, r.iterations)
    rot, trans = pose_error(warm, opose)
    assert rot < 1e-5 and trans < 1e-2, (rot, trans)


def test_early_exit_stays_within_pose_tolerance(of, ora, cuda):
    """The early exit of the C5 comparison (a level ends once the increment
    is below the configured rotation / translation) runs the same iterations
    as the FP64 oracle's early exit and lands within 1e-5 rad / 0.01 mm of
    it, and within 1e-5 rad / 0.01 mm of running every iteration, with fewer
    iterations."""
    import torch
    from openfusion_b200.train_warm_start import eval_config
    ev = eval_config(of)
    cfg = small(of, "c2")
    seq, vol, lam, model, frame = icp_inputs(of, None, cfg, cuda)
    ws = of.icp_workspace(cfg, cuda)
    out = {}
    for stop in (False, True):
        c = dataclasses.replace(cfg, stop_rot_rad=ev.stop_rot_rad if stop else 0.0,
                                stop_trans_mm=ev.stop_trans_mm if stop else 0.0)
        p = dev_pose(seq.poses[3], cuda)
        st = torch.zeros(32, dtype=torch.uint8, device=cuda)
        of.icp_track(c, frame, model, p, ws, st)
        torch.cuda.synchronize()
        out[stop] = (p.cpu().numpy().reshape(4, 4), stats_of(st), c)
    assert out[True][1]["status"] == 0
    assert out[True][1]["iterations"] < out[False][1]["iterations"], out
    fbuf, mbuf = oracle_buffers(of, ora, cfg, frame, model)
    opose, r = ora.icp_track_ex(out[True][2], fbuf, mbuf, seq.poses[3])
    if r.decisions_near == 0:
        assert r.iterations == out[True][1]["iterations"], (r.iterations, out[True][1])
    rot, trans = pose_error(out[True][0], opose)
    assert rot < 1e-5 and trans < 1e-2, ("vs oracle", rot, trans)
    rot, trans = pose_error(out[True][0], out[False][0])
    assert rot < 1e-5 and trans < 1e-2, ("vs every iteration", rot, trans)


def test_learned_warm_start_saves_iterations_at_equal_error(of, cuda):
    """The committed C5 weights through the tracker on a held-out large-motion
    sequence, each frame checked against the FP64 oracle on the tracker's own
    maps: both arms equal the oracle running their own method, both land
    within 1e-5 rad / 0.01 mm of the oracle's plain ICP with every iteration
    (equal pose error), and the warm start saves at least 15 % of the ICP
    iterations and is kept on most frames."""
    import warm_start_c5 as study
    res = study.run([900007], 17, cuda, timed=False)
    for arm in ("plain", "warm"):
        r = res[arm]
        assert r["status_nonzero_frames"] == 0, (arm, r)
        assert r["frames_with_decision_near_threshold"] <= 2, (arm, r)
        assert r["max_rot_rad_vs_own_oracle"] < 1e-5, (arm, r)
        assert r["max_trans_mm_vs_own_oracle"] < 1e-2, (arm, r)
        assert r["max_rot_rad_vs_full_oracle"] < 1e-5, (arm, r)
        assert r["max_trans_mm_vs_full_oracle"] < 1e-2, (arm, r)
    assert res["warm"]["judge_equal_own_oracle_frac"] == 1.0, res["warm"]
    assert res["warm"]["warm_start_kept_frac"] >= 0.8, res["warm"]
    assert res["warm"]["mean_icp_iterations"] <= 0.85 * res["plain"]["mean_icp_iterations"], res
