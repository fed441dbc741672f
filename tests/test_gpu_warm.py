"""Warm-started ICP (of_icp_track_warm): the judge, the early exit and the
tracker-level gain of the learned warm start.

No reference counterpart: the reference always starts ICP from the previous
pose and runs every iteration (Source/src/ICP.cpp:84-182). The bars are
therefore relative to plain ICP on the same inputs: a kept warm start lands
where plain ICP lands, a rejected one is replaced by exactly the plain
result, and the early exit stays within the pose tolerance of running every
iteration.
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


def run_plain_and_warm(of, cfg, cuda, warm_of_truth):
    import torch
    seq, vol, lam, model, frame = icp_inputs(of, None, cfg, cuda)
    ws = of.icp_workspace(cfg, cuda)
    plain = dev_pose(seq.poses[3], cuda)
    st_plain = torch.zeros(32, dtype=torch.uint8, device=cuda)
    of.icp_track(cfg, frame, model, plain, ws, st_plain)
    warm = dev_pose(seq.poses[3], cuda)
    st_warm = torch.zeros(32, dtype=torch.uint8, device=cuda)
    of.icp_track_warm(cfg, frame, model, warm, dev_pose(warm_of_truth(seq.poses[4]), cuda), ws,
                      st_warm)
    torch.cuda.synchronize()
    return (seq, plain.cpu().numpy().reshape(4, 4), stats_of(st_plain),
            warm.cpu().numpy().reshape(4, 4), stats_of(st_warm))


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_kept_warm_start_lands_on_the_plain_result(of, cuda, name):
    """A warm start near the truth is kept and converges to plain ICP's pose."""
    cfg = small(of, name)
    seq, plain, sp, warm, sw = run_plain_and_warm(
        of, cfg, cuda, lambda G: perturbed(G, np.radians(0.3), 5.0))
    assert sp["status"] == 0 and sp["warm"] == 0
    assert sw["status"] == 0 and sw["warm"] == 1, sw
    rot, trans = pose_error(warm, plain)
    assert rot < 1e-4 and trans < 0.1, (rot, trans)
    rot_gt, trans_gt = pose_error(warm, seq.poses[4])
    assert rot_gt < np.radians(0.5) and trans_gt < 10.0


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_rejected_warm_start_is_replaced_by_plain_icp(of, cuda, name):
    """A warm start 200 mm / 6 deg off is rejected (disagreement beyond the
    judge's 50 mm / 0.05 rad) and the result is plain ICP's, bit for bit."""
    cfg = small(of, name)
    seq, plain, sp, warm, sw = run_plain_and_warm(
        of, cfg, cuda, lambda G: perturbed(G, np.radians(6.0), 200.0))
    assert sw["status"] == 0 and sw["warm"] == 2, sw
    assert sw["iterations"] > sp["iterations"]  # both passes are counted
    assert np.array_equal(warm, plain)


def test_early_exit_stays_within_pose_tolerance(of, cuda):
    """Stopping a level once the increment is below 2e-5 rad / 0.02 mm saves
    iterations and stays within 1e-5 rad / 0.1 mm of running all of them."""
    import torch
    cfg = small(of, "c2")
    seq, vol, lam, model, frame = icp_inputs(of, None, cfg, cuda)
    ws = of.icp_workspace(cfg, cuda)
    out = {}
    for stop in (False, True):
        c = dataclasses.replace(cfg, stop_rot_rad=2e-5 if stop else 0.0,
                                stop_trans_mm=0.02 if stop else 0.0)
        p = dev_pose(seq.poses[3], cuda)
        st = torch.zeros(32, dtype=torch.uint8, device=cuda)
        of.icp_track(c, frame, model, p, ws, st)
        torch.cuda.synchronize()
        out[stop] = (p.cpu().numpy().reshape(4, 4), stats_of(st))
    assert out[True][1]["status"] == 0
    assert out[True][1]["iterations"] < out[False][1]["iterations"], out
    rot, trans = pose_error(out[True][0], out[False][0])
    assert rot < 1e-5 and trans < 0.1, (rot, trans)


def test_learned_warm_start_saves_iterations_at_equal_error(of, cuda):
    """The committed C5 weights through the tracker on a held-out large-motion
    sequence: at least 15% fewer ICP iterations than plain ICP, the warm start
    kept on most frames, and the same pose error against the ground truth
    (within 0.01 deg / 0.05 mm of plain's worst frame)."""
    from openfusion_b200 import learned
    from openfusion_b200.train_warm_start import eval_config, pose_errors, run_tracker
    cfg = dataclasses.replace(eval_config(of), seed=900007)
    scene = of.make_scene(cfg.scene_kind, cfg.seed, cfg.size_mm)
    poses = of.make_trajectory(cfg.motion, cfg.seed + 1, cfg.size_mm, 24)
    depth = learned.render_device(cfg, scene, poses, device=cuda)
    res = {}
    for arm, w in (("plain", None), ("warm", learned.load_weights())):
        hist, its, warm, _ = run_tracker(of, cfg, depth, poses, w, timed=False)
        r, t = pose_errors(hist[1:], poses[1:])
        res[arm] = (its, warm, r, t)
    its_p, _, r_p, t_p = res["plain"]
    its_w, kept, r_w, t_w = res["warm"]
    assert its_w.mean() <= 0.85 * its_p.mean(), (its_w.mean(), its_p.mean())
    assert np.mean(kept == 1) >= 0.8, kept
    assert r_w.max() <= r_p.max() + 0.01, (r_w.max(), r_p.max())
    assert t_w.max() <= t_p.max() + 0.05, (t_w.max(), t_p.max())
