"""The learned warm start against plain ICP, frame by frame against the FP64
oracle (large-motion workload: 640x480, 512^3 over 3 m, inter-frame motion
U[0, 10] cm / U[0, 5] deg).

    python tests/warm_start_c5.py [--seeds 910000 910001 910002] [--frames 121]
                                  [--out results.json] [--weights file.npy]

Both arms run through the tracker (one CUDA graph per frame) with the same
early exit. After every frame the tracker's own ICP inputs are read back --
the pre-processed frame pyramid, the model pyramid raycast at the previous
pose, the previous pose and, for the warm arm, the CNN's warm start -- and
the FP64 oracle tracks the same frame twice:
  own   the arm's own method (early exit; warm-started pass on the finest
        level and the judge for the warm arm): the parity check of the arm;
  full  plain ICP from the previous pose with every iteration (10/5/4) and no
        early exit: the frame's FP64 pose, the common bar of both arms.
Decisions (exit, judge) whose quantity lies within 1 % of its threshold can
go either way between FP32 and FP64; those frames are counted and left out of
the `own` maximum. Frames/s are device-timed in a separate pass without the
read-back. Reference for the plain arm's start: Source/src/ICP.cpp:84-182
(ICP from the previous pose).

This is test infrastructure (it runs the oracle); tests/test_gpu_warm.py runs
a short sequence of it.
"""
from __future__ import annotations

import argparse
import ctypes as C
import dataclasses
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pose_error(P, G):
    R = np.asarray(P)[:3, :3].T @ np.asarray(G)[:3, :3]
    c = np.clip((np.trace(R) - 1.0) / 2.0, -1.0, 1.0)
    return float(np.arccos(c)), float(np.linalg.norm(np.asarray(P)[:3, 3] - np.asarray(G)[:3, 3]))


def to_oracle(of, ora, cfg, pyr, with_depth=True):
    pts, deps = [], []
    for lv in range(cfg.levels):
        v, n = of.unpack_points(cfg, pyr, lv)
        pts.append(np.concatenate([v.cpu().numpy(), n.cpu().numpy()], axis=-1))
        deps.append(of.unpack_depth(cfg, pyr, lv).cpu().numpy() if with_depth else None)
    return ora.pack_pyramid(cfg, pts, deps if with_depth else None)


def track_arm(of, ora, cfg, depth, poses, weights, dev):
    """One arm through the tracker with the per-frame oracle checks; returns
    per-frame records."""
    import torch
    from openfusion_b200 import _native as N
    from openfusion_b200 import learned
    from openfusion_b200.api import _ptr, _stream
    full_cfg = dataclasses.replace(cfg, stop_rot_rad=0.0, stop_trans_mm=0.0)
    net = learned.WarmStartNet(dev, weights=weights) if weights is not None else None
    warm_dev = torch.empty(16, dtype=torch.float64, device=dev)
    prev_dev = torch.empty(16, dtype=torch.float64, device=dev)
    tr = of.Tracker(cfg, poses[0], warm_start_weights=weights)
    tr.process(depth[0])
    prev, _ = tr.pose()
    recs = []
    for k in range(1, depth.shape[0]):
        W = None
        if net is not None:
            # the prediction the tracker's CNN branch makes for this pair (the
            # same kernel on the same inputs)
            prev_dev.copy_(torch.from_numpy(prev.reshape(16)))
            N.check("of_cnn_predict", N.lib().of_cnn_predict(
                _ptr(net.params), _ptr(net.master), _ptr(depth[k - 1]), _ptr(depth[k]),
                cfg.width, cfg.height, _ptr(prev_dev), None, _ptr(warm_dev), _stream()))
        tr.process(depth[k])
        b = tr.buffers()
        frame = of.copy_pyramid(cfg, b.frame, dev)
        model = of.copy_pyramid(cfg, b.model, dev)
        P, st = tr.pose()
        if net is not None:
            W = warm_dev.cpu().numpy().reshape(4, 4)
        fbuf = to_oracle(of, ora, cfg, frame)
        mbuf = to_oracle(of, ora, cfg, model, with_depth=False)
        own, r_own = ora.icp_track_ex(cfg, fbuf, mbuf, prev, warm=W)
        full, r_full = ora.icp_track_ex(full_cfg, fbuf, mbuf, prev)
        recs.append({
            "k": k, "pose": P, "status": int(st.status), "iterations": int(st.iterations),
            "warm": int(st.warm), "own": own, "own_iterations": int(r_own.iterations),
            "own_warm": int(r_own.warm), "own_status": int(r_own.status),
            "near": int(r_own.decisions_near), "full": full, "full_status": int(r_full.status),
            "truth": poses[k]})
        prev = P
    tr.close()
    return recs


def timed_arm(of, cfg, depth, poses, weights):
    from openfusion_b200.train_warm_start import run_tracker
    _, _, _, ms = run_tracker(of, cfg, depth, poses, weights, timed=True)
    return ms


def summarise(recs):
    own = [pose_error(r["pose"], r["own"]) for r in recs if r["near"] == 0]
    full = [pose_error(r["pose"], r["full"]) for r in recs]
    truth = [pose_error(r["pose"], r["truth"]) for r in recs]
    ofull = [pose_error(r["full"], r["truth"]) for r in recs]
    out = {
        "frames": len(recs),
        "max_rot_rad_vs_own_oracle": max((a for a, _ in own), default=0.0),
        "max_trans_mm_vs_own_oracle": max((b for _, b in own), default=0.0),
        "frames_with_decision_near_threshold": sum(r["near"] > 0 for r in recs),
        "iterations_equal_own_oracle_frac": float(np.mean(
            [r["iterations"] == r["own_iterations"] for r in recs if r["near"] == 0] or [1.0])),
        "max_rot_rad_vs_full_oracle": max(a for a, _ in full),
        "max_trans_mm_vs_full_oracle": max(b for _, b in full),
        "mean_icp_iterations": float(np.mean([r["iterations"] for r in recs])),
        "max_rot_deg_vs_truth": float(np.degrees(max(a for a, _ in truth))),
        "max_trans_mm_vs_truth": max(b for _, b in truth),
        "oracle_full_max_rot_deg_vs_truth": float(np.degrees(max(a for a, _ in ofull))),
        "oracle_full_max_trans_mm_vs_truth": max(b for _, b in ofull),
        "status_nonzero_frames": sum(r["status"] != 0 for r in recs),
    }
    if any(r["warm"] for r in recs):
        out["warm_start_kept_frac"] = float(np.mean([r["warm"] == 1 for r in recs]))
        out["judge_equal_own_oracle_frac"] = float(np.mean(
            [r["warm"] == r["own_warm"] for r in recs]))
    return out


def run(seeds, frames, dev, timed=True, log=None, weights_path=None):
    import openfusion_b200 as of
    from openfusion_b200 import learned
    from openfusion_b200.train_warm_start import eval_config
    from oracle import Oracle
    ora = Oracle("f64")
    weights = learned.load_weights(weights_path)
    res = {"workload": "c5: 640x480, 512^3 over 3 m, motion U[0,10] cm / U[0,5] deg per frame",
           "seeds": list(seeds), "frames_per_seed": frames - 1}
    cfg0 = eval_config(of)
    res["early_exit"] = {"rot_rad": cfg0.stop_rot_rad, "trans_mm": cfg0.stop_trans_mm,
                         "warm_levels": cfg0.warm_levels}
    per = {"plain": [], "warm": []}
    ms = {"plain": [], "warm": []}
    for seed in seeds:
        cfg = dataclasses.replace(cfg0, seed=seed)
        scene = of.make_scene(cfg.scene_kind, cfg.seed, cfg.size_mm)
        poses = of.make_trajectory(cfg.motion, cfg.seed + 1, cfg.size_mm, frames)
        depth = learned.render_device(cfg, scene, poses, device=dev)
        for arm, w in (("plain", None), ("warm", weights)):
            t0 = time.time()
            recs = track_arm(of, ora, cfg, depth, poses, w, dev)
            per[arm] += recs
            if timed:
                ms[arm].append(timed_arm(of, cfg, depth, poses, w))
            if log:
                log(f"seed {seed} {arm}: {summarise(recs)} ({time.time() - t0:.1f} s)")
    for arm in per:
        res[arm] = summarise(per[arm])
        if timed:
            res[arm]["frames_per_s_per_seed"] = [1e3 / m for m in ms[arm]]
            res[arm]["frames_per_s"] = float(np.mean([1e3 / m for m in ms[arm]]))
    if timed:
        ratios = [p / w for p, w in zip(ms["plain"], ms["warm"])]
        res["warm_over_plain_frames_per_s_per_seed"] = ratios
        res["warm_over_plain_frames_per_s"] = {"mean": float(np.mean(ratios)),
                                               "min": float(np.min(ratios)),
                                               "max": float(np.max(ratios))}
    # the two arms' worst frame against the common FP64 bar
    res["equal_error"] = {
        "bar": "per-frame pose within 1e-5 rad and 0.01 mm of the FP64 oracle's plain ICP "
               "(10/5/4, no early exit) on the same maps",
        "plain_within": bool(res["plain"]["max_rot_rad_vs_full_oracle"] <= 1e-5 and
                             res["plain"]["max_trans_mm_vs_full_oracle"] <= 1e-2),
        "warm_within": bool(res["warm"]["max_rot_rad_vs_full_oracle"] <= 1e-5 and
                            res["warm"]["max_trans_mm_vs_full_oracle"] <= 1e-2)}
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, nargs="+", default=[910000, 910001, 910002])
    ap.add_argument("--frames", type=int, default=121)
    ap.add_argument("--out", type=Path, default=None)
    ap.add_argument("--weights", type=Path, default=None,
                    help="warm-start CNN weights (default: the committed ones)")
    a = ap.parse_args()
    import torch
    dev = torch.device("cuda:0")
    res = run(a.seeds, a.frames, dev, log=lambda m: print(m, file=sys.stderr, flush=True),
              weights_path=a.weights)
    line = json.dumps(res)
    if a.out:
        a.out.parent.mkdir(parents=True, exist_ok=True)
        a.out.write_text(line + "\n")
    print(line, flush=True)


if __name__ == "__main__":
    main()
