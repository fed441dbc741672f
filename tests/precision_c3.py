"""Precision study of the large-volume workload: the full-size scene at
640x480 fused into a 1024^3 volume over 4 m with FP16 tsdf + uint16 weight
(4 GiB), tracked frame by frame through the per-stage calls in the tracker's
order (integrate k-1, raycast k-1, preprocess k, ICP k; bit-identical to the
tracker). At checkpoint frames every stage is compared with the FP64 oracle
on the GPU's own input state:

  TSDF     integration of frame k-1 into the GPU's volume: weights equal,
           tsdf/trunc within one FP16 ulp (2^-11) on every voxel not flagged
           at a rounding boundary
  vertex   raycast of the GPU's volume at pose k-1: within 0.1 mm (1e-4 m),
           99.9th percentile, on rays that hit in both and are not flagged
  pose     3-level ICP of frame k from pose k-1 on the GPU's frame and model
           pyramids: within 1e-5 rad and 0.01 mm
  sums     the 27 J^T J / J^T r sums (and residual, inliers) of one system per
           level, relative to their Cauchy-Schwarz scale (FP32 rows with
           pairwise/Kahan FP32 sums against FP64 sums of the same rows)

and, over every frame, the tracked pose against the ground truth. Test
infrastructure: it runs the oracle as the checker.

    python tests/precision_c3.py [--frames 300] [--checkpoints 10]   (on a GPU)
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def linear_words(cfg, host_words: np.ndarray) -> np.ndarray:
    """Brick-major volume buffer -> uint32 voxel words in x, y, z order (one copy)."""
    n = cfg.resolution
    nb = n // 8
    w = host_words.view(np.uint32)[: n ** 3].reshape(nb, nb, nb, 8, 8, 8)
    return np.ascontiguousarray(w.transpose(0, 3, 1, 4, 2, 5)).reshape(-1)


def brick_flags(cfg, host_words: np.ndarray) -> np.ndarray:
    nb = cfg.resolution // 8
    return host_words.view(np.uint8)[4 * cfg.resolution ** 3:][: nb ** 3].copy()


def pose_error(P, G):
    R = np.asarray(P)[:3, :3].T @ np.asarray(G)[:3, :3]
    c = np.clip((np.trace(R) - 1.0) / 2.0, -1.0, 1.0)
    return float(np.arccos(c)), float(np.linalg.norm(np.asarray(P)[:3, 3] - np.asarray(G)[:3, 3]))


def check_integrate(cfg, ora, before: np.ndarray, after: np.ndarray, depth, pose) -> dict:
    words = before.copy()
    n_ora, amb = ora.integrate(cfg, words, depth, pose, ambig=True)
    ok = amb == 0
    wg, wo = after >> 16, words >> 16
    weights_equal = bool(np.array_equal(wg[ok], wo[ok]))
    upd = ok & (wo > 0)
    g = (after[upd] & 0xFFFF).astype(np.uint16).view(np.float16).astype(np.float64)
    o = (words[upd] & 0xFFFF).astype(np.uint16).view(np.float16).astype(np.float64)
    d = np.abs(g - o)
    return {"voxels_updated_oracle": int(n_ora), "flagged_frac": float((~ok).mean()),
            "weights_equal": weights_equal,
            "max_tsdf_err_fp16_ulp": float(d.max() / 2.0 ** -11) if d.size else 0.0,
            "max_tsdf_err_mm": float(d.max() * cfg.trunc_mm) if d.size else 0.0}


def check_raycast(cfg, ora, words, flags, pose, gv, gn) -> dict:
    import raycast_check
    opts, amb = ora.raycast(cfg, words, pose, ambig=True, flags=flags)
    ok = amb == 0
    hit_g, hit_o = gv[..., 3] > 0, opts[..., 3] > 0
    both = hit_g & hit_o & ok
    r = raycast_check.compare(ora, cfg, words, flags, pose, gv, opts, amb)
    nb = both & (gn[..., 3] > 0) & (opts[..., 7] > 0)
    nerr = np.linalg.norm(gn[..., :3][nb] - opts[..., 4:7][nb], axis=-1)
    return {"hit_frac": float(hit_o.mean()), "hit_mismatch_frac": float((hit_g != hit_o)[ok].mean()),
            "flagged_frac": float((~ok).mean()),
            "vertex_err_mm_max": r["max_err_mm"],
            "vertex_err_mm_q999": r["q999_err_mm"],
            "vertex_err_mm_median": r["median_err_mm"],
            "rounding_sensitive_rays": r["rounding_sensitive"],
            "unexplained_rays": r["unexplained"],
            "normal_err_median": float(np.median(nerr))}


def check_sums(cfg, of, ora, frame, model, fpts, mpts, pose, ws, dev) -> dict:
    import torch
    worst = 0.0
    for level in range(cfg.levels):
        P = torch.tensor(np.asarray(pose).reshape(16), dtype=torch.float64, device=dev)
        g = of.icp_system(cfg, level, frame, model, P, ws).cpu().numpy()
        o, amb = ora.icp_system(cfg, level, fpts[level], mpts[level], pose)
        diag = np.array([o[k] for k in (0, 6, 11, 15, 18, 20)])
        scale = np.zeros(29)
        k = 0
        for i in range(6):
            for j in range(i, 6):
                scale[k] = np.sqrt(diag[i] * diag[j])
                k += 1
        scale[21:27] = np.sqrt(diag * o[27])
        scale[27] = o[27]
        scale[28] = max(o[28], 1.0)
        # beyond the whole contribution of pixels at a rounding boundary
        rel = np.maximum(np.abs(g - o) - amb, 0.0) / (scale + 1e-30)
        worst = max(worst, float(rel.max()))
    return {"sum_err_rel_scale_max": worst}


def run_study(frames: int, checkpoints: list[int], log=print) -> dict:
    import torch
    import openfusion_b200 as of
    from oracle import Oracle
    from test_gpu_parity import gpu_pyramid_to_oracle
    ora = Oracle("f64")
    dev = torch.device("cuda:0")
    cfg = of.CONFIGS["c3"]
    seq = of.make_sequence(cfg, frames=frames)
    vol, lam = of.new_volume(cfg, dev), of.lambda_table(cfg, dev)
    scratch = of.integrate_scratch(cfg, dev)
    frame, model = of.new_pyramid(cfg, dev), of.new_pyramid(cfg, dev)
    ws = of.icp_workspace(cfg, dev)
    pose = torch.tensor(seq.poses[0].reshape(16), dtype=torch.float64, device=dev)
    depth = [torch.from_numpy(seq.depth[k].astype(np.int16)).to(dev) for k in range(frames)]
    hist = [seq.poses[0]]
    out = {"workload": "c3: 640x480, 1024^3 FP16 tsdf + uint16 weight over 4 m (4 GiB), "
                       "20 boxes and spheres, axial noise + 2% dropout",
           "frames": frames, "checkpoints": []}
    t0 = time.time()
    for k in range(1, frames):
        check = k in checkpoints
        prev_pose = pose.cpu().numpy().reshape(4, 4).copy()
        if check:
            torch.cuda.synchronize()
            before = linear_words(cfg, vol.cpu().numpy())
        of.integrate(cfg, vol, depth[k - 1], pose, lam, scratch)
        of.raycast(cfg, vol, pose, model)
        of.preprocess(cfg, depth[k], frame)
        cp = {}
        if check:
            torch.cuda.synchronize()
            host = vol.cpu().numpy()
            after = linear_words(cfg, host)
            cp["frame"] = k
            cp["integrate"] = check_integrate(cfg, ora, before, after, seq.depth[k - 1], prev_pose)
            del before
            gv, gn = (t.cpu().numpy().astype(np.float64) for t in of.unpack_points(cfg, model, 0))
            cp["raycast"] = check_raycast(cfg, ora, after, brick_flags(cfg, host), prev_pose, gv, gn)
            del after, host
            fbuf, fpts = gpu_pyramid_to_oracle(of, ora, cfg, frame)
            mbuf, mpts = gpu_pyramid_to_oracle(of, ora, cfg, model, with_depth=False)
            cp["icp_sums"] = check_sums(cfg, of, ora, frame, model, fpts, mpts, prev_pose, ws, dev)
        of.icp_track(cfg, frame, model, pose, ws)
        P = pose.cpu().numpy().reshape(4, 4).copy()
        hist.append(P)
        if check:
            st, opose, its = ora.icp_track(cfg, fbuf, mbuf, prev_pose)
            rot, trans = pose_error(P, opose)
            cp["icp"] = {"oracle_status": int(st), "rot_err_rad": rot, "trans_err_mm": trans}
            out["checkpoints"].append(cp)
            log(json.dumps(cp))
    gt = [pose_error(hist[k], seq.poses[k]) for k in range(frames)]
    cps = out["checkpoints"]
    out["summary"] = {
        "max_tsdf_err_fp16_ulp": max(c["integrate"]["max_tsdf_err_fp16_ulp"] for c in cps),
        "weights_equal": all(c["integrate"]["weights_equal"] for c in cps),
        "max_vertex_err_mm": max(c["raycast"]["vertex_err_mm_max"] for c in cps),
        "max_rounding_sensitive_rays": max(c["raycast"]["rounding_sensitive_rays"] for c in cps),
        "unexplained_rays": sum(len(c["raycast"]["unexplained_rays"]) for c in cps),
        "max_vertex_err_mm_q999": max(c["raycast"]["vertex_err_mm_q999"] for c in cps),
        "max_pose_err_rad": max(c["icp"]["rot_err_rad"] for c in cps),
        "max_pose_err_mm": max(c["icp"]["trans_err_mm"] for c in cps),
        "max_sum_err_rel_scale": max(c["icp_sums"]["sum_err_rel_scale_max"] for c in cps),
        "gt_max_rot_deg": float(np.degrees(max(g[0] for g in gt))),
        "gt_max_trans_mm": float(max(g[1] for g in gt)),
        "gt_mean_trans_mm": float(np.mean([g[1] for g in gt])),
        "seconds": time.time() - t0,
    }
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=300)
    ap.add_argument("--checkpoints", type=int, default=10)
    a = ap.parse_args(argv)
    cps = sorted({max(1, int(round(x))) for x in np.linspace(1, a.frames - 1, a.checkpoints)})
    res = run_study(a.frames, cps, log=lambda m: print(m, file=sys.stderr, flush=True))
    print(json.dumps(res["summary"]), flush=True)
    print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
