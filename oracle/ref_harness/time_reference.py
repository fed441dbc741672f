"""Frames/s of the reference's own kernels rebuilt for sm_100a, driven in
RunApp::display order (oracle/_ref/libref_kernels.so, ref_pipeline.cu), and of
this repository's tracker on the same frames and volume geometry.

TEST INFRASTRUCTURE ONLY (a reported comparison row, not the benchmark).
Runs on a GPU box:  python oracle/ref_harness/time_reference.py [frames]

Workload: 640x480 uint16 depth (fx = fy = 525, c = (319.5, 239.5)), the
reference's volume (Constants.h: 512^3 voxels over a 1024 mm cube, truncation
10 mm, max weight 120), a seeded scene inside the cube and a camera starting at
the reference's initial pose (768 mm from the centre, MainApp.cpp:613-618)
moving a few mm and a fraction of a degree per frame.
"""
import ctypes as C
import dataclasses
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests" / "golden"))

W, H, F, CX, CY, DMIN, DMAX = 640, 480, 525.0, 319.5, 239.5, 300.0, 4000.0


def trajectory(frames):
    out = []
    for k in range(frames):
        a = 0.002 * k
        R = np.array([[np.cos(a), 0, np.sin(a)], [0, 1, 0], [-np.sin(a), 0, np.cos(a)]])
        T = np.eye(4)
        T[:3, :3] = R
        T[:3, 3] = [3.0 * k * 0.5, 1.0 * np.sin(0.1 * k), 768.0 - 1.0 * k]
        out.append(T)
    return out


def main(frames: int):
    import make_ref_fixtures as mf
    import openfusion_b200 as of
    import openfusion_b200._native as N
    lib = C.CDLL(str(ROOT / "oracle" / "_ref" / "libref_kernels.so"))
    P = C.c_void_p
    lib.ref_pipeline_create.argtypes = [P, P]
    lib.ref_pipeline_frame.argtypes = [P, P, P]
    cam = mf.RefCam(W, H, F, F, CX, CY, 1.0 / F, 1.0 / F, -CX / F, -CY / F, DMIN, DMAX)
    sc = mf.scene()
    poses = trajectory(frames)
    depth = []
    for k, T in enumerate(poses):
        d = np.zeros((H, W), np.uint16)
        Tp = np.ascontiguousarray(T, np.float64)
        N.synth().of_synth_render(C.byref(sc), W, H, F, F, CX, CY, Tp.ctypes.data, 91, k, 1.0,
                                  0.0, d.ctypes.data, None)
        depth.append(d)
    # ---- the reference, display() order, host-synchronous as written
    pose0 = np.asarray(poses[0], np.float32).reshape(16).copy()
    assert lib.ref_pipeline_create(C.byref(cam), pose0.ctypes.data) == 0
    ms = []
    ref_poses = []
    for k in range(frames):
        po = np.zeros(16, np.float32)
        t = C.c_double()
        rc = lib.ref_pipeline_frame(depth[k].ctypes.data, po.ctypes.data, C.byref(t))
        assert rc == 0, rc
        ms.append(t.value)
        ref_poses.append(po.reshape(4, 4).astype(np.float64))
    warm = 3
    ref_ms = float(np.median(ms[warm:]))
    # ---- this repository on the same frames and volume geometry: fixed
    # 10/5/4 iterations, and with the convergence exit of the C5 comparison
    import torch
    base = dataclasses.replace(of.CONFIGS["c2"], resolution=512, size_mm=1024.0, trunc_mm=10.0,
                               max_weight=120, min_depth_mm=DMIN, max_depth_mm=DMAX)
    dev = torch.device("cuda:0")
    dd = torch.from_numpy(np.stack(depth).astype(np.int16)).to(dev)

    def run(cfg):
        tr = of.Tracker(cfg, poses[0], tune=2)  # raycast block shape tuned at frame 2
        tr.process(dd[0])
        for k in range(1, 1 + warm):
            tr.process(dd[k])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(1 + warm, frames):
            tr.process(dd[k])
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / (frames - 1 - warm)
        hist = tr.pose_history(frames)
        tr.close()
        return ms, list(hist)

    def err(Ps):
        rot = max(float(np.degrees(np.arccos(np.clip((np.trace(P[:3, :3].T @ G[:3, :3]) - 1) / 2, -1, 1))))
                  for P, G in zip(Ps, poses))
        tra = max(float(np.linalg.norm(P[:3, 3] - G[:3, 3])) for P, G in zip(Ps, poses))
        return rot, tra
    def stages(cfg):
        # the tracker's stages launched one by one in its order (integrate k-1,
        # raycast k-1, pre-process k, ICP k), each timed with CUDA events; mean
        # over frames 4..60 (before free space saturates) and after frame 130
        vol, lam = of.new_volume(cfg, dev), of.lambda_table(cfg, dev)
        scr = of.integrate_scratch(cfg, dev)
        frame, model, ws = of.new_pyramid(cfg, dev), of.new_pyramid(cfg, dev), of.icp_workspace(cfg, dev)
        pose = torch.tensor(np.asarray(poses[0]).reshape(16), dtype=torch.float64, device=dev)
        names = ["integrate", "raycast", "preprocess", "icp"]
        early, late = [], []
        s = torch.cuda.current_stream()
        for k in range(1, frames):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
            ev[0].record(s)
            of.integrate(cfg, vol, dd[k - 1], pose, lam, scr)
            ev[1].record(s)
            of.raycast(cfg, vol, pose, model)
            ev[2].record(s)
            of.preprocess(cfg, dd[k], frame)
            ev[3].record(s)
            of.icp_track(cfg, frame, model, pose, ws)
            ev[4].record(s)
            s.synchronize()
            t = [ev[i].elapsed_time(ev[i + 1]) * 1e3 for i in range(4)]
            if 3 < k <= 60:
                early.append(t)
            elif k > 130:
                late.append(t)
        out = {}
        for key, rows in (("frames_4_60", early), ("after_frame_130", late)):
            if rows:
                out[key] = dict(zip(names, np.round(np.mean(rows, axis=0), 1).tolist()))
        return out

    ours_ms, hist = run(base)
    exit_ms, hist_exit = run(dataclasses.replace(base, stop_rot_rad=5e-6, stop_trans_mm=0.005))
    stage_us = stages(base)
    print(json.dumps({
        "workload": "640x480, 512^3 over 1024 mm (reference constants), %d frames" % frames,
        "reference_kernels_sm100a": {"ms_per_frame": ref_ms, "frames_per_s": 1e3 / ref_ms,
                                     "max_pose_err_deg_mm": err(ref_poses),
                                     "icp": "1 level x 15 iterations, host solve (ICP.cpp)"},
        "this_repo": {"ms_per_frame": ours_ms, "frames_per_s": 1e3 / ours_ms,
                      "max_pose_err_deg_mm": err(hist),
                      "icp": "3 levels 10/5/4, device solve, CUDA graph"},
        "speedup": ref_ms / ours_ms,
        "this_repo_convergence_exit": {"ms_per_frame": exit_ms, "frames_per_s": 1e3 / exit_ms,
                                       "max_pose_err_deg_mm": err(hist_exit),
                                       "icp": "3 levels, at most 10/5/4, a level ends when an "
                                              "increment is below 5e-6 rad and 0.005 mm"},
        "speedup_convergence_exit": ref_ms / exit_ms,
        "stages_us": stage_us}))


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 40)
