"""Benchmark of the KinectFusion per-frame path (one step = one depth frame).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config c2]

Workload (default): 640x480 uint16 depth, 512^3 int16+uint16 TSDF over a 3 m
cube, 3-level ICP (10/5/4), bilateral filter sigma_s 4.5 px / sigma_r 30 mm,
seeded synthetic room of 20 boxes and spheres with axial noise and 2 %
dropout. Every frame is tracked against the model of the previous one, fused
and raycast. `value` is frames/s with the depth frames resident in HBM; `e2e`
is the same loop through the C-ABI with pinned host depth copied in and the
pose copied out every frame. The volume (512 MiB) is larger than L2.

Multi-GPU: the path does not shard a single sequence; N GPUs run N independent
sequences (different seeds), one process per GPU, no collective on the frame
path (weak scaling); timing is the max over ranks.

`warm_start` compares the learned warm start with plain ICP on the
large-motion workload (same frames, same early exit, device-timed frames/s,
ICP iterations and per-frame pose error against the ground truth).

`batched_streams` runs 64 independent streams of mixed resolution and volume
(the batched-streams workload) through one Batch (one launch per stage, one
graph per step, knobs tuned online) and, beside it, through one single-stream
tracker per stream; with N GPUs the streams are sharded longest-first.

`ref_kernels_b200` (a baseline leg, N = 1): the reference's own CUDA kernels
rebuilt for sm_100a with this workload's volume geometry, driven in the
reference's frame order on the same frames as the timed region.

`roofline` is the integration stage's, `roofline_raycast` the raycast's.

`--impl reference` runs the CPU implementation of the same equations (the
FP32 OpenMP build of the oracle restatement) on the host cores.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "frames/s 640x480 @512³ vol, plain vs learned-warm-start ICP at equal pose error"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--frames", type=int, default=300, help="rendered frames (ping-pong)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-kernels", action="store_true",
                    help="skip the reference's kernels rebuilt for sm_100a (baseline leg)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--warm-frames", type=int, default=121,
                    help="frames of the warm-start comparison (0 = skip it)")
    ap.add_argument("--c4-streams", type=int, default=64,
                    help="streams of the batched-streams measurement (0 = skip it)")
    ap.add_argument("--c4-frames", type=int, default=32, help="rendered frames per stream")
    ap.add_argument("--c4-steps", type=int, default=40, help="timed steps of the batch")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers

def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms during the
    timed region (one background nvidia-smi process)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._p = None

    def __enter__(self):
        try:
            self._p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                        "--format=csv,noheader,nounits", "-lms", "100"],
                                       stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.3)  # first sample before the timed work starts
        except Exception:
            self._p = None
        return self

    def __exit__(self, *a):
        if self._p is None:
            return
        time.sleep(0.15)
        self._p.terminate()
        try:
            out, _ = self._p.communicate(timeout=10)
        except Exception:
            self._p.kill()
            out = ""
        self.rows = [[x.strip() for x in line.split(",")] for line in out.splitlines() if line.strip()]

    def summary(self):
        rows = [r for r in self.rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [v for v in (num(r[1]) for r in rows) if v is not None]
        mx = [v for v in (num(r[2]) for r in rows) if v is not None]
        pw = [v for v in (num(r[3]) for r in rows) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None, "reasons": reasons,
                "samples": len(rows)}


def profile_figure(name: str, key: str = "dram_bytes_per_launch"):
    """A figure from an ncu summary under profiles/ (DRAM bytes per launch)."""
    f = ROOT / "profiles" / name
    try:
        return json.loads(f.read_text()).get(key)
    except (OSError, ValueError):
        return None


def frame_index(i: int, n: int) -> int:
    """Ping-pong through n rendered frames: consecutive steps stay adjacent poses."""
    period = 2 * (n - 1)
    j = i % period
    return j if j < n else period - j


def dist_setup(init: bool = True):
    """World size and ranks from torchrun's environment; the NCCL process
    group only when the ranks exchange anything (`init`)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and init:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def workload_config(cfg, n_frames: int, world: int) -> dict:
    """The `config` of both arms' JSON lines: the same workload, worded once."""
    store = "int16" if cfg.storage == "i16" else "fp16"
    return {"workload": cfg.name, "width": cfg.width, "height": cfg.height,
            "volume": f"{cfg.resolution}^3 {store}+uint16 over {cfg.size_mm / 1000:g} m, "
                      f"truncation {cfg.trunc_mm:g} mm, max weight {cfg.max_weight}",
            "icp": f"{cfg.levels} levels, {'/'.join(str(i) for i in cfg.iters)} iterations, "
                   "plain (no warm start)",
            "frames": f"{n_frames} rendered frames (seed {cfg.seed}), traversed forward and back",
            "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (512 MiB volume)"}


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def pose_errors(hist, gt):
    rots, trans = [], []
    for P, G in zip(hist, gt):
        R = P[:3, :3].T @ G[:3, :3]
        rots.append(float(np.arccos(np.clip((np.trace(R) - 1) / 2, -1, 1))))
        trans.append(float(np.linalg.norm(P[:3, 3] - G[:3, 3])))
    return rots, trans


# ------------------------------------------------------------- CPU baseline

def cpu_frames_per_s(cfg, seq, seconds: float):
    """FP32 OpenMP build of the oracle restatement on the host cores."""
    from oracle import CpuTracker, Oracle
    o = Oracle("f32")
    n_seq = len(seq.depth)
    tr = CpuTracker(o, cfg, seq.poses[0])
    tr.process(seq.depth[0])      # frame 0 (fuse only) is not timed
    n, t0 = 0, time.perf_counter()
    while n < 3 or time.perf_counter() - t0 < seconds:
        tr.process(seq.depth[frame_index(1 + n, n_seq)])
        n += 1
    dt = time.perf_counter() - t0
    tr.close()
    return n / dt, n, dt, o.threads()


# ------------------------------------------------ reference kernels (R1)

def ref_kernels_b200(cfg, seq, order, warmup: int, steps: int) -> dict:
    """Baseline leg: the reference's own CUDA kernels, rebuilt for sm_100a
    from its sources with this workload's volume geometry (512^3 over 3 m,
    truncation 30 mm, max weight 128; raycast step 0.75 voxel), driven in
    RunApp::display order (Source/src/MainApp.cpp:786-964: integrate ->
    raycast -> depth upload + updateCameraData -> 15 single-level ICP
    iterations with the host solve -> UpdateTransforms) on the same frames in
    the same order as the timed region, after the same warm-up. Frame time is
    the host wall time of each synchronous frame (the reference synchronises
    between its stages)."""
    import ctypes as C
    lib_path = ROOT / "oracle" / "_ref" / "libref_kernels_c2.so"
    if not lib_path.exists():
        return {"unavailable": "oracle/_ref/libref_kernels_c2.so not built (the reference "
                               "sources were absent at build time)"}
    lib = C.CDLL(str(lib_path))
    lib.ref_world_volume.restype = C.c_float
    lib.ref_truncation.restype = C.c_float
    geom = (lib.ref_volume_size(), float(lib.ref_world_volume()), float(lib.ref_truncation()),
            lib.ref_max_weight())
    if geom != (cfg.resolution, cfg.size_mm, cfg.trunc_mm, cfg.max_weight):
        return {"unavailable": f"reference kernels built for {geom}, not this workload"}

    class RefCam(C.Structure):
        _fields_ = [(k, C.c_int32) for k in ("w", "h")] + [
            (k, C.c_float) for k in ("fx", "fy", "cx", "cy", "ifx", "ify", "icx", "icy",
                                     "dmin", "dmax")]
    # inverse intrinsics as CameraFromFile.cpp:42-51 forms them (inverse of K)
    cam = RefCam(cfg.width, cfg.height, cfg.fx, cfg.fy, cfg.cx, cfg.cy, 1.0 / cfg.fx,
                 1.0 / cfg.fy, -cfg.cx / cfg.fx, -cfg.cy / cfg.fy, cfg.min_depth_mm,
                 cfg.max_depth_mm)
    P = C.c_void_p
    lib.ref_pipeline_create.argtypes = [P, P]
    lib.ref_pipeline_frame.argtypes = [P, P, P]
    pose0 = np.asarray(seq.poses[order[0]], np.float32).reshape(16).copy()
    if lib.ref_pipeline_create(C.byref(cam), pose0.ctypes.data) != 0:
        return {"unavailable": "ref_pipeline_create failed"}
    depth = [np.ascontiguousarray(seq.depth[j], np.uint16) for j in order]
    po = np.zeros(16, np.float32)
    t = C.c_double()
    ms, hist = [], []
    for i in range(len(order)):
        rc = lib.ref_pipeline_frame(depth[i].ctypes.data, po.ctypes.data, C.byref(t))
        if rc != 0:
            return {"unavailable": f"ref_pipeline_frame returned {rc} at frame {i}"}
        if i > warmup:
            ms.append(t.value)
            hist.append(po.reshape(4, 4).astype(np.float64))
    rots, trans = pose_errors(hist, [seq.poses[j] for j in order[1 + warmup:]])
    total_ms = float(np.sum(ms))
    return {"frames_per_s": len(ms) / (total_ms / 1e3), "ms_per_frame": total_ms / len(ms),
            "frames": len(ms), "warmup": warmup,
            "how": "host wall time per synchronous frame (std::chrono), same frames as the "
                   "timed region",
            "geometry": "512^3 over 3000 mm, truncation 30 mm, max weight 128 (generated "
                        "Constants.h); raycast step 1.5 mm x 3000/1024 = 0.75 voxel",
            "icp": "1 level x 15 iterations, FP32 host solve (ICP.cpp:84-182)",
            "max_rot_err_deg": float(np.degrees(max(rots))), "max_trans_err_mm": float(max(trans))}


def cpp_shim_leg(frames: int) -> dict:
    """The same workload through the reference-shaped C++ classes
    (include/openfusion_b200.hpp) with the reference's own call lines and
    order: Integrate -> Raycast -> synchronous depth upload +
    CameraHandler::updateCameraData -> ICP::Iterate_ICP ->
    General::Instance()->UpdateTransforms, one call per stage per frame on the
    legacy default stream, no graph (tests/cpp/shim_track.cpp; CUDA events
    around the frame loop after two warm-up frames). The drop-in path a
    reference host gets by linking the shim."""
    exe = ROOT / "tests" / "cpp" / "_build" / "shim_track"
    if not exe.exists():
        return {"unavailable": "tests/cpp/_build/shim_track not built"}
    try:
        out = subprocess.run([str(exe), str(frames), "c2"], capture_output=True, text=True,
                             timeout=600)
        res = json.loads(out.stdout.strip().splitlines()[-1])
    except Exception as e:  # report, never fail the bench line
        return {"unavailable": f"shim run failed: {e}"}
    res["how"] = ("reference call lines through include/openfusion_b200.hpp, per-stage calls, "
                  "synchronous pageable depth upload per frame, CUDA events")
    return res


# ------------------------------------------------------------------- arms

def run_reference(args, cfg, world, rank):
    if rank != 0:
        return
    import openfusion_b200 as of
    seq = of.make_sequence(cfg, frames=args.frames)
    n_seq = len(seq.depth)
    from oracle import CpuTracker, Oracle
    o = Oracle("f32")
    tr = CpuTracker(o, cfg, seq.poses[0])
    tr.process(seq.depth[0])
    t_w = time.perf_counter()
    for k in range(args.warmup):
        tr.process(seq.depth[frame_index(1 + k, n_seq)])
    per = (time.perf_counter() - t_w) / max(1, args.warmup)
    # keep the whole run within a few minutes: time at most ~120 s of frames
    steps = args.steps
    if per > 0 and steps * per > 120.0:
        steps = max(3, int(120.0 / per))
    t0 = time.perf_counter()
    for k in range(steps):
        tr.process(seq.depth[frame_index(1 + args.warmup + k, n_seq)])
    dt = time.perf_counter() - t0
    tr.close()
    fps = steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": fps, "unit": "frames/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dt / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded analytic room scene, axial noise + 2% dropout)",
        "config": workload_config(cfg, n_seq, args.gpus),
        "cpu_baseline": {"value": fps, "unit": "frames/s", "cores": o.threads(),
                         "cpu_model": cpu_model(), "kind": "port",
                         "sample": f"{steps} consecutive frames after {args.warmup} warm-up "
                                   "frames (FP32 OpenMP restatement of the same equations)"},
        "e2e": {"value": fps, "unit": "frames/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, cfg, world, rank, local):
    import torch
    import openfusion_b200 as of
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if rank:
        cfg = dataclasses.replace(cfg, seed=cfg.seed + 7919 * rank)
    seq = of.make_sequence(cfg, frames=args.frames)
    n_seq = len(seq.depth)
    total = 1 + args.warmup + args.steps
    order = [frame_index(i, n_seq) for i in range(total)]
    depth_dev = torch.from_numpy(seq.depth.astype(np.int16)).to(dev)
    depth_host = torch.from_numpy(seq.depth.astype(np.int16)).pin_memory()
    stream = torch.cuda.current_stream(dev)

    # the tracker tunes its raycast block shape online at the last warm-up
    # step, before its step graphs are captured (never inside the timed region)
    tune = args.warmup if args.warmup >= 1 else 0
    # ---- device-resident loop: value
    tr = of.Tracker(cfg, seq.poses[0], use_graph=True, pose_history=total, tune=tune)
    tr.process(depth_dev[order[0]])
    for i in range(1, 1 + args.warmup):
        tr.process(depth_dev[order[i]])
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    with sampler:
        ev0.record(stream)
        for i in range(1 + args.warmup, total):
            tr.process(depth_dev[order[i]])
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, world)
    bufs = tr.buffers()
    kernels = bufs.kernels_track * args.steps
    ray_tile, tuned = tr.tuning()
    hist = tr.pose_history(total)
    _, st = tr.pose()
    # ---- per-frame times: CUDA events between the steps of the same tracker,
    # continuing the sequence (every frame is past frame 10)
    nf = min(args.steps, 300)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(nf + 1)]
    evs[0].record(stream)
    for i in range(nf):
        tr.process(depth_dev[frame_index(total + i, n_seq)])
        evs[i + 1].record(stream)
    torch.cuda.synchronize()
    per_frame = np.array([evs[i].elapsed_time(evs[i + 1]) for i in range(nf)])
    tr.close()
    rots, trans = pose_errors(hist, [seq.poses[j] for j in order])

    # ---- end to end through the C-ABI: pinned host depth in, pose out
    tr = of.Tracker(cfg, seq.poses[0], use_graph=True, pose_history=total, tune=tune)
    pose_out = torch.zeros((total, 16), dtype=torch.float64).pin_memory()
    tr.process(depth_host[order[0]])
    for i in range(1, 1 + args.warmup):
        tr.process(depth_host[order[i]])
        tr.pose(out=pose_out[i])
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev2.record(stream)
    for i in range(1 + args.warmup, total):
        tr.process(depth_host[order[i]])
        tr.pose(out=pose_out[i])
    ev3.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = max_over_ranks(ev2.elapsed_time(ev3), world)
    e2e_hist = pose_out.numpy().reshape(total, 4, 4)
    assert np.allclose(e2e_hist[1 + args.warmup:], hist[1 + args.warmup:], atol=1e-6), \
        "end-to-end poses differ from the device-resident run"
    tr.close()

    # ---- per-stage kernel times (stage-wise launches with CUDA events), with
    # the raycast block shape the tracker chose
    stages = stage_times(of, dataclasses.replace(cfg, ray_tile=ray_tile), seq, depth_dev, order,
                         args, dev)

    # ---- the learned warm start against plain ICP (large-motion workload)
    warm = warm_start_comparison(of, args, dev, world, rank) if args.warm_frames > 1 else None
    # ---- many independent streams batched
    batched = batched_streams(of, args, dev, world, rank) if args.c4_streams > 0 else None

    fps = world * args.steps / (ms_max / 1e3)
    e2e_fps = world * args.steps / (e2e_ms / 1e3)
    if rank != 0:
        return
    peak, peak_kind = peaks()
    integ_bytes = stages["integrate_alg_bytes"]
    # the traffic of a kernel that visits every voxel (the reference's), over
    # this stage's time: above the HBM peak because whole bricks are decided
    # from tile bounds and skipped
    sweep_bytes = 8.0 * cfg.resolution ** 3 + 2.0 * cfg.width * cfg.height
    sweep_gbps = sweep_bytes / (stages["integrate_ms"] / 1e3) / 1e9
    achieved = integ_bytes / (stages["integrate_ms"] / 1e3) / 1e9
    traffic = profile_figure("integrate_traffic.json")
    line = {
        "metric": METRIC, "value": fps, "unit": "frames/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded analytic room scene, axial noise + 2% dropout)",
        "config": workload_config(cfg, n_seq, world),
        "stages_ms": {k: v for k, v in stages.items() if k.endswith("_ms")},
        "pose_error": {"max_rot_deg": float(np.degrees(max(rots))),
                       "max_trans_mm": float(max(trans)),
                       "mean_trans_mm": float(np.mean(trans)),
                       "last_icp_status": int(st.status), "last_inliers": int(st.inliers)},
        "roofline": {"kernel": "integrate stage (k_depth_tiles + k_classify_bricks + "
                               "k_integrate_list)", "bound": "hbm", "achieved": achieved,
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "alg_bytes_per_launch": integ_bytes,
                     "alg_units": "8 B per voxel in view (centre inside the 2-pixel border, "
                                  "depth in [min, max]) + 2 B per depth pixel",
                     "visible_voxels_per_launch": stages["integrate_visible_voxels"],
                     "updated_voxels_per_launch": stages["integrate_updated_voxels"],
                     "frac_updated_voxels": stages["integrate_updated_bytes"] /
                                            (stages["integrate_ms"] / 1e3) / 1e9 / peak},
        "roofline_raycast": {
            "kernel": "k_raycast", "bound": "hbm",
            "achieved": stages["raycast_alg_bytes"] / (stages["raycast_ms"] / 1e3) / 1e9,
            "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
            "frac": stages["raycast_alg_bytes"] / (stages["raycast_ms"] / 1e3) / 1e9 / peak,
            "traffic": profile_figure("raycast_traffic.json"),
            "alg_bytes_per_launch": stages["raycast_alg_bytes"],
            "alg_samples_per_launch": stages["raycast_samples"],
            "alg_units": "2 B per sample of a plain march at 0.75 voxel from the ray's entry "
                         "(box of voxel centres, depth range) to its surface or exit, 8 samples "
                         "per hit for the trilinear refinement, + 24 B per pixel out"},
        "frame_ms": {"median": float(np.median(per_frame)), "p10": float(np.percentile(per_frame, 10)),
                     "p90": float(np.percentile(per_frame, 90)), "frames": int(nf),
                     "how": "CUDA events between graph-replayed steps (rank 0)"},
        "integrate_full_sweep": {"bytes_per_frame": sweep_bytes, "equivalent_GBps": sweep_gbps,
                                 "note": "8 B x N^3 + depth (a kernel visiting every voxel, as the "
                                         "reference's does) over this stage's time; not a roofline "
                                         "fraction: whole bricks are skipped"},
        "e2e": {"value": e2e_fps, "unit": "frames/s",
                "h2d_bytes_per_step": cfg.width * cfg.height * 2, "d2h_bytes_per_step": 128},
        "gpu_launches": kernels,
        "tuning": {"raycast_block": ["16x16", "32x8", "8x32", "32x4", "16x8", "8x16", "8x8"][ray_tile],
                   "tuned_online": tuned, "at_warmup_step": tune},
        "clocks": sampler.summary(),
    }
    if warm is not None:
        line["warm_start"] = warm
    if batched is not None:
        line["batched_streams"] = batched
    if world == 1:
        line["e2e_cpp_shim"] = cpp_shim_leg(args.steps + 3)
    if world == 1 and not args.no_ref_kernels:
        ref = ref_kernels_b200(cfg, seq, order, args.warmup, args.steps)
        if "frames_per_s" in ref:
            ref["value_over_reference_kernels"] = fps / ref["frames_per_s"]
            ref["e2e_over_reference_kernels"] = e2e_fps / ref["frames_per_s"]
        line["ref_kernels_b200"] = ref
    if world == 1 and not args.no_cpu_baseline:
        cps, n, dt, cores = cpu_frames_per_s(cfg, seq, args.cpu_seconds)
        line["cpu_baseline"] = {"value": cps, "unit": "frames/s", "cores": cores,
                                "cpu_model": cpu_model(), "kind": "port",
                                "sample": f"{n} consecutive frames ({dt:.1f} s) of the same "
                                          "sequence, FP32 OpenMP restatement"}
    print(json.dumps(line), flush=True)


def warm_start_comparison(of, args, dev, world, rank):
    """The learned warm start against plain ICP on the large-motion workload
    (640x480, 512^3 over 3 m, inter-frame motion up to 10 cm / 5 deg): three
    held-out seeds (910000 + 3 rank + i), both trackers with the same early
    exit over the same rendered frames. Per seed, one synchronous pass per arm
    gives ICP iterations and pose error against the ground truth, then three
    rounds of device-timed passes (CUDA events, max over ranks) alternate the
    arms; a seed's frames/s are the median of its rounds."""
    from openfusion_b200 import learned
    from openfusion_b200.train_warm_start import eval_config, pose_errors, run_tracker
    cfg0 = eval_config(of)
    weights = learned.load_weights()
    seeds = [910000 + 3 * rank + i for i in range(3)]
    out = {"workload": "c5: 640x480, 512^3 over 3 m, motion U[0,10] cm / U[0,5] deg per frame; "
                       f"early exit {cfg0.stop_rot_rad:g} rad / {cfg0.stop_trans_mm:g} mm in both "
                       "arms; warm pass on the finest level",
           "seeds": seeds, "frames_per_seed": args.warm_frames - 1,
           "data": "synthetic (held-out seeds, device renderer)",
           "how": "per seed: median of 3 alternating device-timed passes per arm"}
    arms = {"plain": None, "warm": weights}
    acc = {arm: {"ms": [], "its": [], "rot": [], "trans": [], "kept": []} for arm in arms}
    ratios = []
    for seed in seeds:
        cfg = dataclasses.replace(cfg0, seed=seed)
        scene = of.make_scene(cfg.scene_kind, cfg.seed, cfg.size_mm)
        poses = of.make_trajectory(cfg.motion, cfg.seed + 1, cfg.size_mm, args.warm_frames)
        depth = learned.render_device(cfg, scene, poses, device=dev)
        for arm, w in arms.items():
            hist, its, kept, _ = run_tracker(of, cfg, depth, poses, w, timed=False)
            r, t = pose_errors(hist[1:], poses[1:])
            acc[arm]["its"] += list(its)
            acc[arm]["rot"] += list(r)
            acc[arm]["trans"] += list(t)
            if arm == "warm":
                acc[arm]["kept"] += list(kept == 1)
        per = {arm: [] for arm in arms}
        for _ in range(3):
            for arm, w in arms.items():
                barrier(world)
                _, _, _, ms = run_tracker(of, cfg, depth, poses, w, timed=True)
                per[arm].append(max_over_ranks(ms, world))
        for arm in arms:
            acc[arm]["ms"].append(float(np.median(per[arm])))
        ratios.append(acc["plain"]["ms"][-1] / acc["warm"]["ms"][-1])
    for arm in arms:
        a = acc[arm]
        out[arm] = {"frames_per_s": world * 1e3 / float(np.mean(a["ms"])),
                    "frames_per_s_per_seed": [world * 1e3 / m for m in a["ms"]],
                    "ms_per_frame": float(np.mean(a["ms"])),
                    "mean_icp_iterations": float(np.mean(a["its"])),
                    "max_rot_err_deg": float(np.max(a["rot"])), "mean_rot_err_deg": float(np.mean(a["rot"])),
                    "max_trans_err_mm": float(np.max(a["trans"])), "mean_trans_err_mm": float(np.mean(a["trans"]))}
        if arm == "warm":
            out[arm]["warm_start_kept_frac"] = float(np.mean(a["kept"]))
    out["warm_over_plain_frames_per_s_per_seed"] = ratios
    out["warm_over_plain_frames_per_s"] = float(np.mean(ratios))
    # the per-frame FP64 oracle comparison of both arms is a test run
    # (tests/warm_start_c5.py); its recorded summary is carried here, labelled
    rec = ROOT / "profiles" / "warm_start_c5_oracle_study.json"
    if rec.exists():
        st = json.loads(rec.read_text())
        out["oracle_study_recorded"] = {
            "source": str(rec.relative_to(ROOT)), "command": st["command"],
            "seeds": st["seeds"], "frames_per_seed": st["frames_per_seed"],
            "bar": st["equal_error"]["bar"],
            "plain_within": st["equal_error"]["plain_within"],
            "warm_within": st["equal_error"]["warm_within"],
            **{f"{arm}_max_{k}_vs_fp64_oracle": st[arm][f"max_{k}_vs_full_oracle"]
               for arm in ("plain", "warm") for k in ("rot_rad", "trans_mm")},
            "warm_over_plain_frames_per_s": st["warm_over_plain_frames_per_s"],
            "note": "recorded by the oracle study, not re-measured by this run"}
    return out


def batched_streams(of, args, dev, world, rank):
    """The batched-streams workload: 64 independent seeded streams of mixed
    resolution and volume (c4_configs), sharded over the ranks longest-first,
    one frame of every stream per step through one Batch (one launch per
    stage, CUDA graph per step, knobs tuned online during the warm-up).
    Beside it: the same streams through one single-stream Tracker each, run
    one after another on the same device (the per-stream path). Device time,
    max over ranks; frames/s counts every stream's frames."""
    import torch
    from openfusion_b200 import learned
    cfgs = of.c4_configs(count=args.c4_streams, frames=args.c4_frames)
    plan = of.shard([of.stream_cost(c) for c in cfgs], world)
    mine = [c for c, r in zip(cfgs, plan) if r == rank]
    seqs = []
    for c in mine:
        scene = of.make_scene(c.scene_kind, c.seed, c.size_mm)
        poses = of.make_trajectory(c.motion, c.seed + 1, c.size_mm, c.frames)
        seqs.append((poses, learned.render_device(c, scene, poses, device=dev)))
    n_seq = args.c4_frames
    tune_steps = 30
    warm = max(args.warmup, tune_steps)
    total = 1 + warm + args.c4_steps
    order = [frame_index(i, n_seq) for i in range(total)]
    stream = torch.cuda.current_stream(dev)
    out = {"workload": f"c4: {args.c4_streams} streams, resolution U{{160x120, 320x240, 640x480}}, "
                       "volume U{128^3, 256^3, 512^3} over U[2, 3] m, seeded rooms; one frame of "
                       "every stream per step",
           "streams": args.c4_streams, "streams_this_rank": len(mine), "steps": args.c4_steps,
           "data": "synthetic (device renderer)", "parallelism": f"shard{world}"}
    # ---- batched
    batch = of.Batch(mine, [p[0] for p, _ in seqs], use_graph=True, tune=True)
    for i in range(1 + warm):
        batch.process([d[order[i]] for _, d in seqs])
    torch.cuda.synchronize()
    tun = batch.tuning()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    e0.record(stream)
    for i in range(1 + warm, total):
        batch.process([d[order[i]] for _, d in seqs])
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    P = batch.poses()
    err = [pose_errors([P[k]], [seqs[k][0][order[-1]]]) for k in range(len(mine))]
    launches = batch.buffers(0).kernels_track
    batch.close()
    del batch
    torch.cuda.empty_cache()
    # ---- the same streams, one single-stream tracker each
    trackers = [of.Tracker(c, p[0], use_graph=True, pose_history=8) for c, (p, _) in zip(mine, seqs)]
    for i in range(1 + warm):
        for t, (_, d) in zip(trackers, seqs):
            t.process(d[order[i]])
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    e0.record(stream)
    for i in range(1 + warm, total):
        for t, (_, d) in zip(trackers, seqs):
            t.process(d[order[i]])
    e1.record(stream)
    torch.cuda.synchronize()
    ms_seq = max_over_ranks(e0.elapsed_time(e1), world)
    err_seq = [pose_errors([t.pose()[0]], [seqs[k][0][order[-1]]]) for k, t in enumerate(trackers)]
    for t in trackers:
        t.close()
    del trackers
    torch.cuda.empty_cache()
    frames = args.c4_streams * args.c4_steps
    out.update({
        "frames_per_s": frames / (ms / 1e3), "ms_per_step": ms / args.c4_steps,
        "single_stream_trackers_frames_per_s": frames / (ms_seq / 1e3),
        "batched_over_single_stream": ms_seq / ms,
        "gpu_launches_per_step": launches,
        "tuning": {"ray_tile": int(tun.ray_tile), "list_div": int(tun.list_div),
                   "icp_clusters": int(tun.icp_clusters), "tuned": int(tun.tuned)},
        "max_rot_err_deg_last_step": float(np.degrees(max(e[0][0] for e in err))),
        "max_trans_err_mm_last_step": float(max(e[1][0] for e in err)),
        # the same streams through single-stream trackers: the drift against
        # the ground truth is the method's on that stream, not the batching's
        "single_stream_max_rot_err_deg_last_step": float(np.degrees(max(e[0][0] for e in err_seq))),
        "single_stream_max_trans_err_mm_last_step": float(max(e[1][0] for e in err_seq)),
        "worst_stream": worst_stream(mine, err, err_seq),
    })
    return out


def worst_stream(cfgs, err_batch, err_single):
    """The stream with the largest last-step translation error of the batch,
    with both paths' errors against the ground truth."""
    k = int(np.argmax([e[1][0] for e in err_batch]))
    return {"name": cfgs[k].name, "size_mm": cfgs[k].size_mm, "trunc_mm": cfgs[k].trunc_mm,
            "batched_rot_deg": float(np.degrees(err_batch[k][0][0])),
            "batched_trans_mm": float(err_batch[k][1][0]),
            "single_stream_rot_deg": float(np.degrees(err_single[k][0][0])),
            "single_stream_trans_mm": float(err_single[k][1][0])}


def stage_times(of, cfg, seq, depth_dev, order, args, dev):
    """Average device time of each stage, launched stage by stage on the
    current stream and bracketed by CUDA events, over the same frames."""
    import torch
    vol = of.new_volume(cfg, dev)
    lam = of.lambda_table(cfg, dev)
    scratch = of.integrate_scratch(cfg, dev)
    frame = of.new_pyramid(cfg, dev)
    model = of.new_pyramid(cfg, dev)
    ws = of.icp_workspace(cfg, dev)
    pose = torch.tensor(seq.poses[0].reshape(16), dtype=torch.float64, device=dev)
    of.integrate(cfg, vol, depth_dev[order[0]], pose, lam, scratch)
    of.raycast(cfg, vol, pose, model)
    acc = {"preprocess": 0.0, "icp": 0.0, "integrate": 0.0, "raycast": 0.0}
    s = torch.cuda.current_stream(dev)
    poses = [pose.clone()]
    n = 0
    total = len(order)
    ray_samples, ray_pixels = [], []
    for i in range(1, total):
        d = depth_dev[order[i]]
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
        ev[0].record(s)
        of.preprocess(cfg, d, frame)
        ev[1].record(s)
        of.icp_track(cfg, frame, model, pose, ws)
        ev[2].record(s)
        of.integrate(cfg, vol, d, pose, lam, scratch)
        ev[3].record(s)
        of.raycast(cfg, vol, pose, model)
        ev[4].record(s)
        poses.append(pose.clone())
        if i % 50 == 0 or i == total - 1:
            torch.cuda.synchronize()
        if i > args.warmup:
            s.synchronize()
            for j, name in enumerate(acc):
                acc[name] += ev[j].elapsed_time(ev[j + 1])
            n += 1
            if (i - args.warmup) % 10 == 1:
                # the raycast's algorithmic samples at this frame's pose, from
                # the surface distances the launch found (outside the timing)
                v, _ = of.unpack_points(cfg, model, 0)
                v = v.cpu().numpy().astype(np.float64)
                P = pose.cpu().numpy().reshape(4, 4)
                dist = np.linalg.norm(v[..., :3] - P[:3, 3], axis=-1)
                smp, _ = of.raycast_march_samples(cfg, P, v[..., 3] > 0, dist)
                ray_samples.append(smp)
                ray_pixels.append(cfg.width * cfg.height)
    # Algorithmic bytes of one integration launch: 4 B read + 4 B write per
    # voxel in view (centre inside the 2-pixel border, depth in [min, max])
    # plus 2 B per depth pixel; beside it the stricter count of the voxels the
    # launch actually changes. The census launches count both with the
    # integration's own tests and no writes; they replay the same frames at
    # the same poses on a second volume, outside any timing.
    vol2 = of.new_volume(cfg, dev)
    upd, vis = [], []
    for i in range(total):
        d = depth_dev[order[i]]
        if i > args.warmup and (i - args.warmup) % 10 == 0:
            upd.append(of.integrate_census(cfg, vol2, d, poses[i], lam))
            vis.append(of.integrate_visible_census(cfg, vol2, d, poses[i], lam))
        of.integrate(cfg, vol2, d, poses[i], lam, scratch)
    out = {f"{k}_ms": v / max(n, 1) for k, v in acc.items()}
    # raycast: 2 B (one int16 tsdf) per algorithmic sample + 24 B (vertex and
    # normal, 3 floats each) per pixel written
    out["raycast_samples"] = float(np.mean(ray_samples))
    out["raycast_alg_bytes"] = 2.0 * float(np.mean(ray_samples)) + 24.0 * float(np.mean(ray_pixels))
    out["integrate_alg_bytes"] = 8.0 * float(np.mean(vis)) + 2.0 * cfg.width * cfg.height
    out["integrate_visible_voxels"] = float(np.mean(vis))
    out["integrate_updated_bytes"] = 8.0 * float(np.mean(upd)) + 2.0 * cfg.width * cfg.height
    out["integrate_updated_voxels"] = float(np.mean(upd))
    del vol, vol2
    torch.cuda.empty_cache()
    return out


def main():
    args = parse()
    # the reference arm runs on rank 0 alone and exchanges nothing
    grouped = args.impl != "reference"
    world, rank, local = dist_setup(init=grouped)
    import openfusion_b200 as of
    cfg = of.CONFIGS[args.config]
    try:
        if args.impl == "reference":
            run_reference(args, cfg, world, rank)
        else:
            run_ours(args, cfg, world, rank, local)
    finally:
        if world > 1 and grouped:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
