"""Python mirror of the reference's per-frame interfaces over the C-ABI.

The reference exposes VolumeIntegrator::Integrate, Raycaster::Raycast,
ICP::Iterate_ICP and CameraHandler::updateCameraData over raw device
pointers (Source/include/VolumeIntegrator.h:9-17, Raycaster.h:6-13,
ICP.h:50-70, CameraHandler.h:24). Here the same stages take torch CUDA
tensors (device memory and streams only) and call the CUDA library; the
`Tracker` is the whole frame loop of RunApp::display (MainApp.cpp:786-964).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N

STORAGE = {"i16": 0, "f16": 1}


@dataclass
class Config:
    """One workload: camera, volume and algorithm parameters."""
    name: str
    width: int
    height: int
    fx: float
    fy: float
    cx: float
    cy: float
    resolution: int
    size_mm: float
    trunc_mm: float
    max_weight: int = 128
    storage: str = "i16"
    min_depth_mm: float = 300.0
    max_depth_mm: float = 5000.0
    sigma_space_px: float = 4.5
    sigma_range_mm: float = 30.0
    radius_px: int = 0
    levels: int = 3
    iters: tuple = (10, 5, 4)
    dist_thresh_mm: float = 25.0
    normal_thresh: float = 0.65
    stop_rot_rad: float = 0.0       # early exit (0 = every iteration)
    stop_trans_mm: float = 0.0
    judge_max_rms_mm: float = 10.0  # warm-start judge
    judge_min_inlier_frac: float = 0.3
    judge_max_rot_rad: float = 0.05
    judge_max_trans_mm: float = 50.0
    warm_levels: int = 0            # pyramid levels of a warm-started pass (0 = all)
    min_step_vox: float = 0.75
    far_step_frac: float = 0.8
    refine_iters: int = 3
    ray_tile: int = 0               # raycast block shape (0 16x16, 1 32x8, 2 8x32, 3 32x4,
                                    # 4 16x8, 5 8x16, 6 8x8)
    scene_kind: int = 1
    motion: int = 0
    noise: float = 1.0
    dropout: float = 0.0
    frames: int = 300
    seed: int = 2000

    def camera(self) -> N.Camera:
        return N.Camera(self.width, self.height, self.fx, self.fy, self.cx, self.cy,
                        self.min_depth_mm, self.max_depth_mm)

    def volume(self) -> N.VolumeDesc:
        return N.VolumeDesc(self.resolution, STORAGE[self.storage], self.size_mm, self.trunc_mm,
                            self.max_weight, 0)

    def filter(self) -> N.FilterParams:
        return N.FilterParams(self.sigma_space_px, self.sigma_range_mm, self.radius_px,
                              self.levels)

    def raycast(self) -> N.RaycastParams:
        return N.RaycastParams(self.min_step_vox, self.far_step_frac, self.refine_iters,
                               self.ray_tile)

    def icp(self) -> N.IcpParams:
        it = (C.c_int32 * 4)(*(list(self.iters) + [0] * (4 - len(self.iters))))
        return N.IcpParams(self.levels, it, self.dist_thresh_mm, self.normal_thresh,
                           self.stop_rot_rad, self.stop_trans_mm, self.judge_max_rms_mm,
                           self.judge_min_inlier_frac, self.judge_max_rot_rad,
                           self.judge_max_trans_mm, self.warm_levels)

    def radius(self) -> int:
        return self.radius_px if self.radius_px > 0 else int(np.ceil(2.0 * self.sigma_space_px))


# The workloads of the benchmark configurations: C1 small plain method,
# C2 full-size plain method, C3 precision study (1024^3 fp16), C5 large motion.
CONFIGS = {
    "c1": Config("c1_320x240_128^3", 320, 240, 262.5, 262.5, 160.0, 120.0, 128, 2000.0, 60.0,
                 max_weight=128, scene_kind=0, frames=30, seed=1000, dropout=0.0),
    "c2": Config("c2_640x480_512^3", 640, 480, 525.0, 525.0, 319.5, 239.5, 512, 3000.0, 30.0,
                 max_weight=128, scene_kind=1, frames=300, seed=2000, dropout=0.02),
    "c3": Config("c3_640x480_1024^3_f16", 640, 480, 525.0, 525.0, 319.5, 239.5, 1024, 4000.0,
                 30.0, max_weight=128, storage="f16", scene_kind=1, frames=300, seed=2000,
                 dropout=0.02),
    "c5": Config("c5_640x480_512^3_large_motion", 640, 480, 525.0, 525.0, 319.5, 239.5, 512,
                 3000.0, 30.0, max_weight=128, scene_kind=1, motion=1, frames=300, seed=5000,
                 dropout=0.02),
}


def c4_configs(count: int = 64, seed: int = 4000, frames: int = 100) -> list[Config]:
    """The batched-streams workload: `count` independent seeded scenes (room
    of 20 boxes and spheres), each with a resolution drawn uniformly from
    {160x120, 320x240, 640x480} (intrinsics scaled from 640x480 / 525 px) and
    a volume drawn from {128^3, 256^3, 512^3} over U[2, 3] m (truncation the
    larger of 30 mm and 4 voxels). Stream i: scene seed seed + i."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        w, h = [(160, 120), (320, 240), (640, 480)][int(rng.integers(0, 3))]
        res = [128, 256, 512][int(rng.integers(0, 3))]
        size = float(rng.uniform(2000.0, 3000.0))
        f = 525.0 * w / 640.0
        out.append(Config(f"c4_s{i}_{w}x{h}_{res}^3", w, h, f, f, (w - 1) / 2.0, (h - 1) / 2.0,
                          res, size, max(30.0, 4.0 * size / res), max_weight=128, scene_kind=1,
                          frames=frames, seed=seed + i, dropout=0.02))
    return out


def _stream(stream=None) -> int:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def pyramid_layout(cfg: Config, levels: int | None = None) -> N.PyramidLayout:
    lay = N.PyramidLayout()
    N.check("of_pyramid_layout",
            N.lib().of_pyramid_layout(C.byref(cfg.camera()), levels or cfg.levels, C.byref(lay)))
    return lay


def level_camera(cfg: Config, level: int) -> N.Camera:
    out = N.Camera()
    N.check("of_camera_level", N.lib().of_camera_level(C.byref(cfg.camera()), level, C.byref(out)))
    return out


def volume_bytes(cfg: Config) -> int:
    n = C.c_size_t()
    N.check("of_volume_bytes", N.lib().of_volume_bytes(C.byref(cfg.volume()), C.byref(n)))
    return n.value


# ------------------------------------------------------------------ stages --

def new_volume(cfg: Config, device="cuda"):
    import torch
    vol = torch.empty(volume_bytes(cfg) // 4, dtype=torch.int32, device=device)
    N.check("of_volume_reset", N.lib().of_volume_reset(C.byref(cfg.volume()), _ptr(vol), _stream()))
    return vol


def new_pyramid(cfg: Config, device="cuda"):
    import torch
    return torch.zeros(pyramid_layout(cfg).total_bytes, dtype=torch.uint8, device=device)


def lambda_table(cfg: Config, device="cuda"):
    import torch
    lam = torch.empty(cfg.width * cfg.height * 2, dtype=torch.float32, device=device)
    N.check("of_lambda_table", N.lib().of_lambda_table(C.byref(cfg.camera()), _ptr(lam), _stream()))
    return lam


def preprocess(cfg: Config, depth, frame=None):
    """CameraHandler::updateCameraData: uint16 depth -> filtered pyramid + maps."""
    frame = new_pyramid(cfg, depth.device) if frame is None else frame
    N.check("of_preprocess", N.lib().of_preprocess(C.byref(cfg.camera()), C.byref(cfg.filter()),
                                                   _ptr(depth), cfg.width, _ptr(frame), _stream()))
    return frame


def integrate_scratch(cfg: Config, device="cuda"):
    """Scratch of of_integrate_tiled (tile depth bounds and brick work list)."""
    import torch
    n = C.c_size_t()
    N.check("of_integrate_scratch_bytes",
            N.lib().of_integrate_scratch_bytes(C.byref(cfg.volume()), C.byref(cfg.camera()),
                                               C.byref(n)))
    return torch.empty(n.value, dtype=torch.uint8, device=device)


def integrate(cfg: Config, vol, depth, pose, lam, scratch=None):
    """VolumeIntegrator::Integrate: fuse `depth` at FP64 device pose `pose`.
    With `scratch` (integrate_scratch) whole bricks are decided from per-tile
    depth bounds (of_integrate_tiled); the volume written is the same."""
    if scratch is None:
        N.check("of_integrate", N.lib().of_integrate(C.byref(cfg.volume()), _ptr(vol),
                                                     C.byref(cfg.camera()), _ptr(depth), cfg.width,
                                                     _ptr(pose), _ptr(lam), _stream()))
    else:
        N.check("of_integrate_tiled",
                N.lib().of_integrate_tiled(C.byref(cfg.volume()), _ptr(vol), C.byref(cfg.camera()),
                                           _ptr(depth), cfg.width, _ptr(pose), _ptr(lam),
                                           _ptr(scratch), _stream()))


def integrate_census(cfg: Config, vol, depth, pose, lam) -> int:
    import torch
    cnt = torch.zeros(1, dtype=torch.int64, device=vol.device)
    N.check("of_integrate_census",
            N.lib().of_integrate_census(C.byref(cfg.volume()), _ptr(vol), C.byref(cfg.camera()),
                                        _ptr(depth), cfg.width, _ptr(pose), _ptr(lam), _ptr(cnt),
                                        _stream()))
    return int(cnt.item())

def integrate_visible_census(cfg: Config, vol, depth, pose, lam) -> int:
    """Voxels in view at `pose`: centre inside the 2-pixel image border with a
    depth in [min, max] (the integration's frustum test)."""
    import torch
    cnt = torch.zeros(1, dtype=torch.int64, device=vol.device)
    N.check("of_integrate_visible_census",
            N.lib().of_integrate_visible_census(C.byref(cfg.volume()), _ptr(vol),
                                                C.byref(cfg.camera()), _ptr(depth), cfg.width,
                                                _ptr(pose), _ptr(lam), _ptr(cnt), _stream()))
    return int(cnt.item())


def raycast(cfg: Config, vol, pose, model=None, rgba=None):
    """Raycaster::Raycast: world vertex/normal pyramid of the volume at `pose`."""
    model = new_pyramid(cfg, vol.device) if model is None else model
    N.check("of_raycast", N.lib().of_raycast(C.byref(cfg.volume()), _ptr(vol),
                                             C.byref(cfg.camera()), C.byref(cfg.raycast()),
                                             cfg.levels, _ptr(pose), _ptr(model), _ptr(rgba),
                                             _stream()))
    return model


def raycast_march_samples(cfg: Config, pose: np.ndarray, hit: np.ndarray,
                          hit_dist: np.ndarray) -> tuple[int, int]:
    """The algorithmic sample count of one raycast launch: for every pixel's
    ray (through the pixel at z = -1, Raycaster.cu:112-125), the volume reads
    of a plain march at 0.75 voxel from where the ray enters the box of voxel
    centres within the depth range to its surface (`hit`, at distance
    `hit_dist` mm from the camera) or to where it leaves, counting the sample
    at the start, plus 8 reads for the trilinear refinement of a hit. This is
    what a kernel without empty-space skipping reads; it is the roofline's
    unit, not what this library's raycast reads. Host arithmetic in FP64.
    Returns (samples, rays that enter the box)."""
    P = np.asarray(pose, np.float64).reshape(4, 4)
    ys, xs = np.mgrid[0:cfg.height, 0:cfg.width].astype(np.float64)
    dc = np.stack([-(xs - cfg.cx) / cfg.fx, -(ys - cfg.cy) / cfg.fy, -np.ones_like(xs)], -1)
    lam = np.linalg.norm(dc, axis=-1)
    d = (dc @ P[:3, :3].T) / lam[..., None]
    o = P[:3, 3]
    vs = cfg.size_mm / cfg.resolution
    lo, hi = -0.5 * cfg.size_mm + 0.5 * vs, 0.5 * cfg.size_mm - 0.5 * vs
    with np.errstate(divide="ignore", invalid="ignore"):
        t_a = (lo - o) / d
        t_b = (hi - o) / d
    par = np.abs(d) < 1e-12
    inside = (o >= lo) & (o <= hi)
    t_near = np.where(par, np.where(inside, -np.inf, np.inf), np.minimum(t_a, t_b)).max(-1)
    t_far = np.where(par, np.where(inside, np.inf, -np.inf), np.maximum(t_a, t_b)).min(-1)
    t0 = np.maximum(t_near, cfg.min_depth_mm * lam)
    t1 = np.minimum(t_far, cfg.max_depth_mm * lam)
    enters = t0 < t1
    hit = np.asarray(hit, bool) & enters
    t_end = np.where(hit, np.asarray(hit_dist, np.float64), t1)
    step = 0.75 * vs
    n = np.where(enters & (t_end >= t0), np.floor((t_end - t0) / step) + 1.0, 0.0)
    n += np.where(hit, 8.0, 0.0)
    return int(n.sum()), int(enters.sum())


def icp_workspace(cfg: Config, device="cuda"):
    import torch
    n = C.c_size_t()
    N.check("of_icp_workspace_bytes",
            N.lib().of_icp_workspace_bytes(C.byref(cfg.camera()), C.byref(n)))
    return torch.zeros(n.value, dtype=torch.uint8, device=device)


def icp_track(cfg: Config, frame, model, pose, ws, stats=None):
    """ICP::Iterate_ICP: refine the FP64 device pose in place."""
    N.check("of_icp_track", N.lib().of_icp_track(C.byref(cfg.camera()), C.byref(cfg.icp()),
                                                 _ptr(frame), _ptr(model), _ptr(pose), _ptr(ws),
                                                 _ptr(stats), _stream()))


def icp_track_warm(cfg: Config, frame, model, pose, warm_pose, ws, stats=None):
    """icp_track from a warm start (FP64 device 4x4), judged against the
    previous pose in `pose`; a rejected result is replaced by plain ICP."""
    N.check("of_icp_track_warm",
            N.lib().of_icp_track_warm(C.byref(cfg.camera()), C.byref(cfg.icp()), _ptr(frame),
                                      _ptr(model), _ptr(pose), _ptr(warm_pose), _ptr(ws),
                                      _ptr(stats), _stream()))


def icp_system(cfg: Config, level: int, frame, model, pose, ws):
    """One correspondence + reduction pass (ICP::FindCorresponding): 29 floats."""
    import torch
    out = torch.zeros(29, dtype=torch.float32, device=frame.device)
    N.check("of_icp_system", N.lib().of_icp_system(C.byref(cfg.camera()), C.byref(cfg.icp()),
                                                   level, _ptr(frame), _ptr(model), _ptr(pose),
                                                   _ptr(ws), _ptr(out), _stream()))
    return out


class _DeviceBytes:
    """A device range described by the CUDA array interface (no copy)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1",
                                         "data": (int(ptr), False), "version": 3}


def copy_pyramid(cfg: Config, ptr: int, device="cuda"):
    """A copy (uint8 CUDA tensor) of the frame or model pyramid at device
    address `ptr`, e.g. a Tracker's or a Batch stream's `buffers().frame` /
    `.model`, ordered on the current stream."""
    import torch
    src = torch.as_tensor(_DeviceBytes(ptr, int(pyramid_layout(cfg).total_bytes)), device=device)
    return src.clone()


def unpack_points(cfg: Config, pyr, level: int = 0):
    """(vertex[H,W,4], normal[H,W,4]) views of one level of a pyramid buffer."""
    import torch
    lay = pyramid_layout(cfg)
    w, h = lay.width[level], lay.height[level]
    off = lay.points_offset[level]
    pts = pyr[off: off + w * h * 32].view(torch.float32).view(h, w, 2, 4)
    return pts[:, :, 0, :], pts[:, :, 1, :]


def unpack_depth(cfg: Config, pyr, level: int = 0):
    import torch
    lay = pyramid_layout(cfg)
    w, h = lay.width[level], lay.height[level]
    off = lay.depth_offset[level]
    return pyr[off: off + w * h * 4].view(torch.float32).view(h, w)


def volume_to_linear(cfg: Config, vol_words: np.ndarray):
    """Brick-major voxel words -> (tsdf_q int16 or f16 bits, weight) in x,y,z order.
    `vol_words` is a whole volume buffer (its trailing brick flags are ignored)."""
    n = cfg.resolution
    nb = n // 8
    w = np.asarray(vol_words).view(np.uint32)[: n ** 3].reshape(nb, nb, nb, 8, 8, 8)
    w = w.transpose(0, 3, 1, 4, 2, 5).reshape(n, n, n)
    return (w & 0xFFFF).astype(np.uint16), (w >> 16).astype(np.uint16)


def linear_to_volume(cfg: Config, q: np.ndarray, weight: np.ndarray) -> np.ndarray:
    """(q, weight) in x,y,z order -> a whole volume buffer (int32 words) with
    every brick flagged as near a surface; unobserved voxels (weight 0) hold
    the +1 pattern, as the library's reset writes them."""
    n = cfg.resolution
    nb = n // 8
    one = 0x7FFF if cfg.storage == "i16" else 0x3C00
    q = np.where(np.asarray(weight) == 0, one, np.asarray(q).astype(np.int64) & 0xFFFF)
    words = (q.astype(np.uint32) & 0xFFFF) | (weight.astype(np.uint32) << 16)
    words = words.reshape(nb, 8, nb, 8, nb, 8).transpose(0, 2, 4, 1, 3, 5).reshape(-1)
    # brick and super-brick flags set (near a surface), saturated-brick bytes clear
    nbr = nb ** 3
    ns = (nb + 3) // 4
    tail = np.zeros(volume_bytes(cfg) - 4 * n ** 3, np.uint8)
    tail[:nbr] = 1
    soff = (nbr + 255) // 256 * 256
    tail[soff:soff + ns ** 3] = 1
    return np.concatenate([words.view(np.uint8), tail]).view(np.int32)


# ----------------------------------------------------------------- tracker --

class Tracker:
    """Owns the per-frame state of RunApp (MainApp.cpp:591-647) and runs the
    frame loop (MainApp.cpp:786-964) as one CUDA graph per frame."""

    def __init__(self, cfg: Config, initial_pose: np.ndarray, use_graph: bool = True,
                 pose_history: int = 1024, warm_start_weights: np.ndarray | None = None,
                 depth_filter: N.DepthFilterParams | None = None, tune: int = 0):
        """`warm_start_weights`: FP32 weights of the warm-start CNN (None =
        plain ICP from the previous pose). `tune` = k >= 1: step k times every
        raycast block shape and keeps the fastest before the step graphs are
        captured (of_tracker_desc_t.tune); 0: cfg.ray_tile as given."""
        self.cfg = cfg
        d = N.TrackerDesc()
        d.camera = cfg.camera()
        d.volume = cfg.volume()
        d.filter = cfg.filter()
        d.raycast = cfg.raycast()
        d.icp = cfg.icp()
        d.initial_pose = (C.c_double * 16)(*np.asarray(initial_pose, np.float64).reshape(16))
        d.use_graph = 1 if use_graph else 0
        d.pose_history = pose_history
        d.tune = tune
        if depth_filter is not None:
            d.depth_filter = depth_filter
        self._weights = None
        if warm_start_weights is not None:
            self._weights = np.ascontiguousarray(warm_start_weights, np.float32)
            d.warm_start_weights = self._weights.ctypes.data
        h = C.c_void_p()
        N.check("of_tracker_create", N.lib().of_tracker_create(C.byref(d), C.byref(h)))
        self._h = h
        self.frames = 0

    def close(self):
        if self._h:
            N.lib().of_tracker_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def process(self, depth, stream=None):
        """`depth`: CUDA uint16 tensor, or a (pinned) CPU tensor copied on `stream`."""
        on_host = 0 if depth.is_cuda else 1
        N.check("of_tracker_process",
                N.lib().of_tracker_process(self._h, depth.data_ptr(), on_host, _stream(stream)))
        self.frames += 1

    def flush(self, stream=None):
        """Fuses the last processed frame now (each process() call fuses the
        frame before it); call before reading the volume or the model."""
        N.check("of_tracker_flush", N.lib().of_tracker_flush(self._h, _stream(stream)))

    def save(self, path, stream=None):
        """Checkpoint: volume, pose, history, frame count, last frame (of_tracker_save)."""
        N.check("of_tracker_save", N.lib().of_tracker_save(self._h, str(path).encode(),
                                                           _stream(stream)))

    def load(self, path, stream=None):
        """Resume from a checkpoint of the same configuration (of_tracker_load)."""
        N.check("of_tracker_load", N.lib().of_tracker_load(self._h, str(path).encode(),
                                                           _stream(stream)))
        b = self.buffers()
        self.frames = int(b.frames)

    def set_prior(self, delta: np.ndarray | None):
        arr = None if delta is None else (C.c_double * 16)(*np.asarray(delta, np.float64).reshape(16))
        N.check("of_tracker_set_prior", N.lib().of_tracker_set_prior(self._h, arr))

    def pose(self, out=None, stats_out=None, stream=None):
        """Copies the current pose into `out` (pinned float64 tensor [16]) asynchronously,
        or returns a numpy array after a synchronous copy."""
        import torch
        if out is None:
            buf = (C.c_double * 16)()
            st = N.IcpStats()
            N.check("of_tracker_pose", N.lib().of_tracker_pose(self._h, buf, C.byref(st),
                                                               _stream(stream)))
            torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
            return np.array(buf[:]).reshape(4, 4), st
        N.check("of_tracker_pose", N.lib().of_tracker_pose(self._h, out.data_ptr(),
                                                           _ptr(stats_out), _stream(stream)))
        return out

    def pose_history(self, count: int) -> np.ndarray:
        buf = np.zeros((count, 16), np.float64)
        N.check("of_tracker_pose_history",
                N.lib().of_tracker_pose_history(self._h, buf.ctypes.data, count, _stream()))
        return buf.reshape(count, 4, 4)

    def buffers(self) -> N.TrackerBuffers:
        b = N.TrackerBuffers()
        N.check("of_tracker_buffers", N.lib().of_tracker_buffers(self._h, C.byref(b)))
        return b

    def tuning(self) -> tuple[int, bool]:
        """(raycast block shape in use, whether the online tuning has run)."""
        tile, tuned = C.c_int32(), C.c_int32()
        N.check("of_tracker_tuning", N.lib().of_tracker_tuning(self._h, C.byref(tile),
                                                               C.byref(tuned)))
        return tile.value, bool(tuned.value)


# --------------------------------------------------------------- synthetic --

@dataclass
class Sequence:
    cfg: Config
    scene: N.SynthScene
    poses: np.ndarray            # [F, 4, 4] ground-truth camera-to-world
    depth: np.ndarray = field(default=None)   # [F, H, W] uint16


def make_scene(kind: int, seed: int, cube_mm: float) -> N.SynthScene:
    sc = N.SynthScene()
    if N.synth().of_synth_scene(kind, seed, cube_mm, C.byref(sc)) != 0:
        raise ValueError("of_synth_scene: bad arguments")
    return sc


def make_trajectory(motion: int, seed: int, cube_mm: float, frames: int) -> np.ndarray:
    out = np.zeros((frames, 16), np.float64)
    if N.synth().of_synth_trajectory(motion, seed, cube_mm, frames, out.ctypes.data) != 0:
        raise ValueError("of_synth_trajectory: bad arguments")
    return out.reshape(frames, 4, 4)


def render(cfg: Config, scene: N.SynthScene, pose: np.ndarray, frame: int,
           noise: float | None = None, dropout: float | None = None, exact: bool = False):
    depth = np.zeros((cfg.height, cfg.width), np.uint16)
    ex = np.zeros((cfg.height, cfg.width), np.float32) if exact else None
    P = np.ascontiguousarray(pose, np.float64)
    r = N.synth().of_synth_render(C.byref(scene), cfg.width, cfg.height, cfg.fx, cfg.fy, cfg.cx,
                                  cfg.cy, P.ctypes.data, cfg.seed + 2, frame,
                                  cfg.noise if noise is None else noise,
                                  cfg.dropout if dropout is None else dropout, depth.ctypes.data,
                                  None if ex is None else ex.ctypes.data)
    if r != 0:
        raise ValueError("of_synth_render: bad arguments")
    return (depth, ex) if exact else depth


def make_sequence(cfg: Config, frames: int | None = None, render_depth: bool = True) -> Sequence:
    f = cfg.frames if frames is None else frames
    scene = make_scene(cfg.scene_kind, cfg.seed, cfg.size_mm)
    poses = make_trajectory(cfg.motion, cfg.seed + 1, cfg.size_mm, f)
    seq = Sequence(cfg, scene, poses)
    if render_depth:
        seq.depth = np.stack([render(cfg, scene, poses[k], k) for k in range(f)])
    return seq


# ------------------------------------------------------- camera-side filters --

DEPTH_FILTER = {"median5": 1, "gradient": 2, "average": 4, "undistort": 8}


def depth_filter_params(steps=(), null_value: int = 0, average_passes: int = 1,
                        average_threshold_mm: float = 15.0, gradient_threshold_mm: float = 10.0,
                        k1=0.0, k2=0.0, p1=0.0, p2=0.0) -> N.DepthFilterParams:
    p = N.DepthFilterParams()
    N.lib().of_depth_filter_defaults(C.byref(p))
    p.steps = sum(DEPTH_FILTER[s] for s in steps)
    p.null_value, p.average_passes = null_value, average_passes
    p.average_threshold_mm, p.gradient_threshold_mm = average_threshold_mm, gradient_threshold_mm
    p.k1, p.k2, p.p1, p.p2 = k1, k2, p1, p2
    return p


def depth_filter(cfg: Config, depth, steps=(), out=None, **kw):
    """The camera-side filter chain on a CUDA uint16 (int16-typed) depth image."""
    import torch
    p = depth_filter_params(steps, **kw)
    out = torch.empty_like(depth) if out is None else out
    scratch = torch.empty_like(depth)
    N.check("of_depth_filter", N.lib().of_depth_filter(C.byref(cfg.camera()), C.byref(p),
                                                       _ptr(depth), _ptr(out), _ptr(scratch),
                                                       _stream()))
    return out


# ----------------------------------------------------------- headless views --

def depth_rgba(cfg: Config, depth):
    """RGBA8 words [H, W] (int32 CUDA tensor): gray depth / max depth."""
    import torch
    out = torch.empty((cfg.height, cfg.width), dtype=torch.int32, device=depth.device)
    N.check("of_depth_to_rgba", N.lib().of_depth_to_rgba(C.byref(cfg.camera()), _ptr(depth),
                                                         _ptr(out), _stream()))
    return out


def normals_rgba(cfg: Config, pyramid, pose=None, alpha: float = 1.0):
    """RGBA8 words [H, W] of level-0 normals, (n + 1) / 2 (world space with `pose`)."""
    import torch
    out = torch.empty((cfg.height, cfg.width), dtype=torch.int32, device=pyramid.device)
    N.check("of_normals_to_rgba", N.lib().of_normals_to_rgba(
        C.byref(cfg.camera()), _ptr(pyramid), _ptr(pose), alpha, _ptr(out), _stream()))
    return out


# ------------------------------------------------------------------- mesh --

def extract_mesh(cfg: Config, vol, max_triangles: int | None = None, with_ids: bool = False):
    """Triangles [T, 3, 3] (CUDA float32, world mm) of the volume's surface
    (of_mesh_extract); grows the buffer once if the first guess is short."""
    import torch
    cap = max_triangles or 1 << 20
    count = torch.zeros(1, dtype=torch.int32, device=vol.device)
    for _ in range(2):
        tris = torch.empty((cap, 9), dtype=torch.float32, device=vol.device)
        ids = torch.empty(cap, dtype=torch.int64, device=vol.device) if with_ids else None
        N.check("of_mesh_extract", N.lib().of_mesh_extract(
            C.byref(cfg.volume()), _ptr(vol), _ptr(tris), _ptr(ids), cap, _ptr(count), _stream()))
        n = int(count.item())
        if n <= cap or max_triangles:
            break
        cap = n
    n = min(n, cap)
    out = tris[:n].view(n, 3, 3)
    return (out, ids[:n]) if with_ids else out


def write_obj(path, triangles) -> None:
    """Triangles [T, 3, 3] (host or CUDA) as a Wavefront OBJ file."""
    t = np.ascontiguousarray(triangles.cpu().numpy() if hasattr(triangles, "cpu") else triangles,
                             np.float32)
    N.check("of_mesh_write_obj", N.lib().of_mesh_write_obj(str(path).encode(), t.ctypes.data,
                                                           t.shape[0]))


def save_volume_raw(cfg: Config, vol, path) -> None:
    """The volume as the reference's SavedVolume.raw (N^3 float tsdf mm)."""
    N.check("of_volume_save_raw", N.lib().of_volume_save_raw(C.byref(cfg.volume()), _ptr(vol),
                                                             str(path).encode(), _stream()))


# --------------------------------------------------------------- recordings --

END_OF_SEQUENCE = 7  # of_reader_next after the last frame


def read_recording_info(path) -> N.RecordingInfo:
    """Parameters.txt of a recording directory (CameraFromFile::Init)."""
    info = N.RecordingInfo()
    N.check("of_recording_read_info", N.lib().of_recording_read_info(str(path).encode(),
                                                                     C.byref(info)))
    return info


def write_recording(path, cfg: Config, depth_frames, name: str = "", date: str = "",
                    camera_type: str = "Synthetic", z_offset_mm: float = 0.0) -> None:
    """A recording directory in the reference's format (WriteToFile): host
    uint16 frames [F, H, W] (numpy) or CUDA tensors."""
    import os
    os.makedirs(path, exist_ok=True)
    info = N.RecordingInfo()
    info.camera = cfg.camera()
    info.z_offset_mm = z_offset_mm
    info.frames = len(depth_frames)
    info.name = (name or str(path)).encode()[:255]
    info.date = date.encode()[:63]
    info.camera_type = camera_type.encode()[:63]
    N.check("of_recording_write_info", N.lib().of_recording_write_info(str(path).encode(),
                                                                       C.byref(info)))
    for k, d in enumerate(depth_frames):
        on_dev = hasattr(d, "is_cuda") and d.is_cuda
        if on_dev:
            ptr = d.data_ptr()
        else:
            d = np.ascontiguousarray(d, np.uint16)
            ptr = d.ctypes.data
        N.check("of_recording_write_frame",
                N.lib().of_recording_write_frame(str(path).encode(), k + 1, cfg.width, cfg.height,
                                                 ptr, 1 if on_dev else 0,
                                                 _stream() if on_dev else None))


def read_recording_frame(path, number: int, width: int, height: int) -> np.ndarray:
    out = np.zeros((height, width), np.uint16)
    N.check("of_recording_read_frame", N.lib().of_recording_read_frame(
        str(path).encode(), number, width, height, out.ctypes.data))
    return out


class Reader:
    """A recording as a prefetching frame source (of_reader_*): next() copies
    the next frame into a CUDA tensor asynchronously; None after the last."""

    def __init__(self, path, prefetch: int = 4):
        h = C.c_void_p()
        N.check("of_reader_open", N.lib().of_reader_open(str(path).encode(), prefetch, C.byref(h)))
        self._h = h
        w, hh, f = C.c_int32(), C.c_int32(), C.c_int32()
        N.check("of_reader_info", N.lib().of_reader_info(self._h, C.byref(w), C.byref(hh),
                                                         C.byref(f)))
        self.width, self.height, self.frames = w.value, hh.value, f.value

    def next(self, out=None, stream=None):
        import torch
        if out is None:
            out = torch.empty((self.height, self.width), dtype=torch.int16, device="cuda")
        st = N.lib().of_reader_next(self._h, out.data_ptr(), _stream(stream))
        if st == END_OF_SEQUENCE:
            return None
        N.check("of_reader_next", st)
        return out

    def close(self):
        if self._h:
            N.lib().of_reader_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ batched --

def stream_cost(cfg: Config) -> float:
    """Per-frame work of one stream (voxel-visit units), of_batch_stream_cost."""
    st = N.BatchStream()
    st.camera = cfg.camera()
    st.volume = cfg.volume()
    c = C.c_double()
    N.check("of_batch_stream_cost", N.lib().of_batch_stream_cost(C.byref(st), C.byref(cfg.icp()),
                                                                 C.byref(c)))
    return c.value


def shard(costs, ranks: int) -> list[int]:
    """Longest-first greedy assignment of streams to ranks (of_batch_shard)."""
    n = len(costs)
    arr = (C.c_double * max(n, 1))(*costs)
    out = (C.c_int32 * max(n, 1))()
    N.check("of_batch_shard", N.lib().of_batch_shard(C.cast(arr, C.c_void_p), n, ranks,
                                                     C.cast(out, C.c_void_p)))
    return [int(out[i]) for i in range(n)]


class Batch:
    """Many independent streams (each its own Config: camera, volume) tracked
    and fused together, one launch per stage for all streams (of_batch_*).
    The filter, raycast and ICP parameters are `common`'s (default: the first
    stream's)."""

    def __init__(self, cfgs: list[Config], initial_poses, common: Config | None = None,
                 use_graph: bool = True, tune: bool = False, tuning: tuple | None = None):
        common = common or cfgs[0]
        self.cfgs = list(cfgs)
        n = len(cfgs)
        self._streams = (N.BatchStream * n)()
        for i, (c, P) in enumerate(zip(cfgs, initial_poses)):
            self._streams[i].camera = c.camera()
            self._streams[i].volume = c.volume()
            self._streams[i].initial_pose = (C.c_double * 16)(*np.asarray(P, np.float64).reshape(16))
        d = N.BatchDesc()
        d.count = n
        d.streams = C.cast(self._streams, C.POINTER(N.BatchStream))
        d.filter = common.filter()
        d.raycast = common.raycast()
        d.icp = common.icp()
        d.use_graph = 1 if use_graph else 0
        d.tune = 1 if tune else 0
        t = tuning or (0, 2, 0)
        d.tuning = N.BatchTuning(t[0], t[1], t[2], 0)
        h = C.c_void_p()
        N.check("of_batch_create", N.lib().of_batch_create(C.byref(d), C.byref(h)))
        self._h = h
        self.frames = 0

    def close(self):
        if self._h:
            N.lib().of_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def process(self, depths, stream=None):
        """One frame of every stream: CUDA uint16 tensors, or (pinned) CPU tensors."""
        assert len(depths) == len(self.cfgs)
        on_host = 0 if depths[0].is_cuda else 1
        ptrs = (C.c_void_p * len(depths))(*[d.data_ptr() for d in depths])
        N.check("of_batch_process", N.lib().of_batch_process(self._h, ptrs, on_host,
                                                             _stream(stream)))
        self.frames += 1

    def flush(self, stream=None):
        N.check("of_batch_flush", N.lib().of_batch_flush(self._h, _stream(stream)))

    def poses(self, with_stats: bool = False):
        """(n, 4, 4) current poses (synchronous), and the ICP statistics."""
        import torch
        n = len(self.cfgs)
        out = np.zeros((n, 16), np.float64)
        stats = (N.IcpStats * n)()
        N.check("of_batch_poses", N.lib().of_batch_poses(self._h, out.ctypes.data,
                                                         C.cast(stats, C.c_void_p), _stream()))
        torch.cuda.current_stream().synchronize()
        P = out.reshape(n, 4, 4)
        return (P, list(stats)) if with_stats else P

    def tuning(self) -> N.BatchTuning:
        t = N.BatchTuning()
        N.check("of_batch_tuning", N.lib().of_batch_tuning(self._h, C.byref(t)))
        return t

    def buffers(self, i: int) -> N.TrackerBuffers:
        b = N.TrackerBuffers()
        N.check("of_batch_stream_buffers", N.lib().of_batch_stream_buffers(self._h, i, C.byref(b)))
        return b

