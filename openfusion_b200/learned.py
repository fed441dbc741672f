"""Learned ICP warm start: the BF16 CNN of csrc/of_cnn.cu, its training data
and its training loop, over torch CUDA tensors (device memory and streams
only; every kernel is the library's own).

The network maps a (previous, current) pair of depth frames to the camera
motion between them; the tracker starts ICP from that prediction and keeps
it only when ICP's judge accepts the result (include/openfusion_b200.h,
of_icp_track_warm). Training pairs are rendered on the device from seeded
synthetic trajectories, and their labels are the poses this library's own
ICP produces for them.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _native as N
from .api import Config, _ptr, _stream, make_scene, make_trajectory, new_pyramid, preprocess

ROT_SCALE = 10.0    # network output = rotation vector (rad) x 10
TRANS_SCALE = 0.01  # network output = translation (mm) / 100
IN_ELEMS = 2 * 60 * 80
WEIGHTS = Path(__file__).resolve().parent / "weights" / "warm_start_c5.npy"


def param_count() -> int:
    n = C.c_int64()
    N.check("of_cnn_param_count", N.lib().of_cnn_param_count(C.byref(n)))
    return n.value


# ----------------------------------------------------------- pose algebra --

def log_so3(R: np.ndarray) -> np.ndarray:
    """Rotation vector of a rotation matrix (angle < pi)."""
    c = np.clip((np.trace(R) - 1.0) / 2.0, -1.0, 1.0)
    th = np.arccos(c)
    v = np.array([R[2, 1] - R[1, 2], R[0, 2] - R[2, 0], R[1, 0] - R[0, 1]])
    if th < 1e-6:
        return 0.5 * v
    return th / (2.0 * np.sin(th)) * v


def exp_so3(w: np.ndarray) -> np.ndarray:
    th = np.linalg.norm(w)
    K = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]])
    if th < 1e-8:
        return np.eye(3) + K + 0.5 * K @ K
    return np.eye(3) + np.sin(th) / th * K + (1 - np.cos(th)) / th ** 2 * K @ K


def motion_target(T_prev: np.ndarray, T_cur: np.ndarray) -> np.ndarray:
    """Network target of the motion from T_prev to T_cur (camera-to-world)."""
    D = np.linalg.inv(T_prev) @ T_cur
    return np.concatenate([log_so3(D[:3, :3]) * ROT_SCALE, D[:3, 3] * TRANS_SCALE])


def apply_motion(T_prev: np.ndarray, out: np.ndarray) -> np.ndarray:
    D = np.eye(4)
    D[:3, :3] = exp_so3(np.asarray(out[:3], np.float64) / ROT_SCALE)
    D[:3, 3] = np.asarray(out[3:], np.float64) / TRANS_SCALE
    return T_prev @ D


# ------------------------------------------------------------- rendering --

def render_device(cfg: Config, scene: N.SynthScene, poses: np.ndarray, first_frame: int = 0,
                  device="cuda", stream=None):
    """All frames of a trajectory rendered on the device: uint16 depth as an
    int16 tensor [F, H, W] (the host renderer's scene, noise and dropout)."""
    import torch
    f = len(poses)
    sc = torch.from_numpy(np.frombuffer(bytes(scene), np.uint8).copy()).to(device)
    P = torch.from_numpy(np.ascontiguousarray(poses, np.float64).reshape(f, 16)).to(device)
    out = torch.empty((f, cfg.height, cfg.width), dtype=torch.int16, device=device)
    N.check("of_synth_render_device",
            N.lib().of_synth_render_device(_ptr(sc), cfg.width, cfg.height, cfg.fx, cfg.fy,
                                           cfg.cx, cfg.cy, _ptr(P), f, cfg.seed + 2, first_frame,
                                           cfg.noise, cfg.dropout, _ptr(out), _stream(stream)))
    return out


# --------------------------------------------------------------- network --

class WarmStartNet:
    """Parameters (FP32 master + BF16 copy), Adam state and per-batch
    workspaces of the warm-start CNN."""

    def __init__(self, device="cuda", seed: int = 0, weights: np.ndarray | None = None):
        import torch
        self.device = torch.device(device)
        n = param_count()
        self.n = n
        self.master = torch.empty(n, dtype=torch.float32, device=self.device)
        self.params = torch.empty(n, dtype=torch.int16, device=self.device)  # BF16 bits
        self.m = torch.zeros(n, dtype=torch.float32, device=self.device)
        self.v = torch.zeros(n, dtype=torch.float32, device=self.device)
        self.grad = torch.zeros(n, dtype=torch.float32, device=self.device)
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        self.loss_w = torch.tensor([1.0, 1.0, 1.0, 1.0, 1.0, 1.0], dtype=torch.float32,
                                   device=self.device)
        self.step = 0
        self._ws = {}
        if weights is None:
            N.check("of_cnn_init", N.lib().of_cnn_init(_ptr(self.master), _ptr(self.params),
                                                        seed, _stream()))
        else:
            self.load(weights)

    def load(self, weights: np.ndarray):
        import torch
        w = np.ascontiguousarray(weights, np.float32).reshape(-1)
        assert w.size == self.n, (w.size, self.n)
        self.master.copy_(torch.from_numpy(w))
        N.check("of_cnn_load", N.lib().of_cnn_load(_ptr(self.master), _ptr(self.params), _stream()))

    def weights(self) -> np.ndarray:
        return self.master.cpu().numpy().copy()

    def workspace(self, batch: int):
        import torch
        if batch not in self._ws:
            b = C.c_size_t()
            N.check("of_cnn_workspace_bytes", N.lib().of_cnn_workspace_bytes(batch, C.byref(b)))
            self._ws[batch] = torch.empty(b.value, dtype=torch.uint8, device=self.device)
        return self._ws[batch]

    @staticmethod
    def inputs(prev, cur, out=None):
        """BF16 network inputs [B, 2*60*80] (int16 bits) of depth pairs
        prev[i], cur[i] (int16 tensors [B, H, W] or [H, W])."""
        import torch
        if prev.dim() == 2:
            prev, cur = prev[None], cur[None]
        b, h, w = prev.shape
        assert prev.is_contiguous() and cur.is_contiguous()
        out = torch.empty((b, IN_ELEMS), dtype=torch.int16, device=prev.device) if out is None else out
        cells = torch.empty((b, IN_ELEMS), dtype=torch.float32, device=prev.device)
        N.check("of_cnn_input", N.lib().of_cnn_input(_ptr(prev), _ptr(cur), w, h, b, h * w,
                                                    _ptr(cells), _ptr(out), _stream()))
        return out

    def forward(self, inp):
        import torch
        b = inp.shape[0]
        out = torch.empty((b, 6), dtype=torch.float32, device=self.device)
        N.check("of_cnn_forward", N.lib().of_cnn_forward(_ptr(self.params), _ptr(self.master),
                                                         _ptr(inp), b, _ptr(self.workspace(b)),
                                                         _ptr(out), _stream()))
        return out

    def gradients(self, inp, target):
        """Loss and parameter gradients (self.grad) of one batch."""
        b = inp.shape[0]
        N.check("of_cnn_backward",
                N.lib().of_cnn_backward(_ptr(self.params), _ptr(self.master), _ptr(inp), b,
                                        _ptr(target), _ptr(self.loss_w), _ptr(self.workspace(b)),
                                        _ptr(self.grad), _ptr(self.loss), _stream()))
        return self.loss

    def train_step(self, inp, target, lr: float):
        loss = self.gradients(inp, target)
        self.step += 1
        N.check("of_cnn_adam", N.lib().of_cnn_adam(_ptr(self.master), _ptr(self.params),
                                                   _ptr(self.grad), _ptr(self.m), _ptr(self.v),
                                                   self.step, lr, _stream()))
        return loss


# ------------------------------------------------------------ training data --

def icp_labelled_pairs(cfg: Config, seed: int, frames: int, device="cuda", swap: bool = False):
    """One seeded trajectory: network inputs of its consecutive depth pairs
    and their targets, the motion between each frame's ground-truth pose and
    the pose this library's ICP finds for the next frame (frame-to-frame,
    started at the ground truth, against the previous frame's own maps).
    With `swap` the reversed pairs follow, with the inverse motions."""
    import torch
    import dataclasses
    c = dataclasses.replace(cfg, seed=seed)
    scene = make_scene(c.scene_kind, seed, c.size_mm)
    poses = make_trajectory(c.motion, seed + 1, c.size_mm, frames)
    depth = render_device(c, scene, poses, device=device)
    inp = WarmStartNet.inputs(depth[:-1].contiguous(), depth[1:].contiguous())
    lib = N.lib()
    cam = c.camera()
    frame = new_pyramid(c, device)
    model = new_pyramid(c, device)
    ws = torch.empty(_icp_ws_bytes(c), dtype=torch.uint8, device=device).zero_()
    v3 = torch.empty((c.height * c.width, 3), dtype=torch.float32, device=device)
    n3 = torch.empty_like(v3)
    pose_prev = torch.empty(16, dtype=torch.float64, device=device)
    pose = torch.empty(16, dtype=torch.float64, device=device)
    out = torch.empty((frames - 1, 16), dtype=torch.float64, device=device)
    icp = c.icp()
    preprocess(c, depth[0], frame)
    for k in range(1, frames):
        # model: the previous frame's maps in world space at its true pose
        pose_prev.copy_(torch.from_numpy(poses[k - 1].reshape(16)))
        N.check("of_points_to_reference", lib.of_points_to_reference(
            C.byref(cam), _ptr(frame), _ptr(pose_prev), _ptr(v3), _ptr(n3), _stream()))
        N.check("of_points_from_reference", lib.of_points_from_reference(
            C.byref(cam), c.levels, _ptr(v3), _ptr(n3), _ptr(model), _stream()))
        preprocess(c, depth[k], frame)
        pose.copy_(torch.from_numpy(poses[k].reshape(16)))
        N.check("of_icp_track", lib.of_icp_track(C.byref(cam), C.byref(icp), _ptr(frame),
                                                 _ptr(model), _ptr(pose), _ptr(ws), None,
                                                 _stream()))
        out[k - 1].copy_(pose)
    icp_poses = out.cpu().numpy().reshape(-1, 4, 4)
    target = np.stack([motion_target(poses[k - 1], icp_poses[k - 1]) for k in range(1, frames)])
    if swap:
        inp = torch.cat([inp, WarmStartNet.inputs(depth[1:].contiguous(), depth[:-1].contiguous())])
        back = np.stack([motion_target(icp_poses[k - 1], poses[k - 1]) for k in range(1, frames)])
        target = np.concatenate([target, back])
    return inp, torch.from_numpy(target.astype(np.float32)).to(device), poses, icp_poses


def _icp_ws_bytes(cfg: Config) -> int:
    b = C.c_size_t()
    N.check("of_icp_workspace_bytes", N.lib().of_icp_workspace_bytes(C.byref(cfg.camera()),
                                                                    C.byref(b)))
    return b.value


def training_set(cfg: Config, seeds, frames: int, device="cuda", swap: bool = False):
    import torch
    xs, ys = [], []
    for s in seeds:
        x, y, _, _ = icp_labelled_pairs(cfg, int(s), frames, device, swap)
        xs.append(x)
        ys.append(y)
    return torch.cat(xs), torch.cat(ys)


def train(net: WarmStartNet, x, y, epochs: int, batch: int = 256, lr: float = 1e-3,
          seed: int = 0, log=None):
    """Adam over shuffled mini-batches (a fixed permutation per epoch from
    `seed`); the learning rate decays linearly to 10% over the run."""
    import torch
    n = x.shape[0]
    rng = np.random.default_rng(seed)
    steps = epochs * (n // batch)
    done = 0
    losses = []
    for ep in range(epochs):
        perm = torch.from_numpy(rng.permutation(n)).to(x.device)
        for i in range(n // batch):
            idx = perm[i * batch:(i + 1) * batch]
            cur_lr = lr * (1.0 - 0.9 * done / max(steps, 1))
            loss = net.train_step(x[idx].contiguous(), y[idx].contiguous(), cur_lr)
            done += 1
        losses.append(float(loss.item()))
        if log:
            log(f"epoch {ep}: loss {losses[-1]:.5f}")
    return losses


def load_weights(path: Path | None = None) -> np.ndarray:
    return np.load(path or WEIGHTS).astype(np.float32)
