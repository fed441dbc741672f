"""ctypes front end of the CPU oracle (test infrastructure only).

`Oracle("f64")` loads the FP64 checker, `Oracle("f32")` the FP32 OpenMP CPU
baseline; both are the same restatement (of_oracle.c). Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
LIBS = {"f64": "liboracle_f64.so", "f32": "libcpu_f32_omp.so"}


class Cam(C.Structure):
    _fields_ = [("w", C.c_int32), ("h", C.c_int32), ("fx", C.c_double), ("fy", C.c_double),
                ("cx", C.c_double), ("cy", C.c_double), ("dmin", C.c_double),
                ("dmax", C.c_double)]


class Vol(C.Structure):
    _fields_ = [("n", C.c_int32), ("storage", C.c_int32), ("size", C.c_double),
                ("trunc", C.c_double), ("max_w", C.c_int32), ("pad", C.c_int32)]


class IcpOpts(C.Structure):
    _fields_ = [("stop_rot", C.c_double), ("stop_trans", C.c_double), ("warm_levels", C.c_int32),
                ("pad", C.c_int32), ("judge_rms", C.c_double), ("judge_frac", C.c_double),
                ("judge_rot", C.c_double), ("judge_trans", C.c_double)]


class IcpResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("warm", C.c_int32),
                ("inliers", C.c_int32), ("examined", C.c_int32), ("decisions_near", C.c_int32),
                ("residual_sq", C.c_double)]


class RefCam(C.Structure):
    _fields_ = [("w", C.c_int32), ("h", C.c_int32), ("fx", C.c_double), ("fy", C.c_double),
                ("cx", C.c_double), ("cy", C.c_double), ("ifx", C.c_double), ("ify", C.c_double),
                ("icx", C.c_double), ("icy", C.c_double), ("dmin", C.c_double), ("dmax", C.c_double)]


class RefVol(C.Structure):
    _fields_ = [("n", C.c_int32), ("b1", C.c_int32), ("world", C.c_double), ("trunc", C.c_double),
                ("max_w", C.c_int32), ("pad", C.c_int32)]


class Params(C.Structure):
    _fields_ = [("sigma_s", C.c_double), ("sigma_r", C.c_double), ("radius", C.c_int32),
                ("levels", C.c_int32), ("iters", C.c_int32 * 4), ("dist_thresh", C.c_double),
                ("normal_thresh", C.c_double), ("min_step_vox", C.c_double),
                ("far_step_frac", C.c_double), ("refine_iters", C.c_int32), ("pad", C.c_int32)]


def build() -> None:
    """Compiles the oracle libraries (gcc; see oracle/Makefile)."""
    res = subprocess.run(["make", "-s", "-C", str(HERE)], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + res.stdout + res.stderr)


P = C.c_void_p


class Oracle:
    def __init__(self, kind: str = "f64"):
        path = BUILD / LIBS[kind]
        if not path.exists():
            build()
        self.lib = C.CDLL(str(path))
        L = self.lib
        L.ora_real_bytes.restype = C.c_int32
        L.ora_threads.restype = C.c_int32
        self.real = np.float64 if L.ora_real_bytes() == 8 else np.float32
        L.ora_cam_level.argtypes = [C.POINTER(Cam), C.c_int32, C.POINTER(Cam)]
        L.ora_bilateral.argtypes = [C.POINTER(Cam), P, C.c_double, C.c_double, C.c_int32, P]
        L.ora_pyr_down.argtypes = [P, C.c_int32, C.c_int32, P, C.c_int32, C.c_int32, C.c_double]
        L.ora_vertex_normal.argtypes = [C.POINTER(Cam), P, P]
        L.ora_preprocess.argtypes = [C.POINTER(Cam), C.POINTER(Params), P, P]
        L.ora_pyramid_elems.argtypes = [C.POINTER(Cam), C.c_int32]
        L.ora_pyramid_elems.restype = C.c_int64
        L.ora_integrate.argtypes = [C.POINTER(Vol), P, C.POINTER(Cam), P, P, P]
        L.ora_integrate.restype = C.c_int64
        L.ora_raycast.argtypes = [C.POINTER(Vol), P, P, C.POINTER(Cam), C.POINTER(Params), P, P, P]
        L.ora_tsdf_at.argtypes = [C.POINTER(Vol), P, C.c_int64, P, P]
        L.ora_raycast_pixels.argtypes = [C.POINTER(Vol), P, P, C.POINTER(Cam), C.POINTER(Params), P,
                                         C.c_int32, P, C.c_int32, P, P]
        L.ora_model_down.argtypes = [P, C.c_int32, P, C.c_int32, C.c_int32]
        L.ora_icp_system.argtypes = [C.POINTER(Cam), P, C.c_int32, C.c_int32, P, P, C.c_double,
                                     C.c_double, P, P]
        L.ora_icp_step.argtypes = [P, P, P]
        L.ora_icp_step.restype = C.c_int32
        L.ora_icp_track.argtypes = [C.POINTER(Cam), C.POINTER(Params), P, P, P, P]
        L.ora_icp_track.restype = C.c_int32
        L.ora_icp_track_ex.argtypes = [C.POINTER(Cam), C.POINTER(Params), C.POINTER(IcpOpts), P,
                                       P, P, P, C.POINTER(IcpResult)]
        L.ora_icp_track_ex.restype = C.c_int32
        L.ora_ref_convert.argtypes = [C.POINTER(RefCam), P, P, P, P]
        L.ora_ref_integrate_voxels.argtypes = [C.POINTER(RefVol), C.POINTER(RefCam), P, P, P, P,
                                               C.c_int64, P, P, P, P, P]
        L.ora_ref_integrate_full.argtypes = [C.POINTER(RefVol), C.POINTER(RefCam), P, P, P, P, P]
        L.ora_ref_raycast.argtypes = [C.POINTER(RefVol), P, C.POINTER(RefCam), P, P, P, P, P]
        L.ora_ref_icp_system.argtypes = [C.POINTER(RefCam), P, P, P, P, P, P, P, P, P, P]
        L.ora_ref_compose.argtypes = [P, P, P]
        L.ora_tracker_create.argtypes = [C.POINTER(Cam), C.POINTER(Vol), C.POINTER(Params), P]
        L.ora_tracker_create.restype = C.c_void_p
        L.ora_tracker_destroy.argtypes = [P]
        L.ora_tracker_process.argtypes = [P, P]
        L.ora_tracker_process.restype = C.c_int32
        L.ora_tracker_pose.argtypes = [P, P]
        L.ora_tracker_volume.argtypes = [P]
        L.ora_tracker_volume.restype = C.c_void_p
        L.ora_depth_median5.argtypes = [C.c_int32, C.c_int32, C.c_int32, P, P]
        L.ora_depth_average.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_double, P, P]
        L.ora_depth_gradient.argtypes = [C.c_int32, C.c_int32, C.c_double, P, P, P]
        L.ora_depth_undistort.argtypes = [C.c_int32, C.c_int32] + [C.c_double] * 8 + [
            C.c_int32, P, P, P]
        L.ora_mesh.argtypes = [C.POINTER(Vol), P, P, P, C.c_int64]
        L.ora_mesh.restype = C.c_int64

    # ----------------------------------------------------------- parameters
    @staticmethod
    def cam(cfg, level: int = 0) -> Cam:
        c = Cam(cfg.width, cfg.height, cfg.fx, cfg.fy, cfg.cx, cfg.cy, cfg.min_depth_mm,
                cfg.max_depth_mm)
        if level:
            out = Cam()
            Oracle._any().lib.ora_cam_level(C.byref(c), level, C.byref(out))
            return out
        return c

    _inst = None

    @staticmethod
    def _any() -> "Oracle":
        if Oracle._inst is None:
            Oracle._inst = Oracle("f64")
        return Oracle._inst

    @staticmethod
    def vol(cfg) -> Vol:
        return Vol(cfg.resolution, 0 if cfg.storage == "i16" else 1, cfg.size_mm, cfg.trunc_mm,
                   cfg.max_weight, 0)

    @staticmethod
    def params(cfg) -> Params:
        it = (C.c_int32 * 4)(*(list(cfg.iters) + [0] * (4 - len(cfg.iters))))
        return Params(cfg.sigma_space_px, cfg.sigma_range_mm, cfg.radius_px, cfg.levels, it,
                      cfg.dist_thresh_mm, cfg.normal_thresh, cfg.min_step_vox, cfg.far_step_frac,
                      cfg.refine_iters, 0)

    # --------------------------------------------------------------- stages
    def level_dims(self, cfg):
        out = []
        for l in range(cfg.levels):
            c = self.cam(cfg, l)
            out.append((c.w, c.h))
        return out

    def preprocess(self, cfg, depth: np.ndarray):
        """-> list per level of (depth[h,w], pts[h,w,8])"""
        d = np.ascontiguousarray(depth, np.uint16)
        n = self.lib.ora_pyramid_elems(C.byref(self.cam(cfg)), cfg.levels)
        buf = np.zeros(n, self.real)
        self.lib.ora_preprocess(C.byref(self.cam(cfg)), C.byref(self.params(cfg)), d.ctypes.data,
                                buf.ctypes.data)
        return self.split_pyramid(cfg, buf), buf

    def split_pyramid(self, cfg, buf):
        out, off = [], 0
        for (w, h) in self.level_dims(cfg):
            dep = buf[off: off + w * h].reshape(h, w)
            off += w * h
            pts = buf[off: off + w * h * 8].reshape(h, w, 8)
            off += w * h * 8
            out.append((dep, pts))
        return out

    def pack_pyramid(self, cfg, levels_pts, levels_depth=None) -> np.ndarray:
        parts = []
        for l, (w, h) in enumerate(self.level_dims(cfg)):
            dep = np.zeros(w * h, self.real) if levels_depth is None else \
                np.asarray(levels_depth[l], self.real).reshape(-1)
            parts += [dep, np.asarray(levels_pts[l], self.real).reshape(-1)]
        return np.ascontiguousarray(np.concatenate(parts))

    def vertex_normal(self, cfg, level: int, depth: np.ndarray) -> np.ndarray:
        d = np.ascontiguousarray(depth, self.real)
        pts = np.zeros(d.shape + (8,), self.real)
        self.lib.ora_vertex_normal(C.byref(self.cam(cfg, level)), d.ctypes.data, pts.ctypes.data)
        return pts

    def pyr_down(self, cfg, src: np.ndarray) -> np.ndarray:
        s_ = np.ascontiguousarray(src, self.real)
        h, w = (s_.shape[0] + 1) // 2, (s_.shape[1] + 1) // 2
        dst = np.zeros((h, w), self.real)
        self.lib.ora_pyr_down(s_.ctypes.data, s_.shape[1], s_.shape[0], dst.ctypes.data, w, h,
                              3.0 * cfg.sigma_range_mm)
        return dst

    def integrate(self, cfg, words: np.ndarray, depth: np.ndarray, pose: np.ndarray,
                  ambig: bool = False):
        """In-place update of linear-layout uint32 `words`; returns (updated, ambig mask)."""
        assert words.dtype == np.uint32 and words.flags.c_contiguous
        d = np.ascontiguousarray(depth, np.uint16)
        P_ = np.ascontiguousarray(pose, np.float64)
        am = np.zeros(words.shape, np.uint8) if ambig else None
        n = self.lib.ora_integrate(C.byref(self.vol(cfg)), words.ctypes.data,
                                   C.byref(self.cam(cfg)), d.ctypes.data, P_.ctypes.data,
                                   None if am is None else am.ctypes.data)
        return n, am

    def raycast(self, cfg, words: np.ndarray, pose: np.ndarray, ambig: bool = False,
                flags: np.ndarray | None = None):
        P_ = np.ascontiguousarray(pose, np.float64)
        pts = np.zeros((cfg.height, cfg.width, 8), self.real)
        am = np.zeros((cfg.height, cfg.width), np.uint8) if ambig else None
        fl = None if flags is None else np.ascontiguousarray(flags, np.uint8)
        self.lib.ora_raycast(C.byref(self.vol(cfg)), words.ctypes.data,
                             None if fl is None else fl.ctypes.data, C.byref(self.cam(cfg)),
                             C.byref(self.params(cfg)), P_.ctypes.data, pts.ctypes.data,
                             None if am is None else am.ctypes.data)
        return pts, am

    def raycast_pixels(self, cfg, words: np.ndarray, pose: np.ndarray, flags, pixels,
                       perts) -> np.ndarray:
        """The march of the given (x, y) pixels with every position update
        moved by each perturbation (mm); returns [len(pixels), len(perts), 4]
        vertex + hit flag."""
        P_ = np.ascontiguousarray(pose, np.float64)
        xy = np.ascontiguousarray(np.asarray(pixels, np.int32).reshape(-1, 2))
        pe = np.ascontiguousarray(perts, np.float64)
        out = np.zeros((len(xy), len(pe), 4), self.real)
        fl = None if flags is None else np.ascontiguousarray(flags, np.uint8)
        if len(xy):
            self.lib.ora_raycast_pixels(C.byref(self.vol(cfg)), words.ctypes.data,
                                        None if fl is None else fl.ctypes.data,
                                        C.byref(self.cam(cfg)), C.byref(self.params(cfg)),
                                        P_.ctypes.data, len(xy), xy.ctypes.data, len(pe),
                                        pe.ctypes.data, out.ctypes.data)
        return out

    def tsdf_at(self, cfg, words: np.ndarray, xyz: np.ndarray) -> np.ndarray:
        """The trilinear tsdf / trunc at world points [..., 3] (mm)."""
        pts = np.ascontiguousarray(np.asarray(xyz, np.float64).reshape(-1, 3))
        out = np.zeros(len(pts), self.real)
        if len(pts):
            self.lib.ora_tsdf_at(C.byref(self.vol(cfg)), words.ctypes.data, len(pts),
                                 pts.ctypes.data, out.ctypes.data)
        return out.reshape(np.asarray(xyz).shape[:-1])

    @staticmethod
    def shade_rgba(cfg, pose: np.ndarray, normals: np.ndarray) -> np.ndarray:
        """The raycast's shaded view (showNormal false) in FP64, from world
        normals [H, W, 3] (zero where the ray missed): the ray of pixel (x, y)
        through the pixel at z = -1, rotated by the pose and normalised
        (Raycaster.cu:112-125); g = 0.6 (-d . n) + 0.2, black where |d . n| is
        below epsilon (Raycaster.cu:219-227); packed by rgbaFloatToInt
        (Raycaster.cu:26-33): each channel saturated to [0, 1], times 255,
        truncated; alpha 0. Returns uint32 [H, W]."""
        P = np.asarray(pose, np.float64)
        ys, xs = np.mgrid[0:cfg.height, 0:cfg.width].astype(np.float64)
        dc = np.stack([-(xs - cfg.cx) / cfg.fx, -(ys - cfg.cy) / cfg.fy,
                       -np.ones_like(xs)], -1)
        dw = dc @ P[:3, :3].T
        d = dw / np.linalg.norm(dw, axis=-1, keepdims=True)
        dot = -(d * np.asarray(normals, np.float64)).sum(-1)
        g = np.where(np.abs(dot) < 1e-6, 0.0, 0.6 * dot + 0.2)
        q = np.floor(np.clip(g, 0.0, 1.0) * 255.0).astype(np.uint32)
        return (q << 16) | (q << 8) | q

    def model_pyramid(self, cfg, pts0: np.ndarray):
        lv = [np.ascontiguousarray(pts0, self.real)]
        for (w, h) in self.level_dims(cfg)[1:]:
            src = lv[-1]
            dst = np.zeros((h, w, 8), self.real)
            self.lib.ora_model_down(src.ctypes.data, src.shape[1], dst.ctypes.data, w, h)
            lv.append(dst)
        return lv

    def icp_system(self, cfg, level: int, frame_pts, model_pts, pose):
        f = np.ascontiguousarray(frame_pts, self.real)
        m = np.ascontiguousarray(model_pts, self.real)
        P_ = np.ascontiguousarray(pose, np.float64)
        out = np.zeros(29)
        amb = np.zeros(29)
        self.lib.ora_icp_system(C.byref(self.cam(cfg, level)), f.ctypes.data, m.shape[1],
                                m.shape[0], m.ctypes.data, P_.ctypes.data, cfg.dist_thresh_mm,
                                cfg.normal_thresh, out.ctypes.data, amb.ctypes.data)
        return out, amb

    def icp_step(self, sys: np.ndarray, pose: np.ndarray):
        s = np.ascontiguousarray(sys, np.float64)
        P_ = np.array(pose, np.float64, copy=True)
        mp = C.c_double()
        st = self.lib.ora_icp_step(s.ctypes.data, P_.ctypes.data, C.byref(mp))
        return st, P_, mp.value

    def depth_filter(self, kind: str, depth: np.ndarray, null_value: int = 0, thr: float = 0.0,
                     undistort=None):
        """Camera-side filter of uint16 depth [H, W]: "median5", "average"
        (thr mm), "gradient" (thr mm) or "undistort" (undistort = (fx, fy, cx,
        cy, k1, k2, p1, p2)). Returns (out, ambiguity mask or None)."""
        d = np.ascontiguousarray(depth, np.uint16)
        h, w = d.shape
        out = np.zeros_like(d)
        amb = np.zeros(d.shape, np.uint8)
        if kind == "median5":
            self.lib.ora_depth_median5(w, h, null_value, d.ctypes.data, out.ctypes.data)
            return out, None
        if kind == "average":
            self.lib.ora_depth_average(w, h, null_value, thr, d.ctypes.data, out.ctypes.data)
            return out, None
        if kind == "gradient":
            self.lib.ora_depth_gradient(w, h, thr, d.ctypes.data, out.ctypes.data, amb.ctypes.data)
            return out, amb
        self.lib.ora_depth_undistort(w, h, *[float(x) for x in undistort], null_value,
                                     d.ctypes.data, out.ctypes.data, amb.ctypes.data)
        return out, amb

    def mesh(self, cfg, words: np.ndarray):
        """(triangles [T, 3, 3] mm, ids [T]) of linear-layout uint32 `words`, id order."""
        w = np.ascontiguousarray(words, np.uint32)
        n = self.lib.ora_mesh(C.byref(self.vol(cfg)), w.ctypes.data, None, None, 0)
        tris = np.zeros((max(n, 1), 9), self.real)
        ids = np.zeros(max(n, 1), np.uint64)
        m = self.lib.ora_mesh(C.byref(self.vol(cfg)), w.ctypes.data, tris.ctypes.data,
                              ids.ctypes.data, n)
        assert m == n
        return tris[:n].reshape(n, 3, 3), ids[:n]

    def icp_track(self, cfg, frame_buf: np.ndarray, model_buf: np.ndarray, pose: np.ndarray):
        P_ = np.array(pose, np.float64, copy=True)
        its = C.c_int32()
        st = self.lib.ora_icp_track(C.byref(self.cam(cfg)), C.byref(self.params(cfg)),
                                    frame_buf.ctypes.data, model_buf.ctypes.data, P_.ctypes.data,
                                    C.byref(its))
        return st, P_, its.value

    def icp_track_ex(self, cfg, frame_buf: np.ndarray, model_buf: np.ndarray, pose: np.ndarray,
                     warm: np.ndarray | None = None):
        """ora_icp_track_ex with cfg's early exit (stop_rot_rad, stop_trans_mm),
        warm_levels and judge thresholds; returns (pose, IcpResult)."""
        P_ = np.array(pose, np.float64, copy=True)
        W = None if warm is None else np.ascontiguousarray(warm, np.float64)
        o = IcpOpts(cfg.stop_rot_rad, cfg.stop_trans_mm, cfg.warm_levels, 0, cfg.judge_max_rms_mm,
                    cfg.judge_min_inlier_frac, cfg.judge_max_rot_rad, cfg.judge_max_trans_mm)
        r = IcpResult()
        self.lib.ora_icp_track_ex(C.byref(self.cam(cfg)), C.byref(self.params(cfg)), C.byref(o),
                                  frame_buf.ctypes.data, model_buf.ctypes.data, P_.ctypes.data,
                                  None if W is None else W.ctypes.data, C.byref(r))
        return P_, r

    def threads(self) -> int:
        return self.lib.ora_threads()


class RefSemantics:
    """The reference-semantics functions of the oracle (FP64), for comparison
    with outputs of the reference's own kernels."""

    def __init__(self, oracle: "Oracle"):
        self.L = oracle.lib

    @staticmethod
    def cam(w, h, fx, fy, cx, cy, ifx, ify, icx, icy, dmin, dmax) -> RefCam:
        return RefCam(w, h, fx, fy, cx, cy, ifx, ify, icx, icy, dmin, dmax)

    @staticmethod
    def vol(n, world, trunc, max_w, b1=1) -> RefVol:
        return RefVol(n, b1, world, trunc, max_w, 0)

    def convert(self, cam, depth, T):
        d = np.ascontiguousarray(depth, np.uint16)
        T_ = np.ascontiguousarray(T, np.float64)
        v = np.zeros((cam.h, cam.w, 3))
        n = np.zeros((cam.h, cam.w, 3))
        self.L.ora_ref_convert(C.byref(cam), d.ctypes.data, T_.ctypes.data, v.ctypes.data,
                               n.ctypes.data)
        return v, n

    def integrate_voxels(self, vol, cam, vertex, invT, cpos, storage, prev_t, prev_w):
        vx = np.ascontiguousarray(vertex, np.float64)
        iT = np.ascontiguousarray(invT, np.float64)
        cp = np.ascontiguousarray(cpos, np.float64)
        st = np.ascontiguousarray(storage, np.int64)
        pt = np.ascontiguousarray(prev_t, np.float64)
        pw = np.ascontiguousarray(prev_w, np.int32)
        ot = np.zeros(len(st))
        ow = np.zeros(len(st), np.int32)
        am = np.zeros(len(st), np.uint8)
        self.L.ora_ref_integrate_voxels(C.byref(vol), C.byref(cam), vx.ctypes.data, iT.ctypes.data,
                                        cp.ctypes.data, st.ctypes.data, len(st), pt.ctypes.data,
                                        pw.ctypes.data, ot.ctypes.data, ow.ctypes.data,
                                        am.ctypes.data)
        return ot, ow, am

    def integrate_full(self, vol, cam, vertex, invT, cpos, trunc):
        n = vol.n
        t = np.full((n + 1) * n * n, trunc, np.float32)
        w = np.zeros((n + 1) * n * n, np.uint8)
        vx = np.ascontiguousarray(vertex, np.float64)
        iT = np.ascontiguousarray(invT, np.float64)
        cp = np.ascontiguousarray(cpos, np.float64)
        self.L.ora_ref_integrate_full(C.byref(vol), C.byref(cam), vx.ctypes.data, iT.ctypes.data,
                                      cp.ctypes.data, t.ctypes.data, w.ctypes.data)
        return t, w

    def raycast(self, vol, tsdf, cam, T, cpos):
        T_ = np.ascontiguousarray(T, np.float64)
        cp = np.ascontiguousarray(cpos, np.float64)
        v = np.zeros((cam.h, cam.w, 3))
        nn = np.zeros((cam.h, cam.w, 3))
        am = np.zeros((cam.h, cam.w), np.uint8)
        self.L.ora_ref_raycast(C.byref(vol), tsdf.ctypes.data, C.byref(cam), T_.ctypes.data,
                               cp.ctypes.data, v.ctypes.data, nn.ctypes.data, am.ctypes.data)
        return v, nn, am

    def icp_system(self, cam, depth, new_v, new_n, model_v, model_n, invT):
        args = [np.ascontiguousarray(a, np.float64) for a in (new_v, new_n, model_v, model_n, invT)]
        d = np.ascontiguousarray(depth, np.uint16)
        o36, o6, a36, a6 = np.zeros(36), np.zeros(6), np.zeros(36), np.zeros(6)
        self.L.ora_ref_icp_system(C.byref(cam), d.ctypes.data, *[a.ctypes.data for a in args],
                                  o36.ctypes.data, o6.ctypes.data, a36.ctypes.data, a6.ctypes.data)
        return o36, o6, a36, a6

    def compose(self, xopt, T, full):
        x = np.ascontiguousarray(xopt, np.float64)
        T_ = np.array(T, np.float64, copy=True).reshape(16)
        F = np.array(full, np.float64, copy=True).reshape(16)
        self.L.ora_ref_compose(x.ctypes.data, T_.ctypes.data, F.ctypes.data)
        return T_.reshape(4, 4), F.reshape(4, 4)


class CpuTracker:
    """The whole frame loop on the CPU (FP64 oracle or FP32 OpenMP baseline)."""

    def __init__(self, oracle: Oracle, cfg, pose0):
        self.o = oracle
        self.cfg = cfg
        P_ = np.ascontiguousarray(pose0, np.float64)
        self.h = oracle.lib.ora_tracker_create(C.byref(Oracle.cam(cfg)), C.byref(Oracle.vol(cfg)),
                                               C.byref(Oracle.params(cfg)), P_.ctypes.data)
        if not self.h:
            raise MemoryError("ora_tracker_create failed")

    def process(self, depth: np.ndarray) -> int:
        d = np.ascontiguousarray(depth, np.uint16)
        return self.o.lib.ora_tracker_process(self.h, d.ctypes.data)

    def pose(self) -> np.ndarray:
        P_ = np.zeros(16)
        self.o.lib.ora_tracker_pose(self.h, P_.ctypes.data)
        return P_.reshape(4, 4)

    def close(self):
        if self.h:
            self.o.lib.ora_tracker_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
