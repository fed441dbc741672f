"""The raycast's algorithmic sample count (raycast_march_samples), the unit of
the raycast roofline: against a per-ray scalar march on a small camera, for
rays that hit a surface and rays that leave the box. CPU only."""
import dataclasses
import math

import numpy as np


def scalar_count(cfg, P, hit, dist):
    vs = cfg.size_mm / cfg.resolution
    lo, hi = -0.5 * cfg.size_mm + 0.5 * vs, 0.5 * cfg.size_mm - 0.5 * vs
    step = 0.75 * vs
    total, entered = 0, 0
    for y in range(cfg.height):
        for x in range(cfg.width):
            dc = [-(x - cfg.cx) / cfg.fx, -(y - cfg.cy) / cfg.fy, -1.0]
            lam = math.sqrt(sum(c * c for c in dc))
            d = [sum(P[r][k] * dc[k] for k in range(3)) / lam for r in range(3)]
            o = [P[r][3] for r in range(3)]
            tn, tf = -math.inf, math.inf
            for a in range(3):
                if abs(d[a]) < 1e-12:
                    if not lo <= o[a] <= hi:
                        tn, tf = math.inf, -math.inf
                    continue
                ta, tb = (lo - o[a]) / d[a], (hi - o[a]) / d[a]
                tn, tf = max(tn, min(ta, tb)), min(tf, max(ta, tb))
            t0, t1 = max(tn, cfg.min_depth_mm * lam), min(tf, cfg.max_depth_mm * lam)
            if not t0 < t1:
                continue
            entered += 1
            h = bool(hit[y, x])
            end = dist[y, x] if h else t1
            n, t = 0, t0
            while t <= end + 1e-9:
                n += 1
                t = t0 + n * step
            total += n + (8 if h else 0)
    return total, entered


def test_march_samples_match_a_scalar_march():
    import openfusion_b200 as of
    cfg = dataclasses.replace(of.CONFIGS["c1"], width=16, height=12, fx=13.1, fy=13.1,
                              cx=7.5, cy=5.5)
    rng = np.random.default_rng(7)
    for trial in range(4):
        a = rng.uniform(-0.6, 0.6, 3)
        K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
        th = np.linalg.norm(a)
        R = np.eye(3) + np.sin(th) / th * K + (1 - np.cos(th)) / th ** 2 * K @ K
        P = np.eye(4)
        P[:3, :3] = R
        # inside the cube for the first trials, outside (looking in) for the last
        P[:3, 3] = rng.uniform(-600, 600, 3) if trial < 3 else R @ np.array([0, 0, 1800.0])
        hit = rng.random((cfg.height, cfg.width)) < 0.6
        dist = rng.uniform(400.0, 1500.0, (cfg.height, cfg.width))
        got = of.raycast_march_samples(cfg, P, hit, dist)
        exp = scalar_count(cfg, P.tolist(), hit, dist)
        assert got[1] == exp[1] and got[1] > 0, (trial, got, exp)
        assert abs(got[0] - exp[0]) <= 2, (trial, got, exp)
