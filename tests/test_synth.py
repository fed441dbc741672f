"""Synthetic seeded scenes: deterministic, within the configured motion bounds,
with the axial noise model and dropout rate of the workload description."""
import numpy as np

from conftest import pose_error


def test_render_is_deterministic(of):
    cfg = of.CONFIGS["c2"]
    a = of.make_sequence(cfg, frames=2)
    b = of.make_sequence(cfg, frames=2)
    assert np.array_equal(a.depth, b.depth) and np.array_equal(a.poses, b.poses)


def test_smooth_motion_bounds(of):
    for name in ("c1", "c2"):
        cfg = of.CONFIGS[name]
        P = of.make_trajectory(cfg.motion, cfg.seed + 1, cfg.size_mm, 300)
        for k in range(1, 300):
            rot, trans = pose_error(P[k], P[k - 1])
            assert trans <= 10.0 and np.degrees(rot) <= 0.5
        for k in range(300):
            assert np.allclose(P[k][:3, :3] @ P[k][:3, :3].T, np.eye(3), atol=1e-12)
            assert np.all(np.abs(P[k][:3, 3]) < cfg.size_mm / 2)


def test_large_motion_bounds(of):
    cfg = of.CONFIGS["c5"]
    P = of.make_trajectory(1, cfg.seed + 1, cfg.size_mm, 200)
    rots, transs = zip(*[pose_error(P[k], P[k - 1]) for k in range(1, 200)])
    assert max(transs) <= 110.0 and np.degrees(max(rots)) <= 5.6
    assert np.median(transs) > 20.0


def test_noise_model_and_dropout(of):
    cfg = of.CONFIGS["c2"]
    scene = of.make_scene(cfg.scene_kind, cfg.seed, cfg.size_mm)
    P = of.make_trajectory(0, cfg.seed + 1, cfg.size_mm, 1)[0]
    clean, exact = of.render(cfg, scene, P, 0, noise=0.0, dropout=0.0, exact=True)
    noisy = of.render(cfg, scene, P, 0)
    hit = exact > 0
    assert hit.mean() > 0.95
    assert np.abs(clean[hit].astype(np.float64) - exact[hit]).max() <= 0.5 + 1e-3
    drop = (noisy == 0) & hit
    assert abs(drop.mean() - cfg.dropout) < 0.005
    keep = (noisy > 0) & hit
    z = exact[keep] * 1e-3
    sigma = 1000.0 * (0.0012 + 0.0019 * (z - 0.4) ** 2)
    r = (noisy[keep].astype(np.float64) - exact[keep]) / np.sqrt(sigma ** 2 + 1.0 / 12.0)
    assert abs(r.mean()) < 0.02 and abs(r.std() - 1.0) < 0.03
