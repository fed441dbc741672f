"""The ray-by-ray raycast checker (tests/raycast_check.py) on the CPU, with
the FP64 oracle standing in for the GPU: a march whose positions are all
moved by 0.01 mm is fully explained, and a vertex moved off the surface by
0.5 mm is reported as unexplained."""
import dataclasses

import numpy as np


def test_checker_explains_perturbed_marches_and_catches_a_planted_error(of, ora):
    import raycast_check
    cfg = dataclasses.replace(of.CONFIGS["c1"], resolution=64, width=160, height=120, fx=131.25,
                              fy=131.25, cx=80.0, cy=60.0)
    seq = of.make_sequence(cfg, frames=3)
    n = cfg.resolution
    words = np.full(n ** 3, 0x7FFF, np.uint32)  # unobserved: +1 at weight 0
    for k in range(2):
        ora.integrate(cfg, words, seq.depth[k], seq.poses[k])
    pose = seq.poses[2]
    opts, amb = ora.raycast(cfg, words, pose, ambig=True)
    assert (opts[..., 3] > 0).mean() > 0.5
    ys, xs = np.mgrid[0:cfg.height, 0:cfg.width]
    pix = np.stack([xs.ravel(), ys.ravel()], -1)
    moved = ora.raycast_pixels(cfg, words, pose, None, pix, [1e-2])[:, 0, :]
    fake = np.zeros_like(opts)
    fake[..., :4] = moved.reshape(cfg.height, cfg.width, 4)
    r = raycast_check.compare(ora, cfg, words, None, pose, fake, opts, amb)
    assert not r["unexplained"], r
    # a vertex moved 0.5 mm along its ray, off the surface
    hit = np.argwhere((opts[..., 3] > 0) & (amb == 0) & (np.abs(fake - opts)[..., :3].max(-1) < 1e-6))
    y, x = hit[len(hit) // 2]
    o, d = raycast_check._ray(cfg, pose, x, y)
    fake[y, x, :3] += 0.5 * d
    r = raycast_check.compare(ora, cfg, words, None, pose, fake, opts, amb)
    assert (int(x), int(y)) in [(u, v) for u, v, _ in r["unexplained"]], r
