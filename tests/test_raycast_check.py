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


def test_grazing_reason_needs_a_crossing_of_the_field_within_0_1_mm(of, ora):
    """A ray running along a surface through a field that alternates in sign
    from voxel to voxel (a crossing every 7.8 mm): a vertex on one of the
    crossings is explained as grazing, a vertex 2 mm beside it is not, and a
    vertex on a lone crossing of a plain wall (one crossing, not three) is not
    a grazing ray either."""
    import raycast_check
    cfg = dataclasses.replace(of.CONFIGS["c1"], resolution=128, size_mm=1000.0, trunc_mm=60.0,
                              width=160, height=120, fx=131.25, fy=131.25, cx=80.0, cy=60.0)
    n, vs, org = cfg.resolution, cfg.size_mm / cfg.resolution, -0.5 * cfg.size_mm
    c = org + (np.arange(n) + 0.5) * vs  # voxel centres
    k0 = n // 2
    z0 = c[k0]  # the ray's height: a layer of voxel centres
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")

    def words_of(f):
        q = np.clip(np.round(np.clip(f, -1, 1) * 32767), -32767, 32767).astype(np.int16)
        return (q.view(np.uint16).astype(np.uint32) | np.uint32(1 << 16)).reshape(-1).copy()

    # camera on the x axis at height z0 looking along +x (pixel (80, 60) is the
    # optical axis): camera -z -> world +x
    pose = np.eye(4)
    pose[:3, :3] = [[0, 0, -1], [0, 1, 0], [1, 0, 0]]
    pose[:3, 3] = [-450.0, 0.0, z0]
    o = pose[:3, 3]
    alt = np.where((np.arange(n) % 2) == 0, 0.05, -0.05)[:, None, None]
    words = words_of((Z - z0) / cfg.trunc_mm + alt)
    # crossings midway between voxel centres along x; take one 300 mm ahead
    i = int(np.searchsorted(c, o[0] + 300.0))
    xc = 0.5 * (c[i] + c[i + 1])
    on = np.array([xc, 0.0, z0])
    assert raycast_check.grazing_crossing(ora, cfg, words, pose, 80, 60, on)
    assert not raycast_check.grazing_crossing(ora, cfg, words, pose, 80, 60, on + [2.0, 0, 0])
    # a plain wall across the ray: one crossing
    wall = words_of((X - xc) / cfg.trunc_mm * -1.0)
    assert not raycast_check.grazing_crossing(ora, cfg, wall, pose, 80, 60, on)
