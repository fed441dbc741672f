"""Camera-side depth filters on the device against the oracle (bit for bit;
the undistortion within 1 mm of its FP64 bilinear value), the chain against
its steps one by one, and the tracker with filters against the tracker fed
filtered frames."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def noisy_frame(of):
    d = of.make_sequence(of.CONFIGS["c2"], frames=1).depth[0].astype(np.uint16)
    rng = np.random.default_rng(12)
    m = rng.random(d.shape)
    d[m < 0.01] = 0
    sp = m > 0.995
    d[sp] = np.clip(d[sp].astype(np.int64) + rng.integers(-400, 400, sp.sum()), 0, 65535)
    return d


def dev(x, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int16)).to(cuda)


def host(t):
    return t.cpu().numpy().view(np.uint16)


@pytest.mark.parametrize("kind", ["median5", "average", "gradient", "undistort"])
def test_filter_step_matches_oracle(of, ora, cuda, kind):
    cfg = of.CONFIGS["c2"]
    d = noisy_frame(of)
    kw = dict(k1=-0.12, k2=0.03, p1=0.002, p2=-0.001) if kind == "undistort" else {}
    g = host(of.depth_filter(cfg, dev(d, cuda), [kind], **kw))
    thr = {"average": 15.0, "gradient": 10.0}.get(kind, 0.0)
    und = (cfg.fx, cfg.fy, cfg.cx, cfg.cy, -0.12, 0.03, 0.002, -0.001)
    o, amb = ora.depth_filter(kind, d, null_value=0, thr=thr, undistort=und)
    ok = np.ones(d.shape, bool) if amb is None else amb == 0
    if kind == "undistort":
        both = ok & (g != 0) & (o != 0)
        assert np.abs(g[both].astype(np.int64) - o[both].astype(np.int64)).max() <= 1
        assert ((g == 0) != (o == 0))[ok].mean() < 1e-4
    else:
        assert np.array_equal(g[ok], o[ok])
    assert (g != d).mean() > 0.001


def test_chain_equals_steps(of, ora, cuda):
    """The GIPCam chain (median, gradient, average twice), out of place and in
    place, equals the oracle's filters applied one after another."""
    import torch
    cfg = of.CONFIGS["c2"]
    d = noisy_frame(of)
    steps = ["median5", "gradient", "average"]
    g = host(of.depth_filter(cfg, dev(d, cuda), steps, average_passes=2))
    t = dev(d, cuda)
    of.depth_filter(cfg, t, steps, out=t, average_passes=2)
    torch.cuda.synchronize()
    assert np.array_equal(host(t), g)
    o, _ = ora.depth_filter("median5", d)
    o, amb = ora.depth_filter("gradient", o, thr=10.0)
    o, _ = ora.depth_filter("average", o, thr=15.0)
    o, _ = ora.depth_filter("average", o, thr=15.0)
    # a gradient test on its threshold changes a pixel and its averaged
    # neighbourhood (3x3 after two passes of the 3x3 average)
    assert (g != o).sum() <= 25 * int(amb.sum())


def test_tracker_with_filters_equals_prefiltered_input(of, cuda):
    import torch
    cfg = of.CONFIGS["c1"]
    seq = of.make_sequence(cfg, frames=6)
    p = of.depth_filter_params(["median5", "average"])
    a = of.Tracker(cfg, seq.poses[0], depth_filter=p)
    b = of.Tracker(cfg, seq.poses[0])
    for k in range(6):
        d = torch.from_numpy(seq.depth[k].astype(np.int16)).to(cuda)
        a.process(d)
        b.process(of.depth_filter(cfg, d, ["median5", "average"]))
    assert np.array_equal(a.pose_history(6), b.pose_history(6))
    a.close()
    b.close()
