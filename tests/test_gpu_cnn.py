"""The warm-start CNN kernels against the FP64 oracle (oracle/cnn_oracle.py),
and the device renderer against the host renderer.

Tolerances: the oracle rounds the stored activations to BF16 where the
kernels store them, so the two differ by FP32-versus-FP64 summation only,
plus an occasional activation that lands on the other side of a BF16
rounding boundary; outputs and per-tensor gradients agree to 1% of their
norm (BF16 has 8 significant bits: one step is 0.4%).
"""
import numpy as np
import pytest

from oracle import cnn_oracle as co

pytestmark = pytest.mark.gpu


def _oracle_params(net):
    master = net.master.cpu().numpy().astype(np.float64)
    bits = net.params.cpu().numpy().view(np.uint16)
    p = co.unpack(co.bf16_bits_to_f64(bits))
    pb = co.unpack(master)
    for name, _ in co.layout():
        if name.startswith("b"):
            p[name] = pb[name]  # biases are read from the FP32 master values
    return p


def _random_input(rng, b, device):
    import torch
    x = co.bf16_round(rng.normal(0.0, 0.4, (b,) + co.IN_SHAPE))
    bits = (x.astype(np.float32).view(np.uint32) >> 16).astype(np.uint16)
    return x, torch.from_numpy(bits.view(np.int16).reshape(b, -1).copy()).to(device)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_device_renderer_matches_host(of, cuda):
    from openfusion_b200 import learned
    cfg = of.CONFIGS["c2"]
    scene = of.make_scene(cfg.scene_kind, cfg.seed, cfg.size_mm)
    poses = of.make_trajectory(cfg.motion, cfg.seed + 1, cfg.size_mm, 3)
    dev = learned.render_device(cfg, scene, poses, device=cuda).cpu().numpy().view(np.uint16)
    for k in range(3):
        host = of.render(cfg, scene, poses[k], k)
        d = np.abs(dev[k].astype(np.int32) - host.astype(np.int32))
        assert d.max() <= 1 and (d > 0).mean() < 1e-3, (k, d.max(), (d > 0).mean())
        assert (host > 0).mean() > 0.9


def test_network_input_matches_oracle(of, cuda):
    import torch
    from openfusion_b200 import learned
    cfg = of.CONFIGS["c2"]
    seq = of.make_sequence(cfg, frames=3)
    d = torch.from_numpy(seq.depth.astype(np.int16)).to(cuda)
    bits = learned.WarmStartNet.inputs(d[:-1].contiguous(), d[1:].contiguous()).cpu().numpy()
    got = co.bf16_bits_to_f64(bits.view(np.uint16)).reshape(2, 2, 60, 80)
    for i in range(2):
        ref = co.network_input(seq.depth[i], seq.depth[i + 1])
        # BF16 rounding (at most one spacing, 2^-7 relative) of FP32 sums
        # that differ from the FP64 ones by ~1e-7 m
        tol = np.abs(ref) * 2.0 ** -7 + 1e-6
        assert np.all(np.abs(got[i] - ref) <= tol), np.abs(got[i] - ref).max()
        assert (np.abs(ref[1]) > 0).mean() > 0.5


def test_forward_matches_oracle(of, cuda):
    from openfusion_b200 import learned
    net = learned.WarmStartNet(cuda, seed=3)
    rng = np.random.default_rng(0)
    x, xin = _random_input(rng, 4, cuda)
    out = net.forward(xin).cpu().numpy()
    _, ref = co.forward(_oracle_params(net), x, bf16=True)
    assert _rel(out, ref) < 1e-2, (out, ref)


def test_gradients_match_oracle(of, cuda):
    import torch
    from openfusion_b200 import learned
    net = learned.WarmStartNet(cuda, seed=5)
    rng = np.random.default_rng(1)
    x, xin = _random_input(rng, 8, cuda)
    target = rng.normal(0.0, 1.0, (8, 6))
    tgt = torch.tensor(target, dtype=torch.float32, device=cuda)
    loss = float(net.gradients(xin, tgt).item())
    g = net.grad.cpu().numpy().astype(np.float64)
    wk = net.loss_w.cpu().numpy().astype(np.float64)
    ref_loss, _, ref = co.loss_and_grads(_oracle_params(net), x, target, wk, bf16=True)
    assert abs(loss - ref_loss) <= 1e-2 * ref_loss
    gp = co.unpack(g)
    for name, _ in co.layout():
        assert _rel(gp[name], ref[name]) < 1e-2, (name, _rel(gp[name], ref[name]))


def test_adam_step_matches_formula(of, cuda):
    import torch
    from openfusion_b200 import learned
    net = learned.WarmStartNet(cuda, seed=9)
    rng = np.random.default_rng(2)
    p0 = net.master.cpu().numpy().astype(np.float64)
    g = rng.normal(0.0, 1e-3, p0.size).astype(np.float32)
    net.grad.copy_(torch.from_numpy(g))
    from openfusion_b200 import _native as N
    lr = 1e-3
    assert N.lib().of_cnn_adam(net.master.data_ptr(), net.params.data_ptr(), net.grad.data_ptr(),
                               net.m.data_ptr(), net.v.data_ptr(), 1, lr,
                               torch.cuda.current_stream().cuda_stream) == 0
    p1 = net.master.cpu().numpy().astype(np.float64)
    gd = g.astype(np.float64)
    m = 0.1 * gd
    v = 0.001 * gd * gd
    ref = p0 - lr * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
    assert np.allclose(p1, ref, rtol=0, atol=1e-6)
    bits = net.params.cpu().numpy().view(np.uint16)
    assert np.array_equal(co.bf16_bits_to_f64(bits), co.bf16_round(p1.astype(np.float32)))


def test_training_is_reproducible_and_reduces_the_loss(of, cuda):
    """A short run on ICP-labelled pairs of seeded large-motion sequences
    (320x240 for speed): the loss falls, and a second run from the same
    seeds gives bit-identical weights (fixed-order reductions only)."""
    import dataclasses
    from openfusion_b200 import learned
    cfg = dataclasses.replace(of.CONFIGS["c5"], width=320, height=240, fx=262.5, fy=262.5,
                              cx=159.75, cy=119.75)
    x, y = learned.training_set(cfg, [11, 12, 13, 14], 25, cuda)
    assert x.shape == (96, 9600) and y.shape == (96, 6)
    runs = []
    for _ in range(2):
        net = learned.WarmStartNet(cuda, seed=21)
        losses = learned.train(net, x, y, epochs=40, batch=32, lr=2e-3, seed=4)
        runs.append((losses, net.weights()))
    losses, w = runs[0]
    assert losses[-1] < 0.5 * losses[0], losses
    assert np.array_equal(w, runs[1][1])


def test_fused_prediction_matches_the_staged_path(of, cuda):
    """of_cnn_predict (one cluster launch) against of_cnn_input +
    of_cnn_forward + of_cnn_warm_pose on the trained weights: outputs within
    1% of their norm (same arithmetic, other summation order), warm pose
    within the same tolerance carried through the exponential map."""
    import torch
    from openfusion_b200 import _native as N, learned
    net = learned.WarmStartNet(cuda, weights=learned.load_weights())
    cfg = of.CONFIGS["c5"]
    seq = of.make_sequence(cfg, frames=3)
    d = torch.from_numpy(seq.depth.astype(np.int16)).to(cuda)
    lib, st = N.lib(), torch.cuda.current_stream().cuda_stream
    for k in (1, 2):
        ref = net.forward(net.inputs(d[k - 1].contiguous(), d[k].contiguous()))
        prev = torch.tensor(seq.poses[k - 1].reshape(16), dtype=torch.float64, device=cuda)
        w_ref = torch.empty(16, dtype=torch.float64, device=cuda)
        assert lib.of_cnn_warm_pose(ref.data_ptr(), prev.data_ptr(), w_ref.data_ptr(), st) == 0
        out = torch.zeros(6, dtype=torch.float32, device=cuda)
        warm = torch.zeros(16, dtype=torch.float64, device=cuda)
        assert lib.of_cnn_predict(net.params.data_ptr(), net.master.data_ptr(), d[k - 1].data_ptr(),
                                  d[k].data_ptr(), cfg.width, cfg.height, prev.data_ptr(),
                                  out.data_ptr(), warm.data_ptr(), st) == 0
        torch.cuda.synchronize()
        r, o = ref.cpu().numpy()[0], out.cpu().numpy()
        assert _rel(o, r) < 1e-2, (o, r)
        W, Wr = warm.cpu().numpy().reshape(4, 4), w_ref.cpu().numpy().reshape(4, 4)
        assert np.abs(W[:3, :3] - Wr[:3, :3]).max() < 1e-3 * max(1.0, np.abs(r).max())
        assert np.abs(W[:3, 3] - Wr[:3, 3]).max() < 2.0
