"""The FP64 CNN oracle pinned on its own definitions (CPU).

The warm-start network has no reference counterpart, so its oracle is pinned
by analytic checks: the parameter layout the CUDA code declares, BF16
rounding on known values, and central finite differences of the loss against
the oracle's chain-rule gradients, for every parameter tensor.
"""
import numpy as np

from oracle import cnn_oracle as co


def test_layout_matches_cuda_declaration():
    # of_cnn.cu: static_assert(kParams == 508534)
    assert co.param_count() == 508534
    names = [n for n, _ in co.layout()]
    assert names == ["w0", "b0", "w1", "b1", "w2", "b2", "w3", "b3", "wf1", "bf1", "wf2", "bf2"]


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 3.0e38, 1e-40], np.float64)
    r = co.bf16_round(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: ties to even -> 1
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2.0 ** -6
    assert r[3] == -2.5
    assert np.isfinite(r[4])
    bits = np.array([0x3F80, 0xC020, 0x0000], np.uint16)
    assert np.array_equal(co.bf16_bits_to_f64(bits), [1.0, -2.5, 0.0])


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(7)
    flat = np.zeros(co.param_count())
    p = co.unpack(flat)
    for name, shape in co.layout():
        fan = int(np.prod(shape[1:])) if len(shape) > 1 else 1
        p[name] = rng.normal(0.0, np.sqrt(2.0 / fan), shape) if len(shape) > 1 else \
            rng.normal(0.0, 0.05, shape)
    x = rng.normal(0.0, 0.5, (2,) + co.IN_SHAPE)
    target = rng.normal(0.0, 1.0, (2, 6))
    wk = np.array([1.0, 1.0, 1.0, 0.5, 0.5, 0.5])
    loss, _, g = co.loss_and_grads(p, x, target, wk, bf16=False)
    assert loss > 0
    h = 1e-6
    for name, shape in co.layout():
        for _ in range(3):
            idx = tuple(int(rng.integers(0, s)) for s in shape)
            base = p[name][idx]
            p[name][idx] = base + h
            lp, _, _ = co.loss_and_grads(p, x, target, wk, bf16=False)
            p[name][idx] = base - h
            lm, _, _ = co.loss_and_grads(p, x, target, wk, bf16=False)
            p[name][idx] = base
            num = (lp - lm) / (2 * h)
            ana = g[name][idx]
            # ReLU kinks are measure-zero; the scale guards near-zero entries
            assert abs(num - ana) <= 1e-5 * max(1.0, abs(ana)) + 1e-7, (name, idx, num, ana)
