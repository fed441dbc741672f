"""FP64 CPU restatement of the learned warm-start CNN (test infrastructure).

TEST INFRASTRUCTURE ONLY: the checker for openfusion_b200/csrc/of_cnn.cu,
never used by the product path. The network has no reference counterpart
(gilbs10/OpenFusion tracks with plain ICP, Source/src/ICP.cpp:84-182); this
module restates the same layers from their definitions:

  conv (cross-correlation with zero padding), ReLU, fully connected layers;
  loss  mean_b sum_k w_k (out_bk - target_bk)^2;
  backward by the chain rule (conv weight gradient = correlation of the
  input with the output gradient, input gradient = transposed convolution).

With `bf16=True` the stored activations are rounded to BF16 (round to
nearest even) exactly where the CUDA kernels store them, so the two agree up
to FP32-versus-FP64 summation; weights are passed in already rounded.
"""
from __future__ import annotations

import numpy as np

CONV = [  # ci, co, k, stride, pad
    (2, 16, 5, 2, 2),
    (16, 32, 3, 2, 1),
    (32, 64, 3, 2, 1),
    (64, 128, 3, 2, 1),
]
F1_IN, F1_OUT, F2_OUT = 128 * 4 * 5, 160, 6
IN_SHAPE = (2, 60, 80)


def layout():
    """(name, shape) of every parameter tensor, in storage order."""
    out = []
    for i, (ci, co, k, _, _) in enumerate(CONV):
        out += [(f"w{i}", (co, ci, k, k)), (f"b{i}", (co,))]
    out += [("wf1", (F1_OUT, F1_IN)), ("bf1", (F1_OUT,)), ("wf2", (F2_OUT, F1_OUT)),
            ("bf2", (F2_OUT,))]
    return out


def param_count() -> int:
    return int(sum(np.prod(s) for _, s in layout()))


def unpack(flat: np.ndarray) -> dict:
    p, off = {}, 0
    for name, shape in layout():
        n = int(np.prod(shape))
        p[name] = np.asarray(flat[off:off + n], np.float64).reshape(shape)
        off += n
    return p


def pack(tensors: dict) -> np.ndarray:
    return np.concatenate([np.asarray(tensors[n], np.float64).reshape(-1) for n, _ in layout()])


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits_to_f64(bits: np.ndarray) -> np.ndarray:
    return (np.asarray(bits, np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def network_input(prev: np.ndarray, cur: np.ndarray) -> np.ndarray:
    """Input of one pair of uint16 depth frames (H = 60 k, W = 80 k), before
    BF16 rounding: block means of the valid depths in metres (0 if empty);
    channel 0 the previous block means minus their mean over the non-empty
    blocks, channel 1 current minus previous where both are non-empty."""
    h, w = prev.shape
    k = w // 80

    def cells(d):
        b = np.asarray(d, np.float64).reshape(60, k, 80, k)
        n = (b > 0).sum(axis=(1, 3))
        s = b.sum(axis=(1, 3))
        return np.where(n > 0, s / (1000.0 * np.maximum(n, 1)), 0.0)

    p, q = cells(prev), cells(cur)
    mu = p[p > 0].mean() if (p > 0).any() else 0.0
    x0 = np.where(p > 0, p - mu, 0.0)
    x1 = np.where((p > 0) & (q > 0), q - p, 0.0)
    return np.stack([x0, x1])


def _im2col(x, k, s, p):
    b, c, h, w = x.shape
    ho, wo = (h + 2 * p - k) // s + 1, (w + 2 * p - k) // s + 1
    xp = np.zeros((b, c, h + 2 * p, w + 2 * p))
    xp[:, :, p:p + h, p:p + w] = x
    cols = np.empty((b, c, k, k, ho, wo))
    for ky in range(k):
        for kx in range(k):
            cols[:, :, ky, kx] = xp[:, :, ky:ky + s * ho:s, kx:kx + s * wo:s]
    return cols, ho, wo


def conv_fwd(x, w, b, s, p):
    co, ci, k, _ = w.shape
    cols, ho, wo = _im2col(x, k, s, p)
    y = np.einsum("bcyxhw,ocyx->bohw", cols, w, optimize=True)
    return y + b[None, :, None, None]


def conv_bwd(x, w, s, p, g):
    """Gradients of conv_fwd for the pre-activation gradient g."""
    co, ci, k, _ = w.shape
    b, _, h, wd = x.shape
    cols, ho, wo = _im2col(x, k, s, p)
    gw = np.einsum("bohw,bcyxhw->ocyx", g, cols, optimize=True)
    gb = g.sum(axis=(0, 2, 3))
    gcols = np.einsum("bohw,ocyx->bcyxhw", g, w, optimize=True)
    gxp = np.zeros((b, ci, h + 2 * p, wd + 2 * p))
    for ky in range(k):
        for kx in range(k):
            gxp[:, :, ky:ky + s * ho:s, kx:kx + s * wo:s] += gcols[:, :, ky, kx]
    return gxp[:, :, p:p + h, p:p + wd], gw, gb


def forward(p: dict, x: np.ndarray, bf16: bool = True):
    """Activations (post-ReLU, as stored) and the output, for input x [B,2,60,80]."""
    rnd = bf16_round if bf16 else (lambda a: a)
    acts = [np.asarray(x, np.float64)]
    h = acts[0]
    for i, (_, _, _, s, pad) in enumerate(CONV):
        h = rnd(np.maximum(conv_fwd(h, p[f"w{i}"], p[f"b{i}"], s, pad), 0.0))
        acts.append(h)
    flat = h.reshape(h.shape[0], -1)
    f1 = rnd(np.maximum(flat @ p["wf1"].T + p["bf1"], 0.0))
    acts.append(f1)
    out = f1 @ p["wf2"].T + p["bf2"]
    return acts, out


def loss_and_grads(p: dict, x: np.ndarray, target: np.ndarray, wk: np.ndarray, bf16: bool = True):
    acts, out = forward(p, x, bf16)
    b = out.shape[0]
    e = out - target
    loss = float(np.mean(np.sum(wk[None, :] * e * e, axis=1)))
    gout = 2.0 * wk[None, :] * e / b
    g = {}
    f1 = acts[5]
    g["wf2"] = gout.T @ f1
    g["bf2"] = gout.sum(axis=0)
    gf1 = (gout @ p["wf2"]) * (f1 > 0)
    a4 = acts[4].reshape(b, -1)
    g["wf1"] = gf1.T @ a4
    g["bf1"] = gf1.sum(axis=0)
    gh = (gf1 @ p["wf1"]).reshape(acts[4].shape)
    for i in range(3, -1, -1):
        _, _, _, s, pad = CONV[i]
        gpre = gh * (acts[i + 1] > 0)
        gin, g[f"w{i}"], g[f"b{i}"] = conv_bwd(acts[i], p[f"w{i}"], s, pad, gpre)
        gh = gin
    return loss, out, g
