"""ORACLE (test infrastructure only; never imported by the product).

CPU restatement of the learned warm start's network and its gradients
(egspice_b200/csrc/mlp.cu): in -> 128 -> 128 -> out with tanh hidden
layers, mean squared error on standardized targets. The GEMM operands are
rounded to BF16 exactly where the GPU rounds them (inputs, weights, hidden
activations, output and hidden gradients); everything else is FP64, so the
GPU's FP32 accumulation and its tanhf differ from this by rounding only.
There is no reference counterpart: ESPice has no learned start point.
"""
from __future__ import annotations

import numpy as np

H = 128


def bf16(a) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    a32 = np.ascontiguousarray(a, dtype=np.float32)
    b = a32.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(p: np.ndarray, d: int, o: int):
    """Split a parameter vector in the C API's order."""
    p = np.asarray(p, dtype=np.float64)
    k = 0
    out = []
    for shape in ((H, d), (H,), (H, H), (H,), (o, H), (o,)):
        n = int(np.prod(shape))
        out.append(p[k:k + n].reshape(shape))
        k += n
    assert k == p.size
    return out


def scaling(a: np.ndarray):
    """Per-column mean and population std as float32 (a constant column gets 1)."""
    mu = a.mean(axis=0)
    sd = np.sqrt(((a - mu) ** 2).mean(axis=0))
    sd = np.where(sd > 1e-12, sd, 1.0)
    return mu.astype(np.float32), sd.astype(np.float32)


def standardize(a, mu32, sd32):
    return ((np.asarray(a, dtype=np.float64) - mu32.astype(np.float64)) / sd32.astype(np.float64)).astype(
        np.float32).astype(np.float64)


def loss_grad(p, x, y, in_scale, out_scale, rounding: bool = True):
    """Loss and gradient (C API order) of one batch, as the GPU computes them;
    rounding=False keeps every value FP64 (the plain network, for checking
    the gradient itself by finite differences)."""
    ident = lambda a: np.asarray(a, dtype=np.float64)  # noqa: E731
    rb = bf16 if rounding else ident
    f32 = (lambda a: a.astype(np.float32).astype(np.float64)) if rounding else ident
    return _loss_grad(p, x, y, in_scale, out_scale, rounding, rb, f32)


def _loss_grad(p, x, y, in_scale, out_scale, rounding, bf16, f32):
    d, o = x.shape[1], y.shape[1]
    W1, b1, W2, b2, W3, b3 = unpack(p, d, o)
    xs = bf16(standardize(x, *in_scale) if rounding else (x - in_scale[0]) / in_scale[1])
    ts = standardize(y, *out_scale) if rounding else (y - out_scale[0]) / out_scale[1]
    W1b, W2b, W3b = bf16(W1), bf16(W2), bf16(W3)
    h1 = f32(np.tanh(xs @ W1b.T + b1))
    h1b = bf16(h1)
    h2 = f32(np.tanh(h1b @ W2b.T + b2))
    h2b = bf16(h2)
    yh = h2b @ W3b.T + b3
    n = len(x)
    e = yh - ts
    loss = float((e ** 2).sum() / (n * o))
    dy = f32(2.0 * e / (n * o))
    dyb = bf16(dy)
    dW3 = dyb.T @ h2b
    db3 = dy.sum(axis=0)
    dz2 = f32((dyb @ W3b) * (1.0 - h2 ** 2))
    dz2b = bf16(dz2)
    dW2 = dz2b.T @ h1b
    db2 = dz2.sum(axis=0)
    dz1 = f32((dz2b @ W2b) * (1.0 - h1 ** 2))
    dz1b = bf16(dz1)
    dW1 = dz1b.T @ xs
    db1 = dz1.sum(axis=0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
    return loss, g


def predict(p, x, in_scale, out_scale, o):
    d = x.shape[1]
    W1, b1, W2, b2, W3, b3 = unpack(p, d, o)
    xs = bf16(standardize(x, *in_scale))
    h1b = bf16(np.tanh(xs @ bf16(W1).T + b1).astype(np.float32))
    h2b = bf16(np.tanh(h1b @ bf16(W2).T + b2).astype(np.float32))
    ys = h2b @ bf16(W3).T + b3
    return ys * out_scale[1].astype(np.float64) + out_scale[0].astype(np.float64)
