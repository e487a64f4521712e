"""CPU reference of the learned warm start's network -- TEST INFRASTRUCTURE.

The MLP d0 -> d1 -> d2 -> d3 of include/eigen_GPU_learned.h (tanh, tanh,
linear; mean squared error over all outputs) in FP64 numpy: forward,
backward (the gradient the library's eigen_GPU_mlp_gradient computes) and
one Adam step.  With bf16=True every product's operands are rounded to
BF16 (round to nearest even) where the library's tensor-core products round
them, so the GPU gradient can be compared at FP32-accumulation accuracy.
The gradient itself is checked against central finite differences by
tests/test_mlp_ref.py.  Only tests/ use this module.
"""
import numpy as np


def to_bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(flat, dims):
    d0, d1, d2, d3 = dims
    out, o = [], 0
    for shape in ((d1, d0), (d1,), (d2, d1), (d2,), (d3, d2), (d3,)):
        k = int(np.prod(shape))
        out.append(np.asarray(flat[o:o + k], dtype=np.float64).reshape(shape))
        o += k
    return out


def forward(flat, dims, x, bf16=False):
    """Returns (y, cache)."""
    W1, b1, W2, b2, W3, b3 = unpack(flat, dims)
    r = to_bf16 if bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    x = np.asarray(x, dtype=np.float64)
    h1 = np.tanh(r(x) @ r(W1).T + b1)
    h2 = np.tanh(r(h1) @ r(W2).T + b2)
    y = r(h2) @ r(W3).T + b3
    return y, (x, h1, h2, y)


def gradient(flat, dims, x, t, bf16=False):
    """Gradient of mean((y - t)^2) over all entries, flat (W1 b1 W2 b2 W3 b3),
    and the sum of squared errors."""
    W1, b1, W2, b2, W3, b3 = unpack(flat, dims)
    r = to_bf16 if bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    y, (x, h1, h2, _) = forward(flat, dims, x, bf16)
    d = y - np.asarray(t, dtype=np.float64)
    sse = float((d * d).sum())
    dy = 2.0 * d / d.size
    if bf16:
        dy = np.asarray(dy, dtype=np.float32).astype(np.float64)  # FP32 for the bias, BF16 for products
    gW3 = r(dy).T @ r(h2)
    gb3 = dy.sum(axis=0)
    dh2 = r(dy) @ r(W3)
    dz2 = dh2 * (1.0 - h2 * h2)
    gW2 = r(dz2).T @ r(h1)
    gb2 = dz2.sum(axis=0)
    dh1 = r(dz2) @ r(W2)
    dz1 = dh1 * (1.0 - h1 * h1)
    gW1 = r(dz1).T @ r(x)
    gb1 = dz1.sum(axis=0)
    return np.concatenate([g.reshape(-1) for g in (gW1, gb1, gW2, gb2, gW3, gb3)]), sse


def adam(flat, grad, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (moments updated in place); returns the new weights."""
    m[:] = b1 * m + (1 - b1) * grad
    v[:] = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return flat - lr * mh / (np.sqrt(vh) + eps)
