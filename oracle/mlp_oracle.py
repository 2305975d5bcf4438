"""CPU oracle of the scheduler network (TEST INFRASTRUCTURE ONLY).

Restates, in numpy, the forward and backward pass that scaph_b200/csrc/mlp.cu
runs on the GPU: in -> 64 -> 64 -> out with ReLU, sigmoid cross-entropy
(weighted per output), every GEMM operand rounded to bfloat16 (round to
nearest even) with float32 accumulation, exactly where the GPU rounds.  The
parameter layout is W1[in][64] b1[64] W2[64][64] b2[64] W3[64][out] b3[out].

The restatement itself is pinned by finite differences (float64, no
rounding) in tests/test_mlp.py.  There is no reference counterpart: the
reference has no learned scheduler.
"""
from __future__ import annotations

import numpy as np

H = 64


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 to the nearest bfloat16 (ties to even), as float32."""
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray, n_in: int, n_out: int):
    o = 0
    W1 = p[o:o + n_in * H].reshape(n_in, H); o += n_in * H
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + H * n_out].reshape(H, n_out); o += H * n_out
    b3 = p[o:o + n_out]
    return W1, b1, W2, b2, W3, b3


def num_params(n_in: int, n_out: int) -> int:
    return n_in * H + H + H * H + H + H * n_out + n_out


def _mm(a, b, rnd):
    if rnd:
        return bf16(a).astype(np.float32) @ bf16(b).astype(np.float32)
    return a @ b


def forward(p, X, n_in, n_out, rnd=True, dtype=np.float32):
    W1, b1, W2, b2, W3, b3 = (a.astype(dtype) for a in unpack(p, n_in, n_out))
    X = X.astype(dtype)
    H1 = np.maximum(_mm(X, W1, rnd).astype(dtype) + b1, 0)
    H2 = np.maximum(_mm(H1, W2, rnd).astype(dtype) + b2, 0)
    Y = _mm(H2, W3, rnd).astype(dtype) + b3
    return H1, H2, Y


def loss_grad(p, X, T, W, n_in, n_out, rnd=True, dtype=np.float32):
    """Loss sum(W * BCE-with-logits(Y, T)) and its gradient (flat, same layout)."""
    W1, b1, W2, b2, W3, b3 = (a.astype(dtype) for a in unpack(p, n_in, n_out))
    X, T, W = X.astype(dtype), T.astype(dtype), W.astype(dtype)
    H1, H2, Y = forward(p, X, n_in, n_out, rnd, dtype)
    s = 1 / (1 + np.exp(-Y))
    loss = float(np.sum(W * (np.maximum(Y, 0) - Y * T + np.log1p(np.exp(-np.abs(Y))))))
    dY = W * (s - T)
    gW3 = _mm(H2.T, dY, rnd)
    gb3 = dY.sum(0)
    dH2 = _mm(dY, W3.T, rnd) * (H2 > 0)
    gW2 = _mm(H1.T, dH2, rnd)
    gb2 = dH2.sum(0)
    dH1 = _mm(dH2, W2.T, rnd) * (H1 > 0)
    gW1 = _mm(X.T, dH1, rnd)
    gb1 = dH1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3]).astype(dtype)
    return loss, g
