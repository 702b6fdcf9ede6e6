"""CPU restatement of the learned-split MLP (forward and backward).

TEST INFRASTRUCTURE ONLY: the checker for fkdtree_b200/csrc/fkd_mlp.cu.  The
network has no reference counterpart; this file states its mathematics in
float64 numpy, rounding to bfloat16 exactly where the GPU kernels feed the
tensor cores, so that GPU gradients can be compared element by element:

  parameters: W1[48][64] (rows 40..47 zero), b1[64], W2[64][64], b2[64], w3[64], b3
  forward:    Z1 = bf(X) bf(W1) + b1,  H1 = gelu(Z1)
              Z2 = bf(H1) bf(W2) + b2, H2 = gelu(Z2),  y = H2 . w3 + b3
  loss:       mean((y - t)^2) / 2
  backward:   dy = (y - t) / n
              dw3 = H2^T dy, db3 = sum dy
              dZ2 = (dy w3^T) * gelu'(Z2),  db2 = sum dZ2
              dW2 = bf(H1)^T bf(dZ2),  dH1 = bf(dZ2) bf(W2)^T
              dZ1 = dH1 * gelu'(Z1),  db1 = sum dZ1
              dW1 = bf(X)^T bf(dZ1)
with gelu(x) = x/2 (1 + erf(x/sqrt 2)), bf() = round-to-nearest-even bfloat16.
"""
from __future__ import annotations

import math

import numpy as np

IN, K1, H = 40, 48, 64
OFF_W1 = 0
OFF_B1 = K1 * H
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NPARAM = OFF_B3 + 1

_erf = np.vectorize(math.erf)


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float values to bfloat16 (nearest, ties to even), as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def unpack(p: np.ndarray):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(K1, H), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H), p[OFF_B2:OFF_W3],
            p[OFF_W3:OFF_B3], p[OFF_B3])


def _pad(x):
    x = np.asarray(x, dtype=np.float64).reshape(-1, IN)
    return np.concatenate([x, np.zeros((x.shape[0], K1 - IN))], axis=1)


def forward(p, x, mirror_bf16: bool = True):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    bf = bf16 if mirror_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    X = bf(_pad(x))
    Z1 = X @ bf(W1) + b1
    H1 = gelu(Z1)
    Z2 = bf(H1) @ bf(W2) + b2
    H2 = gelu(Z2)
    y = H2 @ w3 + b3
    return y, (X, Z1, H1, Z2, H2)


def grad(p, x, t, mirror_bf16: bool = True):
    """(gradient (NPARAM,), loss) of mean((y - t)^2)/2."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    bf = bf16 if mirror_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    t = np.asarray(t, dtype=np.float64)
    n = t.shape[0]
    y, (X, Z1, H1, Z2, H2) = forward(p, x, mirror_bf16)
    loss = 0.5 * np.mean((y - t) ** 2)
    dy = (y - t) / n
    g = np.zeros(NPARAM)
    g[OFF_W3:OFF_B3] = H2.T @ dy
    g[OFF_B3] = dy.sum()
    dZ2 = np.outer(dy, w3) * gelu_grad(Z2)
    g[OFF_B2:OFF_W3] = dZ2.sum(axis=0)
    dZ2b = bf(dZ2)
    g[OFF_W2:OFF_B2] = (bf(H1).T @ dZ2b).reshape(-1)
    dH1 = dZ2b @ bf(W2).T
    dZ1 = dH1 * gelu_grad(Z1)
    g[OFF_B1:OFF_W2] = dZ1.sum(axis=0)
    g[OFF_W1:OFF_B1] = (X.T @ bf(dZ1)).reshape(-1)
    g[OFF_W1 + IN * H:OFF_B1] = 0.0
    return g, loss
