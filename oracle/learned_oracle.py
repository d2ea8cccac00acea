"""CPU oracle of the learned hypothesis proposal -- TEST INFRASTRUCTURE ONLY.

Float64 numpy restatements of what rvpoint_b200/csrc/learned.cu computes:

* ``features``: the eight per-point plane features from a point's k nearest
  neighbours (self included) -- |normal| (3), curvature l0/(l0+l1+l2),
  planarity (l1-l0)/l2, log(r + 1e-6) with r the k-th neighbour distance,
  |n . (centroid - p)| / r and |centroid - p| / r, with the eigen-system of
  the neighbourhood covariance (divided by the count, about the centroid);
* ``forward`` / ``loss_and_grad``: the MLP 8 -> 64 -> 64 -> 1 (ReLU) with
  weights rounded to BF16 (round to nearest even) and inputs normalised by a
  per-feature mean and standard deviation, and the mean binary cross-entropy
  with logits with its exact gradient w.r.t. the FP32 master parameters (the
  rounding is treated as the identity, as the GPU training does);
* ``brute_knn``: k nearest neighbours in (d2, index) order with the
  reference's d2 arithmetic ((dx*dx + dy*dy) + dz*dz in float32).

The reference has no learned component; these functions pin the GPU
kernels against their own mathematical definition. Only tests/ and
bench.py's CPU leg use this module.
"""
from __future__ import annotations

import numpy as np

MI, MH = 8, 64
NP = MH * MI + MH + MH * MH + MH + MH + 1  # 4801
OW1, OB1 = 0, MH * MI
OW2 = OB1 + MH
OB2 = OW2 + MH * MH
OW3 = OB2 + MH
OB3 = OW3 + MH


def bf16_round(w: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 (round to nearest even) -> float32."""
    b = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def unpack(params: np.ndarray):
    p = np.asarray(params, dtype=np.float64)
    W1 = p[OW1:OB1].reshape(MH, MI)
    b1 = p[OB1:OW2]
    W2 = p[OW2:OB2].reshape(MH, MH)
    b2 = p[OB2:OW3]
    w3 = p[OW3:OB3]
    b3 = p[OB3]
    return W1, b1, W2, b2, w3, b3


def tf32_round(x: np.ndarray) -> np.ndarray:
    """float32 -> TF32 (10 mantissa bits, round to nearest, ties away from
    zero: cvt.rna.tf32.f32) -> float32."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x1000) & 0xFFFFE000
    return b.astype(np.uint32).view(np.float32)


def forward(params, mean, std, feat, tensor_core: bool = False):
    """Logits (float64) of feat (n x 8) with the BF16-rounded weights.

    tensor_core: the roundings of the GPU's tensor-core forward pass --
    normalised inputs computed in float32 ((feat - mean) * (1 / std)) and
    rounded to TF32, hidden layer 1 rounded to BF16 after its bias and ReLU;
    every sum in float64."""
    W1, b1, W2, b2, w3, b3 = unpack(bf16_round(params))
    if tensor_core:
        inv = (np.float32(1.0) / np.asarray(std, np.float32)).astype(np.float32)
        x32 = (np.asarray(feat, np.float32) - np.asarray(mean, np.float32)) * inv
        xn = tf32_round(x32.astype(np.float32)).astype(np.float64)
    else:
        xn = (np.asarray(feat, np.float64) - np.asarray(mean, np.float64)) / \
            np.asarray(std, np.float64)
    z1 = xn @ W1.T + b1
    h1 = np.maximum(z1, 0.0)
    if tensor_core:
        h1 = bf16_round(h1.astype(np.float32)).astype(np.float64)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0.0)
    return h2 @ w3 + b3


def _b(a):
    """float64 -> float32 -> BF16 -> float64."""
    return bf16_round(np.asarray(a, np.float32)).astype(np.float64)


def loss_and_grad(params, mean, std, feat, labels, tensor_core: bool = False):
    """Mean BCE-with-logits and its gradient (NP floats, float64).

    tensor_core: the roundings of the GPU's tensor-core training step -- the
    forward pass's (see forward), delta2 rounded to BF16 before it meets W2,
    and the operands of the weight-gradient products (delta2, h1, delta1 and
    the normalised inputs) rounded to BF16; the bias and w3 sums use the
    unrounded values. Every sum in float64."""
    W1, b1, W2, b2, w3, b3 = unpack(bf16_round(params))
    if tensor_core:
        inv = (np.float32(1.0) / np.asarray(std, np.float32)).astype(np.float32)
        x32 = ((np.asarray(feat, np.float32) - np.asarray(mean, np.float32)) * inv).astype(
            np.float32)
        xn = tf32_round(x32).astype(np.float64)
    else:
        xn = (np.asarray(feat, np.float64) - np.asarray(mean, np.float64)) / \
            np.asarray(std, np.float64)
    y = np.asarray(labels, np.float64)
    n = xn.shape[0]
    z1 = xn @ W1.T + b1
    h1 = np.maximum(z1, 0.0)
    if tensor_core:
        h1 = _b(h1)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0.0)
    out = h2 @ w3 + b3
    loss = np.mean(np.maximum(out, 0.0) - y * out + np.log1p(np.exp(-np.abs(out))))
    g = (1.0 / (1.0 + np.exp(-out)) - y) / n
    d2 = np.outer(g, w3) * (h2 > 0)
    d1 = ((_b(d2) if tensor_core else d2) @ W2) * (h1 > 0)
    grad = np.zeros(NP)
    if tensor_core:
        grad[OW1:OB1] = (_b(d1).T @ _b(x32)).ravel()
        grad[OB1:OW2] = d1.sum(0)
        grad[OW2:OB2] = (_b(d2).T @ h1).ravel()
        grad[OB2:OW3] = d2.sum(0)
        grad[OW3:OB3] = h2.T @ g
        grad[OB3] = g.sum()
        return loss, grad
    grad[OW1:OB1] = (d1.T @ xn).ravel()
    grad[OB1:OW2] = d1.sum(0)
    grad[OW2:OB2] = (d2.T @ h1).ravel()
    grad[OB2:OW3] = d2.sum(0)
    grad[OW3:OB3] = h2.T @ g
    grad[OB3] = g.sum()
    return loss, grad


def brute_knn(x, y, z, k: int):
    """Indices (n x k) of the k nearest points in (d2, index) order."""
    P = np.stack([x, y, z], 1).astype(np.float32)
    n = P.shape[0]
    out = np.empty((n, k), np.int64)
    for i in range(n):
        d = P - P[i]
        d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        order = np.lexsort((np.arange(n), d2))
        out[i] = order[:k]
    return out


def features(x, y, z, nbrs):
    """The eight features of every point from its neighbour rows (n x k)."""
    P = np.stack([x, y, z], 1).astype(np.float64)
    n, k = nbrs.shape
    f = np.zeros((n, MI))
    for i in range(n):
        d = P[nbrs[i]] - P[i]
        c = d.mean(0)
        e = d - c
        A = e.T @ e
        lam, V = np.linalg.eigh(A)
        nrm = V[:, 0]
        l0, l1, l2 = max(lam[0], 0.0), lam[1], lam[2]
        r = np.sqrt(np.sum(d[-1] ** 2)) + 1e-6
        s = l0 + l1 + l2
        f[i, 0:3] = np.abs(nrm)
        f[i, 3] = l0 / s if s > 0 else 1.0
        f[i, 4] = (l1 - l0) / l2 if l2 > 0 else 0.0
        f[i, 5] = np.log(r)
        f[i, 6] = abs(nrm @ c) / r
        f[i, 7] = np.linalg.norm(c) / r
    return f
