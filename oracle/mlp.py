"""CPU oracle of the learned opening-angle controller -- TEST INFRASTRUCTURE ONLY.

float64 numpy restatement of the network, loss and gradients that
cosmo-nbody_b200/csrc/controller.cu computes on the GPU (the controller has
no counterpart in the reference), and of the bucket features.  Used by the
tests to check the GPU gradients; its own gradient is checked against
central finite differences in tests/test_oracle_mlp.py.

Network: 12 -> 64 -> 64 -> 1, SiLU, theta = 0.2 + 0.8 sigmoid(z).
Parameter vector (5057): W1[64][12], b1[64], W2[64][64], b2[64], w3[64], b3.
Loss: mean over samples of c (theta - y)^2, c = over_weight if theta > y.
"""
from __future__ import annotations

import numpy as np

N_IN, N_H = 12, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_H * N_IN
OFF_W2 = OFF_B1 + N_H
OFF_B2 = OFF_W2 + N_H * N_H
OFF_W3 = OFF_B2 + N_H
OFF_B3 = OFF_W3 + N_H
N_PARAMS = OFF_B3 + 1
THETA_LO, THETA_HI = 0.2, 1.0


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OFF_W1:OFF_B1].reshape(N_H, N_IN), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(N_H, N_H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x))


def silu(x):
    return x * sigmoid(x)


def dsilu(x):
    s = sigmoid(x)
    return s * (1.0 + x * (1.0 - s))


def forward(p, X, hidden_bf16=False):
    """theta and the activations; hidden_bf16: round the first layer's SiLU
    outputs to bfloat16, as the fused inference kernel feeds them to the
    tensor cores."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    a1 = X @ W1.T + b1
    h1 = silu(a1)
    if hidden_bf16:
        h1 = bf16_round(h1.astype(np.float32)).astype(np.float64)
    a2 = h1 @ W2.T + b2
    h2 = silu(a2)
    z = h2 @ w3 + b3
    theta = THETA_LO + (THETA_HI - THETA_LO) * sigmoid(z)
    return theta, (X, a1, h1, a2, h2, z)


def loss_and_grad(p, X, y, over_weight=1.0):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    theta, (X, a1, h1, a2, h2, z) = forward(p, X)
    n = X.shape[0]
    diff = theta - np.asarray(y, np.float64)
    c = np.where(diff > 0, over_weight, 1.0)
    loss = float(np.mean(c * diff * diff))
    sg = sigmoid(z)
    dz = 2.0 * c * diff / n * (THETA_HI - THETA_LO) * sg * (1.0 - sg)
    g = np.zeros(N_PARAMS)
    g[OFF_W3:OFF_B3] = dz @ h2
    g[OFF_B3] = dz.sum()
    da2 = np.outer(dz, w3) * dsilu(a2)
    g[OFF_W2:OFF_B2] = (da2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = da2.sum(axis=0)
    da1 = (da2 @ W2) * dsilu(a1)
    g[OFF_W1:OFF_B1] = (da1.T @ X).ravel()
    g[OFF_B1:OFF_W2] = da1.sum(axis=0)
    return loss, g


def loss_and_grad_tc(p, X, y, over_weight=1.0):
    """Loss and gradient of the tensor-core training path: the operands of
    the four 64-wide contractions rounded to bfloat16 (H1 and W2 in the
    forward second layer, dA2 and W2 in dH1 = dA2 W2, dA2 and H1 in dW2, dA1
    and X in dW1), everything else in float64."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    X = np.asarray(X, np.float64)

    def bf(a):
        return bf16_round(np.asarray(a, np.float32)).astype(np.float64)
    a1 = X @ W1.T + b1
    h1b, W2b = bf(silu(a1)), bf(W2)
    a2 = h1b @ W2b.T + b2
    h2 = silu(a2)
    z = h2 @ w3 + b3
    theta = THETA_LO + (THETA_HI - THETA_LO) * sigmoid(z)
    n = X.shape[0]
    diff = theta - np.asarray(y, np.float64)
    c = np.where(diff > 0, over_weight, 1.0)
    loss = float(np.mean(c * diff * diff))
    sg = sigmoid(z)
    dz = 2.0 * c * diff / n * (THETA_HI - THETA_LO) * sg * (1.0 - sg)
    g = np.zeros(N_PARAMS)
    g[OFF_W3:OFF_B3] = dz @ h2
    g[OFF_B3] = dz.sum()
    da2 = np.outer(dz, w3) * dsilu(a2)
    g[OFF_W2:OFF_B2] = (bf(da2).T @ h1b).ravel()
    g[OFF_B2:OFF_W3] = da2.sum(axis=0)
    da1 = (bf(da2) @ W2b) * dsilu(a1)
    g[OFF_W1:OFF_B1] = (bf(da1).T @ bf(X)).ravel()
    g[OFF_B1:OFF_W2] = da1.sum(axis=0)
    return loss, g


def bf16_round(a):
    """float32 -> bfloat16 -> float32, round to nearest even."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounding = ((u >> 16) & 1) + 0x7FFF
    r = ((u + rounding) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def bucket_features(rec, aabb, parents, bucket, accel, perm=None):
    """Features of one bucket (first, count, node, _) from the node table
    records rec [M,2,4] / boxes aabb [M,2,4], parents and the previous step's
    accelerations accel [N,3] (row perm[i] for sorted body i; perm None:
    identity), in float64."""
    first, count, v = int(bucket[0]), int(bucket[1]), int(bucket[2])

    def extent(u):
        lo, hi = aabb[u, 0].astype(np.float64), aabb[u, 1].astype(np.float64)
        return float(np.max(hi[:3] - lo[:3]))
    A = rec[v, 0].astype(np.float64)
    m_body = A[3] / count
    s = np.cbrt(max(m_body, 1e-30))
    lo, hi = aabb[v, 0].astype(np.float64), aabb[v, 1].astype(np.float64)
    ext = max(extent(v), 1e-3 * s)
    vol = np.prod(hi[:3] - lo[:3] + s)
    f = [np.log2(ext / s), 0.0, np.log2(count * s ** 3 / vol)]
    p = v
    pe, pm = ext, A[3]
    for _ in range(3):
        q = int(parents[p])
        if q >= 0:
            p = q
        P = rec[p, 0].astype(np.float64)
        pe = max(extent(p), ext)
        pm = max(P[3], A[3])
        f += [np.log2(pe / ext), np.log2(pm / A[3]),
              float(np.linalg.norm(P[:3] - A[:3]) / pe)]
    rows = np.arange(first, first + count)
    if perm is not None:
        rows = np.asarray(perm, np.int64)[rows]
    amean = np.linalg.norm(np.asarray(accel, np.float64)[rows], axis=1).mean()
    # mean |a| over the third ancestor's force scale G M / l^2 (G = 1)
    f[1] = 0.25 * np.log2(max(amean * pe * pe / pm, 1e-6))
    return np.array(f)
