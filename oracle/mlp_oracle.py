"""CPU oracle for the learned photon-energy sampler -- TEST INFRASTRUCTURE ONLY.

A float64 numpy restatement of the network that sfparticles_b200/csrc/sfp_mlp.cu
trains and runs.  The GPU kernels are checked against it:

* ``loss_and_grad``: the training kernel's forward and backward pass.  It uses
  the BF16-rounded weights and FP32-free float64 activations; the gradient is
  taken with respect to the rounded weights.
* ``forward_infer``: the inference kernel's arithmetic.  Activations are also
  rounded to BF16 between layers, as the tensor-core fragments carry them.

The network has no reference counterpart; its training data comes from the
optical-depth inverse-CDF table (``_bisect_interp``,
qed/optical_depth_tables.py:59-102), which the oracle's C restatement checks.
"""
from __future__ import annotations

import numpy as np

H = 64
NPARAM = 8577
OFF = {"W0": 0, "b0": 128, "W1": 192, "b1": 4288, "W2": 4352, "b2": 8448, "W3": 8512, "b3": 8576}


def bf16_round(x):
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(P, round_weights=True):
    P = np.asarray(P, dtype=np.float32)
    rw = bf16_round if round_weights else (lambda v: np.asarray(v, dtype=np.float64))
    W0 = rw(P[OFF["W0"]:OFF["b0"]]).reshape(H, 2)
    W1 = rw(P[OFF["W1"]:OFF["b1"]]).reshape(H, H)
    W2 = rw(P[OFF["W2"]:OFF["b2"]]).reshape(H, H)
    W3 = rw(P[OFF["W3"]:OFF["b3"]])
    b0 = P[OFF["b0"]:OFF["W1"]].astype(np.float64)
    b1 = P[OFF["b1"]:OFF["W2"]].astype(np.float64)
    b2 = P[OFF["b2"]:OFF["W3"]].astype(np.float64)
    b3 = float(P[OFF["b3"]])
    return W0, b0, W1, b1, W2, b2, W3, b3


def _silu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return z * s, s * (1.0 + z * (1.0 - s))


def loss_and_grad(P, feat, target):
    """(sum (y - t)^2, gradient [8577]) for features [n, 2] and targets [n]."""
    W0, b0, W1, b1, W2, b2, W3, b3 = unpack(P)
    x = np.asarray(feat, dtype=np.float64).reshape(-1, 2)
    t = np.asarray(target, dtype=np.float64)
    a1, d1 = _silu(x @ W0.T + b0)
    a2, d2 = _silu(a1 @ W1.T + b1)
    a3, d3 = _silu(a2 @ W2.T + b2)
    y = a3 @ W3 + b3
    e = y - t
    dy = 2.0 * e
    g = np.zeros(NPARAM)
    g[OFF["W3"]:OFF["b3"]] = a3.T @ dy
    g[OFF["b3"]] = dy.sum()
    dz3 = np.outer(dy, W3) * d3
    g[OFF["W2"]:OFF["b2"]] = (dz3.T @ a2).ravel()
    g[OFF["b2"]:OFF["W3"]] = dz3.sum(0)
    dz2 = (dz3 @ W2) * d2
    g[OFF["W1"]:OFF["b1"]] = (dz2.T @ a1).ravel()
    g[OFF["b1"]:OFF["W2"]] = dz2.sum(0)
    dz1 = (dz2 @ W1) * d1
    g[OFF["W0"]:OFF["b0"]] = (dz1.T @ x).ravel()
    g[OFF["b0"]:OFF["W1"]] = dz1.sum(0)
    return float((e * e).sum()), g


def features(log_chi, u):
    """The network's input features, as the kernels compute them (float32)."""
    f0 = (np.asarray(log_chi, dtype=np.float64) / 3.0).astype(np.float32)
    u = np.clip(np.asarray(u, dtype=np.float64), 2.0 ** -53, 1.0 - 2.0 ** -53)
    lu = np.log(u.astype(np.float32))
    lv = np.log((1.0 - u).astype(np.float32))
    f1 = ((lu - lv) * np.float32(0.125)).astype(np.float32)
    return np.stack([f0, f1], axis=1)


def forward_infer(P, log_chi, u):
    """δ as the inference kernel computes it (BF16 weights and activations)."""
    W0, b0, W1, b1, W2, b2, W3, b3 = unpack(P)
    x = features(log_chi, u).astype(np.float64)
    a1 = bf16_round(_silu(x @ W0.T + b0)[0])
    a2 = bf16_round(_silu(a1 @ W1.T + b1)[0])
    a3 = _silu(a2 @ W2.T + b2)[0]
    y = (a3 @ W3 + b3).astype(np.float32)
    d = np.exp2((y - np.float32(1.0)) * np.float32(3.0 * np.log2(10.0))).astype(np.float64)
    return np.clip(d, 1e-6, 1.0)
