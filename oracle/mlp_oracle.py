"""CPU restatement (numpy, float64) of the learned troubled-cell indicator: features, labels and
the MLP's forward / backward passes.

TEST INFRASTRUCTURE ONLY: the checker for the library's indicator kernels (dgb_indicator_features,
dgb_indicator_labels, dgb_mlp_forward / _backward / _adam, the BF16 scoring inside the limiter).
The network and its inputs are this project's own (no counterpart in the reference); the labels
come from the reference limiter as restated in oracle/dg_oracle.py.
"""
from __future__ import annotations

from math import erf, factorial, sqrt, pi

import numpy as np

from oracle import dg_oracle as O

N_IN, N_H = 225, 64
_erf = np.vectorize(erf)


def split(params):
    p = np.asarray(params, np.float64)
    o = 0
    W1 = p[o:o + N_H * N_IN].reshape(N_H, N_IN); o += N_H * N_IN
    b1 = p[o:o + N_H]; o += N_H
    W2 = p[o:o + N_H * N_H].reshape(N_H, N_H); o += N_H * N_H
    b2 = p[o:o + N_H]; o += N_H
    w3 = p[o:o + N_H]; o += N_H
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / sqrt(2.0))) + x * np.exp(-0.5 * x * x) / sqrt(2.0 * pi)


def forward(params, X):
    W1, b1, W2, b2, w3, b3 = split(params)
    A1 = X @ W1.T + b1
    H1 = gelu(A1)
    A2 = H1 @ W2.T + b2
    H2 = gelu(A2)
    z = H2 @ w3 + b3
    return 1.0 / (1.0 + np.exp(-z)), (A1, H1, A2, H2)


def loss_and_grad(params, X, y, pos_weight):
    """Weighted binary cross-entropy (mean over samples) and its gradient, flat layout."""
    W1, b1, W2, b2, w3, b3 = split(params)
    p, (A1, H1, A2, H2) = forward(params, X)
    n = X.shape[0]
    w = np.where(y > 0.5, pos_weight, 1.0)
    pc = np.clip(p, 1e-7, 1 - 1e-7)
    loss = float(np.sum(-w * (y * np.log(pc) + (1 - y) * np.log(1 - pc))) / n)
    dz = w * (p - y) / n
    dA2 = dz[:, None] * w3[None, :] * gelu_grad(A2)
    dA1 = (dA2 @ W2) * gelu_grad(A1)
    g = np.concatenate([(dA1.T @ X).ravel(), dA1.sum(0), (dA2.T @ H1).ravel(), dA2.sum(0), H2.T @ dz,
                        [dz.sum()]])
    return loss, g


def taylor_transform(order: int) -> np.ndarray:
    """T with a = T u: nodal values at the equispaced 1D nodes -> scaled Taylor coefficients
    (u(x) = sum_m a_m x^m / m!)."""
    x = np.linspace(-1.0, 1.0, order + 1)
    V = np.array([[xi ** m / factorial(m) for m in range(order + 1)] for xi in x])
    return np.linalg.inv(V)


def modes(U, n_elem, perm, order=2):
    """a[e, f, mx + (p+1) my] of every element (perm: tensor node -> reference node index)."""
    n1 = order + 1
    T = taylor_transform(order)
    V = np.asarray(U).reshape(n_elem, 5, n1 * n1)[:, :, perm].reshape(n_elem, 5, n1, n1)  # [e, f, iy, ix]
    tx = np.einsum("mi,efyi->efym", T, V)
    a = np.einsum("ny,efym->efnm", T, tx)  # [e, f, my, mx]
    return a.reshape(n_elem, 5, n1 * n1)


def scales(a):
    s = np.empty(a.shape[:2])
    s[:, 0] = np.abs(a[:, 0, 0])
    s[:, 3] = np.abs(a[:, 3, 0])
    s[:, 4] = np.abs(a[:, 4, 0])
    s[:, 1] = s[:, 2] = np.sqrt(np.abs(a[:, 0, 0] * a[:, 3, 0]))
    return s + 1e-300


FEAT_FLOOR = 5e-5  # rounding floor of the normalised inputs
FEAT_S0 = 1e-5


def compress(x):
    """The fixed input compression: soft threshold at the rounding floor, then a signed log,
    sign(x) log(1 + max(|x| - 5e-5, 0) / 1e-5) / log(1 + 1e5)."""
    return np.sign(x) * np.log1p(np.maximum(np.abs(x) - FEAT_FLOOR, 0.0) / FEAT_S0) / np.log1p(1.0 / FEAT_S0)


def features(S: O.Setup, U, perm):
    a = modes(U, S.N_E, perm)
    s = scales(a)
    nb = S.a["neighbors"].reshape(S.N_E, S.N_N)
    idx = np.arange(S.N_E)
    els = [idx] + [np.where(nb[:, k] >= 0, nb[:, k], idx) for k in range(4)]
    X = np.empty((S.N_E, 5, 5, 9))
    for n, el in enumerate(els):
        v = a[el].copy()
        v[:, :, 0] -= a[:, :, 0]
        X[:, n] = compress(v / s[:, :, None])
    return X.reshape(S.N_E, N_IN)


def labels(S: O.Setup, U, perm, tol=1e-8):
    """1 where the full limiter changes a non-constant mode by more than tol of the field scale, in
    an element whose own non-constant modes rise above the rounding floor of the inputs."""
    a = modes(U, S.N_E, perm)
    b = modes(O.limit(S, U), S.N_E, perm)
    s = scales(a)
    changed = (np.abs(b - a)[:, :, 1:] > tol * s[:, :, None]).any(axis=(1, 2))
    above = (np.abs(a)[:, :, 1:] > FEAT_FLOOR * s[:, :, None]).any(axis=(1, 2))
    return (changed & above).astype(np.float64)


def band(S: O.Setup, flags):
    """The flagged elements and their face neighbours: the set the gated limiter works on when the
    flags are taken once per time step (dg_b200/csrc/device/learned.cuh, indicator_band_kernel)."""
    f = np.asarray(flags, bool)
    nb = S.a["neighbors"].reshape(S.N_E, S.N_N)
    b = f.copy()
    for k in range(S.N_N):
        n = nb[:, k]
        ok = n >= 0
        b[ok] |= f[n[ok]]
    return b


def gated_m2(S: O.Setup, U, flags):
    """The m2 limiter on the flagged elements only (m2i arithmetic, x then y pass), given flags."""
    U = np.asarray(U, np.float64)
    fl = np.repeat(np.asarray(flags, bool), S.N_F * S.N_s)
    n1 = S.order + 1
    a = S.a
    W = U.copy()
    for off, L2M, M2L in ((0, a["Lag2MonoX"], a["MonoX2Lag"]), (2, a["Lag2MonoY"], a["MonoY2Lag"])):
        W = np.where(fl, O._m2i_pass(S, W, off, L2M, M2L, n1), W)
    return W
