"""CPU restatement of the learned-closure network and its training gradient.  TEST INFRASTRUCTURE ONLY.

Only tests/ use this module, as the checker of the GPU training and inference kernels.  FP64
numpy, written out layer by layer (no autodiff), for the 10 -> 32 -> 32 -> 1 perceptron with
SiLU hidden units and a softplus output scaled by a fixed factor:

    z1 = x W1 + b1,  h1 = silu(z1)
    z2 = h1 W2 + b2, h2 = silu(z2)
    y  = h2 W3 + b3, nu = s * softplus(y)
    loss = sum_n w_n (nu_n - t_n)^2 / sum_n w_n

The parameter block is one float vector: W1[10][32], b1[32], W2[32][32], b2[32], W3[32], b3, s.
The closure replaces the closed-form eddy viscosity of lbmpy's Smagorinsky model
(turbulence_models.py:25-84).  Parity: the gradient is pinned by central finite differences
(tests/test_closure.py); the features by the C restatement in lbm_oracle.c (om_mlp_features).
"""
from __future__ import annotations

import numpy as np

NIN, NH = 10, 32
W1, B1 = 0, NIN * NH
W2 = B1 + NH
B2 = W2 + NH * NH
W3 = B2 + NH
B3 = W3 + NH
SCALE = B3 + 1
NPARAM = SCALE + 1
NTRAIN = SCALE


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[W1:B1].reshape(NIN, NH), p[B1:W2], p[W2:B2].reshape(NH, NH), p[B2:W3], p[W3:B3], p[B3], p[SCALE])


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def forward(p, X):
    """nu_t for samples X [n, 10]."""
    w1, b1, w2, b2, w3, b3, s = unpack(p)
    z1 = X @ w1 + b1
    h1 = z1 * _sig(z1)
    z2 = h1 @ w2 + b2
    h2 = z2 * _sig(z2)
    y = h2 @ w3 + b3
    return s * np.where(y > 20, y, np.log1p(np.exp(np.minimum(y, 20))))


def loss_and_grad(p, X, t, w=None):
    """Weighted mean squared error of nu_t against targets t and its gradient with respect to the
    trained parameters (the output scale gets gradient 0)."""
    X = np.asarray(X, np.float64)
    t = np.asarray(t, np.float64)
    w = np.ones_like(t) if w is None else np.asarray(w, np.float64)
    w1, b1, w2, b2, w3, b3, s = unpack(p)
    z1 = X @ w1 + b1
    s1 = _sig(z1)
    h1 = z1 * s1
    z2 = h1 @ w2 + b2
    s2 = _sig(z2)
    h2 = z2 * s2
    y = h2 @ w3 + b3
    sp = np.where(y > 20, y, np.log1p(np.exp(np.minimum(y, 20))))
    nu = s * sp
    W = w.sum()
    r = nu - t
    loss = float((w * r * r).sum() / W)
    dnu = 2.0 * w * r / W
    dy = dnu * s * np.where(y > 20, 1.0, _sig(y))
    g = np.zeros(NPARAM)
    g[W3:B3] = h2.T @ dy
    g[B3] = dy.sum()
    dh2 = np.outer(dy, w3)
    dz2 = dh2 * s2 * (1.0 + z2 * (1.0 - s2))
    g[W2:B2] = (h1.T @ dz2).reshape(-1)
    g[B2:W3] = dz2.sum(0)
    dh1 = dz2 @ w2.T
    dz1 = dh1 * s1 * (1.0 + z1 * (1.0 - s1))
    g[W1:B1] = (X.T @ dz1).reshape(-1)
    g[B1:W2] = dz1.sum(0)
    return loss, g


def features(P6, rho, u):
    """Vectorised closure features; P6 [n, 6] = (Pxx, Pyy, Pzz, Pxy, Pxz, Pyz), rho [n], u [n, 3]."""
    P6 = np.asarray(P6, np.float64)
    pxx, pyy, pzz, pxy, pxz, pyz = P6.T
    rho = np.asarray(rho, np.float64)
    u = np.asarray(u, np.float64)
    off2 = pxy ** 2 + pxz ** 2 + pyz ** 2
    s2 = pxx ** 2 + pyy ** 2 + pzz ** 2 + 2 * off2
    pim = np.sqrt(2 * s2) / rho
    tr = pxx + pyy + pzz
    dxx, dyy, dzz = pxx - tr / 3, pyy - tr / 3, pzz - tr / 3
    D = np.stack([np.stack([dxx, pxy, pxz], -1), np.stack([pxy, dyy, pyz], -1), np.stack([pxz, pyz, dzz], -1)], -2)
    d2 = (D ** 2).sum((-1, -2))
    dn = np.sqrt(d2)
    tr3 = np.einsum("nab,nbc,nca->n", D, D, D)
    u2 = (u ** 2).sum(-1)
    uau = np.einsum("na,nab,nb->n", u, D, u)
    mx = np.abs(np.stack([dxx, dyy, dzz], -1)).max(-1)
    return np.stack([np.log(pim + 1e-9), 100 * pim, tr / (np.sqrt(s2) + 1e-12),
                     np.sqrt(6.0) * tr3 / (d2 * dn + 1e-30), 30 * np.sqrt(u2), 1000 * (rho - 1),
                     uau / ((u2 + 1e-12) * dn + 1e-30), off2 / (s2 + 1e-30), mx / (dn + 1e-30), 1000 * u2], -1)
