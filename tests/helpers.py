"""Shared set-up for parity tests: identical initial fields on the oracle and on the GPU."""
import numpy as np

from oracle import oracle as O


def tgv_velocity(n, u0=0.05, noise=0.0, seed=0):
    """Taylor-Green vortex in x/y (cell-index coordinates), optional Gaussian noise."""
    nx, ny, nz = n
    x = np.arange(nx)[:, None, None]
    y = np.arange(ny)[None, :, None]
    kx, ky = 2 * np.pi / nx, 2 * np.pi / ny
    u = np.zeros((nx, ny, nz, 3))
    u[..., 0] = u0 * np.sin(kx * x) * np.cos(ky * y)
    u[..., 1] = -u0 * np.cos(kx * x) * np.sin(ky * y)
    if noise:
        u += noise * np.random.default_rng(seed).standard_normal(u.shape)
    return u


def random_velocity(n, amp=1e-2, seed=0):
    return amp * np.random.default_rng(seed).uniform(-1, 1, tuple(n) + (3,))


def rel_linf(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
