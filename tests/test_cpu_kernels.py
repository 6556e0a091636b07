"""The closed-form CPU kernels (oracle/lbm_cpu.c: the timed CPU baseline and the fast checker of
long runs) against the generic oracle, which the golden states pin to lbmpy.

Both restate the same update; the closed form must reproduce the generic moment-space oracle to
round-off in FP64 (1e-13 of the population scale) on every path it has: the vectorised row path,
the single-cell path at periodic seams and next to walls, NoSlip and UBB links.
"""
import numpy as np
import pytest

from oracle import cpu as C
from oracle import oracle as O
from tests.helpers import random_velocity

TOL64 = 1e-13
TOL32 = 2e-6


def _state(n, seed=1):
    u = random_velocity(n, 2e-2, seed=seed)
    rho = 1 + 1e-3 * np.random.default_rng(seed + 1).uniform(-1, 1, n)
    return rho, u


def _ldc_flags(n):
    fl = np.zeros(tuple(s + 2 for s in n), np.uint8)
    fl[:, -1, :] = 2
    fl[0] = fl[-1] = 1
    fl[:, 0, :] = fl[:, :, 0] = fl[:, :, -1] = 1
    return fl


@pytest.mark.parametrize("stencil", ["D3Q19", "D3Q27"])
@pytest.mark.parametrize("compressible", [True, False])
@pytest.mark.parametrize("dtype,tol", [(np.float64, TOL64), (np.float32, TOL32)])
def test_trt_pull_periodic(stencil, compressible, dtype, tol):
    n = (13, 10, 8)                      # odd row length: vector path plus scalar remainder
    rho, u = _state(n)
    orc = O.make(stencil, "trt", relaxation_rate=1.8, compressible=compressible)
    fc = C.FastCPU("trt", orc, dtype=dtype)
    f = orc.new_field(n)
    orc.set_equilibrium(f, rho, u)
    g = fc.new_field(n)
    g[...] = f
    ref, _ = orc.run(f, 40, "pull", 0, periodic=(1, 1, 1))
    got, _ = fc.run(g, 40, periodic=(1, 1, 1))
    w = np.array([float(x) for x in orc.spec.weights])
    err = np.abs(got[1:-1, 1:-1, 1:-1] - ref[1:-1, 1:-1, 1:-1]).max() / (np.abs(ref[1:-1, 1:-1, 1:-1]) + w).max()
    assert err < tol


def test_trt_pull_lid_driven_cavity():
    n = (12, 10, 9)
    orc = O.make("D3Q19", "trt", relaxation_rate=1.7, compressible=True)
    fc = C.FastCPU("trt", orc, ubb=(0.03, 0, 0))
    f = orc.new_field(n)
    orc.set_equilibrium(f, np.ones(n), np.zeros(n + (3,)))
    g = fc.new_field(n)
    g[...] = f
    fl = _ldc_flags(n)
    ref, _ = orc.run(f, 60, "pull", 0, periodic=(0, 0, 0), flags=fl, ubb_velocity=(0.03, 0, 0))
    got, _ = fc.run(g, 60, periodic=(0, 0, 0), flags=fl)
    assert np.abs(got[1:-1, 1:-1, 1:-1] - ref[1:-1, 1:-1, 1:-1]).max() < TOL64


@pytest.mark.parametrize("walls", ["none", "y", "z", "yz", "x"])
@pytest.mark.parametrize("galilean,force", [(False, (0.0, 0.0, 0.0)), (True, (1e-5, 2e-6, -1e-6))])
def test_cumulant_aa(walls, galilean, force):
    n = (14, 9, 7)
    periodic = tuple(int(a not in walls) for a in "xyz")
    rho, u = _state(n, seed=3)
    orc = O.make("D3Q27", "cumulant", relaxation_rate=1.85, compressible=True, galilean_correction=galilean,
                 force=force)
    fc = C.FastCPU("cumulant", orc)
    fl = None
    if walls != "none":
        fl = np.zeros(tuple(s + 2 for s in n), np.uint8)
        for a in walls:
            idx = "xyz".index(a)
            sl0 = [slice(None)] * 3
            sl1 = [slice(None)] * 3
            sl0[idx], sl1[idx] = 0, -1
            fl[tuple(sl0)] = fl[tuple(sl1)] = 1
    # the oracle's state after an EVEN step lies inside the domain (no ghost-layer writes), so
    # both start from the same memory; the next step is ODD
    f = orc.new_field(n)
    orc.set_equilibrium(f, rho, u, "aa", 0)
    g = fc.new_field(n)
    g[...] = f
    for steps in (1, 2, 21):
        f1, g1 = orc.new_field(n), fc.new_field(n)      # copies in the fzyx layout
        f1[...], g1[...] = f, g
        ref, par = orc.run(f1, steps, "aa", 0, periodic=periodic, flags=fl)
        orc.periodic_sync(ref, "aa", par, periodic)
        got, par2 = fc.run(g1, steps, 1, periodic=periodic, flags=fl)
        assert par2 == 1 - par
        assert np.abs(got[1:-1, 1:-1, 1:-1] - ref[1:-1, 1:-1, 1:-1]).max() < TOL64


def test_cumulant_aa_float32_channel():
    n = (16, 8, 8)
    rho, u = _state(n, seed=5)
    orc = O.make("D3Q27", "cumulant", relaxation_rate=1.95, compressible=True, galilean_correction=True,
                 force=(1e-6, 0, 0))
    fc = C.FastCPU("cumulant", orc, dtype=np.float32)
    fl = np.zeros(tuple(s + 2 for s in n), np.uint8)
    fl[:, 0, :] = fl[:, -1, :] = fl[:, :, 0] = fl[:, :, -1] = 1
    f = orc.new_field(n)
    orc.set_equilibrium(f, rho, u, "aa", 0)
    g = fc.new_field(n)
    g[...] = f
    ref, par = orc.run(f, 30, "aa", 0, periodic=(1, 0, 0), flags=fl)
    orc.periodic_sync(ref, "aa", par, (1, 0, 0))
    got, _ = fc.run(g, 30, 1, periodic=(1, 0, 0), flags=fl)
    w = np.array([float(x) for x in orc.spec.weights])
    err = np.abs(got[1:-1, 1:-1, 1:-1] - ref[1:-1, 1:-1, 1:-1]).max() / (np.abs(ref[1:-1, 1:-1, 1:-1]) + w).max()
    assert err < TOL32


def test_rejects_what_it_does_not_restate():
    orc = O.make("D3Q19", "trt", relaxation_rate=1.8, compressible=True, force=(1e-5, 0, 0))
    with pytest.raises(AssertionError):
        C.FastCPU("trt", orc)
    orc = O.make("D3Q27", "cumulant", relaxation_rates=[1.8, 1.0, 1.3] + [1.0] * 7, compressible=True)
    with pytest.raises(AssertionError):
        C.FastCPU("cumulant", orc)
