"""The learned closure without a GPU: the CPU oracle pinned by finite differences and by two
independent restatements, and the product's header (lbm_closure.cuh / the cumulant collision
with the closure, compiled for the host) against the oracle."""
import ctypes

import numpy as np
import pytest

from oracle import mlp_oracle as M
from oracle import oracle as O
from tests.test_collision_host import Physics, host, physics_for, random_state  # noqa: F401  (fixture)


def random_params(seed=0, scale=2e-3):
    rng = np.random.default_rng(seed)
    p = np.zeros(M.NPARAM, np.float32)
    p[M.W1:M.B1] = rng.normal(0, 0.3, M.NIN * M.NH)
    p[M.B1:M.W2] = rng.normal(0, 0.1, M.NH)
    p[M.W2:M.B2] = rng.normal(0, 0.2, M.NH * M.NH)
    p[M.B2:M.W3] = rng.normal(0, 0.1, M.NH)
    p[M.W3:M.B3] = rng.normal(0, 0.3, M.NH)
    p[M.B3] = -1.0
    p[M.SCALE] = scale
    return p


def random_cells(n, seed=1):
    rng = np.random.default_rng(seed)
    P6 = rng.normal(0, 1e-3, (n, 6))
    rho = 1 + rng.uniform(-0.01, 0.01, n)
    u = rng.uniform(-0.05, 0.05, (n, 3))
    return P6, rho, u


def test_oracle_gradient_matches_finite_differences():
    p = random_params(3).astype(np.float64)
    P6, rho, u = random_cells(64)
    X = M.features(P6, rho, u)
    X = (X - X.mean(0)) / X.std(0)
    rng = np.random.default_rng(5)
    t = np.abs(rng.normal(1e-3, 5e-4, 64))
    w = rng.uniform(0.5, 2, 64)
    loss, g = M.loss_and_grad(p, X, t, w)
    assert loss > 0
    idx = list(range(0, M.NTRAIN, 37)) + [M.B1, M.W2 + 5, M.B2 + 3, M.W3 + 7, M.B3]
    for i in idx:
        h = 1e-6 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (M.loss_and_grad(pp, X, t, w)[0] - M.loss_and_grad(pm, X, t, w)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * abs(g).max() + 1e-5 * abs(fd), (i, fd, g[i])
    assert g[M.SCALE] == 0.0


def test_oracle_features_and_network_two_restatements_agree():
    """numpy (vectorised) against C (lbm_oracle.c, per cell)."""
    p = random_params(4)
    P6, rho, u = random_cells(40, seed=7)
    P6[0] = 0.0                    # a cell at rest: the guarded divisions
    u[1] = 0.0
    X = M.features(P6, rho, u)
    nu = M.forward(p, X)
    for i in range(40):
        xc = O.mlp_features(P6[i], rho[i], u[i])
        np.testing.assert_allclose(xc, X[i], rtol=1e-13, atol=1e-13)
        assert abs(O.mlp_nu_t(p, xc) - nu[i]) <= 1e-14 * abs(nu[i]) + 1e-18


def test_host_header_matches_oracle(host):  # noqa: F811
    host.host_closure_nu_t.restype = ctypes.c_double
    host.host_collide_closure.restype = ctypes.c_double
    dp = ctypes.POINTER(ctypes.c_double)
    fp = ctypes.POINTER(ctypes.c_float)
    p = random_params(6)
    P6, rho, u = random_cells(30, seed=8)
    X = M.features(P6, rho, u)
    nu = M.forward(p, X)
    for i in range(30):
        s10 = np.concatenate([P6[i], [rho[i]], u[i]])
        x = np.zeros(10)
        host.host_closure_features(s10.ctypes.data_as(dp), x.ctypes.data_as(dp))
        np.testing.assert_allclose(x, X[i], rtol=1e-13, atol=1e-13)
        v = host.host_closure_nu_t(x.ctypes.data_as(dp), p.ctypes.data_as(fp))
        assert abs(v - nu[i]) <= 1e-13 * abs(nu[i])


@pytest.mark.parametrize("force", [None, (1e-5, -2e-6, 3e-6)])
@pytest.mark.parametrize("galilean", [False, True])
def test_host_closure_collision_matches_oracle(host, force, galilean):  # noqa: F811
    p = random_params(9, scale=5e-3)
    kw = dict(relaxation_rate=1.99, compressible=True, mlp=p, galilean_correction=galilean)
    if force is not None:
        kw["force"] = force
    orc = O.make("D3Q27", "cumulant", **kw)
    phys = physics_for(orc, 3, orc.spec.rates, force, "centralmoment" if force else None, None, galilean)
    phys.sgs = 2
    phys.tau0 = 1 / orc.spec.shear_rate
    phys.sgs_mask = sum(1 << k for k, r in enumerate(orc.spec.rates) if r == orc.spec.shear_rate)
    dp = ctypes.POINTER(ctypes.c_double)
    wp = p.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    oms = []
    for seed in range(6):
        f = random_state(orc, seed, amp=2e-3)
        om_ref = ctypes.c_double(0)
        ref = np.zeros_like(f)
        O.lib().om_collide(ctypes.byref(orc._m), f.ctypes.data_as(dp), ref.ctypes.data_as(dp), ctypes.byref(om_ref))
        g = f.copy()
        om = host.host_collide_closure(0, g.ctypes.data_as(dp), ctypes.byref(phys), wp)
        np.testing.assert_allclose(g, ref, rtol=0, atol=2e-15)
        assert abs(om - om_ref.value) < 1e-13
        h = f.copy()
        host.host_collide_closure(1, h.ctypes.data_as(dp), ctypes.byref(phys), wp)
        scale = np.abs(ref + np.array([float(w) for w in orc.spec.weights])).max()
        assert np.abs(h - ref).max() / scale < 2e-7
        oms.append(om)
    assert min(oms) < 1.99 - 1e-3            # the closure is active: omega below the base rate
