"""The CPU oracle against the reference's golden data and its known-answer tests (no GPU)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from oracle import oracle_spec as S
from tests.helpers import random_velocity, tgv_velocity

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_golden_getter_mrt_incompressible():
    """lbmpy regression data (D3Q19, zero-centred incompressible storage, no force): the oracle's
    getter reproduces the stored density and velocity exactly -- this pins the walberla
    direction order and the incompressible zero-centred getter."""
    d = np.load(os.path.join(GOLDEN, "ldc_d3q19_mrt_incompressible_slab.npz"))
    o = O.make("D3Q19", "mrt", relaxation_rates=[1.7, 1.5, 1.0, 1.0], compressible=False)
    n = d["rho"].shape
    f = o.new_field(n)
    f[1:-1, 1:-1, 1:-1] = d["pdfs"]
    rho, u = o.get_macroscopic(f)
    np.testing.assert_allclose(rho, d["rho"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(u, d["vel"], rtol=0, atol=1e-16)


def test_golden_direction_order_compressible():
    """Absolute (non zero-centred) compressible storage: rho = sum f exactly; the velocity differs
    from sum(c f)/rho only by the force model's half-force shift (|F| = 1e-4 in that run)."""
    d = np.load(os.path.join(GOLDEN, "ldc_d3q19_trt_compressible_slab.npz"))
    o = O.Oracle(S.resolve("D3Q19", "trt", relaxation_rate=1.8, compressible=True, zero_centered=False))
    n = d["rho"].shape
    f = o.new_field(n)
    f[1:-1, 1:-1, 1:-1] = d["pdfs"]
    rho, u = o.get_macroscopic(f)
    np.testing.assert_allclose(rho, d["rho"], rtol=0, atol=1e-14)
    assert np.abs(u - d["vel"]).max() < 5.1e-5 * 1.01
    # another direction order breaks the velocity by far more than the force shift
    perm = list(range(19))
    perm[1], perm[3] = perm[3], perm[1]
    f[1:-1, 1:-1, 1:-1] = d["pdfs"][..., perm]
    _, u_bad = o.get_macroscopic(f)
    assert np.abs(u_bad - d["vel"]).max() > 2e-4


def _run(o, f, steps, pattern, periodic=(1, 1, 1), flags=None, ubb=(0, 0, 0)):
    prev = 1 if pattern in ("aa", "esotwist") else 0
    res, par = o.run(f, steps, pattern, prev, periodic=periodic, flags=flags, ubb_velocity=ubb)
    o.periodic_sync(res, pattern, par, periodic)
    return res, par


@pytest.mark.parametrize("stencil,method,kw", [
    ("D3Q27", "srt", dict(relaxation_rate=1.7)),
    ("D3Q19", "mrt", dict(relaxation_rates=[1.7, 1.5, 1.2, 1.1])),
    ("D3Q27", "cumulant", dict(relaxation_rate=1.8, compressible=True)),
])
def test_zero_centering_identity(stencil, method, kw):
    """tests/test_zero_centering.py:14-62: absolute storage minus zero-centred storage == w_i."""
    n = (10, 6, 6)
    u = random_velocity(n, 0.02, seed=4)
    rho = 1 + 0.01 * np.random.default_rng(3).uniform(-1, 1, n)
    zc = O.Oracle(S.resolve(stencil, method, zero_centered=True, **kw))
    ab = O.Oracle(S.resolve(stencil, method, zero_centered=False, **kw))
    fz, fa = zc.new_field(n), ab.new_field(n)
    zc.set_equilibrium(fz, rho, u)
    ab.set_equilibrium(fa, rho, u)
    rz, _ = _run(zc, fz, 20, "pull")
    ra, _ = _run(ab, fa, 20, "pull")
    w = np.array([float(x) for x in zc.spec.weights])
    diff = ra[1:-1, 1:-1, 1:-1] - rz[1:-1, 1:-1, 1:-1]
    np.testing.assert_allclose(diff, np.broadcast_to(w, diff.shape), rtol=1e-7, atol=1e-13)


@pytest.mark.parametrize("stencil,method,kw", [
    ("D3Q19", "trt", dict(relaxation_rate=1.8, compressible=True)),
    ("D3Q27", "cumulant", dict(relaxation_rate=1.9, compressible=True, galilean_correction=True)),
])
def test_streaming_patterns_agree(stencil, method, kw):
    """tests/advanced_streaming/test_fully_periodic_flow.py: every pattern gives the same flow."""
    n = (8, 6, 6)
    u = random_velocity(n, 0.02, seed=7)
    res = {}
    for pattern in ("pull", "aa", "esotwist"):
        o = O.make(stencil, method, **kw)
        f = o.new_field(n)
        prev = 1 if pattern != "pull" else 0
        o.set_equilibrium(f, np.ones(n), u, pattern, prev)
        r, par = _run(o, f, 10, pattern)
        res[pattern] = o.get_macroscopic(r, pattern, par)[1]
    for p in ("aa", "esotwist"):
        np.testing.assert_allclose(res[p], res["pull"], rtol=0, atol=1e-15)


def test_patterns_agree_with_force_and_noslip():
    """tests/advanced_streaming/test_periodic_pipe_with_force.py:173-192 (duct variant)."""
    n = (6, 8, 7)
    flags = np.zeros((8, 10, 9), np.uint8)
    flags[:, 0, :] = flags[:, -1, :] = flags[:, :, 0] = flags[:, :, -1] = 1
    out = {}
    for pattern in ("pull", "aa", "esotwist"):
        o = O.make("D3Q19", "srt", relaxation_rate=1.0, compressible=False, force=(1e-4, 0, 0))
        f = o.new_field(n)
        prev = 1 if pattern != "pull" else 0
        o.set_equilibrium(f, np.ones(n), np.zeros(n + (3,)), pattern, prev)
        r, par = _run(o, f, 30, pattern, periodic=(1, 0, 0), flags=flags)
        out[pattern] = o.get_macroscopic(r, pattern, par)[1]
    for p in ("aa", "esotwist"):
        np.testing.assert_allclose(out[p], out["pull"], rtol=0, atol=1e-16)


def test_pull_streams_each_population_to_its_neighbour():
    """tests/test_update_kernel.py:12-42: with omega = 0 the sweep is pure streaming."""
    n = (5, 4, 3)
    o = O.make("D3Q27", "srt", relaxation_rate=0.0, compressible=True)
    f = o.new_field(n)
    f[1:-1, 1:-1, 1:-1] = np.random.default_rng(0).uniform(-1e-3, 1e-3, n + (27,))
    start = f[1:-1, 1:-1, 1:-1].copy()
    r, _ = _run(o, f, 1, "pull")
    for i, c in enumerate(o.spec.dirs):
        np.testing.assert_allclose(r[1:-1, 1:-1, 1:-1, i], np.roll(start[..., i], c, axis=(0, 1, 2)), rtol=0, atol=1e-16)


def test_setter_getter_round_trip():
    n = (5, 4, 3)
    u = random_velocity(n, 0.03, seed=1)
    rho = 1 + 0.02 * np.random.default_rng(0).uniform(-1, 1, n)
    for stencil, method, kw in (("D3Q19", "trt", dict(relaxation_rate=1.7, compressible=True, force=(1e-4, 0, 0))),
                                ("D3Q27", "cumulant", dict(relaxation_rate=1.7, compressible=True)),
                                ("D3Q19", "mrt", dict(relaxation_rates=[1.7, 1.5, 1, 1]))):
        o = O.make(stencil, method, **kw)
        for pattern, prev in (("pull", 0), ("aa", 0), ("aa", 1), ("esotwist", 1)):
            f = o.new_field(n)
            o.set_equilibrium(f, rho, u, pattern, prev)
            o.periodic_sync(f, pattern, prev, (1, 1, 1))
            r2, u2 = o.get_macroscopic(f, pattern, prev)
            np.testing.assert_allclose(r2, rho, atol=1e-15)
            np.testing.assert_allclose(u2, u, atol=1e-15)


def test_tgv_viscous_decay_matches_analytic_viscosity():
    """Kinetic energy of a small-amplitude Taylor-Green vortex decays with nu = (1/omega - 1/2)/3."""
    n = (32, 32, 1)
    omega = 1.6
    o = O.make("D3Q19", "trt", relaxation_rate=omega, compressible=True)
    f = o.new_field(n)
    o.set_equilibrium(f, np.ones(n), tgv_velocity(n, 1e-3))
    e0 = o.reduce(f)[4]
    steps = 300
    r, _ = _run(o, f, steps, "pull")
    e1 = o.reduce(r)[4]
    nu = (1 / omega - 0.5) / 3
    k2 = 2 * (2 * np.pi / 32) ** 2
    nu_measured = -np.log(e1 / e0) / (2 * k2 * steps)
    # 32 cells per wavelength and an equilibrium start leave a sub-percent discretisation offset
    assert abs(nu_measured / nu - 1) < 1e-2


def test_plane_poiseuille_profile():
    """tests/poiseuille.py:17-132 restated: width-41 box with 2-cell NoSlip walls on each side,
    rho_0 = 1.2, kinematic viscosity 0.2, TRT + Guo, force 0.2/39^2; the velocity minus the half-force
    shift F/(2 rho_0) matches the analytic parabola within rtol 6e-3."""
    width, wall = 41, 2
    actual = width - 2
    rho0, eta = 1.2, 0.2
    F = 0.2 / actual ** 2
    n = (4, width, 4)
    omega = 2 / (6 * eta + 1)
    o = O.make("D3Q19", "trt", relaxation_rate=omega, compressible=True, force=(F, 0, 0), force_model="guo")
    f = o.new_field(n)
    o.set_equilibrium(f, np.full(n, rho0), np.zeros(n + (3,)))
    flags = np.zeros((6, width + 2, 6), np.uint8)
    flags[:, :wall, :] = 1          # ghost row + first interior row
    flags[:, -wall:, :] = 1
    r, _ = _run(o, f, 8000, "pull", periodic=(1, 0, 1), flags=flags)
    _, u = o.get_macroscopic(r)
    prof = u.mean(axis=(0, 2))[wall:-wall]
    prof[:, 0] -= F / 2 / rho0
    y = np.arange(len(prof))
    mid = (y[-1] - y[0]) / 2
    expected = F / (2 * rho0 * eta) * (actual ** 2 / 4 - (y - mid) ** 2)
    np.testing.assert_allclose(prof[:, 0], expected, rtol=0.006)
    np.testing.assert_allclose(prof[:, 1:], 0, atol=1e-9)


def test_cumulant_generic_recursion_matches_closed_forms():
    """The oracle's generic moment/cumulant recursion agrees with the closed-form Geier relations
    the CUDA kernel uses (checked here on random zero-mean moments, via the oracle library)."""
    o = O.make("D3Q27", "cumulant", relaxation_rate=1.0, compressible=True)
    # a collision with every rate 1 maps any state onto the product-form equilibrium
    f = o.equilibrium(1.02, [0.03, -0.01, 0.02]) + 1e-3 * np.random.default_rng(1).standard_normal(27)
    fe = O.Oracle(S.resolve("D3Q27", "cumulant", relaxation_rates=[1.0] * 27, compressible=True)).collide(f)
    rho = 1 + f.sum()
    c = np.array(o.spec.dirs, float)
    u = c.T @ f / rho
    np.testing.assert_allclose(fe, o.equilibrium(rho, u), atol=1e-15)
