"""The sweep's collision operators (lbm_collide.cuh, compiled for the host with g++) against the
oracle, cell by cell, on random states -- the kernel arithmetic checked without a GPU."""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest
import sympy as sp

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
MK_POP, MK_MRT, MK_CUM, MK_CUM1 = 0, 1, 2, 3
FM = {None: 0, "guo": 1, "centralmoment": 2, "simple": 3, "luo": 4}


class Physics(ctypes.Structure):
    _fields_ = [("rates", ctypes.c_double * 27), ("force", ctypes.c_double * 3), ("force_model", ctypes.c_int),
                ("compressible", ctypes.c_int), ("continuous_eq", ctypes.c_int), ("sgs", ctypes.c_int),
                ("sgs_c18", ctypes.c_double), ("tau0", ctypes.c_double), ("sgs_mask", ctypes.c_uint32),
                ("galilean", ctypes.c_int), ("ubb", (ctypes.c_double * 3) * 4), ("fixed_density", ctypes.c_double),
                ("fixed_density1", ctypes.c_double), ("ubb_density", ctypes.c_double * 4),
                ("ubb_link_mask", ctypes.c_uint32), ("ubb_adapt_mask", ctypes.c_uint32),
                ("foc_limiter", ctypes.c_double), ("foc_a", ctypes.c_double), ("foc_b", ctypes.c_double)]


@pytest.fixture(scope="module")
def host():
    out = os.path.join(tempfile.mkdtemp(), "collide_host.so")
    subprocess.run(["/usr/bin/g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-I/usr/local/cuda/include", "-o", out,
                    os.path.join(HERE, "host", "collide_host.cpp")], check=True)
    lib = ctypes.CDLL(out)
    lib.host_collide.restype = ctypes.c_double
    lib.host_collide.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(Physics)]
    assert lib.host_sizeof_physics() == ctypes.sizeof(Physics)
    return lib


def physics_for(orc, kind, rates, force=None, fm=None, sgs=None, galilean=False):
    p = Physics()
    for k, r in enumerate(rates):
        p.rates[k] = r
    if force is not None:
        for k in range(3):
            p.force[k] = force[k]
        p.force_model = FM[fm]
    p.compressible = int(orc.spec.compressible)
    p.continuous_eq = 1
    p.galilean = int(galilean)
    if sgs is not None:
        p.sgs = 1
        p.sgs_c18 = 18 * sgs * sgs
        p.tau0 = 1 / orc.spec.shear_rate
        native = rates
        mask = 0
        for k, r in enumerate(native):
            if r == orc.spec.shear_rate:
                mask |= 1 << k
        p.sgs_mask = mask
    return p


def random_state(orc, seed, amp=1e-3):
    rng = np.random.default_rng(seed)
    u = rng.uniform(-0.05, 0.05, 3)
    rho = 1 + rng.uniform(-0.02, 0.02)
    return orc.equilibrium(rho, u) + amp * rng.standard_normal(orc.Q)


CASES = [
    ("D3Q19", "trt", MK_POP, dict(relaxation_rate=1.8, compressible=True), None, None, None),
    ("D3Q19", "srt", MK_POP, dict(relaxation_rate=1.3, compressible=False), (1e-4, 2e-5, -3e-5), "guo", None),
    ("D3Q19", "trt", MK_POP, dict(relaxation_rate=1.7, compressible=True), (1e-4, 0, 0), "luo", 0.12),
    ("D3Q19", "mrt", MK_MRT, dict(relaxation_rates=[1.7, 1.5, 1.2, 1.1], compressible=False), (1e-4, 0, 2e-5),
     "guo", None),
    ("D3Q27", "trt", MK_POP, dict(relaxation_rate=1.9, compressible=True), (1e-4, 0, 0), "simple", None),
    ("D3Q27", "mrt", MK_MRT, dict(relaxation_rates=[1.8, 1.4, 1.1, 1.2, 1.3, 1.05], compressible=True), None,
     None, 0.1),
    ("D3Q27", "cumulant", MK_CUM, dict(relaxation_rates=[1.9, 1.3, 1.2, 1.1, 1.05, 1.15, 1.25, 1.35, 1.45, 1.5]
                                       + [1.0] * 0, compressible=True), (1e-4, -2e-5, 3e-5), "centralmoment",
     None),
    ("D3Q27", "cumulant", MK_CUM, dict(relaxation_rate=1.95, compressible=True), (1e-5, 0, 0), "centralmoment",
     0.1),
    ("D3Q27", "cumulant", MK_CUM1, dict(relaxation_rate=1.95, compressible=True), (1e-5, 2e-6, 0),
     "centralmoment", None),
    ("D3Q27", "cumulant", MK_CUM1, dict(relaxation_rate=1.99, compressible=True), None, None, 0.1),
]


@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}-{c[1]}-mk{c[2]}-{i}" for i, c in enumerate(CASES)])
@pytest.mark.parametrize("galilean", [False, True])
def test_collision_matches_oracle(host, case, galilean):
    stencil, method, mk, kw, force, fm, sgs = case
    if galilean and method != "cumulant":
        pytest.skip("Galilean correction is cumulant-only")
    okw = dict(kw)
    if force is not None:
        okw["force"] = force
        okw["force_model"] = fm
    if sgs is not None:
        okw["smagorinsky"] = sgs
    if galilean:
        okw["galilean_correction"] = True
    orc = O.make(stencil, method, **okw)
    rates = orc.spec.rates
    if method in ("srt", "trt"):
        # the population-space kernel takes (omega_even, omega_odd)
        degrees = [sp.Poly(m, *sp.symbols("x y z")).total_degree() for m in orc.spec.moments]
        even = next(r for r, d in zip(orc.spec.rates, degrees) if d > 0 and d % 2 == 0)
        odd = next(r for r, d in zip(orc.spec.rates, degrees) if d % 2 == 1)
        rates = [even, odd]
    p = physics_for(orc, mk, rates, force, fm, sgs, galilean)
    for seed in range(5):
        f = random_state(orc, seed)
        ref = orc.collide(f)
        g = f.copy()
        host.host_collide(orc.Q, mk, 0, g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(p))
        np.testing.assert_allclose(g, ref, rtol=0, atol=2e-15)
        h = f.copy()
        host.host_collide(orc.Q, mk, 1, h.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(p))
        scale = np.abs(ref + np.array([float(w) for w in orc.spec.weights])).max()
        # FP32 single-collision error relative to the populations; the general cumulant path adds
        # and removes the O(1) lattice-weight background in FP32, the other paths never form it
        tol = 5e-7 if mk == MK_CUM else 2e-7
        assert np.abs(h - ref).max() / scale < tol


@pytest.mark.parametrize("limiter", [0.1, True])
@pytest.mark.parametrize("galilean", [False, True])
@pytest.mark.parametrize("rates", [[1.95], [1.8, 1.3]])
def test_fourth_order_correction_matches_oracle(host, limiter, galilean, rates):
    """The fourth-order cumulant correction (limited third-order rates, corrected fourth-order
    polynomial cumulants) of the general cumulant collision against the oracle's restatement of
    methods/cumulantbased/fourth_order_correction.py, on states far enough from equilibrium for the
    limiters to act."""
    from oracle import oracle_spec as OS
    orc = O.make("D3Q27", "cumulant", relaxation_rates=rates, compressible=True, galilean_correction=galilean,
                 fourth_order_correction=limiter)
    w1 = rates[0]
    w2 = rates[1] if len(rates) > 1 else 1.0
    _, (a, b) = OS.fourth_order_rates(w1, w2)
    p = physics_for(orc, MK_CUM, orc.spec.rates, galilean=galilean)
    p.foc_limiter = 1e6 if limiter is True else limiter
    p.foc_a, p.foc_b = a, b
    for seed in range(5):
        f = random_state(orc, seed, amp=3e-3)
        ref = orc.collide(f)
        g = f.copy()
        host.host_collide(27, MK_CUM, 0, g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(p))
        np.testing.assert_allclose(g, ref, rtol=0, atol=2e-15)
    # the correction changes the collision
    plain_rates = rates if len(rates) == 1 else rates + [1.0] * 8
    plain = O.make("D3Q27", "cumulant", relaxation_rates=plain_rates, compressible=True,
                   galilean_correction=galilean)
    f = random_state(orc, 7, amp=3e-3)
    assert np.abs(plain.collide(f) - orc.collide(f)).max() > 1e-6
