"""FreeSlip, SimpleExtrapolationOutflow, ExtrapolationOutflow and NoSlipLinearBouzidi on the GPU
(per-link tables read by the fused boundary handling of the sweep) against the FP64 oracle, and
lbmpy's own free-slip scenario (tests/test_free_slip.py) through the lbmpy-compatible API."""
import numpy as np
import pytest

import lbmpy_b200 as L
from lbmpy_b200.boundaries import (ExtrapolationOutflow, FreeSlip, NoSlip, NoSlipLinearBouzidi,
                                   SimpleExtrapolationOutflow, UBB, slice_from_direction)
from oracle import oracle as O
from tests.helpers import random_velocity
from tests.test_gpu_parity import _interior, pop_rel_linf

pytestmark = pytest.mark.gpu


def _step(n, periodic, stencil, method, pattern, dtype, **kw):
    return L.LatticeBoltzmannStep(domain_size=n, periodicity=periodic, stencil=getattr(L.Stencil, stencil),
                                  method=getattr(L.Method, method.upper()), streaming_pattern=pattern,
                                  config=L.CreateKernelConfig(data_type=dtype), **kw)


def _parity(step, stencil, method, kw, steps, pattern, periodic, dtype, u, rho, **orun):
    bh = step.boundary_handling
    step.velocity_array[...] = u
    step.density_array[...] = rho
    step.set_pdf_fields_from_macroscopic_values()
    step.run(steps)
    assert step.sweep_status() == 0
    orc = O.make(stencil, method, **kw)
    prev = 0 if pattern == "pull" else 1
    f = orc.new_field(step.domain_size)
    orc.set_equilibrium(f, rho, u, pattern, prev)
    orc.periodic_sync(f, pattern, prev, periodic)
    vel, code, value = bh.link_tables_dense(pdfs=f, previous_timestep=prev, pattern=pattern)
    callable_ubb = any(x.velocity_is_callable for x in bh._ubbs)
    flags = (bh.flag_array & 15).astype(np.uint8)
    res, par = orc.run(f, steps, pattern, prev, periodic=periodic, flags=flags, link_code=code, link_value=value,
                       ubb_link=vel if callable_ubb else None, **orun)
    orc.periodic_sync(res, pattern, par, periodic)
    fluid = flags[1:-1, 1:-1, 1:-1] == 0
    err = pop_rel_linf(_interior(step.pdfs)[fluid], res[1:-1, 1:-1, 1:-1][fluid], step.method.weights)
    assert err < (1e-12 if dtype == "float64" else 1e-5), f"{err:.3e}"
    return res


PATTERNS = [("pull", "float64"), ("aa", "float64"), ("pull", "float32"), ("esotwist", "float64")]


@pytest.mark.parametrize("pattern,dtype", PATTERNS)
@pytest.mark.parametrize("given_normal", [True, False])
def test_free_slip_channel(cuda, pattern, dtype, given_normal, monkeypatch):
    monkeypatch.setenv("LBM_B200_PAIR", "0")
    n = (10, 8, 6)
    periodic = (True, False, True)
    kw = dict(relaxation_rate=1.8, compressible=True, force=(2e-5, 0, 0))
    step = _step(n, periodic, "D3Q19", "trt", pattern, dtype, **kw)
    st = list(step.method.stencil)
    step.boundary_handling.set_boundary(NoSlip(), slice_from_direction("S", 3))
    step.boundary_handling.set_boundary(FreeSlip(st, (0, -1, 0) if given_normal else None),
                                        slice_from_direction("N", 3))
    steps = 40 if pattern == "pull" else 41
    _parity(step, "D3Q19", "trt", kw, steps, pattern, periodic, dtype, random_velocity(n, 1e-2, seed=2),
            1 + 1e-3 * np.random.default_rng(3).uniform(-1, 1, n))


@pytest.mark.parametrize("pattern,dtype", PATTERNS)
def test_free_slip_box_corners(cuda, pattern, dtype, monkeypatch):
    """A closed box with FreeSlip on five faces (normals found per link, so edges and corners reflect
    along every wall they touch) under a moving lid; D3Q27 cumulant."""
    monkeypatch.setenv("LBM_B200_PAIR", "0")
    n = (8, 8, 6)
    periodic = (False, False, False)
    kw = dict(relaxation_rate=1.9, compressible=True, galilean_correction=True)
    step = _step(n, periodic, "D3Q27", "cumulant", pattern, dtype, **kw)
    st = list(step.method.stencil)
    bh = step.boundary_handling
    fs = FreeSlip(st)
    for d in ("W", "E", "S", "N", "B"):
        bh.set_boundary(fs, slice_from_direction(d, 3))
    bh.set_boundary(UBB((0.02, 0, 0)), slice_from_direction("T", 3))
    steps = 30 if pattern == "pull" else 31
    _parity(step, "D3Q27", "cumulant", kw, steps, pattern, periodic, dtype, random_velocity(n, 5e-3, seed=4),
            np.ones(n), ubb_velocity=(0.02, 0, 0))


@pytest.mark.parametrize("pattern,dtype", PATTERNS)
@pytest.mark.parametrize("kind", ["simple", "extrapolation"])
def test_outflows_behind_a_profile_inlet(cuda, pattern, dtype, kind, monkeypatch):
    monkeypatch.setenv("LBM_B200_PAIR", "0")
    n = (16, 8, 8)
    periodic = (False, False, False)
    kw = dict(relaxation_rate=1.6, compressible=False)
    step = _step(n, periodic, "D3Q19", "srt", pattern, dtype, **kw)
    bh = step.boundary_handling
    L.geometry.add_pipe_inflow_boundary(bh, 0.03, slice_from_direction("W", 3))
    out = (SimpleExtrapolationOutflow("E", list(step.method.stencil)) if kind == "simple"
           else ExtrapolationOutflow("E", step.method, streaming_pattern=pattern))
    bh.set_boundary(out, slice_from_direction("E", 3))
    for d in ("N", "S", "T", "B"):
        bh.set_boundary(NoSlip(), slice_from_direction(d, 3))
    steps = 60 if pattern == "pull" else 61
    _parity(step, "D3Q19", "srt", kw, steps, pattern, periodic, dtype, random_velocity(n, 3e-3, seed=6),
            np.ones(n))


@pytest.mark.parametrize("pattern,dtype", PATTERNS)
def test_bouzidi_obstacle(cuda, pattern, dtype, monkeypatch):
    """A block obstacle inside a periodic channel whose links carry wall distances from 0.1 to 0.9
    (all three cases of the interpolation), NoSlip channel walls."""
    monkeypatch.setenv("LBM_B200_PAIR", "0")
    n = (14, 10, 8)
    periodic = (True, False, True)
    kw = dict(relaxation_rate=1.7, compressible=True, force=(1e-5, 0, 0))
    step = _step(n, periodic, "D3Q19", "trt", pattern, dtype, **kw)
    bh = step.boundary_handling

    def wall_distance(bd):
        k = np.arange(len(bd["q"]))
        bd["q"] = 0.1 + 0.8 * ((k * 7919) % 97) / 96.0

    bh.set_boundary(NoSlip(), slice_from_direction("S", 3))
    bh.set_boundary(NoSlip(), slice_from_direction("N", 3))
    bh.set_boundary(NoSlipLinearBouzidi(init_wall_distance=wall_distance), slice_obj=(slice(6, 9), slice(4, 7), slice(3, 6)))
    steps = 40 if pattern == "pull" else 41
    _parity(step, "D3Q19", "trt", kw, steps, pattern, periodic, dtype, random_velocity(n, 5e-3, seed=9),
            1 + 1e-3 * np.random.default_rng(10).uniform(-1, 1, n))


def test_lbmpy_free_slip_scenario(cuda):
    """lbmpy's tests/test_free_slip.py through this package: D3Q27 SRT 1.8, 30 x 15 x 30, linear
    inflow profile by UBB callback on W, ExtrapolationOutflow on E, NoSlip S/T/B, FreeSlip N,
    2000 steps; the velocity profile next to the outlet has zero gradient at the free-slip wall."""
    n = (30, 15, 30)
    step = L.LatticeBoltzmannStep(domain_size=n, periodicity=False, stencil=L.Stencil.D3Q27, method=L.Method.SRT,
                                  relaxation_rate=1.8, config=L.CreateKernelConfig(data_type="float64"))
    st = list(step.method.stencil)

    def velocity_info_callback(bd, **_):
        bd["vel_1"] = 0
        bd["vel_2"] = 0
        y = bd.link_positions(1)
        bd["vel_0"] = 0.1 * (1 - (15 - y) / 15)

    bh = step.boundary_handling
    bh.set_boundary(UBB(velocity_info_callback, dim=3), slice_from_direction("W", 3))
    bh.set_boundary(ExtrapolationOutflow(st[4], step.method), slice_from_direction("E", 3))
    for d in ("S", "T", "B"):
        bh.set_boundary(NoSlip("wall"), slice_from_direction(d, 3))
    bh.set_boundary(FreeSlip(st, (0, -1, 0)), slice_from_direction("N", 3))
    step.run(2000)
    vel_profile = step.velocity_array[-2, :, n[2] // 2, 0]
    np.testing.assert_almost_equal(np.gradient(vel_profile)[-1], 0, decimal=3)
