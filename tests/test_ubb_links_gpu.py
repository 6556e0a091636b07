"""Velocity profiles at UBB walls (per-link velocities from callbacks), prescribed wall densities,
adapt_velocity_to_force and two-density pressure-driven channels on the GPU, against the FP64
oracle (boundaries/boundaryconditions.py:724-841, 1044-1099; scenarios.py:104-172)."""
import numpy as np
import pytest

import lbmpy_b200 as L
from lbmpy_b200.boundaries import FixedDensity, NoSlip, UBB, slice_from_direction
from oracle import oracle as O
from tests.helpers import random_velocity, rel_linf
from tests.test_gpu_parity import _interior, pop_rel_linf

pytestmark = pytest.mark.gpu

CASES = [
    ("d3q19-trt-comp-pull", "D3Q19", "trt", "pull", dict(relaxation_rate=1.8, compressible=True)),
    ("d3q19-mrt-incomp-aa", "D3Q19", "mrt", "aa", dict(relaxation_rates=[1.7, 1.5, 1.0, 1.0], compressible=False)),
    ("d3q27-cum-aa", "D3Q27", "cumulant", "aa", dict(relaxation_rate=1.9, compressible=True, galilean_correction=True)),
    ("d3q19-trt-esotwist", "D3Q19", "trt", "esotwist", dict(relaxation_rate=1.7, compressible=True)),
]


def _compare(step, orc, flags, steps, pattern, rho, u, dtype, **orun):
    prev = 0 if pattern == "pull" else 1
    f = orc.new_field(step.domain_size)
    orc.set_equilibrium(f, rho, u, pattern, prev)
    res, par = orc.run(f, steps, pattern, prev, periodic=(False,) * 3, flags=flags, **orun)
    fluid = flags[1:-1, 1:-1, 1:-1] == 0
    err = pop_rel_linf(_interior(step.pdfs)[fluid], res[1:-1, 1:-1, 1:-1][fluid], step.method.weights)
    rho_o, u_o = orc.get_macroscopic(res, pattern, par)
    uerr = rel_linf(step.velocity_array[fluid], u_o[fluid])
    return err, uerr, u_o


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_pipe_inflow_channel_matches_oracle(cuda, case, dtype, monkeypatch):
    """create_channel(u_max=...): parabolic pipe inflow on W (one velocity per link, set by the
    geometry callback), FixedDensity 1 on E, pipe walls."""
    name, stencil, method, pattern, kw = case
    monkeypatch.setenv("LBM_B200_PAIR", "0")
    n = (14, 10, 10)
    step = L.create_channel(domain_size=n, u_max=0.03, stencil=getattr(L.Stencil, stencil),
                            method=getattr(L.Method, method.upper()), streaming_pattern=pattern,
                            config=L.CreateKernelConfig(data_type=dtype), **kw)
    bh = step.boundary_handling
    u = random_velocity(n, 5e-3, seed=3)
    rho = 1.0 + 1e-3 * np.random.default_rng(4).uniform(-1, 1, n)
    step.velocity_array[...] = u
    step.density_array[...] = rho
    step.set_pdf_fields_from_macroscopic_values()
    steps = 60 if pattern == "pull" else 61              # in place: end on an even step
    step.run(steps)
    flags = (bh.flag_array & 15).astype(np.uint8)
    assert set(np.unique(flags)) <= {0, 1, 2, 6}
    links = bh.ubb_link_velocities_dense()
    assert np.abs(links).max() > 0.02                     # the profile reaches its centre value
    err, uerr, u_o = _compare(step, O.make(stencil, method, **kw), flags, steps, pattern, rho, u, dtype,
                              ubb_link=links, fixed_density=1.0)
    assert err < (1e-12 if dtype == "float64" else 1e-5), f"{name} {dtype}: {err:.3e}"
    assert uerr < (1e-11 if dtype == "float64" else 1e-4)
    assert u_o[0, :, :, 0].max() > 0.01                   # the inflow has entered the pipe


@pytest.mark.parametrize("pattern", ["pull", "aa"])
def test_pressure_driven_channel_with_two_densities(cuda, pattern, monkeypatch):
    """create_channel(pressure_difference=...): FixedDensity 1 + dp on W and 1 on E (flag types 6
    and 7, the plan's two densities)."""
    monkeypatch.setenv("LBM_B200_PAIR", "0")
    n = (16, 8, 8)
    kw = dict(relaxation_rate=1.8, compressible=True)
    step = L.create_channel(domain_size=n, pressure_difference=3e-3, duct=True, stencil=L.Stencil.D3Q19,
                            method=L.Method.TRT, streaming_pattern=pattern,
                            config=L.CreateKernelConfig(data_type="float64"), **kw)
    step.set_pdf_fields_from_macroscopic_values()
    steps = 80 if pattern == "pull" else 81
    step.run(steps)
    flags = (step.boundary_handling.flag_array & 15).astype(np.uint8)
    assert set(np.unique(flags)) == {0, 1, 6, 7}
    err, uerr, u_o = _compare(step, O.make("D3Q19", "trt", **kw), flags, steps, pattern, np.ones(n),
                              np.zeros(n + (3,)), "float64", fixed_density=1.003, fixed_density1=1.0)
    assert err < 1e-12, f"{pattern}: {err:.3e}"
    assert u_o[..., 0].mean() > 1e-5                      # the pressure drop drives the flow along +x


@pytest.mark.parametrize("compressible", [True, False])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_adapted_lid_with_force_and_wall_density(cuda, compressible, dtype, monkeypatch):
    """A lid with adapt_velocity_to_force=True under a Guo body force, with a prescribed wall density
    (used by compressible methods), against the oracle."""
    monkeypatch.setenv("LBM_B200_PAIR", "0")
    n = (10, 9, 8)
    F = (1e-5, -2e-6, 0.0)
    kw = dict(relaxation_rate=1.75, compressible=compressible, force=F)
    step = L.LatticeBoltzmannStep(domain_size=n, periodicity=False, stencil=L.Stencil.D3Q19, method=L.Method.TRT,
                                  config=L.CreateKernelConfig(data_type=dtype), **kw)
    bh = step.boundary_handling
    bh.set_boundary(UBB((0.02, 0.0, 0.0), density=1.01, adapt_velocity_to_force=True),
                    slice_from_direction("N", 3))
    for d in ("W", "E", "S", "T", "B"):
        bh.set_boundary(NoSlip(), slice_from_direction(d, 3))
    u = random_velocity(n, 5e-3, seed=8)
    rho = np.ones(n)
    step.velocity_array[...] = u
    step.set_pdf_fields_from_macroscopic_values()
    step.run(50)
    flags = (bh.flag_array & 15).astype(np.uint8)
    err, uerr, _ = _compare(step, O.make("D3Q19", "trt", **kw), flags, 50, "pull", rho, u, dtype,
                            ubb_velocity=(0.02, 0.0, 0.0), ubb_adapt=True, ubb_density=1.01)
    assert err < (1e-12 if dtype == "float64" else 1e-5), f"{dtype}: {err:.3e}"
