"""FixedDensity outlets on the GPU (the boundary pre-pass k_boundary_prepass plus the sweep) against the FP64
oracle: velocity inlet, density outlet, no-slip channel walls; SRT/TRT, MRT and cumulant, pull
and in-place patterns, FP64 and FP32 storage."""
import numpy as np
import pytest

import lbmpy_b200 as L
from lbmpy_b200.boundaries import FixedDensity, NoSlip, UBB, slice_from_direction
from oracle import oracle as O
from tests.helpers import random_velocity, rel_linf
from tests.test_gpu_parity import _interior, pop_rel_linf

pytestmark = pytest.mark.gpu

CASES = [
    ("d3q19-trt-comp", "D3Q19", "trt", "pull", dict(relaxation_rate=1.8, compressible=True)),
    ("d3q19-mrt-incomp", "D3Q19", "mrt", "aa", dict(relaxation_rates=[1.7, 1.5, 1.0, 1.0], compressible=False)),
    ("d3q27-cum", "D3Q27", "cumulant", "aa", dict(relaxation_rate=1.9, compressible=True, galilean_correction=True)),
    ("d3q19-trt-esopull", "D3Q19", "trt", "esopull", dict(relaxation_rate=1.7, compressible=True)),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_density_outlet_matches_oracle(cuda, case, dtype, monkeypatch):
    name, stencil, method, pattern, kw = case
    monkeypatch.setenv("LBM_B200_PAIR", "0")
    n = (14, 8, 6)
    step = L.LatticeBoltzmannStep(domain_size=n, periodicity=False, stencil=getattr(L.Stencil, stencil),
                                  method=getattr(L.Method, method.upper()), streaming_pattern=pattern,
                                  config=L.CreateKernelConfig(data_type=dtype), **kw)
    bh = step.boundary_handling
    for d in ("N", "S", "T", "B"):
        bh.set_boundary(NoSlip(), slice_from_direction(d, 3))
    bh.set_boundary(UBB((0.02, 0.0, 0.0)), slice_from_direction("W", 3))
    bh.set_boundary(FixedDensity(0.998), slice_from_direction("E", 3))
    u = random_velocity(n, 1e-2, seed=5)
    rho = 1.0 + 1e-3 * np.random.default_rng(6).uniform(-1, 1, n)
    step.velocity_array[...] = u
    step.density_array[...] = rho
    step.set_pdf_fields_from_macroscopic_values()
    steps = 60 if pattern == "pull" else 61              # in place: end on an even step
    step.run(steps)
    assert step.sweep_status() == 0

    orc = O.make(stencil, method, **kw)
    prev = 0 if pattern == "pull" else 1
    f = orc.new_field(n)
    orc.set_equilibrium(f, rho, u, pattern, prev)
    flags = (bh.flag_array & 7).astype(np.uint8)
    res, par = orc.run(f, steps, pattern, prev, periodic=(False,) * 3, flags=flags, ubb_velocity=(0.02, 0, 0),
                       fixed_density=0.998)
    fluid = flags[1:-1, 1:-1, 1:-1] == 0
    err = pop_rel_linf(_interior(step.pdfs)[fluid], res[1:-1, 1:-1, 1:-1][fluid], step.method.weights)
    assert err < (1e-12 if dtype == "float64" else 1e-5), f"{name} {dtype}: {err:.3e}"
    rho_o, u_o = orc.get_macroscopic(res, pattern, par)
    assert rel_linf(step.velocity_array[fluid], u_o[fluid]) < (1e-11 if dtype == "float64" else 1e-4)


def test_density_outlet_rejects_forces(cuda):
    step = L.LatticeBoltzmannStep(domain_size=(8, 6, 6), periodicity=False, stencil=L.Stencil.D3Q19,
                                  method=L.Method.TRT, relaxation_rate=1.7, force=(1e-5, 0, 0),
                                  config=L.CreateKernelConfig(data_type="float32"))
    step.boundary_handling.set_boundary(FixedDensity(1.0), slice_from_direction("E", 3))
    with pytest.raises(Exception, match="force-free"):
        step.run(1)
