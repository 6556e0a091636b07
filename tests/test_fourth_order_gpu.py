"""Fourth-order cumulant correction on the GPU: the sweep against the FP64 oracle (limited third-order
rates and corrected fourth-order cumulants, with and without the Galilean correction, pull and AA,
FP64 / FP32) and lbmpy's shear-wave scenario, where the corrected method's viscosity error matches
the oracle's and is an order of magnitude below the uncorrected method's."""
import numpy as np
import pytest

import lbmpy_b200 as L
from tests import shear_wave as SW
from tests.helpers import random_velocity
from tests.test_gpu_parity import FP32_TOL, FP64_TOL, _interior, make_pair, pop_rel_linf, run_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("pattern", ["pull", "aa"])
@pytest.mark.parametrize("limiter,galilean,rates", [(0.1, False, [1.95]), (True, True, [1.9, 1.3]),
                                                     (0.02, True, [1.99])])
def test_fourth_order_sweep_parity(cuda, dtype, pattern, limiter, galilean, rates):
    n = (12, 10, 8)
    periodic = (True, True, True)
    kw = dict(relaxation_rates=rates, compressible=True, galilean_correction=galilean,
              fourth_order_correction=limiter)
    # a rough velocity field, so that the third-order cumulants reach the limiter scale
    step, orc, f, flags, ubb, prev = make_pair("D3Q27", "cumulant", n, pattern, dtype, periodic=periodic,
                                               u=random_velocity(n, 4e-2, seed=3), **kw)
    steps = 40 if pattern == "pull" else 41
    res, _ = run_pair(step, orc, f, flags, ubb, prev, steps, pattern, periodic)
    err = pop_rel_linf(_interior(step.pdfs), res[1:-1, 1:-1, 1:-1], step.method.weights)
    assert err < (FP64_TOL if dtype == "float64" else FP32_TOL), f"{err:.3e}"


def _gpu_shear_wave(nu, foc, l=32):
    omega = 1.0 / (3 * nu + 0.5)
    u = SW.initial_velocity(l)
    kw = dict(relaxation_rate=omega, compressible=True)
    if foc:
        kw["fourth_order_correction"] = foc
    step = L.LatticeBoltzmannStep(domain_size=u.shape[:3], periodicity=True, stencil=L.Stencil.D3Q27,
                                  method=L.Method.CUMULANT, config=L.CreateKernelConfig(data_type="float64"), **kw)
    step.velocity_array[...] = u
    step.set_pdf_fields_from_macroscopic_values()
    first, total, every = SW.schedule(l)
    step.run(first)
    amps = []
    while step.time_steps_run < total:
        step.run(every)
        amps.append(SW.amplitude(step.velocity_array[:, 0, :, 1]))
    return SW.viscosity_error(amps, every, l, nu)


def test_shear_wave_viscosity_error():
    """nu = 1e-3, l = 32 (lbmpy's scenario, shortened as its integration test): ER_nu of the oracle
    is 6.3e-3 without and 4.1e-4 with the correction (limiter 0.1)."""
    plain = _gpu_shear_wave(1e-3, False)
    corrected = _gpu_shear_wave(1e-3, 0.1)
    assert abs(plain - 6.27e-3) < 5e-5
    assert abs(corrected - 4.13e-4) < 5e-5
