"""Fourth-order cumulant correction (LBMConfig(fourth_order_correction=...),
methods/cumulantbased/fourth_order_correction.py:21-237) on the host: the method's rates against the
oracle, the argument checks, and the oracle on lbmpy's shear-wave scenario, where the correction cuts
the viscosity error of the D3Q27 cumulant method by an order of magnitude (Geier et al. 2017: fourth
order accurate diffusion).  The collision itself is checked against the oracle in
tests/test_collision_host.py."""
import numpy as np
import pytest

import lbmpy_b200 as L
from oracle import oracle as O
from oracle import oracle_spec as OS
from tests import shear_wave as SW


@pytest.mark.parametrize("rates", [[1.8], [1.9, 1.2]])
def test_rates_match_oracle(rates):
    cfg = L.LBMConfig(stencil=L.Stencil.D3Q27, method=L.Method.CUMULANT, relaxation_rates=rates,
                      compressible=True, fourth_order_correction=0.05)
    rule = L.create_lb_collision_rule(lbm_config=cfg)
    assert rule.fourth_order_limiter == 0.05
    ref = OS.resolve("D3Q27", "cumulant", relaxation_rates=rates, compressible=True, fourth_order_correction=0.05)
    np.testing.assert_allclose([float(r) for r in rule.method.relaxation_rates], ref.rates, rtol=0, atol=1e-15)
    cfg = L.LBMConfig(stencil=L.Stencil.D3Q27, method=L.Method.CUMULANT, relaxation_rate=1.8, compressible=True,
                      fourth_order_correction=True)
    assert L.create_lb_collision_rule(lbm_config=cfg).fourth_order_limiter == 1e6


def test_argument_checks():
    with pytest.raises(ValueError):
        L.create_lb_method(lbm_config=L.LBMConfig(stencil=L.Stencil.D3Q19, method=L.Method.SRT, relaxation_rate=1.8,
                                                  fourth_order_correction=True))
    with pytest.raises(AssertionError):
        L.create_lb_method(lbm_config=L.LBMConfig(stencil=L.Stencil.D3Q27, method=L.Method.CUMULANT,
                                                  relaxation_rates=[1.8, 1.0, 1.0], compressible=True,
                                                  fourth_order_correction=True))
    with pytest.raises(NotImplementedError):
        L.create_lb_collision_rule(lbm_config=L.LBMConfig(
            stencil=L.Stencil.D3Q27, method=L.Method.CUMULANT, relaxation_rate=1.8, compressible=True,
            fourth_order_correction=True, subgrid_scale_model=L.SubgridScaleModel.SMAGORINSKY))


def _oracle_shear_wave(nu, foc, l=32):
    omega = 1.0 / (3 * nu + 0.5)
    kw = dict(relaxation_rate=omega, compressible=True)
    if foc:
        kw["fourth_order_correction"] = foc
    orc = O.make("D3Q27", "cumulant", **kw)
    u = SW.initial_velocity(l)
    n = u.shape[:3]
    f = orc.new_field(n)
    orc.set_equilibrium(f, np.ones(n), u)
    first, total, every = SW.schedule(l)
    f, _ = orc.run(f, first, "pull", 0, periodic=(True, True, True))
    amps, t = [], first
    while t < total:
        f, _ = orc.run(f, every, "pull", 0, periodic=(True, True, True))
        t += every
        amps.append(SW.amplitude(orc.get_macroscopic(f)[1][:, 0, :, 1]))
    return SW.viscosity_error(amps, every, l, nu)


def test_shear_wave_viscosity_error_on_the_oracle():
    """nu = 1e-3 (omega 1.988), l = 32: ER_nu 6.3e-3 without the correction, 4e-4 with limiter 0.1."""
    plain = _oracle_shear_wave(1e-3, False)
    corrected = _oracle_shear_wave(1e-3, 0.1)
    assert plain > 3e-3
    assert corrected < 1e-3
    assert corrected < 0.2 * plain
