"""FixedDensity boundaries (boundaries/boundaryconditions.py:1044-1099) on the CPU oracle: a fluid
at rest between density walls at its own density stays at rest, and a channel with a velocity
inlet and a density outlet settles to the outlet density next to the outlet.  The GPU sweeps are
held to these oracle runs in tests/test_fixed_density_gpu.py."""
import numpy as np
import pytest

from oracle import oracle as O

FD = 6


def _channel_flags(n, inlet):
    flags = np.zeros(tuple(s + 2 for s in n), np.uint8)
    flags[:, 0, :] = flags[:, -1, :] = 1
    flags[:, :, 0] = flags[:, :, -1] = 1
    flags[0, :, :] = 2 if inlet else FD
    flags[-1, :, :] = FD
    return flags


@pytest.mark.parametrize("case", [
    ("D3Q19", "trt", dict(relaxation_rate=1.7, compressible=True)),
    ("D3Q19", "mrt", dict(relaxation_rates=[1.7, 1.5, 1.0, 1.0], compressible=False)),
    ("D3Q27", "cumulant", dict(relaxation_rate=1.8, compressible=True, galilean_correction=True)),
], ids=["d3q19-trt", "d3q19-mrt", "d3q27-cum"])
@pytest.mark.parametrize("pattern", ["pull", "aa"])
def test_rest_state_between_density_walls_is_kept(case, pattern):
    stencil, method, kw = case
    n = (8, 6, 5)
    orc = O.make(stencil, method, **kw)
    prev = 0 if pattern == "pull" else 1
    f = orc.new_field(n)
    orc.set_equilibrium(f, np.ones(n), np.zeros(n + (3,)), pattern, prev)
    res, par = orc.run(f, 40, pattern, prev, periodic=(False,) * 3, flags=_channel_flags(n, inlet=False),
                       fixed_density=1.0)
    rho, u = orc.get_macroscopic(res, pattern, par)
    assert np.abs(u).max() < 1e-14 and np.abs(rho - 1).max() < 1e-14


def test_density_outlet_sets_the_outlet_density():
    n = (24, 8, 8)
    orc = O.make("D3Q19", "trt", relaxation_rate=1.6, compressible=True)
    f = orc.new_field(n)
    orc.set_equilibrium(f, np.ones(n), np.zeros(n + (3,)), "pull", 0)
    res, par = orc.run(f, 600, "pull", 0, periodic=(False,) * 3, flags=_channel_flags(n, inlet=True),
                       ubb_velocity=(0.02, 0.0, 0.0), fixed_density=0.998)
    rho, u = orc.get_macroscopic(res, "pull", par)
    core = (slice(None), slice(2, 6), slice(2, 6))
    assert abs(rho[-1][core[1:]].mean() - 0.998) < 1e-3          # the layer next to the outlet
    assert rho[0][core[1:]].mean() > rho[-1][core[1:]].mean()     # pressure falls along the channel
    assert u[..., 0][core].min() > 0                                # through-flow everywhere in the core
