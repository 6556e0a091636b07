"""The oracle's collision, forcing and boundaries reproduce states that lbmpy's own generated
kernels wrote (its regression files ``tests/reference_files/*.npz``, sampled into
``tests/golden/lbmpy_states.npz`` by ``tests/golden/make_golden.py``).

lbmpy does not record how those files were made.  The run parameters below were identified by
re-running the scenarios from rest and matching the stored PDFs; each reproduces its file to
round-off (about 1e-15 of the population scale), so the oracle is pinned to lbmpy's arithmetic
for the methods they cover:

- 2-D lid-driven cavity 16 x 19 (``create_lid_driven_cavity``, scenarios.py:72-101; lid 0.005 on
  N, NoSlip W/E/S), D2Q9 SRT omega = 1.8, force (1e-4, -2e-5) with the Guo, Luo and Simple force
  models (forcemodels.py:179-317), 100 steps;
- 2-D force-driven channel 40 x 80 (``create_channel(force=1e-4)``, scenarios.py:104-172; periodic
  in x, NoSlip N/S), D2Q9 SRT omega = 1.8, same three force models, 500 steps;
- 3-D lid-driven cavity 16 x 17 x 18, D3Q19 TRT with rates (1.8, 1.3), the discrete Maxwellian
  equilibrium (maxwellian_equilibrium.py:64-104), Luo force (1e-4, -2e-5, 1.24e-5), 100 steps.

Compressible states are stored absolute (f), incompressible ones zero-centred (f - w).  The
D3Q19 MRT file is not matched: no parameter set tried reproduced it (the best fit of the four
MRT rates left 4e-5), so it is not used here.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from oracle import oracle_spec as S

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "lbmpy_states.npz"))
TOL = 1e-13


def _sample(name):
    return tuple(GOLDEN[name + "__shape"]), GOLDEN[name + "__idx"], GOLDEN[name + "__val"]


def _run_2d(name, steps, omega=1.8, flags_fn=None, periodic=(0, 0, 0), force=(1e-4, -2e-5), ubb=(0.005, 0, 0),
            **kw):
    shape, idx, val = _sample(name)
    n = shape[:2]
    fm = kw.pop("force_model")
    comp = kw.pop("compressible")
    o = O.Oracle(S.resolve("D2Q9", "srt", relaxation_rate=omega, compressible=comp, zero_centered=not comp,
                           force=force, force_model=fm, **kw))
    f = o.new_field(n)
    o.set_equilibrium(f, np.ones(n), np.zeros(n + (2,)))
    res, _ = o.run(f, steps, "pull", 0, periodic=periodic, flags=flags_fn(n), ubb_velocity=ubb)
    got = np.ascontiguousarray(res[1:-1, 1:-1]).reshape(shape).reshape(-1)[idx]
    return got, val


def _ldc_flags_2d(n):
    fl = np.zeros((n[0] + 2, n[1] + 2), np.uint8)
    fl[:, -1] = 2                                # UBB on N first, NoSlip overrides the corners
    fl[0, :] = fl[-1, :] = fl[:, 0] = 1
    return fl


def _channel_flags_2d(n):
    fl = np.zeros((n[0] + 2, n[1] + 2), np.uint8)
    fl[:, 0] = fl[:, -1] = 1
    return fl


@pytest.mark.parametrize("force_model", ["guo", "luo", "simple"])
@pytest.mark.parametrize("compressible", [True, False])
def test_lid_driven_cavity_2d(force_model, compressible):
    name = f"LidDrivenCavity_SRT_{force_model}_{'compressible' if compressible else 'incompressible'}"
    got, ref = _run_2d(name, 100, flags_fn=_ldc_flags_2d, force_model=force_model, compressible=compressible)
    assert np.abs(got - ref).max() < TOL


@pytest.mark.parametrize("force_model", ["guo", "luo", "simple"])
@pytest.mark.parametrize("compressible", [True, False])
def test_force_driven_channel_2d(force_model, compressible):
    name = f"ForceDrivenChannel_{force_model}_{'compressible' if compressible else 'incompressible'}"
    got, ref = _run_2d(name, 500, flags_fn=_channel_flags_2d, periodic=(1, 0, 0), force=(1e-4, 0),
                       ubb=(0, 0, 0), force_model=force_model, compressible=compressible)
    assert np.abs(got - ref).max() < TOL


def ldc_flags_3d(n):
    """lbmpy's lid-driven cavity in the ghost layers: UBB on N, then NoSlip on W, E, S, T, B."""
    fl = np.zeros(tuple(s + 2 for s in n), np.uint8)
    fl[:, -1, :] = 2
    fl[0, :, :] = fl[-1, :, :] = fl[:, 0, :] = fl[:, :, 0] = fl[:, :, -1] = 1
    return fl


TRT_RATES = [1.8, 1.3]
TRT_FORCE = (1e-4, -2e-5, 1.24e-5)


def run_trt_ldc_3d(compressible, steps=100, rates=TRT_RATES, continuous=False, force_model="luo"):
    name = f"LidDrivenCavity_TRT_luo_{'compressible' if compressible else 'incompressible'}"
    shape, idx, val = _sample(name)
    n = shape[:3]
    o = O.Oracle(S.resolve("D3Q19", "trt", relaxation_rates=rates, compressible=compressible,
                           zero_centered=not compressible, force=TRT_FORCE, force_model=force_model,
                           continuous_equilibrium=continuous))
    f = o.new_field(n)
    o.set_equilibrium(f, np.ones(n), np.zeros(n + (3,)))
    res, _ = o.run(f, steps, "pull", 0, periodic=(0, 0, 0), flags=ldc_flags_3d(n), ubb_velocity=(0.005, 0, 0))
    got = np.ascontiguousarray(res[1:-1, 1:-1, 1:-1]).reshape(-1)[idx]
    return got, val


@pytest.mark.parametrize("compressible", [True, False])
def test_lid_driven_cavity_d3q19_trt(compressible):
    got, ref = run_trt_ldc_3d(compressible)
    assert np.abs(got - ref).max() < TOL


@pytest.mark.parametrize("wrong", ["continuous_equilibrium", "odd_rate", "guo_force", "one_step_more"])
def test_golden_state_rejects_a_wrong_method(wrong):
    """The golden state separates methods that differ only slightly: each variant below misses it
    by more than 1e-9 (the Guo instead of the Luo force model by 1.6e-9, the others by 2e-7 or
    more), four orders of magnitude above the tolerance."""
    kw = {"continuous_equilibrium": dict(continuous=True), "odd_rate": dict(rates=[1.8, 1.3 + 1e-3]),
          "guo_force": dict(force_model="guo"), "one_step_more": dict(steps=101)}[wrong]
    got, ref = run_trt_ldc_3d(False, **kw)
    assert np.abs(got - ref).max() > 1e-9
