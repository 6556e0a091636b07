"""The row-staged sweep: persistent CTAs, the Q population rows of each row segment bulk-copied
into shared-memory stages ahead of the collision.

Held to the FP64 oracle like every sweep (1e-12 for FP64 storage, 1e-5 for FP32), and to the
one-cell sweep it restructures (same collision code; FP32 and 16-bit storage within a few
rounding steps).  Rows longer than one segment (the halo values at segment edges), the periodic
wrap across a row's ends, walls, moving walls, every stage count and the device status word are
covered; each test checks that the staged kernel is the one that ran.
"""
import numpy as np
import pytest
import torch

import lbmpy_b200 as L
from tests.test_gpu_parity import _boundaries, _interior, make_pair, pop_rel_linf, run_pair

pytestmark = pytest.mark.gpu

STAGED_CASES = [
    # id, stencil, method, pattern, n, periodic, boundaries, kwargs
    ("d3q19-trt-pull-periodic", "D3Q19", "trt", "pull", (136, 6, 5), (1, 1, 1), None,
     dict(relaxation_rate=1.8, compressible=True)),
    ("d3q19-srt-pull-guo", "D3Q19", "srt", "pull", (24, 10, 8), (1, 1, 1), None,
     dict(relaxation_rate=1.6, compressible=False, force=(1e-5, -2e-6, 3e-6))),
    ("d3q19-mrt-pull-ldc", "D3Q19", "mrt", "pull", (16, 10, 8), (0, 0, 0), "ldc",
     dict(relaxation_rates=[1.7, 1.5, 1.0, 1.0], compressible=False)),
    ("d3q19-trt-aa-ldc-comp", "D3Q19", "trt", "aa", (16, 12, 8), (0, 0, 0), "ldc",
     dict(relaxation_rate=1.9, compressible=True)),
    ("d3q27-trt-aa-periodic", "D3Q27", "trt", "aa", (264, 4, 4), (1, 1, 1), None,
     dict(relaxation_rate=1.8, compressible=True)),
    ("d3q27-cum-aa-channel", "D3Q27", "cumulant", "aa", (136, 6, 6), (1, 0, 0), "duct",
     dict(relaxation_rate=1.95, compressible=True, galilean_correction=True, force=(1e-5, 0, 0))),
    ("d3q27-cum-pull-smag", "D3Q27", "cumulant", "pull", (16, 10, 8), (1, 1, 1), None,
     dict(relaxation_rate=1.99, compressible=True, subgrid_scale_model=(L.SubgridScaleModel.SMAGORINSKY, 0.1))),
    ("d3q27-mrt-pull", "D3Q27", "mrt", "pull", (16, 8, 8), (1, 1, 1), None,
     dict(relaxation_rates=[1.8, 1.4, 1.1, 1.2, 1.0, 1.0], compressible=True)),
]


def _run_case(case, dtype, monkeypatch, staged="1", ns=None, storage=None):
    name, stencil, method, pattern, n, periodic, bkind, kw = case
    monkeypatch.setenv("LBM_B200_STAGED", staged)
    monkeypatch.setenv("LBM_B200_PAIR", "0")
    monkeypatch.setenv("LBM_B200_QUAD", "0")
    if ns is not None:
        monkeypatch.setenv("LBM_B200_NS", str(ns))
    else:
        monkeypatch.delenv("LBM_B200_NS", raising=False)
    step, orc, f, flags, ubb, prev = make_pair(stencil, method, n, pattern, dtype, storage=storage,
                                               periodic=periodic, boundaries=_boundaries(bkind), **kw)
    assert step.sweep_variant() == ("staged" if staged == "1" else "cell")
    return step, orc, f, flags, ubb, prev


@pytest.mark.parametrize("case", STAGED_CASES, ids=[c[0] for c in STAGED_CASES])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_staged_sweep_matches_oracle(cuda, case, dtype, monkeypatch):
    name, stencil, method, pattern, n, periodic, bkind, kw = case
    step, orc, f, flags, ubb, prev = _run_case(case, dtype, monkeypatch)
    res, _ = run_pair(step, orc, f, flags, ubb, prev, 60, pattern, periodic)
    assert step.sweep_status() == 0
    got = _interior(step.pdfs)
    ref = res[1:-1, 1:-1, 1:-1]
    fluid = np.ones(n, bool) if flags is None else (flags[1:-1, 1:-1, 1:-1] == 0)
    err = pop_rel_linf(got[fluid], ref[fluid], step.method.weights)
    tol = 1e-12 if dtype == "float64" else 1e-5
    assert err < tol, f"{name} {dtype}: {err:.3e}"


@pytest.mark.parametrize("case", [STAGED_CASES[i] for i in (0, 3, 4, 5)],
                         ids=[STAGED_CASES[i][0] for i in (0, 3, 4, 5)])
@pytest.mark.parametrize("storage", [None, "float16", "bfloat16"])
def test_staged_sweep_matches_cell_sweep(cuda, case, storage, monkeypatch):
    """FP32 arithmetic on FP32 / FP16 / BF16 storage: the staged and the one-cell sweep differ by
    rounding at most (same collision code, scheduled differently)."""
    outs = []
    for staged in ("1", "0"):
        step, *_ = _run_case(case, "float32", monkeypatch, staged=staged, storage=storage)
        step.run(40)
        assert step.sweep_status() == 0
        outs.append(_interior(step.pdfs))
    scale = 1.0 + max(step.method.weights)
    err = np.abs(outs[0] - outs[1]).max() / scale
    assert err <= (1e-6 if storage is None else 1e-5), err


@pytest.mark.parametrize("ns", [3, 4, 5])
def test_stage_count_does_not_change_results(cuda, ns, monkeypatch):
    case = STAGED_CASES[5]                       # D3Q27 cumulant AA channel, two segments per row in FP64
    outs = {}
    for k in (ns, 2):
        step, *_ = _run_case(case, "float32", monkeypatch, ns=k)
        step.run(30)
        assert step.sweep_status() == 0
        outs[k] = step.pdfs.clone()
    assert torch.equal(outs[ns], outs[2])


def test_staged_compressible_moving_wall(cuda, monkeypatch):
    """Compressible UBB (the wall density pre-pass) through the staged sweep, AA, FP64."""
    case = ("d3q27-cum-aa-ldc", "D3Q27", "cumulant", "aa", (16, 10, 8), (0, 0, 0), "ldc",
            dict(relaxation_rate=1.9, compressible=True, galilean_correction=True))
    step, orc, f, flags, ubb, prev = _run_case(case, "float64", monkeypatch)
    res, _ = run_pair(step, orc, f, flags, ubb, prev, 50, "aa", (0, 0, 0))
    assert step.sweep_status() == 0
    fluid = flags[1:-1, 1:-1, 1:-1] == 0
    err = pop_rel_linf(_interior(step.pdfs)[fluid], res[1:-1, 1:-1, 1:-1][fluid], step.method.weights)
    assert err < 1e-12, err


def test_staged_not_used_where_it_does_not_apply(cuda, monkeypatch):
    """Rows whose length is not a whole number of 16-byte units, and EsoTwist, fall back."""
    monkeypatch.setenv("LBM_B200_STAGED", "1")
    monkeypatch.setenv("LBM_B200_PAIR", "0")
    s = L.LatticeBoltzmannStep(domain_size=(10, 6, 4), periodicity=True, stencil=L.Stencil.D3Q19,
                               method=L.Method.TRT, relaxation_rate=1.7,
                               config=L.CreateKernelConfig(data_type="float32"))
    assert s.sweep_variant() == "cell"
    s = L.LatticeBoltzmannStep(domain_size=(16, 6, 4), periodicity=True, stencil=L.Stencil.D3Q19,
                               method=L.Method.TRT, relaxation_rate=1.7, streaming_pattern="esotwist",
                               config=L.CreateKernelConfig(data_type="float32"))
    assert s.sweep_variant() == "cell"


def test_staged_wait_runs_out_and_reports(cuda, monkeypatch):
    """lbm_plan_set_stage_wait: every CTA waits, before its last tile, on a barrier that nothing
    arrives at; the wait runs out after 2 ms, the sweep sets LBM_STATUS_STAGE_TIMEOUT and returns
    with that tile unswept.  The context stays usable: with the probe off the next sweeps complete
    and match the oracle again from a fresh state."""
    from lbmpy_b200 import _native as N
    case = STAGED_CASES[0]
    step, orc, f, flags, ubb, prev = _run_case(case, "float64", monkeypatch)
    plan = step._bound().plan
    N.check(N.lib().lbm_plan_set_stage_wait(plan.handle, 2_000_000, 1), "lbm_plan_set_stage_wait")
    step.run(1)
    torch.cuda.synchronize()
    assert step.sweep_status() == N.STATUS_STAGE_TIMEOUT
    assert step.sweep_status() == 0            # the read above cleared it
    N.check(N.lib().lbm_plan_set_stage_wait(plan.handle, 0, 0), "lbm_plan_set_stage_wait")
    with pytest.raises(ValueError):
        N.check(N.lib().lbm_plan_set_stage_wait(plan.handle, 61 * 10 ** 9, 0), "lbm_plan_set_stage_wait")
    name, stencil, method, pattern, n, periodic, bkind, kw = case
    step2, orc2, f2, flags2, ubb2, prev2 = _run_case(case, "float64", monkeypatch)
    res, _ = run_pair(step2, orc2, f2, flags2, ubb2, prev2, 20, pattern, periodic)
    assert step2.sweep_status() == 0
    assert pop_rel_linf(_interior(step2.pdfs), res[1:-1, 1:-1, 1:-1], step2.method.weights) < 1e-12
