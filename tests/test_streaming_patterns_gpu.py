"""Push, EsoPull and EsoPush sweeps on the GPU against the FP64 oracle (whose accessors are pinned
to lbmpy's in tests/test_streaming_patterns.py): periodic boxes, lid-driven cavities with
compressible and incompressible moving walls, a forced cumulant channel; FP64 and FP32 storage."""
import numpy as np
import pytest

import lbmpy_b200 as L
from tests.test_gpu_parity import _boundaries, _interior, make_pair, run_pair
from tests.helpers import rel_linf

pytestmark = pytest.mark.gpu


def _written_by_fluid(flags, dirs, periodic):
    """[nx, ny, nz, Q]: interior slot (x, q) whose push writer x - c_q is a fluid cell.  A slot
    whose writer is a wall holds whatever it held before (nothing writes it) until the next
    step's bounce-back replaces it, so it takes no part in the comparison."""
    f = flags.copy()
    n = [s - 2 for s in f.shape]
    for ax in range(3):
        if periodic[ax]:
            lo, hi = [slice(None)] * 3, [slice(None)] * 3
            lo[ax], hi[ax] = 0, n[ax]
            f[tuple(lo)] = f[tuple(hi)]
            lo[ax], hi[ax] = n[ax] + 1, 1
            f[tuple(lo)] = f[tuple(hi)]
    out = np.zeros(tuple(n) + (len(dirs),), bool)
    for q, c in enumerate(dirs):
        out[..., q] = f[1 - c[0]:1 - c[0] + n[0], 1 - c[1]:1 - c[1] + n[1], 1 - c[2]:1 - c[2] + n[2]] == 0
    return out

CASES = [
    ("d3q19-trt-periodic", "D3Q19", "trt", (12, 10, 8), (1, 1, 1), None,
     dict(relaxation_rate=1.8, compressible=True)),
    ("d3q19-trt-ldc-comp", "D3Q19", "trt", (10, 12, 8), (0, 0, 0), "ldc",
     dict(relaxation_rate=1.9, compressible=True)),
    ("d3q19-mrt-ldc", "D3Q19", "mrt", (12, 10, 8), (0, 0, 0), "ldc",
     dict(relaxation_rates=[1.7, 1.5, 1.0, 1.0], compressible=False)),
    ("d3q27-cum-channel", "D3Q27", "cumulant", (12, 10, 8), (1, 0, 0), "duct",
     dict(relaxation_rate=1.95, compressible=True, galilean_correction=True, force=(1e-5, 0, 0))),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("pattern", ["push", "esopull", "esopush"])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_pattern_matches_oracle(cuda, case, pattern, dtype, monkeypatch):
    name, stencil, method, n, periodic, bkind, kw = case
    monkeypatch.setenv("LBM_B200_PAIR", "0")
    step, orc, f, flags, ubb, prev = make_pair(stencil, method, n, pattern, dtype, periodic=periodic,
                                               boundaries=_boundaries(bkind), **kw)
    assert step.sweep_variant() == "cell"
    res, par = run_pair(step, orc, f, flags, ubb, prev, 50, pattern, periodic)
    fluid = np.ones(n, bool) if flags is None else (flags[1:-1, 1:-1, 1:-1] == 0)
    got, ref = _interior(step.pdfs), res[1:-1, 1:-1, 1:-1]
    mask = np.broadcast_to(fluid[..., None], got.shape).copy()
    if pattern == "push" and flags is not None:
        mask &= _written_by_fluid(flags, orc.spec.dirs, periodic)
    err = np.abs(got - ref)[mask].max() / np.abs(ref + np.asarray(step.method.weights)).max()
    assert err < (1e-12 if dtype == "float64" else 1e-5), f"{name} {pattern} {dtype}: {err:.3e}"
    rho_o, u_o = orc.get_macroscopic(res, pattern, par)
    assert rel_linf(step.velocity_array[fluid], u_o[fluid]) < (1e-11 if dtype == "float64" else 1e-4)
    assert step.sweep_status() == 0


@pytest.mark.parametrize("pattern", ["push", "esopull", "esopush"])
def test_patterns_need_32_or_64_bit_storage(cuda, pattern):
    with pytest.raises(NotImplementedError):
        L.LatticeBoltzmannStep(domain_size=(8, 8, 8), periodicity=True, stencil=L.Stencil.D3Q19,
                               method=L.Method.TRT, relaxation_rate=1.8, streaming_pattern=pattern,
                               optimization={"storage_dtype": "float16"},
                               config=L.CreateKernelConfig(data_type="float32"))
