"""The D3Q27 central-moment sweep (collide_cm) against the FP64 oracle's generic restatement:
periodic boxes and walled channels, Guo / Luo / Simple forcing, pull and AA, FP64 and FP32."""
import numpy as np
import pytest

import lbmpy_b200 as L
from tests.test_gpu_parity import _boundaries, _interior, make_pair, pop_rel_linf, run_pair

pytestmark = pytest.mark.gpu

CASES = [
    ("periodic-unforced", "pull", (10, 8, 6), (1, 1, 1), None, dict(relaxation_rate=1.8)),
    ("periodic-guo", "aa", (10, 8, 6), (1, 1, 1), None, dict(relaxation_rate=1.9, force=(1e-5, -2e-6, 3e-6))),
    ("channel-luo", "pull", (12, 8, 8), (1, 0, 0), "duct",
     dict(relaxation_rate=1.7, force=(2e-5, 0, 0), force_model="luo")),
    ("channel-simple-aa", "aa", (12, 8, 8), (1, 0, 0), "duct",
     dict(relaxation_rate=1.6, force=(2e-5, 0, 0), force_model="simple")),
    ("ldc-rates", "pull", (10, 10, 8), (0, 0, 0), "ldc",
     dict(relaxation_rates=[1.8, 1.4, 1.2, 1.1, 1.0, 1.05, 1.0, 1.0, 1.0, 1.0])),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_central_moment_sweep_matches_oracle(cuda, case, dtype):
    name, pattern, n, periodic, bkind, kw = case
    step, orc, f, flags, ubb, prev = make_pair("D3Q27", "central_moment", n, pattern, dtype,
                                               periodic=periodic, boundaries=_boundaries(bkind),
                                               compressible=True, **kw)
    steps = 40 if pattern == "pull" else 41
    res, par = run_pair(step, orc, f, flags, ubb, prev, steps, pattern, periodic)
    fluid = np.ones(n, bool) if flags is None else (flags[1:-1, 1:-1, 1:-1] == 0)
    err = pop_rel_linf(_interior(step.pdfs)[fluid], res[1:-1, 1:-1, 1:-1][fluid], step.method.weights)
    assert err < (1e-12 if dtype == "float64" else 1e-5), f"{name} {dtype}: {err:.3e}"
