"""Rows without flagged cells skip their flag loads (the row summary lbm_flags_finalize builds).

An obstacle inside a periodic box mixes flagged and unflagged rows in every plane; results are
held to the FP64 oracle for every sweep variant, and after a second obstacle is added (the step
re-finalizes the flags, which rebuilds the summary).

AA runs end on an even step.  After an odd step the slot (x, i) of a fluid cell x next to a wall
cell w = x - c_i holds whatever w wrote there: nothing for the one-cell sweep and the oracle,
w's own collision for the pair and quad sweeps (which collide a wall cell with its fluid
partner).  No fluid cell uses that value: the next even step replaces it by the bounce-back."""
import numpy as np
import pytest

import lbmpy_b200 as L
from lbmpy_b200.boundaries import NoSlip
from tests.test_gpu_parity import _interior, make_pair, pop_rel_linf, run_pair

pytestmark = pytest.mark.gpu

OBSTACLE = (slice(6, 10), slice(4, 7), slice(3, 6))        # ghost-inclusive x, y, z


@pytest.mark.parametrize("variant", ["cell", "pair", "staged"])
@pytest.mark.parametrize("case", [
    ("D3Q19", "trt", "pull", dict(relaxation_rate=1.8, compressible=True)),
    ("D3Q27", "cumulant", "aa", dict(relaxation_rate=1.95, compressible=True, galilean_correction=True,
                                      force=(1e-5, 0, 0))),
], ids=["d3q19-trt-pull", "d3q27-cum-aa"])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_obstacle_matches_oracle(cuda, case, dtype, variant, monkeypatch):
    stencil, method, pattern, kw = case
    if variant == "pair" and dtype == "float64":
        pytest.skip("no FP64 pair sweep")
    monkeypatch.setenv("LBM_B200_PAIR", "1" if variant == "pair" else "0")
    monkeypatch.setenv("LBM_B200_STAGED", "1" if variant == "staged" else "0")
    n = (16, 10, 8)
    step, orc, f, flags, ubb, prev = make_pair(stencil, method, n, pattern, dtype, periodic=(1, 1, 1),
                                               boundaries=[(NoSlip(), OBSTACLE)], **kw)
    assert step.sweep_variant() == variant
    res, _ = run_pair(step, orc, f, flags, ubb, prev, 61 if pattern == "aa" else 60, pattern, (1, 1, 1))
    fluid = flags[1:-1, 1:-1, 1:-1] == 0
    err = pop_rel_linf(_interior(step.pdfs)[fluid], res[1:-1, 1:-1, 1:-1][fluid], step.method.weights)
    assert err < (1e-12 if dtype == "float64" else 1e-5), err


def test_adding_an_obstacle_rebuilds_the_row_summary(cuda, monkeypatch):
    monkeypatch.setenv("LBM_B200_PAIR", "0")
    n = (16, 10, 8)
    kw = dict(relaxation_rate=1.8, compressible=True)
    step, orc, f, flags, ubb, prev = make_pair("D3Q19", "trt", n, "pull", "float64", periodic=(1, 1, 1),
                                               boundaries=[(NoSlip(), OBSTACLE)], **kw)
    res, _ = run_pair(step, orc, f, flags, ubb, prev, 30, "pull", (1, 1, 1))
    # a second obstacle: rows that had no flagged cell get walls and near-wall cells
    bh = step.boundary_handling
    bh.set_boundary(NoSlip(), (slice(2, 5), slice(7, 10), slice(5, 8)))
    flags2 = (bh.flag_array & 7).astype(np.uint8)
    step.run(30)
    res2, _ = orc.run(res, 30, "pull", 0, periodic=(1, 1, 1), flags=flags2, ubb_velocity=ubb)
    orc.periodic_sync(res2, "pull", 0, (1, 1, 1))
    fluid = (flags[1:-1, 1:-1, 1:-1] == 0) & (flags2[1:-1, 1:-1, 1:-1] == 0)
    err = pop_rel_linf(_interior(step.pdfs)[fluid], res2[1:-1, 1:-1, 1:-1][fluid], step.method.weights)
    assert err < 1e-12, err
