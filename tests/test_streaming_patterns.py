"""Streaming patterns beyond pull / AA / EsoTwist: push (two fields) and the in-place EsoPull and
EsoPush (fieldaccess.py:78-87, 184-318), on the CPU oracle.

The oracle's accessor tables are checked against lbmpy's rules evaluated on lbmpy's own
'walberla' and 'lehmann' orderings (tests/golden/stencil_orderings.json, read from the
reference's stencils.py by tests/golden/make_orderings.py), and every pattern must produce the
physics of the pull pattern: lbmpy's advanced-streaming tests hold all patterns to the same
result the same way."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
ORDERINGS = json.load(open(os.path.join(HERE, "golden", "stencil_orderings.json")))


def _reference_table(stencil, pattern, parity, rw):
    """lbmpy's EsoPull / EsoPush accessors (fieldaccess.py:184-318) on the fixture orderings."""
    wal = [tuple(d) for d in ORDERINGS[stencil]["walberla"]]
    leh = [tuple(d) for d in ORDERINGS[stencil]["lehmann"]]
    inv = [wal.index(tuple(-c for c in d)) for d in wal]
    off, slot = [], []
    for i, d in enumerate(wal):
        even = leh.index(d) % 2 == 0
        neg, zero, pos = [-c for c in d], [0, 0, 0], list(d)
        if pattern == "esopull":
            if rw == 0:
                o, s = (neg if even else zero), (i if parity == 0 else inv[i])
            else:
                o, s = (zero if even else pos), (inv[i] if parity == 0 else i)
        else:
            if rw == 0:
                o, s = (zero if even else neg), (inv[i] if parity == 0 else i)
            else:
                o, s = (pos if even else zero), (i if parity == 0 else inv[i])
        off.append(o)
        slot.append(s)
    return np.array(off), np.array(slot)


@pytest.mark.parametrize("stencil", ["D3Q19", "D3Q27"])
@pytest.mark.parametrize("pattern", ["esopull", "esopush"])
def test_eso_accessors_follow_the_lehmann_ordering(stencil, pattern):
    orc = O.make(stencil, "srt", relaxation_rate=1.5)
    assert [list(c) for c in orc.spec.dirs] == ORDERINGS[stencil]["walberla"]
    for parity in (0, 1):
        for rw in (0, 1):
            off, slot = orc.accessor_table(pattern, parity, rw)
            ref_off, ref_slot = _reference_table(stencil, pattern, parity, rw)
            np.testing.assert_array_equal(off, ref_off)
            np.testing.assert_array_equal(slot, ref_slot)


def _ldc_flags(n):
    flags = np.zeros(tuple(s + 2 for s in n), np.uint8)
    flags[0, :, :] = flags[-1, :, :] = 1
    flags[:, 0, :] = 1
    flags[:, :, 0] = flags[:, :, -1] = 1
    flags[1:-1, -1, 1:-1] = 2           # the lid: UBB 0
    return flags


@pytest.mark.parametrize("case", [
    ("D3Q19", "trt", dict(relaxation_rate=1.8, compressible=True), False),
    ("D3Q27", "cumulant", dict(relaxation_rate=1.9, compressible=True, galilean_correction=True), False),
    ("D3Q19", "mrt", dict(relaxation_rates=[1.7, 1.5, 1.0, 1.0], compressible=False), True),
], ids=["d3q19-trt-periodic", "d3q27-cum-periodic", "d3q19-mrt-ldc"])
def test_every_pattern_gives_the_pull_result(case):
    stencil, method, kw, walls = case
    n = (8, 6, 5)
    rng = np.random.default_rng(3)
    u = rng.uniform(-0.02, 0.02, n + (3,))
    rho = 1 + rng.uniform(-1e-3, 1e-3, n)
    periodic = (False,) * 3 if walls else (True,) * 3
    flags = _ldc_flags(n) if walls else None
    out = {}
    for pattern in ("pull", "push", "aa", "esotwist", "esopull", "esopush"):
        orc = O.make(stencil, method, **kw)
        prev = 0 if pattern in ("pull", "push") else 1
        f = orc.new_field(n)
        orc.set_equilibrium(f, rho, u, pattern, prev)
        orc.periodic_sync(f, pattern, prev, periodic)
        res, par = orc.run(f, 12, pattern, prev, periodic=periodic, flags=flags, ubb_velocity=(0.03, 0, 0))
        orc.periodic_sync(res, pattern, par, periodic)
        out[pattern] = orc.get_macroscopic(res, pattern, par)
    rho_p, u_p = out["pull"]
    assert np.abs(u_p).max() > 1e-3
    for pattern, (r, v) in out.items():
        assert np.abs(r - rho_p).max() < 1e-13, pattern
        assert np.abs(v - u_p).max() < 1e-13, pattern
