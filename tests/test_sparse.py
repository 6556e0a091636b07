"""Sparse (list-based) LBM on the host: the cell list and pull index against lbmpy's own
SparseLbMapper output (tests/golden/sparse_index.npz, written by tests/golden/make_sparse.py), and
the oracle's sparse update (lbmpy's update_rule_sparse) against the dense oracle on the same
geometry — lbmpy's sparse notebook test compares the sparse channel with the dense one."""
import os

import numpy as np
import pytest

import lbmpy_b200 as L
from lbmpy_b200.boundaries import UBB
from lbmpy_b200.sparse import NOT_FOUND, SparseLbBoundaryMapper, SparseLbMapper
from oracle import oracle as O

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "sparse_index.npz"))
FLUID, NOSLIP, UBB_FLAG = 1, 2, 4
CASES = {"channel": "D3Q19", "cavity": "D3Q19", "periodic27": "D3Q27"}


def _stencil(name):
    m = L.create_lb_method(lbm_config=L.LBMConfig(stencil=getattr(L.Stencil, name), method=L.Method.SRT,
                                                  relaxation_rate=1.5))
    return [tuple(int(v) for v in d) for d in m.stencil]


def _mapper(case):
    return SparseLbMapper(_stencil(CASES[case]), GOLDEN[f"{case}_flags"], FLUID, NOSLIP, UBB_FLAG)


@pytest.mark.parametrize("case", sorted(CASES))
def test_index_array_matches_lbmpy(case):
    m = _mapper(case)
    assert m.num_fluid_cells == int(GOLDEN[f"{case}_num_fluid"])
    coords = np.stack([m.coordinates[c] for c in ("x", "y", "z")], axis=-1)
    np.testing.assert_array_equal(coords, GOLDEN[f"{case}_coords"])
    idx = m.create_index_array(1)
    assert idx.dtype == np.uint32 and idx.shape == GOLDEN[f"{case}_index"].shape
    np.testing.assert_array_equal(idx, GOLDEN[f"{case}_index"])


def test_cell_lookup():
    m = _mapper("cavity")
    for k in (0, 7, m.num_fluid_cells, len(m) - 1):
        c = m.coordinate(k)
        assert m.cell_idx((c["x"], c["y"], c["z"])) == k
    with pytest.raises(IndexError):
        m.cell_idx((0, 0, 0))                         # a NoSlip cell is not listed
    bulk = m.cell_idx_bulk(m.coordinates[:5])
    np.testing.assert_array_equal(bulk, np.arange(5))
    probe = np.zeros(2, dtype=m.coordinates.dtype)
    probe[1] = m.coordinates[3]
    np.testing.assert_array_equal(m.cell_idx_bulk(probe), [NOT_FOUND, 3])


def test_missing_neighbour_raises():
    """A fluid cell next to an unflagged cell that is no periodic image: lbmpy raises ValueError."""
    flags = np.zeros((6, 6, 6), dtype=np.uint16)
    flags[1:-1, 1:-1, 1:-1] = FLUID
    flags[2, 2, 2] = 0                                 # a hole inside the domain
    m = SparseLbMapper(_stencil("D3Q19"), flags, FLUID, NOSLIP, UBB_FLAG)
    with pytest.raises(ValueError):
        m.create_index_array(1)


def _lists_from_dense(f, coords):
    return np.stack([f[x, y, z] for x, y, z in coords])


def _dense_flags(flags):
    out = np.zeros(flags.shape, np.uint8)
    out[(flags & NOSLIP) != 0] = 1
    out[(flags & UBB_FLAG) != 0] = 2
    return out


@pytest.mark.parametrize("case,method,kw,periodic,steps", [
    ("channel", "trt", dict(relaxation_rate=1.7, compressible=True, force=(2e-5, 0, 0)), (True, False, True), 25),
    ("cavity", "srt", dict(relaxation_rate=1.6, compressible=True), (False, False, False), 20),
    ("periodic27", "cumulant", dict(relaxation_rate=1.8, compressible=True), (True, True, True), 15),
])
def test_oracle_sparse_update_equals_dense(case, method, kw, periodic, steps):
    """The oracle's sparse stream-pull-collide (plus the sparse UBB) reproduces the dense oracle with
    the same walls: the index array streams, bounces back and wraps as the dense grid does."""
    stencil = CASES[case]
    flags = GOLDEN[f"{case}_flags"]
    m = _mapper(case)
    idx = m.create_index_array(1)
    n = tuple(s - 2 for s in flags.shape)
    orc = O.make(stencil, method, **kw)
    rng = np.random.default_rng(5)
    f = orc.new_field(n)
    orc.set_equilibrium(f, 1 + 1e-3 * rng.uniform(-1, 1, n), 1e-2 * rng.uniform(-1, 1, n + (3,)))
    orc.periodic_sync(f, "pull", 0, periodic)
    coords = [tuple(int(v) for v in (c["x"], c["y"], c["z"])) for c in m.coordinates]
    lst = _lists_from_dense(f, coords)
    links = None
    u_lid = (0.03, 0.01, 0.0)
    if case == "cavity":
        mapper = SparseLbBoundaryMapper(UBB(u_lid), L.create_lb_method(lbm_config=L.LBMConfig(
            stencil=L.Stencil.D3Q19, method=L.Method.SRT, relaxation_rate=1.6, compressible=True)))
        arr = mapper.create_index_arr(m, UBB_FLAG)
        links = np.stack([arr["dir"], arr["nidx0"], arr["nidx1"]], axis=-1)
    res_s = orc.sparse_run(lst, idx, steps, ubb_links=links, ubb_velocity=u_lid)
    res_d, _ = orc.run(f, steps, "pull", 0, periodic=periodic, flags=_dense_flags(flags), ubb_velocity=u_lid)
    ref = _lists_from_dense(res_d, coords[:m.num_fluid_cells])
    got = res_s[:m.num_fluid_cells]
    assert np.abs(got - ref).max() < 1e-13          # zero-centred populations, |f~| < 0.4


def test_ubb_links_of_the_cavity_lid():
    m = _mapper("cavity")
    method = L.create_lb_method(lbm_config=L.LBMConfig(stencil=L.Stencil.D3Q19, method=L.Method.SRT,
                                                       relaxation_rate=1.6))
    arr = SparseLbBoundaryMapper(UBB((0.05, 0, 0)), method).create_index_arr(m, UBB_FLAG)
    st = _stencil("D3Q19")
    # every fluid cell of the top layer links to the lid in the 5 directions with c_z = +1
    top = sum(1 for c in m.fluid_coordinates if c["z"] == 5)
    assert top == 25 and len(arr) == 5 * top
    for rec in arr:
        c, b = m.coordinate(rec["nidx0"]), m.coordinate(rec["nidx1"])
        d = st[rec["dir"]]
        assert (int(b["x"]) - int(c["x"]), int(b["y"]) - int(c["y"]), int(b["z"]) - int(c["z"])) == d
        assert GOLDEN["cavity_flags"][b["x"], b["y"], b["z"]] & UBB_FLAG
    with pytest.raises(NotImplementedError):
        SparseLbBoundaryMapper(UBB(lambda *a: None, dim=3), method)
