"""Sparse (list-based) LBM on the GPU through lbmpy's sparse API (lbmpy_b200.sparse, C ABI
lbm_sparse_*): the sweep against the oracle's restatement of lbmpy's sparse update on lbmpy's own
index arrays (tests/golden/sparse_index.npz), the setter / getter, the sparse UBB, and a porous
medium where the sparse sweep matches the dense sweep on the same walls."""
import os

import numpy as np
import pytest
import torch

import lbmpy_b200 as L
from lbmpy_b200 import sparse as S
from lbmpy_b200.boundaries import NoSlip, UBB
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "sparse_index.npz"))
FLUID, NOSLIP, UBB_FLAG = 1, 2, 4
TOL = {"float64": 1e-12, "float32": 1e-5}


def _method(stencil, method, **kw):
    return L.create_lb_method(lbm_config=L.LBMConfig(stencil=getattr(L.Stencil, stencil),
                                                     method=getattr(L.Method, method.upper()), **kw))


def _rule(stencil, method, **kw):
    cfg = L.LBMConfig(stencil=getattr(L.Stencil, stencil), method=getattr(L.Method, method.upper()), **kw)
    return L.create_lb_collision_rule(lbm_config=cfg)


def _pop_err(got, ref, weights):
    return float(np.abs(got - ref).max() / np.abs(ref + np.asarray(weights)).max())


CASES = [
    ("channel", "D3Q19", "trt", dict(relaxation_rate=1.7, compressible=True, force=(2e-5, 0, 0)), 25),
    ("cavity", "D3Q19", "srt", dict(relaxation_rate=1.6, compressible=True), 20),
    ("periodic27", "D3Q27", "cumulant", dict(relaxation_rate=1.8, compressible=True), 15),
    ("periodic27", "D3Q27", "central_moment", dict(relaxation_rate=1.7, compressible=True), 15),
    ("channel", "D3Q19", "mrt", dict(relaxation_rates=[1.7, 1.5, 1.2, 1.1], compressible=False), 20),
]


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("case,stencil,method,kw,steps", CASES)
def test_sparse_sweep_against_oracle(cuda, case, stencil, method, kw, steps, dtype):
    flags = GOLDEN[f"{case}_flags"]
    rule = _rule(stencil, method, **kw)
    m = rule.method
    mapper = S.SparseLbMapper(list(m.stencil), flags, FLUID, NOSLIP, UBB_FLAG)
    idx = mapper.create_index_array(1)
    np.testing.assert_array_equal(idx, GOLDEN[f"{case}_index"])
    q, n = m.stencil.Q, len(mapper)
    rng = np.random.default_rng(11)
    okind = "central_moment" if method == "central_moment" else method
    orc = O.make(stencil, okind, **kw)
    init = np.stack([orc.equilibrium(1 + 1e-3 * rng.uniform(-1, 1), 1e-2 * rng.uniform(-1, 1, 3))
                     for _ in range(n)])
    tdt = torch.float64 if dtype == "float64" else torch.float32
    init = init.astype(np.float32).astype(np.float64) if dtype == "float32" else init
    f = S.pdf_list(n, q, tdt)
    f.copy_(torch.from_numpy(init).to(tdt))
    d = S.pdf_list(n, q, tdt)
    d.copy_(f)
    kernel = S.create_lb_function_sparse(S.create_lb_update_rule_sparse(rule, "f", "d", "idx"))
    links, u_lid = None, (0.03, 0.01, 0.0)
    ubb = None
    if case == "cavity":
        ubb = S.SparseLbBoundaryMapper(UBB(u_lid), m, "f")
        arr = ubb.create_index_arr(mapper, UBB_FLAG)
        links = np.stack([arr["dir"], arr["nidx0"], arr["nidx1"]], axis=-1)
    for _ in range(steps):
        if ubb is not None:
            ubb(f=f, indexField=arr)
        kernel(f=f, d=d, idx=idx)
        f, d = d, f
    torch.cuda.synchronize()
    ref = orc.sparse_run(init, idx, steps, ubb_links=links, ubb_velocity=u_lid)
    nf = mapper.num_fluid_cells
    got = f.double().cpu().numpy()[:nf]
    err = _pop_err(got, ref[:nf], m.weights)
    assert err < TOL[dtype], f"{err:.3e}"


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_sparse_setter_getter(cuda, dtype):
    m = _method("D3Q19", "trt", relaxation_rate=1.7, compressible=True)
    orc = O.make("D3Q19", "trt", relaxation_rate=1.7, compressible=True)
    n, q = 300, 19
    rng = np.random.default_rng(3)
    rho = 1 + 1e-2 * rng.uniform(-1, 1, n)
    u = 3e-2 * rng.uniform(-1, 1, (n, 3))
    tdt = torch.float64 if dtype == "float64" else torch.float32
    f = S.pdf_list(n, q, tdt)
    S.create_macroscopic_value_setter_sparse(m, "f", rho, u)(f)
    ref = np.stack([orc.equilibrium(r, v) for r, v in zip(rho, u)])
    assert _pop_err(f.double().cpu().numpy(), ref, m.weights) < TOL[dtype]
    vel = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    out = S.create_macroscopic_value_getter_sparse(m, "f", {"density": True, "velocity": vel})(f)
    assert out["velocity"] is vel
    tol = 1e-13 if dtype == "float64" else 1e-6
    assert np.abs(out["density"].cpu().numpy() - rho).max() < tol
    assert np.abs(vel.cpu().numpy() - u).max() < tol


def test_sparse_argument_errors(cuda):
    rule = _rule("D3Q19", "srt", relaxation_rate=1.5)
    kernel = S.create_lb_function_sparse(S.create_lb_update_rule_sparse(rule, "f", "d", "idx"))
    f = S.pdf_list(10, 19)
    idx = np.zeros((10, 18), np.uint32)
    with pytest.raises(ValueError):
        kernel(f=f, d=torch.zeros((10, 19), dtype=torch.float64, device="cuda"), idx=idx)   # AoS list
    with pytest.raises(ValueError):
        kernel(f=f, d=S.pdf_list(10, 19, torch.float32), idx=idx)                          # dtype mismatch
    with pytest.raises(ValueError):
        kernel(f=f, d=f, idx=idx)                                                           # src == dst
    with pytest.raises(NotImplementedError):
        S.create_lb_update_rule_sparse(rule, "f", "d", "idx", kernel_type="collide_only")


def test_porous_medium_sparse_equals_dense(cuda, monkeypatch):
    """40 x 32 x 24 channel with random spheres (about a third of the cells solid), periodic in
    x, walls on the four other faces, force driven, D3Q19 TRT FP32: 200 sparse sweeps over the
    fluid-cell list equal 200 dense sweeps of LatticeBoltzmannStep on the same walls."""
    for var in ("LBM_B200_PAIR", "LBM_B200_QUAD", "LBM_B200_STAGED"):
        monkeypatch.setenv(var, "0")
    n = (40, 32, 24)
    kw = dict(relaxation_rate=1.6, compressible=False, force=(5e-6, 0, 0))
    step = L.LatticeBoltzmannStep(domain_size=n, periodicity=(True, False, False), stencil=L.Stencil.D3Q19,
                                  method=L.Method.TRT, config=L.CreateKernelConfig(data_type="float32"), **kw)
    rng = np.random.default_rng(8)
    ext = tuple(s + 2 for s in n)
    X, Y, Z = np.meshgrid(*[np.arange(s) for s in ext], indexing="ij")
    solid = np.zeros(ext, bool)
    for _ in range(60):
        c = np.array([rng.uniform(6, n[0] - 5), rng.uniform(1, n[1]), rng.uniform(1, n[2])])
        r = rng.uniform(3, 5)
        solid |= (X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 < r * r
    solid[:, 0, :] = solid[:, -1, :] = solid[:, :, 0] = solid[:, :, -1] = True
    solid[0, 1:-1, 1:-1] = solid[-1, 1:-1, 1:-1] = False     # periodic ghost planes
    bh = step.boundary_handling
    bh.set_boundary(NoSlip(), mask_callback=lambda x, y, z: solid[(x + 0.5).astype(int), (y + 0.5).astype(int),
                                                                   (z + 0.5).astype(int)])
    flags = np.zeros(ext, np.uint16)
    flags[1:-1, 1:-1, 1:-1] = FLUID
    flags[solid] = NOSLIP
    assert ((bh.flag_array & 15) == 1).sum() == solid.sum()
    mapper = S.SparseLbMapper(list(step.method.stencil), flags, FLUID, NOSLIP, UBB_FLAG)
    idx = mapper.create_index_array(1)
    nf = mapper.num_fluid_cells
    assert 0.5 * np.prod(n) < nf < 0.8 * np.prod(n)
    step.set_pdf_fields_from_macroscopic_values()
    coords = torch.from_numpy(np.stack([mapper.coordinates[c].astype(np.int64) for c in "xyz"])).cuda()
    f = S.pdf_list(len(mapper), 19, torch.float32)
    f.copy_(step.pdfs[coords[0], coords[1], coords[2]])
    d = S.pdf_list(len(mapper), 19, torch.float32)
    rule = L.create_lb_collision_rule(lbm_config=L.LBMConfig(stencil=L.Stencil.D3Q19, method=L.Method.TRT, **kw))
    kernel = S.create_lb_function_sparse(S.create_lb_update_rule_sparse(rule, "f", "d", "idx"))
    for _ in range(200):
        kernel(f=f, d=d, idx=idx)
        f, d = d, f
    step.run(200)
    dense = step.pdfs[coords[0, :nf], coords[1, :nf], coords[2, :nf]].double().cpu().numpy()
    got = f[:nf].double().cpu().numpy()
    err = _pop_err(got, dense, step.method.weights)
    assert err < 1e-6, f"{err:.3e}"
    u = S.create_macroscopic_value_getter_sparse(step.method, "f", {"velocity": True})(f, num_fluid_cells=nf)
    assert float(u["velocity"][:, 0].mean()) > 0          # the flow runs along the force
