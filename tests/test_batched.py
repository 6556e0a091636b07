"""Batched domains: one persistent launch per step over many independent fields of uneven size.

Every domain of a batch must evolve exactly as the same domain run alone through
LatticeBoltzmannStep (itself held to the oracle in test_gpu_parity.py), and an FP64 batch is
compared with the oracle directly.  Tiling, CUDA-graph replay and autotuning must not change
results.
"""
import ctypes

import numpy as np
import pytest
import sympy as sp
import torch

import lbmpy_b200 as L
from lbmpy_b200 import _native as N
from lbmpy_b200.batched import LatticeBoltzmannBatch, Tiling, lid_driven_cavity_batch
from lbmpy_b200.boundaries import NoSlip, UBB, slice_from_direction
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SIZES = [(16, 24, 8), (10, 12, 14), (24, 16, 16), (8, 8, 8), (18, 10, 12)]
RATES = [(1.6, 1.5), (1.9, 1.7), (1.75, 1.55), (1.5, 1.95), (1.85, 1.6)]


def _interior(t):
    return t[1:-1, 1:-1, 1:-1].detach().cpu().double().numpy()


def _ldc(bh, lid=0.05):
    bh.set_boundary(UBB((lid, 0.0, 0.0)), slice_from_direction("N", 3))
    for d in ("W", "E", "S", "T", "B"):
        bh.set_boundary(NoSlip(), slice_from_direction(d, 3))


def _mrt_batch(dtype, pattern="pull", tiling=Tiling(), **kw):
    ws, wb = sp.Symbol("omega_shear"), sp.Symbol("omega_bulk")
    cfg = L.LBMConfig(stencil=L.Stencil.D3Q19, method=L.Method.MRT, relaxation_rates=[ws, wb, 1, 1],
                      compressible=False, streaming_pattern=pattern)
    b = LatticeBoltzmannBatch(SIZES, kernel_params=[{"omega_shear": a, "omega_bulk": c} for a, c in RATES],
                              lbm_config=cfg, config=L.CreateKernelConfig(data_type=dtype), tiling=tiling, **kw)
    for k in range(len(SIZES)):
        _ldc(b.boundary_handling(k))
    return b


def _scale(weights):
    return 1.0 + max(weights)


@pytest.mark.parametrize("graph", [True, False])
def test_mrt_cavities_match_single_domain_runs(cuda, graph, monkeypatch):
    monkeypatch.setenv("LBM_B200_PAIR", "0")     # the one-cell-per-thread sweep, as the batch uses
    steps = 40
    b = _mrt_batch("float32", use_cuda_graph=graph)
    b.run(steps)
    torch.cuda.synchronize()
    for k, (size, (ws, wb)) in enumerate(zip(SIZES, RATES)):
        s = L.LatticeBoltzmannStep(domain_size=size, periodicity=False, stencil=L.Stencil.D3Q19,
                                   method=L.Method.MRT, relaxation_rates=[ws, wb, 1, 1], compressible=False,
                                   config=L.CreateKernelConfig(data_type="float32"))
        _ldc(s.boundary_handling)
        s.run(steps)
        got, ref = _interior(b.pdfs(k)), _interior(s.pdfs)
        err = np.abs(got - ref).max() / _scale(s.method.weights)
        assert err <= 1e-6, f"domain {k} {size}: {err:.3e}"
        rho, u = b.macroscopic_values(k)
        assert np.abs(u.cpu().numpy() - s.velocity_array).max() < 1e-6
        assert np.abs(s.velocity_array).max() > 1e-3      # the lid has set the fluid moving


def test_fp64_batch_matches_oracle(cuda):
    steps = 30
    b = _mrt_batch("float64")
    b.run(steps)
    torch.cuda.synchronize()
    for k in (0, 1, 4):
        ws, wb = RATES[k]
        orc = O.make("D3Q19", "mrt", relaxation_rates=[ws, wb, 1.0, 1.0], compressible=False)
        f = orc.new_field(SIZES[k])
        orc.set_equilibrium(f, np.ones(SIZES[k]), np.zeros(SIZES[k] + (3,)))
        flags = (b._handlings[k].flag_array & 7).astype(np.uint8)
        res, _ = orc.run(f, steps, "pull", 0, periodic=(False,) * 3, flags=flags, ubb_velocity=(0.05, 0.0, 0.0))
        fluid = flags[1:-1, 1:-1, 1:-1] == 0
        got = _interior(b.pdfs(k))[fluid]
        ref = res[1:-1, 1:-1, 1:-1][fluid]
        assert np.abs(got - ref).max() / _scale(b.method.weights) < 1e-12, k


def test_cumulant_aa_channels_with_per_domain_periodicity(cuda, monkeypatch):
    """In-place AA streaming, D3Q27 cumulant, a body force, and periodicity set per domain."""
    monkeypatch.setenv("LBM_B200_PAIR", "0")
    sizes = [(16, 10, 8), (12, 14, 10), (20, 8, 12)]
    periodic = [(True, False, False), (True, False, True), (False, False, False)]
    kw = dict(stencil=L.Stencil.D3Q27, method=L.Method.CUMULANT, relaxation_rate=1.95, compressible=True,
              galilean_correction=True, force=(1e-5, 0, 0), streaming_pattern="aa")
    b = LatticeBoltzmannBatch(sizes, periodicity=periodic, config=L.CreateKernelConfig(data_type="float32"),
                              tiling=Tiling(16, 8, 2, 4), **kw)
    rng = np.random.default_rng(4)
    us = [torch.tensor(rng.uniform(-0.02, 0.02, s + (3,)), device="cuda") for s in sizes]
    walls = [("N", "S"), ("N", "S"), ("N", "S", "W", "E", "T", "B")]
    for k in range(3):
        b.set_pdf_fields_from_macroscopic_values(k, 1.0, us[k])
        for d in walls[k]:
            b.boundary_handling(k).set_boundary(NoSlip(), slice_from_direction(d, 3))
    b.run(9)
    torch.cuda.synchronize()
    for k, size in enumerate(sizes):
        s = L.LatticeBoltzmannStep(domain_size=size, periodicity=periodic[k],
                                   config=L.CreateKernelConfig(data_type="float32"), **kw)
        for d in walls[k]:
            s.boundary_handling.set_boundary(NoSlip(), slice_from_direction(d, 3))
        s.velocity_array[...] = us[k].cpu().numpy()
        s.set_pdf_fields_from_macroscopic_values()
        s.run(9)
        got, ref = _interior(b.pdfs(k)), _interior(s.pdfs)
        assert np.abs(got - ref).max() / _scale(s.method.weights) <= 1e-6, k
        assert b.previous_timestep == s.previous_timestep


@pytest.mark.parametrize("pattern", ["pull", "aa"])
def test_tilings_agree_and_autotune_keeps_state(cuda, pattern):
    ref = _mrt_batch("float32", pattern, Tiling(32, 8, 1, 0))
    ref.run(6)
    before = ref._buf[0].clone()
    cands = (Tiling(16, 16, 1, 0), Tiling(32, 4, 4, 16), Tiling(8, 8, 3, 2))
    best = ref.autotune(cands, sweeps=2, repeats=1)
    assert best in cands and len(ref.tuning) == 3
    assert torch.equal(ref._buf[0], before)           # tuning left the state as it was
    ref.run(7)
    for t in cands:
        other = _mrt_batch("float32", pattern, t)
        other.run(13)
        for k in range(len(SIZES)):
            assert torch.equal(other.pdfs(k), ref.pdfs(k)), (t, k)


def test_cavity_batch_builder_and_info(cuda):
    b = lid_driven_cavity_batch(12, seed=3, edges=(8, 16, 24), tiling=Tiling(16, 8, 1, 2))
    info = b.info()
    assert info["cells"] == b.number_of_cells
    assert info["blocks"] <= 2 * torch.cuda.get_device_properties(0).multi_processor_count
    assert info["thread_slots"] >= info["cells"]
    b.run(20)
    torch.cuda.synchronize()
    rates = {tuple(p.values()) for p in b.kernel_params}
    assert len(rates) == 12 and all(1.5 <= v <= 1.95 for r in rates for v in r)
    _, u = b.macroscopic_values(0)
    assert torch.isfinite(u).all() and u[..., 0].abs().max() > 1e-3


def _raw_create(common, domains, a, bb, elems, flags=None, flag_bytes=0, tiling=(32, 8, 1, 0)):
    t = N.LbmBatchTiling(*tiling)
    h = ctypes.c_void_p()
    rc = N.lib().lbm_batch_create(ctypes.byref(common), domains, len(domains), ctypes.c_void_p(a),
                                  ctypes.c_void_p(bb), elems, ctypes.c_void_p(flags), flag_bytes, ctypes.byref(t),
                                  ctypes.byref(h))
    if rc == 0:
        N.lib().lbm_batch_destroy(h)
    return rc


def test_batch_rejects_bad_layouts(cuda):
    common = N.LbmPlanDesc()
    common.stencil, common.method, common.store_dtype = 19, N.METHOD_TRT, N.DTYPE_F32
    common.rates[0], common.rates[1] = 1.8, 1.0
    n, q = 6, 19
    ex = n + 2
    strides = (1, ex, ex * ex, ex ** 3)
    extent = (q - 1) * strides[3] + (ex - 1) * (strides[2] + strides[1]) + ex
    doms = (N.LbmDomainDesc * 2)()
    for k in range(2):
        for i in range(3):
            doms[k].dims[i] = n
        for i in range(4):
            doms[k].strides[i] = strides[i]
        doms[k].rates[0], doms[k].rates[1] = 1.8, 1.0
        doms[k].flags_offset = -1
        doms[k].offset = k * extent
    a = torch.zeros(2 * extent, device="cuda")
    bb = torch.zeros(2 * extent, device="cuda")
    assert _raw_create(common, doms, a.data_ptr(), bb.data_ptr(), 2 * extent) == N.LBM_OK
    doms[1].offset = extent - 5                                        # overlaps domain 0
    assert _raw_create(common, doms, a.data_ptr(), bb.data_ptr(), 2 * extent) == N.LBM_E_INVALID
    doms[1].offset = extent + 1                                        # runs past the buffer
    assert _raw_create(common, doms, a.data_ptr(), bb.data_ptr(), 2 * extent) == N.LBM_E_INVALID
    doms[1].offset = extent
    doms[1].flags_offset = 0                                           # flags but no flag buffer
    assert _raw_create(common, doms, a.data_ptr(), bb.data_ptr(), 2 * extent) == N.LBM_E_INVALID
    doms[1].flags_offset = -1
    assert _raw_create(common, doms, a.data_ptr(), a.data_ptr(), 2 * extent) == N.LBM_E_INVALID  # pull, one buffer
    host = np.zeros(2 * extent, dtype=np.float32)
    assert _raw_create(common, doms, host.ctypes.data, bb.data_ptr(), 2 * extent) == N.LBM_E_INVALID
    assert _raw_create(common, doms, a.data_ptr(), bb.data_ptr(), 2 * extent,
                       tiling=(32, 16, 1, 0)) == N.LBM_E_INVALID     # 512 threads per block
