"""Parity of the CUDA sweep (through the C ABI, via the lbmpy-compatible API) with the CPU oracle.

Bars (all against the FP64 oracle): FP64 storage 1e-12 relative L-infinity of the populations
after 100 steps, FP32 storage 1e-5 -- relative to the largest population f = f~ + w_i; the stored
zero-centred values f~ are also held to 1e-9 (FP64) relative to their own maximum; 16-bit storage:
relative L2 velocity error against the FP64 oracle (1e-3 for FP16).
"""
import numpy as np
import pytest
import torch

import lbmpy_b200 as L
from lbmpy_b200.boundaries import NoSlip, UBB, slice_from_direction
from oracle import oracle as O
from tests.helpers import random_velocity, rel_linf, tgv_velocity

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-5


def _interior(t):
    return t[1:-1, 1:-1, 1:-1].detach().cpu().double().numpy()


def pop_rel_linf(got, ref, weights):
    """Relative L-infinity error of the populations f = f~ + w (lbmpy's absolute PDFs)."""
    w = np.asarray(weights)
    return float(np.abs(got - ref).max() / np.abs(ref + w).max())


def make_pair(stencil, method, n, pattern="pull", dtype="float64", storage=None, periodic=(True, True, True),
              boundaries=None, u=None, rho=None, **method_kw):
    """Same initial state on a LatticeBoltzmannStep (GPU) and on the oracle."""
    cfg = dict(stencil=getattr(L.Stencil, stencil), method=getattr(L.Method, method.upper()),
               streaming_pattern=pattern, **method_kw)
    opt = {"storage_dtype": storage} if storage else {}
    step = L.LatticeBoltzmannStep(domain_size=n, periodicity=periodic, optimization=opt,
                                  config=L.CreateKernelConfig(data_type=dtype), **cfg)
    if boundaries:
        for obj, sl in boundaries:
            step.boundary_handling.set_boundary(obj, sl)
    if u is None:
        u = random_velocity(n, 1e-2, seed=1)
    if rho is None:
        rho = 1.0 + 1e-3 * np.random.default_rng(2).uniform(-1, 1, n)
    step.velocity_array[...] = u
    step.density_array[...] = rho
    step.set_pdf_fields_from_macroscopic_values()

    okw = {k: v for k, v in method_kw.items() if k in ("relaxation_rate", "relaxation_rates", "compressible",
                                                       "galilean_correction", "force", "force_model",
                                                       "fourth_order_correction")}
    if "subgrid_scale_model" in method_kw:
        sgs = method_kw["subgrid_scale_model"]
        okw["smagorinsky"] = sgs[1] if isinstance(sgs, tuple) else True
    if isinstance(okw.get("force_model"), str):
        okw["force_model"] = okw["force_model"]
    orc = O.make(stencil, method, **okw)
    f = orc.new_field(n)
    prev = 1 if pattern != "pull" else 0
    orc.set_equilibrium(f, rho, u, pattern, prev)
    # the oracle keeps values written across a periodic face in the ghost layer until its next
    # communication step; the GPU writes them to the periodic image directly
    orc.periodic_sync(f, pattern, prev, periodic)
    flags = None
    if boundaries:
        flags = (step.boundary_handling.flag_array & 7).astype(np.uint8)
    ubb = step.boundary_handling.ubb_velocities
    return step, orc, f, flags, (ubb[0] if ubb else (0.0, 0.0, 0.0)), prev


def run_pair(step, orc, f, flags, ubb, prev, steps, pattern, periodic):
    """Runs both; returns the oracle field (periodic write-backs applied) and its last parity."""
    step.run(steps)
    res, par = orc.run(f, steps, pattern, prev, periodic=periodic, flags=flags, ubb_velocity=ubb)
    orc.periodic_sync(res, pattern, par, periodic)
    return res, par


CASES = [
    # id, stencil, method, pattern, n, periodic, boundaries, kwargs
    ("d3q19-trt-pull-tgv", "D3Q19", "trt", "pull", (16, 16, 8), (1, 1, 1), None,
     dict(relaxation_rate=1.8, compressible=True)),
    ("d3q19-srt-pull-guo", "D3Q19", "srt", "pull", (12, 10, 8), (1, 1, 1), None,
     dict(relaxation_rate=1.6, compressible=False, force=(1e-5, -2e-6, 3e-6))),
    ("d3q19-mrt-pull-ldc", "D3Q19", "mrt", "pull", (12, 10, 8), (0, 0, 0), "ldc",
     dict(relaxation_rates=[1.7, 1.5, 1.0, 1.0], compressible=False)),
    ("d3q19-trt-aa-ldc-comp", "D3Q19", "trt", "aa", (10, 12, 8), (0, 0, 0), "ldc",
     dict(relaxation_rate=1.9, compressible=True)),
    ("d3q19-trt-esotwist", "D3Q19", "trt", "esotwist", (12, 10, 8), (1, 1, 1), None,
     dict(relaxation_rate=1.7, compressible=True)),
    ("d3q19-trt-pull-smag-guo", "D3Q19", "trt", "pull", (12, 10, 8), (1, 1, 1), None,
     dict(relaxation_rate=1.95, compressible=True, force=(2e-5, 0, 0),
          subgrid_scale_model=(L.SubgridScaleModel.SMAGORINSKY, 0.14))),
    ("d3q27-trt-aa", "D3Q27", "trt", "aa", (12, 10, 8), (1, 1, 1), None,
     dict(relaxation_rate=1.8, compressible=True)),
    ("d3q27-mrt-pull", "D3Q27", "mrt", "pull", (10, 8, 8), (1, 1, 1), None,
     dict(relaxation_rates=[1.8, 1.4, 1.1, 1.2, 1.0, 1.0], compressible=True)),
    ("d3q27-cum-aa-channel", "D3Q27", "cumulant", "aa", (12, 10, 8), (1, 0, 0), "duct",
     dict(relaxation_rate=1.95, compressible=True, galilean_correction=True, force=(1e-5, 0, 0))),
    ("d3q27-cum-pull-smag", "D3Q27", "cumulant", "pull", (10, 10, 8), (1, 1, 1), None,
     dict(relaxation_rate=1.99, compressible=True, subgrid_scale_model=(L.SubgridScaleModel.SMAGORINSKY, 0.1))),
    ("d3q27-cum-esotwist-ldc", "D3Q27", "cumulant", "esotwist", (10, 10, 8), (0, 0, 0), "ldc",
     dict(relaxation_rate=1.9, compressible=True, galilean_correction=True)),
]


def _boundaries(kind):
    if kind == "ldc":
        b = [(UBB((0.02, 0.0, 0.0)), slice_from_direction("N", 3))]
        b += [(NoSlip(), slice_from_direction(d, 3)) for d in ("W", "E", "S", "T", "B")]
        return b
    if kind == "duct":
        return [(NoSlip(), slice_from_direction(d, 3)) for d in ("N", "S", "T", "B")]
    return None


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("dtype,kernel", [("float64", "cell"), ("float32", "pair"), ("float32", "cell"),
                                          ("float32", "zpipe")])
def test_sweep_parity(cuda, case, dtype, kernel, monkeypatch):
    """kernel='pair': two cells per thread with packed FP32x2 arithmetic (the default for even nx);
    kernel='cell': one cell per thread (forced with LBM_B200_PAIR=0); kernel='zpipe': columns of
    3 cells along z per thread with the next cell's loads in flight (D3Q27 cumulant FP32 only;
    the other methods fall back to the one-cell sweep)."""
    name, stencil, method, pattern, n, periodic, bkind, kw = case
    monkeypatch.setenv("LBM_B200_PAIR", "1" if kernel == "pair" else "0")
    if kernel == "zpipe":
        monkeypatch.setenv("LBM_B200_ZPIPE", "3")
    if dtype == "float32" and stencil == "D3Q27" and method == "mrt" and pattern not in ("pull", "aa"):
        pytest.skip("not built")
    steps = 100
    step, orc, f, flags, ubb, prev = make_pair(stencil, method, n, pattern, dtype, periodic=periodic,
                                               boundaries=_boundaries(bkind), **kw)
    if kernel == "zpipe" and method == "cumulant" and pattern in ("pull", "aa"):
        assert step.sweep_variant() == "zpipe"
    # the setter first
    fluid0 = np.ones(n, bool) if bkind is None else \
        ((step.boundary_handling.flag_array & 7)[1:-1, 1:-1, 1:-1] == 0)
    w = step.method.weights
    assert pop_rel_linf(_interior(step.pdfs)[fluid0], f[1:-1, 1:-1, 1:-1][fluid0], w) < \
        (FP64_TOL if dtype == "float64" else 1e-7)
    res, par = run_pair(step, orc, f, flags, ubb, prev, steps, pattern, periodic)
    got = _interior(step.pdfs)
    ref = res[1:-1, 1:-1, 1:-1]
    fluid = np.ones(n, bool) if flags is None else (flags[1:-1, 1:-1, 1:-1] == 0)
    err = pop_rel_linf(got[fluid], ref[fluid], w)
    tol = FP64_TOL if dtype == "float64" else FP32_TOL
    assert err < tol, f"{name} {dtype}: relative L-inf error {err:.3e} >= {tol}"
    if dtype == "float64":
        zc = rel_linf(got[fluid], ref[fluid])
        assert zc < 1e-9, f"{name}: zero-centred relative error {zc:.3e}"
    # macroscopic values through both getters
    rho_o, u_o = orc.get_macroscopic(res, pattern, par)
    assert rel_linf(step.velocity_array[fluid], u_o[fluid]) < (1e-11 if dtype == "float64" else 1e-4)


@pytest.mark.parametrize("storage,bound", [("float16", 1e-3), ("bfloat16", 5e-3), ("e3m12", 2.5e-4)])
@pytest.mark.parametrize("kernel", ["quad", "pair", "cell"])
def test_low_precision_storage_l2_velocity(cuda, storage, bound, kernel, monkeypatch):
    """Zero-centred 16-bit storage with FP32 collision vs the FP64 oracle (TGV + noise).
    FP16 meets the 1e-3 bar; BF16's 8-bit mantissa leaves a few 1e-3; e3m12's two extra mantissa
    bits cut FP16's error by about four (bound stated per type)."""
    monkeypatch.setenv("LBM_B200_PAIR", "1" if kernel == "pair" else "0")
    monkeypatch.setenv("LBM_B200_QUAD", "1" if kernel == "quad" else "0")
    n = (32, 32, 16)
    u = tgv_velocity(n, 0.04, noise=1e-3, seed=0)
    rho = np.ones(n)
    step, orc, f, flags, ubb, prev = make_pair("D3Q19", "trt", n, "pull", "float32", storage=storage,
                                               u=u, rho=rho, relaxation_rate=1.8, compressible=True)
    res, _ = run_pair(step, orc, f, flags, ubb, prev, 200, "pull", (1, 1, 1))
    _, u_ref = orc.get_macroscopic(res)
    err = np.linalg.norm(step.velocity_array - u_ref) / np.linalg.norm(u_ref)
    assert err <= bound, f"{storage}: relative L2 velocity error {err:.3e}"


def test_conserved_reduction_matches_oracle(cuda):
    n = (16, 12, 10)
    step, orc, f, flags, ubb, prev = make_pair("D3Q19", "trt", n, "pull", "float64", relaxation_rate=1.8,
                                               compressible=True, force=(1e-5, 0, 0))
    red0 = step.reduce_conserved()
    ref0 = orc.reduce(f)
    np.testing.assert_allclose(red0, ref0, rtol=1e-12, atol=1e-15)
    res, _ = run_pair(step, orc, f, flags, ubb, prev, 20, "pull", (1, 1, 1))
    red = step.reduce_conserved()
    np.testing.assert_allclose(red, orc.reduce(res), rtol=1e-11, atol=1e-14)
    # mass conserved; momentum grows by F per cell and step
    assert abs(red[0] - red0[0]) < 1e-10 * red0[0]
    ncell = np.prod(n)
    assert abs((red[1] - red0[1]) - 20 * 1e-5 * ncell) < 1e-9


def test_getter_setter_round_trip(cuda):
    """set -> get returns the prescribed fields (tests/test_macroscopic_value_kernels.py:13-56)."""
    n = (8, 6, 4)
    for method, kw in (("trt", dict(relaxation_rate=1.8, compressible=True, force=(1e-4, 2e-4, 0))),
                       ("mrt", dict(relaxation_rates=[1.7, 1.5, 1.0, 1.0], compressible=False)),
                       ("cumulant", dict(relaxation_rate=1.9, compressible=True, force=(1e-4, 0, 1e-4)))):
        for pattern in ("pull", "aa", "esotwist"):
            stencil = "D3Q27" if method == "cumulant" else "D3Q19"
            cfg = L.LBMConfig(stencil=getattr(L.Stencil, stencil), method=getattr(L.Method, method.upper()), **kw)
            m = L.create_lb_method(cfg)
            pdfs = L.create_pdf_array(n, m.stencil.Q)
            u = torch.tensor(random_velocity(n, 0.02, seed=3), device="cuda")
            rho = 1 + 0.01 * torch.rand(n, dtype=torch.float64, device="cuda")
            for prev in (L.Timestep.EVEN, L.Timestep.ODD) if pattern != "pull" else (L.Timestep.BOTH,):
                L.macroscopic_values_setter(m, rho, u, pdfs, pattern, prev)
                r2 = torch.empty_like(rho)
                u2 = torch.empty_like(u)
                L.macroscopic_values_getter(m, r2, u2, pdfs, pattern, prev)
                assert torch.allclose(r2, rho, rtol=0, atol=1e-14), (method, pattern, prev)
                assert torch.allclose(u2, u, rtol=0, atol=1e-14), (method, pattern, prev)


def test_host_side_errors(cuda):
    cfg = L.LBMConfig(stencil=L.Stencil.D3Q19, method=L.Method.TRT, relaxation_rate=1.8)
    k = L.create_lb_function(lbm_config=cfg)
    a = L.create_pdf_array((8, 8, 8), 19)
    b = L.create_pdf_array((8, 8, 8), 19)
    with pytest.raises(ValueError):
        k(src=a.cpu(), dst=b)                        # host tensor
    with pytest.raises(ValueError):
        k(src=a, dst=L.create_pdf_array((8, 8, 9), 19))   # shape mismatch
    with pytest.raises(ValueError):
        k(src=a.float(), dst=b.float())              # dtype mismatch
    with pytest.raises(ValueError):
        k(src=a, dst=a)                              # pull needs two fields
    with pytest.raises(ValueError):
        k(src=a, dst=b, omega=1.0)                   # unknown parameter
    k(src=a, dst=b)
    torch.cuda.synchronize()


def test_symbolic_relaxation_rate(cuda):
    """Free symbols of the method are kernel keyword arguments (lbstep.py:269 kernel_params)."""
    import sympy as sp
    cfg = L.LBMConfig(stencil=L.Stencil.D3Q19, method=L.Method.SRT, relaxation_rate=sp.Symbol("omega"),
                      compressible=True)
    k = L.create_lb_function(lbm_config=cfg)
    assert k.parameters == {"omega"}
    n = (8, 8, 8)
    a, b = L.create_pdf_array(n, 19), L.create_pdf_array(n, 19)
    u = torch.tensor(random_velocity(n, 0.02, seed=5), device="cuda")
    L.macroscopic_values_setter(k.method, 1.0, u, a)
    k(src=a, dst=b, omega=1.3, periodicity=(True, True, True))
    orc = O.make("D3Q19", "srt", relaxation_rate=1.3, compressible=True)
    f = orc.new_field(n)
    orc.set_equilibrium(f, np.ones(n), u.cpu().numpy())
    res, _ = orc.run(f, 1, "pull", 0, periodic=(True, True, True))
    assert pop_rel_linf(_interior(b), res[1:-1, 1:-1, 1:-1], k.method.weights) < 1e-13
    with pytest.raises(ValueError):
        k(src=a, dst=b)


QUAD_CASES = [("d3q19-trt-aa-ldc", "D3Q19", "trt", "aa", (16, 12, 8), (0, 0, 0), "ldc",
               dict(relaxation_rate=1.9, compressible=True)),
              ("d3q19-trt-pull-periodic", "D3Q19", "trt", "pull", (20, 10, 6), (1, 1, 1), None,
               dict(relaxation_rate=1.8, compressible=True, force=(1e-5, 0, 0))),
              ("d3q27-cum-aa-channel", "D3Q27", "cumulant", "aa", (12, 10, 8), (1, 0, 0), "duct",
               dict(relaxation_rate=1.95, compressible=True, galilean_correction=True, force=(1e-5, 0, 0))),
              ("d3q19-srt-aa-periodic", "D3Q19", "srt", "aa", (8, 6, 6), (1, 1, 1), None,
               dict(relaxation_rate=1.6, compressible=False))]


@pytest.mark.parametrize("case", QUAD_CASES, ids=[c[0] for c in QUAD_CASES])
@pytest.mark.parametrize("storage", ["float16", "bfloat16", "e3m12"])
def test_quad_sweep_matches_pair_sweep(cuda, case, storage, monkeypatch):
    """The four-cells-per-thread sweep against the two-cells-per-thread sweep on 16-bit storage
    (the same packed FP32x2 collision, so the fields agree to the last 16-bit digit), 30 steps,
    with walls, periodic wrap across the row ends and both AA parities."""
    name, stencil, method, pattern, n, periodic, bkind, kw = case
    fields = {}
    for kernel in ("quad", "pair"):
        monkeypatch.setenv("LBM_B200_PAIR", "1")
        monkeypatch.setenv("LBM_B200_QUAD", "1" if kernel == "quad" else "0")
        cfg = dict(stencil=getattr(L.Stencil, stencil), method=getattr(L.Method, method.upper()),
                   streaming_pattern=pattern, **kw)
        step = L.LatticeBoltzmannStep(domain_size=n, periodicity=periodic, optimization={"storage_dtype": storage},
                                      config=L.CreateKernelConfig(data_type="float32"), **cfg)
        for obj, sl in (_boundaries(bkind) or []):
            step.boundary_handling.set_boundary(obj, sl)
        step.velocity_array[...] = random_velocity(n, 2e-2, seed=3)
        step.set_pdf_fields_from_macroscopic_values()
        step.run(30)
        if storage == "e3m12":
            from tests import e3m12 as E
            fields[kernel] = E.decode(step.pdfs[1:-1, 1:-1, 1:-1].cpu().numpy()).astype(np.float64)
        else:
            fields[kernel] = _interior(step.pdfs)
    fluid = np.ones(n, bool) if bkind is None else \
        ((step.boundary_handling.flag_array & 7)[1:-1, 1:-1, 1:-1] == 0)
    diff = np.abs(fields["quad"] - fields["pair"])[fluid].max()
    scale = np.abs(fields["pair"][fluid]).max()
    assert diff <= 1e-6 * scale, f"{name} {storage}: max difference {diff:.3e} (scale {scale:.3e})"
