"""The learned closure on the GPU: the training kernels' gradient checked against the CPU oracle,
the in-sweep inference checked cell by cell against the oracle's sweep, and the trained network's
gain over the method without it."""
import numpy as np
import pytest
import torch

import lbmpy_b200 as L
from lbmpy_b200 import closure as C
from lbmpy_b200.enums import SubgridScaleModel
from oracle import mlp_oracle as M
from oracle import oracle as O
from tests.helpers import random_velocity
from tests.test_closure import random_cells, random_params

pytestmark = pytest.mark.gpu


def _state(P6, rho, u):
    return torch.tensor(np.concatenate([P6, rho[:, None], u], 1).T.copy(), dtype=torch.float32, device="cuda")


def test_feature_and_forward_kernels_match_oracle(cuda):
    P6, rho, u = random_cells(5000, seed=11)
    X = M.features(P6.astype(np.float32).astype(np.float64), rho.astype(np.float32).astype(np.float64),
                   u.astype(np.float32).astype(np.float64))
    feats = C.closure_features(_state(P6, rho, u))
    got = feats.cpu().double().numpy().T
    scale = np.abs(X).max(0) + 1e-3
    assert (np.abs(got - X) / scale).max() < 2e-5
    p = random_params(12)
    clo = C.MLPClosure(params=torch.from_numpy(p))
    nu = clo.predict(feats).cpu().double().numpy()
    ref = M.forward(p, got)
    np.testing.assert_allclose(nu, ref, rtol=2e-5, atol=1e-9)


@pytest.mark.parametrize("weighted", [False, True])
def test_training_gradient_matches_oracle(cuda, weighted):
    """lbm_mlp_loss_grad (FP32, block partials summed in FP64) against the FP64 oracle."""
    rng = np.random.default_rng(13)
    n = 3000                                            # several chunks and a ragged last one
    X = rng.standard_normal((n, 10)).astype(np.float32)
    t = np.abs(rng.normal(2e-3, 1e-3, n)).astype(np.float32)
    w = rng.uniform(0.2, 3.0, n).astype(np.float32) if weighted else None
    p = random_params(14)
    clo = C.MLPClosure(params=torch.from_numpy(p))
    feats = torch.from_numpy(X.T.copy()).cuda()
    loss, grad = clo.loss_and_grad(feats, torch.from_numpy(t).cuda(),
                                   torch.from_numpy(w).cuda() if weighted else None)
    ref_loss, ref_grad = M.loss_and_grad(p, X.astype(np.float64), t, w)
    assert abs(loss.item() - ref_loss) <= 1e-5 * ref_loss
    g = grad.cpu().double().numpy()
    assert np.abs(g - ref_grad).max() <= 1e-4 * np.abs(ref_grad).max()
    assert g[M.SCALE] == 0.0
    # deterministic: the same call gives the same bits
    _, grad2 = clo.loss_and_grad(feats, torch.from_numpy(t).cuda(), torch.from_numpy(w).cuda() if weighted else None)
    assert torch.equal(grad, grad2)


def test_adam_step_matches_reference(cuda):
    from lbmpy_b200 import _native as N
    import ctypes
    rng = np.random.default_rng(15)
    p = random_params(16)
    g = rng.normal(0, 1e-2, M.NPARAM).astype(np.float32)
    m1 = rng.normal(0, 1e-3, M.NPARAM).astype(np.float32)
    m2 = np.abs(rng.normal(0, 1e-5, M.NPARAM)).astype(np.float32)
    dp, dg, d1, d2 = (torch.from_numpy(a.copy()).cuda() for a in (p, g, m1, m2))
    step, lr, b1, b2, eps = 7, 1e-3, 0.9, 0.999, 1e-8
    N.check(N.lib().lbm_mlp_adam(ctypes.c_void_p(dg.data_ptr()), ctypes.c_void_p(dp.data_ptr()),
                                 ctypes.c_void_p(d1.data_ptr()), ctypes.c_void_p(d2.data_ptr()), lr, b1, b2, eps, step,
                                 None))
    torch.cuda.synchronize()
    e1 = b1 * m1.astype(np.float64) + (1 - b1) * g
    e2 = b2 * m2.astype(np.float64) + (1 - b2) * g.astype(np.float64) ** 2
    ref = p - lr * (e1 / (1 - b1 ** step)) / (np.sqrt(e2 / (1 - b2 ** step)) + eps)
    ref[M.SCALE] = p[M.SCALE]
    np.testing.assert_allclose(dp.cpu().numpy(), ref, rtol=1e-5, atol=1e-8)


def test_fit_learns_a_teacher_network(cuda):
    """Targets from a fixed teacher network on closure features: training must recover them."""
    P6, rho, u = random_cells(40000, seed=17)
    feats = C.closure_features(_state(P6, rho, u))
    Xs = feats.cpu().double().numpy().T
    mu, sd = Xs.mean(0), Xs.std(0)
    teacher = random_params(18, scale=2e-3)
    target = torch.tensor(M.forward(teacher, (Xs - mu) / sd), dtype=torch.float32, device="cuda")
    student = C.MLPClosure(seed=19, nu_scale=2e-3)
    before = float(((student.predict(feats) - target) ** 2).mean())
    student.fit(feats, target, steps=600, batch=8192, lr=3e-3, lr_final=3e-4, seed=0)
    after = float(((student.predict(feats) - target) ** 2).mean())
    assert after < 0.05 * before, (before, after)
    assert student.history[-1][1] < student.history[0][1]


CLOSURE_CASES = [("pull", None), ("aa", None), ("pull", (1e-5, -2e-6, 3e-6)), ("aa", (1e-5, 0, 0))]


@pytest.mark.parametrize("pattern,force", CLOSURE_CASES)
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_closure_sweep_matches_oracle(cuda, pattern, force, dtype):
    """The in-sweep inference (constant-memory parameters, fused into the cumulant collision)
    cell by cell against the oracle's sweep with the same parameters, 50 steps."""
    from tests.test_gpu_parity import pop_rel_linf, run_pair
    n = (12, 10, 8)
    p = random_params(20, scale=5e-3)
    clo = C.MLPClosure(params=torch.from_numpy(p))
    kw = dict(relaxation_rate=1.99, compressible=True, galilean_correction=True)
    if force is not None:
        kw["force"] = force
    step = L.LatticeBoltzmannStep(domain_size=n, periodicity=True, stencil=L.Stencil.D3Q27,
                                  method=L.Method.CUMULANT, streaming_pattern=pattern,
                                  subgrid_scale_model=(SubgridScaleModel.LEARNED, clo),
                                  config=L.CreateKernelConfig(data_type=dtype), **kw)
    u = random_velocity(n, 2e-2, seed=21)
    rho = 1.0 + 1e-3 * np.random.default_rng(22).uniform(-1, 1, n)
    step.velocity_array[...] = u
    step.density_array[...] = rho
    step.set_pdf_fields_from_macroscopic_values()
    orc = O.make("D3Q27", "cumulant", mlp=p, **kw)
    f = orc.new_field(n)
    prev = 1 if pattern != "pull" else 0
    orc.set_equilibrium(f, rho, u, pattern, prev)
    orc.periodic_sync(f, pattern, prev, (1, 1, 1))
    res, _ = run_pair(step, orc, f, None, (0.0, 0.0, 0.0), prev, 50, pattern, (1, 1, 1))
    got = step.pdfs[1:-1, 1:-1, 1:-1].detach().cpu().double().numpy()
    err = pop_rel_linf(got, res[1:-1, 1:-1, 1:-1], step.method.weights)
    assert err < (1e-12 if dtype == "float64" else 1e-5), err
    # the closure changed the result: the plain method differs by far more than the bar
    plain = O.make("D3Q27", "cumulant", **kw)
    f2 = plain.new_field(n)
    plain.set_equilibrium(f2, rho, u, pattern, prev)
    plain.periodic_sync(f2, pattern, prev, (1, 1, 1))
    res2, _ = plain.run(f2, 50, pattern, prev, periodic=(1, 1, 1))
    assert pop_rel_linf(res2[1:-1, 1:-1, 1:-1], res[1:-1, 1:-1, 1:-1], step.method.weights) > 1e-6


def test_trained_closure_gains_over_the_plain_method(cuda):
    """A small closure study: 32^3 coarse runs, training data from box-filtered 128^3 runs of the
    same method, reference a 64^3 plain run.  What the network gains over the method without it
    (nu_t = 0), measured on the filtered fine data: its eddy viscosity explains the subgrid stress
    with a weighted error well below no closure's and below Smagorinsky's (C = 0.1) on the same
    cells.  The coarse runs with either closure stay finite and keep their energy spectra within
    a factor of the reference's; the spectral errors are reported, not ranked (at this
    resolution the coarse cumulant run is already more dissipative than the reference at high
    wavenumbers, which no eddy viscosity can correct)."""
    from lbmpy_b200.turbulence import closure_study
    res = closure_study(n=32, omega=1.99, steps=240, r_train=4, r_ref=2, snapshots=4, train_steps=600,
                        batch=16384, log=lambda *a: None)
    assert res["train_loss_learned"] < 0.6 * res["train_loss_zero"], res
    assert res["train_loss_learned"] < res["train_loss_smagorinsky"], res
    for name in ("plain", "smagorinsky", "learned"):
        E = np.asarray(res[f"E_{name}"])
        assert np.isfinite(E).all()
        assert res[f"err_{name}"] < 0.5          # mean |log10| error: within ~3x over k = 1..n/3
