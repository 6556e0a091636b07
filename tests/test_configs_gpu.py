"""The benchmark configurations at their stated sizes, on the GPU.

- c1: D3Q19 TRT (omega 1.8, magic odd rate), compressible, FP64, pull, periodic 64^3 Taylor-Green
  vortex (u0 0.05, k = 2 pi / 64), 1000 steps, cell by cell against the CPU restatement (the
  closed-form kernel, itself pinned to the generic oracle and, through it, to lbmpy's stored
  states), with mass and momentum checked after every step.
- c2: D3Q27 cumulant, Galilean-corrected, FP32, AA, 256 x 128 x 128 channel (NoSlip y/z walls,
  periodic x, CentralMoment force 1e-7, omega 1.95, seeded velocity noise 1e-4), 20000 steps; the
  axial velocity against the start-up solution of the rectangular duct (tests/analytic.py).
- c3: D3Q19 TRT periodic Taylor-Green box stored in FP16, BF16 and e3m12 (zero-centred, FP32
  collision) against the same run in FP64: relative L2 velocity error.
- c4: the 512-cavity D3Q19 MRT batch (lid_driven_cavity_batch(512, seed=0)), 2000 steps in one
  persistent launch per step, eight seeded cavities against the same cavity run alone.
"""
import numpy as np
import pytest
import torch

import lbmpy_b200 as L
from lbmpy_b200.boundaries import NoSlip, slice_from_direction
from oracle import cpu as C
from oracle import oracle as O
from tests.analytic import duct_startup_velocity
from tests.helpers import tgv_velocity

pytestmark = pytest.mark.gpu


def test_c1_tgv_d3q19_trt_fp64_64cube_1000_steps(cuda):
    n = (64, 64, 64)
    u = tgv_velocity(n, u0=0.05)
    step = L.LatticeBoltzmannStep(domain_size=n, periodicity=True, stencil=L.Stencil.D3Q19, method=L.Method.TRT,
                                  relaxation_rate=1.8, compressible=True,
                                  config=L.CreateKernelConfig(data_type="float64"))
    step.velocity_array[...] = u
    step.set_pdf_fields_from_macroscopic_values()
    orc = O.make("D3Q19", "trt", relaxation_rate=1.8, compressible=True)
    fc = C.FastCPU("trt", orc)
    f = orc.new_field(n)
    orc.set_equilibrium(f, np.ones(n), u)
    g = fc.new_field(n)
    g[...] = f
    w = np.asarray(step.method.weights)
    m0 = step.reduce_conserved()
    scale = 1.0 + w.max()
    for t in range(1, 1001):
        step.time_step()
        red = step.reduce_conserved()                 # FP64 sums on the GPU, every step
        assert abs(red[0] - m0[0]) < 1e-9 * m0[0], f"mass drifted at step {t}"
        assert np.abs(red[1:4] - m0[1:4]).max() < 1e-12 * m0[0], f"momentum drifted at step {t}"
        if t in (100, 1000):
            g, _ = fc.run(g, 100 if t == 100 else 900, periodic=(1, 1, 1))
            got = step.pdfs[1:-1, 1:-1, 1:-1].double().cpu().numpy()
            err = np.abs(got - g[1:-1, 1:-1, 1:-1]).max() / scale
            assert err < 1e-12, f"step {t}: relative L-infinity {err:.3e}"
            keep = fc.new_field(n)
            keep[...] = g
            g = keep
    # the vortex decays at the rate nu k^2 per velocity component (2 nu k^2 for the energy)
    nu = (1 / 1.8 - 0.5) / 3
    k2 = 2 * (2 * np.pi / 64) ** 2
    assert abs(red[4] / m0[4] / np.exp(-2 * nu * k2 * 1000) - 1) < 1e-2


def test_c2_channel_256x128x128_20000_steps_matches_duct_flow(cuda):
    n = (256, 128, 128)
    omega, force = 1.95, 1e-7
    step = L.LatticeBoltzmannStep(domain_size=n, periodicity=(True, False, False), stencil=L.Stencil.D3Q27,
                                  method=L.Method.CUMULANT, relaxation_rate=omega, compressible=True,
                                  galilean_correction=True, force=(force, 0, 0), streaming_pattern="aa",
                                  config=L.CreateKernelConfig(data_type="float32"))
    for d in ("N", "S", "T", "B"):
        step.boundary_handling.set_boundary(NoSlip(), slice_from_direction(d, 3))
    rng = np.random.default_rng(0)
    step.velocity_array[...] = rng.uniform(-1e-4, 1e-4, n + (3,)).astype(np.float32)
    step.set_pdf_fields_from_macroscopic_values()
    steps = 20000
    step.run(steps)
    ux = step.velocity_array[..., 0].astype(np.float64).mean(axis=0)
    nu = (1 / omega - 0.5) / 3
    ref = duct_startup_velocity(n[1], n[2], nu, force, steps)
    err = np.abs(ux - ref).max() / ref.max()
    print(f"duct profile after {steps} steps: max error {err:.3e} of the peak velocity, peak ratio "
          f"{ux.max() / ref.max():.5f}")
    assert err < 2e-2, f"duct profile: max error {err:.3e} of the peak velocity"
    assert abs(ux.max() / ref.max() - 1) < 5e-3
    assert np.isfinite(step.velocity_array).all()


@pytest.mark.parametrize("storage,bound", [("float32", 1e-4), ("float16", 2e-3), ("bfloat16", 3e-2),
                                           ("e3m12", 5e-4)])
def test_c3_16bit_storage_error_against_fp64(cuda, storage, bound):
    from lbmpy_b200.precision import precision_study
    res = precision_study(128, 1000, 1000, storages=(storage,), device="cuda", log=lambda *_: None)
    err = res[storage]["final_l2_velocity_error"]
    print(f"{storage}: L2 velocity error vs FP64 after 1000 steps at 128^3: {err:.3e}")
    assert err < bound


def test_c4_512_cavity_batch_sampled_against_single_domains(cuda, monkeypatch):
    from lbmpy_b200.batched import lid_driven_cavity_batch
    monkeypatch.setenv("LBM_B200_PAIR", "0")   # the one-cell sweep, whose per-cell code the batch shares
    b = lid_driven_cavity_batch(512, seed=0)
    b.finalize()
    steps = 2000
    b.run(steps)
    torch.cuda.synchronize()
    picks = np.random.default_rng(7).choice(512, 8, replace=False)
    for k in picks:
        size = b.domain_sizes[k]
        p = b.kernel_params[k]
        s = L.LatticeBoltzmannStep(domain_size=size, periodicity=False, stencil=L.Stencil.D3Q19,
                                   method=L.Method.MRT, relaxation_rates=[p["omega_shear"], p["omega_bulk"], 1, 1],
                                   compressible=False, config=L.CreateKernelConfig(data_type="float32"))
        s.boundary_handling.set_boundary(L.UBB((0.05, 0.0, 0.0)), slice_from_direction("N", 3))
        for d in ("W", "E", "S", "T", "B"):
            s.boundary_handling.set_boundary(NoSlip(), slice_from_direction(d, 3))
        s.run(steps)
        got = b.pdfs(int(k))[1:-1, 1:-1, 1:-1].double().cpu().numpy()
        ref = s.pdfs[1:-1, 1:-1, 1:-1].double().cpu().numpy()
        err = np.abs(got - ref).max() / (1.0 + max(s.method.weights))
        assert err <= 1e-6, f"cavity {k} {size}: {err:.3e}"
        assert np.abs(s.velocity_array).max() > 1e-3
        del s
