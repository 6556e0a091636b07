"""The e3m12 16-bit storage format: its steps and range (NumPy restatement, no GPU) and, on the
GPU, the codes the setter writes and the values the getter reads back."""
import numpy as np
import pytest

from tests import e3m12 as E


def test_round_trip_step_and_range():
    rng = np.random.default_rng(0)
    v = rng.uniform(-0.06, 0.06, 200000).astype(np.float32)
    back = E.decode(E.encode(v))
    big = np.abs(v) >= 2.0 ** -11                 # normal range: relative step 2^-12
    rel = np.abs(back[big] - v[big]) / np.abs(v[big])
    assert rel.max() <= 2.0 ** -13 * (1 + 1e-6)   # round to nearest: half a step
    small = ~big                                  # gradual underflow: absolute step 2^-23
    assert np.abs(back[small] - v[small]).max() <= 2.0 ** -24 * (1 + 1e-3)
    # four times finer than IEEE half on the same values
    half = v.astype(np.float16).astype(np.float32)
    assert np.abs(back - v).mean() < 0.3 * np.abs(half - v).mean()


def test_codes_are_monotone_and_saturate():
    v = np.linspace(-0.0625, 0.0625, 4097, dtype=np.float32)
    d = E.decode(E.encode(v))
    assert (np.diff(d) >= 0).all()
    assert E.decode(E.encode(np.float32(0.2))) == E.decode(np.uint16(0x7FFF))      # saturates
    assert E.decode(E.encode(np.float32(-0.2))) == -E.decode(np.uint16(0x7FFF))
    assert E.encode(np.float32(0.0)) == 0 and E.decode(np.uint16(0)) == 0.0
    assert abs(E.decode(np.uint16(0x7FFF)) - 0.0625) < 1e-5


def test_rounds_half_to_even():
    step = 2.0 ** -12 * 2.0 ** -5                  # code step for values in [2^-5, 2^-4)
    base = np.float32(2.0 ** -5)
    tie = np.float32(base + 0.5 * step)            # between codes c and c + 1 (c even)
    assert E.decode(E.encode(tie)) == base
    tie2 = np.float32(base + 1.5 * step)           # between c + 1 (odd) and c + 2 (even)
    assert E.decode(E.encode(tie2)) == np.float32(base + 2 * step)


@pytest.mark.gpu
def test_setter_writes_the_codes_and_getter_reads_them(cuda):
    import torch
    import lbmpy_b200 as L
    from oracle import oracle as O
    from tests.helpers import random_velocity
    n = (12, 8, 6)
    u = random_velocity(n, 0.03, seed=2)
    rho = 1 + 1e-3 * np.random.default_rng(3).uniform(-1, 1, n)
    for stencil in ("D3Q19", "D3Q27"):
        step = L.LatticeBoltzmannStep(domain_size=n, periodicity=True, stencil=getattr(L.Stencil, stencil),
                                      method=L.Method.TRT, relaxation_rate=1.8, compressible=True,
                                      optimization={"storage_dtype": "e3m12"},
                                      config=L.CreateKernelConfig(data_type="float32"))
        step.velocity_array[...] = u
        step.density_array[...] = rho
        step.set_pdf_fields_from_macroscopic_values()
        codes = step.pdfs[1:-1, 1:-1, 1:-1].cpu().numpy().view(np.uint16)
        orc = O.make(stencil, "trt", relaxation_rate=1.8, compressible=True)
        f = orc.new_field(n)
        orc.set_equilibrium(f, rho, u)
        ref = E.encode(f[1:-1, 1:-1, 1:-1].astype(np.float32))
        mism = np.abs(codes.astype(np.int32) - ref.astype(np.int32))
        assert mism.max() <= 1 and (mism == 0).mean() > 0.99     # FP64 equilibria round alike
        step.post_run()
        vals = E.decode(codes).astype(np.float64)
        w = np.asarray(step.method.weights)
        dirs = np.asarray(list(step.method.stencil), np.float64)
        rho_h = 1 + vals.sum(-1)
        u_h = (vals @ dirs) / rho_h[..., None]
        assert np.abs(step.density_array - rho_h).max() < 1e-6
        assert np.abs(step.velocity_array - u_h).max() < 1e-6
        assert np.abs(step.velocity_array - u).max() < 2e-5      # the format's step at |f - w| ~ w u
