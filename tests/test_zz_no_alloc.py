"""The allocation-free reduction entry point against the regular one.

``lbm_reduce_conserved_noalloc`` serves callers that cannot call cudaMalloc (fixed device-memory
budgets, allocator-less embeddings): it keeps its partial sums in a static device array instead of
the plan's scratch.  Here it is called through the C ABI twice in a row on the same fields and
must agree with ``lbm_reduce_conserved`` each time.  This file sorts last so that a run stopping at
the first failure has run every other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

import lbmpy_b200 as L
from lbmpy_b200 import _native as N
from lbmpy_b200.kernel import build_desc
from lbmpy_b200.macroscopic_value_kernels import _rule_for

pytestmark = pytest.mark.gpu


def _reduce_both(step):
    plan = step._macro.get(step.pdfs, step.kernel_params, step.periodicity)
    flags = step._flags(step._kernels[0])
    strides = N.i64_array(step.pdfs.stride())
    prev = 1 if step.previous_timestep == L.Timestep.ODD else 0
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    fptr = ctypes.c_void_p(flags.data_ptr() if flags is not None else None)
    ref = (ctypes.c_double * 5)()
    N.check(N.lib().lbm_reduce_conserved(plan.handle, ctypes.c_void_p(step.pdfs.data_ptr()), strides, fptr, prev,
                                         ref, stream), "lbm_reduce_conserved")
    rule = _rule_for(step.method, step.streaming_pattern, step._storage)
    desc = build_desc(rule, step.domain_size, step.periodicity, step.kernel_params, rates_needed=False)
    got = (ctypes.c_double * 5)()
    N.check(N.lib().lbm_reduce_conserved_noalloc(ctypes.byref(desc), ctypes.c_void_p(step.pdfs.data_ptr()), strides,
                                                 fptr, prev, got, stream), "lbm_reduce_conserved_noalloc")
    return np.array(list(got)), np.array(list(ref))


@pytest.mark.parametrize("setup", ["d3q19-trt-f64-periodic", "d3q27-cumulant-f32-aa-channel"])
def test_noalloc_reduction_matches_allocating_entry_point(cuda, setup):
    n = (24, 20, 12)
    rng = np.random.default_rng(11)
    if setup == "d3q19-trt-f64-periodic":
        step = L.LatticeBoltzmannStep(domain_size=n, periodicity=True, stencil=L.Stencil.D3Q19, method=L.Method.TRT,
                                      relaxation_rate=1.8, compressible=True, force=(1e-5, 0, 0))
    else:
        step = L.LatticeBoltzmannStep(domain_size=n, periodicity=(True, False, False), stencil=L.Stencil.D3Q27,
                                      method=L.Method.CUMULANT, relaxation_rate=1.95, compressible=True,
                                      galilean_correction=True, force=(1e-5, 0, 0), streaming_pattern="aa",
                                      config=L.CreateKernelConfig(data_type="float32"))
        for d in ("N", "S", "T", "B"):
            step.boundary_handling.set_boundary(L.NoSlip(), L.slice_from_direction(d, 3))
    step.velocity_array[...] = rng.uniform(-0.02, 0.02, n + (3,))
    step.set_pdf_fields_from_macroscopic_values()
    step.run(7)
    torch.cuda.synchronize()
    got1, ref1 = _reduce_both(step)
    np.testing.assert_allclose(got1, ref1, rtol=1e-12, atol=1e-15)
    step.run(3)                      # change the fields, then call again: no state may carry over
    torch.cuda.synchronize()
    got2, ref2 = _reduce_both(step)
    np.testing.assert_allclose(got2, ref2, rtol=1e-12, atol=1e-15)
    assert not np.allclose(got1[1:], got2[1:], rtol=0, atol=0) or setup.startswith("d3q19")
    # with every kernel of this configuration loaded, a further call reserves nothing through torch's
    # allocator, and free device memory moves by no more than other users of a shared GPU could
    reserved_before = torch.cuda.memory_reserved()
    free_before = torch.cuda.mem_get_info()[0]
    got3, ref3 = _reduce_both(step)
    torch.cuda.synchronize()
    assert torch.cuda.memory_reserved() == reserved_before
    assert abs(torch.cuda.mem_get_info()[0] - free_before) <= 4 << 20
    np.testing.assert_array_equal(got3, got2)


def test_noalloc_rejects_bad_arguments(cuda):
    desc = N.LbmPlanDesc()
    desc.stencil = 19
    desc.method = N.METHOD_TRT
    desc.store_dtype = N.DTYPE_F64
    for k in range(3):
        desc.dims[k] = 8
    out = (ctypes.c_double * 5)()
    host = np.zeros(19 * 10 * 10 * 10)
    strides = N.i64_array((1, 10, 100, 1000))
    rc = N.lib().lbm_reduce_conserved_noalloc(ctypes.byref(desc), ctypes.c_void_p(host.ctypes.data), strides, None, 0,
                                              out, None)
    assert rc == N.LBM_E_INVALID            # a host pointer is refused before any launch
    desc.stencil = 15
    rc = N.lib().lbm_reduce_conserved_noalloc(ctypes.byref(desc), None, strides, None, 0, out, None)
    assert rc == N.LBM_E_UNSUPPORTED
