"""FP64 global reductions of mass, momentum and kinetic energy (one FP64 pass over the PDFs).

lbmpy has no on-device reduction of its own; its step reduces on the host through the data
handling (lbstep.py:400).  ``lbm_reduce_conserved`` sums per block in FP64 and adds the block
partials in a fixed order, so the result is reproducible run to run.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native as N
from .enums import Timestep


def reduce_pdfs(plan: N.Plan, pdfs: torch.Tensor, previous_timestep=Timestep.BOTH, flags=None, stream=None):
    out = (ctypes.c_double * 5)()
    s = torch.cuda.current_stream().cuda_stream if stream is None else stream.cuda_stream
    N.check(N.lib().lbm_reduce_conserved(plan.handle, ctypes.c_void_p(pdfs.data_ptr()), N.i64_array(pdfs.stride()),
                                         ctypes.c_void_p(flags.data_ptr() if flags is not None else None),
                                         1 if previous_timestep == Timestep.ODD else 0, out, ctypes.c_void_p(s)),
            "lbm_reduce_conserved")
    return np.array(list(out))


def reduce_conserved(step):
    """[mass, momentum_x, momentum_y, momentum_z, kinetic energy] of a LatticeBoltzmannStep."""
    plan = step._macro.get(step.pdfs, step.kernel_params, step.periodicity)
    flags = step._flags(step._kernels[0])
    return reduce_pdfs(plan, step.pdfs, step.previous_timestep, flags)
