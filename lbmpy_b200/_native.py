"""ctypes binding of liblbmb200.so (C ABI in include/lbm_b200.h).

The library is built in-tree by ``python -m lbmpy_b200.build``.  There is no fallback: if the
library is missing or a CUDA device is unavailable, every kernel call raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblbmb200.so")

LBM_OK, LBM_E_INVALID, LBM_E_CUDA, LBM_E_UNSUPPORTED, LBM_E_DEVICE = 0, 1, 2, 3, 4
METHOD_SRT, METHOD_TRT, METHOD_MRT, METHOD_CUMULANT, METHOD_CENTRAL_MOMENT = 0, 1, 2, 3, 4
DTYPE_F64, DTYPE_F32, DTYPE_F16, DTYPE_BF16, DTYPE_E3M12 = 0, 1, 2, 3, 4
PATTERN_PULL, PATTERN_AA, PATTERN_ESOTWIST, PATTERN_PUSH, PATTERN_ESOPULL, PATTERN_ESOPUSH = 0, 1, 2, 3, 4, 5
FORCE_NONE, FORCE_GUO, FORCE_CENTRAL_MOMENT, FORCE_SIMPLE, FORCE_LUO = 0, 1, 2, 3, 4
SGS_NONE, SGS_SMAGORINSKY, SGS_MLP = 0, 1, 2
STATUS_STAGE_TIMEOUT = 1
VARIANT_CELL, VARIANT_PAIR, VARIANT_QUAD, VARIANT_STAGED, VARIANT_ZPIPE = 0, 1, 2, 3, 4
VARIANT_NAMES = {0: "cell", 1: "pair", 2: "quad", 3: "staged", 4: "zpipe"}
MLP_PARAMS = 1442

# exported symbols, one per declaration in include/lbm_b200.h
EXPORTS = ("lbm_plan_create", "lbm_plan_destroy", "lbm_plan_update", "lbm_plan_status", "lbm_sweep_variant",
           "lbm_sweep", "lbm_run",
           "lbm_set_equilibrium", "lbm_get_macroscopic", "lbm_reduce_conserved", "lbm_reduce_conserved_noalloc",
           "lbm_flags_finalize", "lbm_plan_set_links", "lbm_closure_set_weights", "lbm_closure_features", "lbm_mlp_forward",
           "lbm_mlp_create", "lbm_mlp_destroy", "lbm_mlp_loss_grad", "lbm_mlp_adam", "lbm_batch_create", "lbm_batch_sweep", "lbm_batch_info", "lbm_batch_destroy",
           "lbm_sparse_sweep", "lbm_sparse_set_equilibrium", "lbm_sparse_get_macroscopic", "lbm_sparse_ubb",
           "lbm_plan_set_stage_wait", "lbm_halo_copy",
           "lbm_last_error", "lbm_version")


class LbmPlanDesc(ctypes.Structure):
    _fields_ = [
        ("stencil", ctypes.c_int32), ("method", ctypes.c_int32), ("store_dtype", ctypes.c_int32),
        ("pattern", ctypes.c_int32), ("compressible", ctypes.c_int32),
        ("continuous_equilibrium", ctypes.c_int32),
        ("rates", ctypes.c_double * 27),
        ("force_model", ctypes.c_int32),
        ("force", ctypes.c_double * 3),
        ("galilean_correction", ctypes.c_int32),
        ("sgs", ctypes.c_int32),
        ("sgs_constant", ctypes.c_double),
        ("shear_rate", ctypes.c_double),
        ("sgs_mask", ctypes.c_uint32),
        ("ubb_velocity", (ctypes.c_double * 3) * 4),
        ("dims", ctypes.c_int32 * 3),
        ("periodic", ctypes.c_int32 * 3),
        ("fixed_density", ctypes.c_double),
        ("fixed_density1", ctypes.c_double),
        ("ubb_density", ctypes.c_double * 4),
        ("ubb_adapt_mask", ctypes.c_uint32),
        ("fourth_order_limiter", ctypes.c_double),
    ]


class LbmLinkTables(ctypes.Structure):
    _fields_ = [("cell_block", ctypes.c_void_p), ("n_blocks", ctypes.c_int64), ("ubb_velocity", ctypes.c_void_p),
                ("ubb_mask", ctypes.c_uint32), ("link_code", ctypes.c_void_p), ("link_value", ctypes.c_void_p)]


class LbmDomainDesc(ctypes.Structure):
    _fields_ = [
        ("dims", ctypes.c_int32 * 3), ("periodic", ctypes.c_int32 * 3),
        ("strides", ctypes.c_int64 * 4), ("offset", ctypes.c_int64), ("flags_offset", ctypes.c_int64),
        ("rates", ctypes.c_double * 27), ("ubb_velocity", (ctypes.c_double * 3) * 4),
    ]


HALO_MAX_JOBS = 4


class LbmHaloJob(ctypes.Structure):
    _fields_ = [("z", ctypes.c_int32), ("unpack", ctypes.c_int32), ("n_slots", ctypes.c_int32),
                ("slots", ctypes.c_int32 * 27), ("buffer", ctypes.c_void_p)]


class LbmBatchTiling(ctypes.Structure):
    _fields_ = [("tile_x", ctypes.c_int32), ("tile_y", ctypes.c_int32), ("cells_z", ctypes.c_int32),
                ("blocks_per_sm", ctypes.c_int32)]


class LbmError(RuntimeError):
    """A CUDA-side failure reported by liblbmb200."""


_lib = None


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m lbmpy_b200.build` "
                              "(there is no CPU fallback for the B200 sweep)")
        L = ctypes.CDLL(LIB_PATH)
        vp, i64p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)
        L.lbm_plan_create.argtypes = [ctypes.POINTER(LbmPlanDesc), ctypes.POINTER(ctypes.c_void_p)]
        L.lbm_plan_destroy.argtypes = [vp]
        L.lbm_plan_update.argtypes = [vp, ctypes.POINTER(LbmPlanDesc)]
        L.lbm_plan_status.argtypes = [vp, ctypes.POINTER(ctypes.c_uint32), ctypes.c_int]
        L.lbm_sweep_variant.argtypes = [vp, vp, vp, i64p, ctypes.c_int, vp, ctypes.POINTER(ctypes.c_int)]
        L.lbm_sweep.argtypes = [vp, vp, vp, i64p, vp, ctypes.c_int, vp, vp]
        L.lbm_run.argtypes = [vp, vp, vp, i64p, vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int), vp]
        L.lbm_set_equilibrium.argtypes = [vp, vp, i64p, vp, i64p, vp, i64p, ctypes.c_int, vp]
        L.lbm_get_macroscopic.argtypes = [vp, vp, i64p, vp, i64p, vp, i64p, ctypes.c_int, vp]
        L.lbm_reduce_conserved.argtypes = [vp, vp, i64p, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double), vp]
        L.lbm_reduce_conserved_noalloc.argtypes = [ctypes.POINTER(LbmPlanDesc), vp, i64p, vp, ctypes.c_int,
                                                   ctypes.POINTER(ctypes.c_double), vp]
        L.lbm_flags_finalize.argtypes = [vp, vp, vp]
        L.lbm_plan_set_links.argtypes = [vp, ctypes.POINTER(LbmLinkTables)]
        L.lbm_closure_set_weights.argtypes = [vp, ctypes.c_int, vp]
        L.lbm_closure_features.argtypes = [vp, ctypes.c_int64, vp, vp]
        L.lbm_mlp_forward.argtypes = [vp, vp, ctypes.c_int64, vp, vp]
        L.lbm_mlp_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        L.lbm_mlp_destroy.argtypes = [vp]
        L.lbm_mlp_loss_grad.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int64, ctypes.c_double, vp, vp, vp]
        L.lbm_mlp_adam.argtypes = [vp, vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_int, vp]
        L.lbm_batch_create.argtypes = [ctypes.POINTER(LbmPlanDesc), ctypes.POINTER(LbmDomainDesc), ctypes.c_int, vp,
                                       vp, ctypes.c_int64, vp, ctypes.c_int64, ctypes.POINTER(LbmBatchTiling),
                                       ctypes.POINTER(ctypes.c_void_p)]
        L.lbm_batch_sweep.argtypes = [vp, ctypes.c_int, vp]
        L.lbm_batch_info.argtypes = [vp, i64p]
        L.lbm_batch_destroy.argtypes = [vp]
        L.lbm_sparse_sweep.argtypes = [vp, vp, vp, vp, ctypes.c_int64, ctypes.c_int64, vp]
        L.lbm_sparse_set_equilibrium.argtypes = [vp, vp, vp, vp, ctypes.c_int64, ctypes.c_int64, vp]
        L.lbm_sparse_get_macroscopic.argtypes = [vp, vp, vp, vp, ctypes.c_int64, ctypes.c_int64, vp]
        L.lbm_sparse_ubb.argtypes = [vp, vp, vp, ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(ctypes.c_double), vp]
        L.lbm_plan_set_stage_wait.argtypes = [vp, ctypes.c_uint64, ctypes.c_int]
        L.lbm_halo_copy.argtypes = [vp, i64p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                    ctypes.c_int32, ctypes.POINTER(LbmHaloJob), ctypes.c_int32, vp]
        L.lbm_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        for name in EXPORTS:
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    lib().lbm_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int, what: str = ""):
    if rc == LBM_OK:
        return
    msg = last_error()
    if what:
        msg = f"{what}: {msg}"
    if rc in (LBM_E_INVALID, LBM_E_DEVICE):
        raise ValueError(msg)
    if rc == LBM_E_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise LbmError(msg)


def i64_array(values):
    return (ctypes.c_int64 * len(values))(*[int(v) for v in values])


class Plan:
    """Owns an LbmPlan handle."""

    def __init__(self, desc: LbmPlanDesc):
        self.desc = desc
        h = ctypes.c_void_p()
        check(lib().lbm_plan_create(ctypes.byref(desc), ctypes.byref(h)), "lbm_plan_create")
        self.handle = h

    def update(self, desc: LbmPlanDesc):
        check(lib().lbm_plan_update(self.handle, ctypes.byref(desc)), "lbm_plan_update")
        self.desc = desc

    def status(self, clear: bool = True) -> int:
        """Device status word OR-ed by the plan's sweeps (0: every sweep completed)."""
        v = ctypes.c_uint32(0)
        check(lib().lbm_plan_status(self.handle, ctypes.byref(v), int(clear)), "lbm_plan_status")
        return v.value

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and _lib is not None:
            _lib.lbm_plan_destroy(h)
            self.handle = None
