"""The callable returned by ``create_lb_function``: launches the fused sm_100a sweep.

lbmpy's ``create_lb_function`` returns a pystencils ``KernelWrapper`` that is called with the
fields by name and free symbols as keyword arguments (``lbstep.py:269,280``).  ``LbKernel`` keeps
that calling convention: ``kernel(src=pdfs, dst=tmp, omega=1.8)`` for two-field pull,
``kernel(src=pdfs)`` for in-place AA / EsoTwist.  Extra keyword arguments beyond lbmpy's:
``flags`` (uint8 cell flags), ``ubb_velocities`` (wall velocities of UBB numbers 0..3),
``periodicity`` (overrides ``builtin_periodicity``), ``omega_out`` (float32 field receiving the
effective shear rate) and ``stream`` (a ``torch.cuda.Stream``).
"""
from __future__ import annotations

import ctypes
from typing import Dict, Optional, Sequence

import torch

from . import _native as N
from .enums import Timestep, is_inplace
from .fields import check_pdf_tensor
from . import forcemodels

_METHOD = {"srt": N.METHOD_SRT, "trt": N.METHOD_TRT, "mrt": N.METHOD_MRT, "cumulant": N.METHOD_CUMULANT,
           "central_moment": N.METHOD_CENTRAL_MOMENT}
_PATTERN = {"pull": N.PATTERN_PULL, "aa": N.PATTERN_AA, "esotwist": N.PATTERN_ESOTWIST, "push": N.PATTERN_PUSH,
            "esopull": N.PATTERN_ESOPULL, "esopush": N.PATTERN_ESOPUSH}
_DT = {"float64": N.DTYPE_F64, "float32": N.DTYPE_F32, "float16": N.DTYPE_F16, "bfloat16": N.DTYPE_BF16,
       "e3m12": N.DTYPE_E3M12}


def _evaluate(value, params: Dict, placeholder=None):
    if isinstance(value, (int, float)):
        return float(value)
    try:
        return float(value)
    except (TypeError, ValueError):
        pass
    import sympy as sp
    expr = sp.sympify(value)
    subs = {}
    for s in expr.free_symbols:
        if s.name not in params and placeholder is not None:
            return float(placeholder)
        if s.name not in params:
            raise ValueError(f"kernel parameter {s.name!r} has no value: pass {s.name}=... when calling the kernel")
        subs[s] = params[s.name]
    return float(expr.subs(subs))


def free_parameters(update_rule) -> set:
    names = set()
    for r in update_rule.method.relaxation_rates:
        if not isinstance(r, (int, float)):
            try:
                float(r)
            except (TypeError, ValueError):
                import sympy as sp
                names |= {s.name for s in sp.sympify(r).free_symbols}
    return names


def build_desc(update_rule, dims, periodic, params: Dict, ubb_velocities=None,
               rates_needed: bool = True, fixed_density=None, ubb_options=None) -> N.LbmPlanDesc:
    """Resolves an update rule plus parameter values into the C plan descriptor.  Plans that only
    run the getter / setter do not need relaxation rates (rates_needed=False).  ubb_options:
    {"densities": prescribed wall density per UBB number (0: none), "adapt_mask": bit u set when
    UBB number u adapts its velocity to the force}."""
    rule = update_rule.collision_rule
    m = rule.method
    d = N.LbmPlanDesc()
    d.stencil = m.stencil.Q
    d.method = _METHOD[m.kind]
    d.store_dtype = _DT[update_rule.storage_dtype]
    d.pattern = _PATTERN[update_rule.streaming_pattern]
    d.compressible = int(bool(m.compressible))
    d.continuous_equilibrium = int(bool(m.continuous_equilibrium))
    ph = None if rates_needed else 1.0
    rates = [_evaluate(r, params, ph) for r in m.relaxation_rates]
    if m.kind in ("srt", "trt"):
        from . import methods as M
        monos = M.default_monomials(m.stencil.name)
        even = next(r for r, e in zip(rates, monos) if sum(e) % 2 == 0 and sum(e) > 0)
        odd = next(r for r, e in zip(rates, monos) if sum(e) % 2 == 1)
        native_rates = [even, odd]
    else:
        native_rates = rates
    for k, r in enumerate(native_rates):
        d.rates[k] = r
    fm = m.force_model
    if fm is not None:
        d.force_model = fm.native_id
        f = [_evaluate(v, params) for v in fm.force] + [0.0] * 3
        for k in range(3):
            d.force[k] = f[k]
    d.galilean_correction = int(bool(rule.galilean_correction))
    d.fourth_order_limiter = float(getattr(rule, "fourth_order_limiter", 0.0))
    shear = _evaluate(m.shear_relaxation_rate, params, ph)
    d.shear_rate = shear
    if rule.subgrid_scale_model is not None:
        from .enums import SubgridScaleModel
        learned = rule.subgrid_scale_model == SubgridScaleModel.LEARNED
        d.sgs = N.SGS_MLP if learned else N.SGS_SMAGORINSKY
        d.sgs_constant = 0.0 if learned else float(rule.smagorinsky_constant)
        mask = 0
        # every moment whose (numeric) rate equals the shear rate is adapted, as lbmpy substitutes the
        # shared rate symbol (methods/abstractlbmethod.py:102-131, turbulence_models.py:55-63)
        for k, r in enumerate(native_rates):
            if r == shear:
                mask |= 1 << k
        d.sgs_mask = mask
    for u, vel in enumerate((ubb_velocities or [])[:4]):
        vel = list(vel) + [0.0] * 3
        for k in range(3):
            d.ubb_velocity[u][k] = float(vel[k])
    if fixed_density is not None:
        fd = list(fixed_density) if isinstance(fixed_density, (tuple, list)) else [fixed_density]
        d.fixed_density = float(fd[0] or 0.0)
        d.fixed_density1 = float(fd[1] or 0.0) if len(fd) > 1 else 0.0
    if ubb_options:
        for u, rho in enumerate(list(ubb_options.get("densities", ()))[:4]):
            d.ubb_density[u] = float(rho or 0.0)
        d.ubb_adapt_mask = int(ubb_options.get("adapt_mask", 0))
    for k in range(3):
        d.dims[k] = int(dims[k])
        d.periodic[k] = int(bool(periodic[k]))
    return d


def _stream_handle(stream) -> Optional[int]:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, torch.cuda.Stream):
        return stream.cuda_stream
    return int(stream)


class BoundSweep:
    """A sweep with its plan, strides, flags and stream resolved once: launching it costs one
    ctypes call (the per-step path of LatticeBoltzmannStep)."""

    def __init__(self, plan: N.Plan, strides, flags, stream_handle):
        self.plan = plan
        self._strides = N.i64_array(strides)
        self._flags = ctypes.c_void_p(flags.data_ptr() if flags is not None else None)
        self._flags_ref = flags
        self._stream = ctypes.c_void_p(stream_handle)
        self._lib = N.lib()

    def sweep(self, src_ptr: int, dst_ptr: int, parity: int):
        rc = self._lib.lbm_sweep(self.plan.handle, ctypes.c_void_p(src_ptr), ctypes.c_void_p(dst_ptr),
                                 self._strides, self._flags, parity, None, self._stream)
        if rc:
            N.check(rc, "lbm_sweep")

    def variant(self, src_ptr: int, dst_ptr: int, parity: int) -> str:
        """Name of the sweep kernel a launch with these fields uses ("cell", "pair", "quad",
        "staged")."""
        v = ctypes.c_int(-1)
        N.check(self._lib.lbm_sweep_variant(self.plan.handle, ctypes.c_void_p(src_ptr), ctypes.c_void_p(dst_ptr),
                                            self._strides, parity, None, ctypes.byref(v)), "lbm_sweep_variant")
        return N.VARIANT_NAMES[v.value]

    def run(self, a_ptr: int, b_ptr: int, first_parity: int, steps: int) -> bool:
        """`steps` sweeps in one call; returns True if a pull result ended in `b`."""
        in_b = ctypes.c_int(0)
        N.check(self._lib.lbm_run(self.plan.handle, ctypes.c_void_p(a_ptr), ctypes.c_void_p(b_ptr),
                                  self._strides, self._flags, first_parity, int(steps), ctypes.byref(in_b),
                                  self._stream), "lbm_run")
        return bool(in_b.value)


class LbKernel:
    def __init__(self, update_rule):
        self.update_rule = update_rule
        self.method = update_rule.method
        self._plans = {}
        self.parameters = free_parameters(update_rule)

    @property
    def q(self):
        return self.method.stencil.Q

    def plan(self, dims, periodic, params=None, ubb_velocities=None, fixed_density=None, ubb_options=None) -> N.Plan:
        desc = build_desc(self.update_rule, dims, periodic, params or {}, ubb_velocities,
                          fixed_density=fixed_density, ubb_options=ubb_options)
        closure = self.update_rule.collision_rule.closure
        if closure is not None:
            closure.ensure_uploaded()
        key = (tuple(dims), tuple(bool(p) for p in periodic), torch.cuda.current_device())
        p = self._plans.get(key)
        if p is None:
            p = N.Plan(desc)
            self._plans[key] = p
        elif bytes(p.desc) != bytes(desc):
            p.update(desc)
        return p

    def status(self, clear: bool = True) -> int:
        """OR of the device status words of every plan of this kernel (0: every sweep ran to
        completion; N.STATUS_STAGE_TIMEOUT: a staged sweep stopped waiting for its data)."""
        v = 0
        for p in self._plans.values():
            v |= p.status(clear)
        return v

    def bind(self, pdfs: torch.Tensor, periodic, flags=None, ubb_velocities=None, params=None,
             stream=None, fixed_density=None, ubb_options=None) -> BoundSweep:
        check_pdf_tensor(pdfs, self.q, self.update_rule.storage_dtype, "pdfs")
        dims = [s - 2 for s in pdfs.shape[:3]]
        plan = self.plan(dims, periodic, params or {}, ubb_velocities, fixed_density, ubb_options)
        return BoundSweep(plan, pdfs.stride(), flags, _stream_handle(stream))

    def _parity(self):
        ts = self.update_rule.timestep
        return 1 if ts == Timestep.ODD else 0

    def __call__(self, **kwargs):
        ur = self.update_rule
        src = kwargs.pop(ur.field_name, None)
        if src is None:
            src = kwargs.pop("pdfs", None)
        if src is None:
            raise ValueError(f"missing PDF field {ur.field_name!r}")
        inplace = is_inplace(ur.streaming_pattern)
        dst = kwargs.pop(ur.temporary_field_name, None)
        if inplace:
            dst = src
        elif dst is None:
            raise ValueError(f"missing temporary PDF field {ur.temporary_field_name!r} for the pull pattern")
        flags = kwargs.pop("flags", None)
        ubb = kwargs.pop("ubb_velocities", None)
        fixed_density = kwargs.pop("fixed_density", None)
        periodic = kwargs.pop("periodicity", ur.builtin_periodicity)
        omega_out = kwargs.pop("omega_out", None)
        stream = kwargs.pop("stream", None)
        parity = kwargs.pop("parity", None)
        unknown = set(kwargs) - self.parameters
        if unknown:
            raise ValueError(f"unknown kernel arguments {sorted(unknown)}; parameters are {sorted(self.parameters)}")
        check_pdf_tensor(src, self.q, ur.storage_dtype, ur.field_name)
        check_pdf_tensor(dst, self.q, ur.storage_dtype, ur.temporary_field_name)
        if dst.shape != src.shape or dst.stride() != src.stride():
            raise ValueError("src and dst must have the same shape and strides")
        dims = [s - 2 for s in src.shape[:3]]
        if flags is not None:
            if flags.dtype != torch.uint8 or tuple(flags.shape) != tuple(src.shape[:3]) or not flags.is_cuda:
                raise ValueError("flags must be a CUDA uint8 tensor over the ghost-inclusive domain")
            if flags.stride() != (1, flags.shape[0], flags.shape[0] * flags.shape[1]):
                raise ValueError("flags must be contiguous with x fastest")
        if omega_out is not None:
            if omega_out.dtype != torch.float32 or omega_out.numel() != dims[0] * dims[1] * dims[2]:
                raise ValueError("omega_out must be a float32 tensor with one entry per interior cell")
        plan = self.plan(dims, periodic, kwargs, ubb, fixed_density)
        strides = N.i64_array(src.stride())
        par = self._parity() if parity is None else int(parity)
        N.check(N.lib().lbm_sweep(plan.handle, ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()),
                                  strides, ctypes.c_void_p(flags.data_ptr() if flags is not None else None),
                                  par, ctypes.c_void_p(omega_out.data_ptr() if omega_out is not None else None),
                                  ctypes.c_void_p(_stream_handle(stream))), "lbm_sweep")

    def __repr__(self):
        ur = self.update_rule
        return (f"LbKernel({self.method!r}, pattern={ur.streaming_pattern}, timestep={ur.timestep!s}, "
                f"storage={ur.storage_dtype})")
