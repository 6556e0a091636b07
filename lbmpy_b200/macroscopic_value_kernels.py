"""Density / velocity getter and equilibrium setter on the GPU.

lbmpy ``macroscopic_value_kernels.py``: ``pdf_initialization_assignments`` (:29-45),
``macroscopic_values_getter`` (:48-61), ``compile_macroscopic_values_getter`` (:88-167) and
``compile_macroscopic_values_setter`` (:170-242).  The setter writes the method's equilibrium
through the write accessor of the previous time step; the getter reads the values the previous
step wrote (``get_field_accesses`` :14-26).  Velocities carry the force model's half-force
shift F/(2 rho) (``forcemodels.py:592-593``).
"""
from __future__ import annotations

import ctypes

import torch

from . import _native as N
from .enums import Target, Timestep
from .fields import check_pdf_tensor, dtype_name

_PATTERNS = ("pull", "push", "aa", "esotwist", "esopull", "esopush")


def _rule_for(lb_method, streaming_pattern, storage_dtype, collision_rule=None):
    from .creationfunctions import LbmCollisionRule, LbmUpdateRule
    if streaming_pattern not in _PATTERNS:
        raise NotImplementedError(f"streaming pattern {streaming_pattern!r} is not built")
    rule = collision_rule or LbmCollisionRule(lb_method)
    data_type = "float64" if storage_dtype == "float64" else "float32"
    return LbmUpdateRule(rule, streaming_pattern, Timestep.BOTH, "pdfs", "pdfs_tmp", data_type, storage_dtype,
                         (False, False, False))


class _MacroPlanCache:
    def __init__(self, lb_method, streaming_pattern, collision_rule=None):
        self.lb_method = lb_method
        self.pattern = streaming_pattern
        self.collision_rule = collision_rule
        self._plans = {}

    def get(self, pdfs, params=None, periodicity=(False, False, False)):
        from .kernel import build_desc
        storage = dtype_name(pdfs.dtype)
        dims = tuple(int(s) - 2 for s in pdfs.shape[:3])
        key = (storage, dims, tuple(periodicity), torch.cuda.current_device())
        rule = _rule_for(self.lb_method, self.pattern, storage, self.collision_rule)
        desc = build_desc(rule, dims, periodicity, params or {}, rates_needed=False)
        p = self._plans.get(key)
        if p is None:
            p = N.Plan(desc)
            self._plans[key] = p
        elif bytes(p.desc) != bytes(desc):
            p.update(desc)
        return p


def _compute_dtype(pdfs):
    return torch.float64 if pdfs.dtype == torch.float64 else torch.float32


def _interior(t, dims):
    """Accept interior-shaped or ghost-inclusive macroscopic arrays."""
    if tuple(t.shape[:3]) == tuple(d + 2 for d in dims):
        return t[1:-1, 1:-1, 1:-1]
    if tuple(t.shape[:3]) != tuple(dims):
        raise ValueError(f"macroscopic field of shape {tuple(t.shape)} matches neither the interior {dims} "
                         f"nor the ghost-inclusive domain")
    return t


def _prev_parity(previous_timestep) -> int:
    return 1 if previous_timestep == Timestep.ODD else 0


def set_equilibrium(plan_cache, pdfs, density, velocity, previous_timestep=Timestep.BOTH, params=None,
                    periodicity=(False, False, False), stream=None):
    m = plan_cache.lb_method
    check_pdf_tensor(pdfs, m.stencil.Q, dtype_name(pdfs.dtype))
    dims = tuple(int(s) - 2 for s in pdfs.shape[:3])
    cd = torch.float64          # the setter evaluates the equilibrium in FP64 for every storage type
    dev = pdfs.device
    if isinstance(density, torch.Tensor):
        rho = _interior(density.to(device=dev, dtype=cd), dims)
        if rho.dim() == 4:
            rho = rho[..., 0]
    else:
        rho = torch.full(dims, float(density), dtype=cd, device=dev)
    if isinstance(velocity, torch.Tensor):
        u = _interior(velocity.to(device=dev, dtype=cd), dims)
    else:
        vel = [float(v) for v in velocity] + [0.0] * 3
        u = torch.tensor(vel[:3], dtype=cd, device=dev).expand(*dims, 3)
    if u.shape[-1] != 3:
        raise ValueError("velocity must have 3 components")
    plan = plan_cache.get(pdfs, params, periodicity)
    s = torch.cuda.current_stream().cuda_stream if stream is None else stream.cuda_stream
    N.check(N.lib().lbm_set_equilibrium(plan.handle, ctypes.c_void_p(pdfs.data_ptr()), N.i64_array(pdfs.stride()),
                                        ctypes.c_void_p(rho.data_ptr()), N.i64_array(rho.stride()),
                                        ctypes.c_void_p(u.data_ptr()), N.i64_array(u.stride()),
                                        _prev_parity(previous_timestep), ctypes.c_void_p(s)), "lbm_set_equilibrium")


def get_macroscopic(plan_cache, pdfs, density=None, velocity=None, previous_timestep=Timestep.BOTH, params=None,
                    periodicity=(False, False, False), stream=None):
    """Writes density / velocity into the given tensors (any float dtype, interior or ghost-inclusive)."""
    m = plan_cache.lb_method
    check_pdf_tensor(pdfs, m.stencil.Q, dtype_name(pdfs.dtype))
    dims = tuple(int(s) - 2 for s in pdfs.shape[:3])
    cd = _compute_dtype(pdfs)
    targets = []
    rho_t = u_t = None
    if density is not None:
        d = _interior(density, dims)
        if d.dim() == 4:
            d = d[..., 0]
        rho_t = d if (d.dtype == cd and d.is_cuda and d.device == pdfs.device) else torch.empty(dims, dtype=cd,
                                                                                             device=pdfs.device)
        targets.append((d, rho_t))
    if velocity is not None:
        v = _interior(velocity, dims)
        u_t = v if (v.dtype == cd and v.is_cuda and v.device == pdfs.device) else torch.empty(
            dims + (3,), dtype=cd, device=pdfs.device)
        targets.append((v, u_t))
    plan = plan_cache.get(pdfs, params, periodicity)
    s = torch.cuda.current_stream().cuda_stream if stream is None else stream.cuda_stream
    N.check(N.lib().lbm_get_macroscopic(
        plan.handle, ctypes.c_void_p(pdfs.data_ptr()), N.i64_array(pdfs.stride()),
        ctypes.c_void_p(rho_t.data_ptr() if rho_t is not None else None),
        N.i64_array(rho_t.stride()) if rho_t is not None else None,
        ctypes.c_void_p(u_t.data_ptr() if u_t is not None else None),
        N.i64_array(u_t.stride()) if u_t is not None else None,
        _prev_parity(previous_timestep), ctypes.c_void_p(s)), "lbm_get_macroscopic")
    for user, tmp in targets:
        if user is not tmp:
            user.copy_(tmp)


def compile_macroscopic_values_getter(lb_method, output_quantities, pdf_arr=None, ghost_layers=1,
                                      iteration_slice=None, field_layout="numpy", target=Target.GPU,
                                      streaming_pattern="pull", previous_timestep=Timestep.BOTH):
    """Returns ``getter(pdfs, density=..., velocity=...)`` (macroscopic_value_kernels.py:88-167)."""
    if not isinstance(output_quantities, (list, tuple)):
        output_quantities = [output_quantities]
    known = lb_method.conserved_quantity_computation.conserved_quantities
    unknown = [q for q in output_quantities if q not in known]
    if unknown:
        raise ValueError(f"No such conserved quantity: {unknown}, conserved quantities are {list(known)}")
    if ghost_layers != 1 or iteration_slice is not None:
        raise NotImplementedError("the getter iterates over the whole interior")
    cache = _MacroPlanCache(lb_method, streaming_pattern)

    def getter(pdfs, **kwargs):
        if pdf_arr is not None and (pdfs.shape != pdf_arr.shape or pdfs.stride() != pdf_arr.stride()):
            raise AssertionError("Pdf array not matching blueprint which was used to compile")
        if not set(output_quantities).issubset(kwargs.keys()):
            raise ValueError(f"You have to specify the output field for each of the following quantities: "
                             f"{output_quantities}")
        get_macroscopic(cache, pdfs, kwargs.get("density"), kwargs.get("velocity"), previous_timestep)

    return getter


def compile_macroscopic_values_setter(lb_method, quantities_to_set, pdf_arr=None, ghost_layers=1,
                                      iteration_slice=None, field_layout="numpy", target=Target.GPU,
                                      streaming_pattern="pull", previous_timestep=Timestep.BOTH):
    """Returns ``setter(pdfs)`` writing the equilibrium of the given density / velocity
    (macroscopic_value_kernels.py:170-242)."""
    if ghost_layers != 1 or iteration_slice is not None:
        raise NotImplementedError("the setter iterates over the whole interior")
    cache = _MacroPlanCache(lb_method, streaming_pattern)
    density = quantities_to_set.get("density", 1.0)
    velocity = quantities_to_set.get("velocity", (0.0, 0.0, 0.0))

    def setter(pdfs, **kwargs):
        if pdf_arr is not None and (pdfs.shape != pdf_arr.shape or pdfs.stride() != pdf_arr.stride()):
            raise AssertionError("Pdf array not matching blueprint which was used to compile")
        set_equilibrium(cache, pdfs, kwargs.get("density", density), kwargs.get("velocity", velocity),
                        previous_timestep)

    return setter


def macroscopic_values_setter(lb_method, density, velocity, pdfs, streaming_pattern="pull",
                              previous_timestep=Timestep.BOTH, set_pre_collision_pdfs=False):
    """Immediate form of lbmpy's ``macroscopic_values_setter``: writes the equilibrium into ``pdfs``."""
    if set_pre_collision_pdfs:
        raise NotImplementedError("setting pre-collision PDFs is not built")
    set_equilibrium(_MacroPlanCache(lb_method, streaming_pattern), pdfs, density, velocity, previous_timestep)


pdf_initialization_assignments = macroscopic_values_setter


def macroscopic_values_getter(lb_method, density, velocity, pdfs, streaming_pattern="pull",
                              previous_timestep=Timestep.BOTH, use_pre_collision_pdfs=False):
    """Immediate form of lbmpy's ``macroscopic_values_getter``: fills ``density`` / ``velocity``."""
    if use_pre_collision_pdfs:
        raise NotImplementedError("reading pre-collision PDFs is not built")
    get_macroscopic(_MacroPlanCache(lb_method, streaming_pattern), pdfs, density, velocity, previous_timestep)
