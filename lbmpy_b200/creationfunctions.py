"""lbmpy's kernel-creation API, resolved to a B200 sweep instead of generated code.

Mirrors lbmpy ``creationfunctions.py``: ``LBMConfig`` (:100-484), ``LBMOptimisation`` (:487-540),
``create_lb_function`` (:543-559), ``create_lb_ast`` (:562-582), ``create_lb_update_rule``
(:585-638), ``create_lb_collision_rule`` (:641-770), ``create_lb_method`` (:773-868) and
``update_with_default_parameters`` (:920-971).  The normalisation rules of ``LBMConfig`` are kept
(delta-equilibrium inference, TRT magic number, default force models, kernel_type aliases), but
the result of the pipeline is a numeric method description plus a callable that launches the
hand-written sm_100a sweep, not sympy assignments.
"""
from __future__ import annotations

import math
from collections import OrderedDict
from dataclasses import dataclass, field, replace
from fractions import Fraction
from typing import Any, Iterable, List, Optional, Tuple, Union

from . import _native as N
from . import forcemodels
from . import methods as M
from .enums import CollisionSpace, ForceModel, Method, Stencil, SubgridScaleModel, Target, Timestep, is_inplace
from .stencils import LBStencil

__all__ = ["LBMConfig", "LBMOptimisation", "CreateKernelConfig", "create_lb_function", "create_lb_ast",
           "create_lb_update_rule", "create_lb_collision_rule", "create_lb_method",
           "update_with_default_parameters", "LbMethod", "LbmCollisionRule", "LbmUpdateRule", "LbKernel"]


def _is_symbolic(v) -> bool:
    return not isinstance(v, (int, float)) and v is not None and not _is_number(v)


def _is_number(v) -> bool:
    try:
        float(v)
        return True
    except (TypeError, ValueError):
        return False


def _omega_symbol():
    try:
        import sympy as sp
        return sp.Symbol("omega")
    except ImportError:  # pragma: no cover - sympy ships with the image
        return "omega"


@dataclass
class CollisionSpaceInfo:
    collision_space: CollisionSpace


@dataclass
class LBMConfig:
    stencil: Any = field(default_factory=lambda: LBStencil(Stencil.D2Q9))
    method: Any = Method.SRT
    relaxation_rates: Any = None
    relaxation_rate: Any = None
    compressible: bool = False
    zero_centered: bool = True
    delta_equilibrium: Optional[bool] = None
    equilibrium_order: int = 2
    c_s_sq: Any = Fraction(1, 3)
    weighted: bool = True
    nested_moments: Any = None
    force_model: Any = None
    force: Tuple = (0, 0, 0)
    continuous_equilibrium: bool = True
    maxwellian_moments: Optional[bool] = None
    initial_velocity: Any = None
    galilean_correction: bool = False
    fourth_order_correction: Union[float, bool] = False
    collision_space_info: Any = None
    entropic: bool = False
    entropic_newton_iterations: Any = None
    omega_output_field: Any = None
    eddy_viscosity_field: Any = None
    subgrid_scale_model: Any = None
    cassons: Any = False
    fluctuating: Any = False
    temperature: Any = None
    psm_config: Any = None
    output: dict = field(default_factory=dict)
    velocity_input: Any = None
    density_input: Any = None
    conserved_moments: bool = True
    kernel_type: Any = "default_stream_collide"
    streaming_pattern: str = "pull"
    timestep: Timestep = Timestep.BOTH
    field_name: str = "src"
    temporary_field_name: str = "dst"
    lb_method: Any = None
    collision_rule: Any = None
    update_rule: Any = None
    ast: Any = None

    def __post_init__(self):
        # creationfunctions.py:347-484
        if isinstance(self.method, str):
            self.method = Method[self.method.upper()]
        if self.maxwellian_moments is not None:
            self.continuous_equilibrium = self.maxwellian_moments
        if not isinstance(self.stencil, LBStencil):
            self.stencil = LBStencil(self.stencil)
        if self.relaxation_rates is None and self.relaxation_rate is None:
            self.relaxation_rate = _omega_symbol()
        if self.relaxation_rate is not None:
            if self.method in (Method.TRT, Method.TRT_KBC_N1, Method.TRT_KBC_N2, Method.TRT_KBC_N3,
                               Method.TRT_KBC_N4):
                self.relaxation_rates = [self.relaxation_rate,
                                         M.relaxation_rate_from_magic_number(self.relaxation_rate)]
            else:
                self.relaxation_rates = [self.relaxation_rate]
        if not self.compressible and self.method in (Method.MONOMIAL_CUMULANT, Method.CUMULANT):
            raise ValueError("Incompressible cumulant-based methods are not supported (yet).")
        if self.zero_centered and self.entropic:
            raise ValueError("Entropic methods can only be created with `zero_centered=False`.")
        if self.delta_equilibrium is not None:
            if self.delta_equilibrium:
                if not self.zero_centered:
                    raise ValueError("`delta_equilibrium=True` requires `zero_centered=True`!")
                if self.method in (Method.MONOMIAL_CUMULANT, Method.CUMULANT):
                    raise ValueError("Cannot create a cumulant-based method from a delta-equilibrium!")
        else:
            if self.zero_centered:
                self.delta_equilibrium = self.method not in (Method.CENTRAL_MOMENT, Method.MONOMIAL_CUMULANT,
                                                             Method.CUMULANT)
            else:
                self.delta_equilibrium = False
        if isinstance(self.collision_space_info, CollisionSpace):
            self.collision_space_info = CollisionSpaceInfo(self.collision_space_info)
        if self.collision_space_info is None:
            if self.method in (Method.SRT, Method.TRT):
                space = CollisionSpace.POPULATIONS
            elif self.method in (Method.MRT_RAW, Method.MRT):
                space = CollisionSpace.RAW_MOMENTS
            elif self.method == Method.CENTRAL_MOMENT:
                space = CollisionSpace.CENTRAL_MOMENTS
            else:
                space = CollisionSpace.CUMULANTS
            self.collision_space_info = CollisionSpaceInfo(space)
        elif not self.collision_space_info.collision_space.compatible(self.method):
            raise ValueError("Given method is not compatible with given collision space.")
        aliases = {"stream_pull_collide": ("pull", Timestep.BOTH), "collide_stream_push": ("push", Timestep.BOTH),
                   "aa_even": ("aa", Timestep.EVEN), "aa_odd": ("aa", Timestep.ODD),
                   "esotwist_even": ("esotwist", Timestep.EVEN), "esotwist_odd": ("esotwist", Timestep.ODD)}
        if isinstance(self.kernel_type, str) and self.kernel_type in aliases:
            self.streaming_pattern, self.timestep = aliases[self.kernel_type]
            self.kernel_type = "default_stream_collide"
        force_not_zero = any(f != 0 for f in self.force)
        if self.force_model is None and force_not_zero:
            if self.method == Method.CUMULANT:
                self.force_model = forcemodels.CentralMoment(self.force[:self.stencil.D])
            else:
                self.force_model = forcemodels.Guo(self.force[:self.stencil.D])
        classes = {"simple": forcemodels.Simple, "luo": forcemodels.Luo, "guo": forcemodels.Guo,
                   "schiller": forcemodels.Guo, "centralmoment": forcemodels.CentralMoment}
        if isinstance(self.force_model, str):
            name = ForceModel[self.force_model.upper()].name.lower()
            if name not in classes:
                raise NotImplementedError(f"force model {name} is not supported by the B200 sweep")
            self.force_model = classes[name](force=self.force[:self.stencil.D])
        elif isinstance(self.force_model, ForceModel):
            name = self.force_model.name.lower()
            if name not in classes:
                raise NotImplementedError(f"force model {name} is not supported by the B200 sweep")
            self.force_model = classes[name](force=self.force[:self.stencil.D])
        if self.density_input is not None or self.velocity_input is not None:
            self.conserved_moments = False


@dataclass
class LBMOptimisation:
    cse_pdfs: bool = False
    cse_global: bool = False
    simplification: Any = "auto"
    pre_simplification: bool = True
    split: bool = False
    field_size: Any = None
    field_layout: str = "fzyx"
    symbolic_field: Any = None
    symbolic_temporary_field: Any = None
    builtin_periodicity: Tuple[bool, ...] = (False, False, False)
    storage_dtype: Any = None
    """PDF storage type when it differs from the arithmetic type (``CreateKernelConfig.data_type``):
    'float16' / 'bfloat16' / 'e3m12' store zero-centred PDFs in 16 bits and collide in FP32.  e3m12
    (sign, 3 exponent, 12 mantissa bits, scaled by 16) keeps four times finer steps than float16 for
    |f - w| < 1/16 and saturates beyond."""


@dataclass
class CreateKernelConfig:
    """Subset of pystencils' ``CreateKernelConfig`` that applies to the B200 sweep."""
    target: Target = Target.GPU
    data_type: Any = "float64"
    gpu_indexing_params: Any = None
    cpu_openmp: Any = False
    backend: Any = None
    ghost_layers: Any = None

    def __post_init__(self):
        if self.target not in (Target.GPU,):
            raise NotImplementedError("the B200 package only generates GPU sweeps (target=Target.GPU)")


# ------------------------------------------------------------------------------- method
class DensityVelocityComputation:
    """Conserved-quantity conventions of a method (methods/conservedquantitycomputation.py:84-374)."""

    def __init__(self, stencil, compressible, zero_centered, force_model=None):
        self._stencil = stencil
        self.compressible = compressible
        self.zero_centered_pdfs = zero_centered
        self.force_model = force_model
        self.background_density = 1

    @property
    def conserved_quantities(self):
        return {"density": 1, "density_deviation": 1, "velocity": self._stencil.D}


class LbMethod:
    """Numeric description of an lbmpy method: moments (or cumulants), their relaxation rates and
    the storage / equilibrium conventions that the sweep implements."""

    def __init__(self, stencil: LBStencil, kind: str, groups, rates, compressible, zero_centered,
                 delta_equilibrium, equilibrium_order, continuous_equilibrium, force_model, method_enum):
        self.stencil = stencil
        self.kind = kind                       # 'srt', 'trt', 'mrt', 'cumulant'
        self.groups = groups                   # nested list of Poly
        self.relaxation_rates = tuple(rates)   # one per moment, in group order
        self.compressible = compressible
        self.zero_centered = zero_centered
        self.delta_equilibrium = delta_equilibrium
        self.equilibrium_order = equilibrium_order
        self.continuous_equilibrium = continuous_equilibrium
        self.force_model = force_model
        self.method = method_enum
        self.conserved_quantity_computation = DensityVelocityComputation(stencil, compressible, zero_centered,
                                                                         force_model)

    @property
    def dim(self):
        return self.stencil.D

    @property
    def weights(self):
        return [float(w) for w in M.weights(self.stencil.name)]

    @property
    def zero_centered_pdfs(self):
        return self.zero_centered

    @property
    def moments(self):
        """Moment (or cumulant) polynomials as sympy expressions, in relaxation order."""
        import sympy as sp
        x, y, z = sp.symbols("x y z")
        out = []
        for g in self.groups:
            for p in g:
                out.append(sum(sp.Rational(v.numerator, v.denominator) * x ** e[0] * y ** e[1] * z ** e[2]
                               for e, v in p.items()))
        return tuple(out)

    cumulants = moments

    @property
    def relaxation_rate_dict(self):
        return OrderedDict(zip(self.moments, self.relaxation_rates))

    @property
    def shear_relaxation_rate(self):
        rates = {r for g in self.groups for p, r in zip(g, self._group_rates(g)) if M.is_shear(p, self.dim)}
        if len(rates) != 1:
            raise ValueError(f"Shear moments are relaxed with different relaxation times: {rates}")
        return rates.pop()

    def _group_rates(self, group):
        flat = [p for g in self.groups for p in g]
        start = flat.index(group[0])
        return self.relaxation_rates[start:start + len(group)]

    def __repr__(self):
        return (f"LbMethod({self.stencil.name}, {self.kind}, compressible={self.compressible}, "
                f"zero_centered={self.zero_centered}, rates={self.relaxation_rates})")


def create_lb_method(lbm_config=None, **params):
    """creationfunctions.py:773-868 for SRT, TRT, MRT (weighted orthogonal) and CUMULANT."""
    lbm_config, _, _ = update_with_default_parameters(params, lbm_config=lbm_config)
    st = lbm_config.stencil
    if st.name not in ("D3Q19", "D3Q27"):
        raise NotImplementedError(f"the B200 sweep is built for D3Q19 and D3Q27, not {st.name}")
    if lbm_config.entropic or lbm_config.fluctuating or lbm_config.cassons or lbm_config.psm_config:
        raise NotImplementedError("entropic, fluctuating, Casson and PSM collision add-ons are not built")
    if lbm_config.nested_moments is not None:
        raise NotImplementedError("custom moment sets are not built; the default bases are")
    if not lbm_config.zero_centered:
        raise NotImplementedError("the B200 sweep stores zero-centred PDFs (zero_centered=True)")
    if lbm_config.fourth_order_correction and (lbm_config.method != Method.CUMULANT or st.name != "D3Q27"):
        raise ValueError("Fourth-order correction can only be applied to D3Q27 cumulant methods.")
    rates = list(lbm_config.relaxation_rates)
    method = lbm_config.method
    dim = st.D
    if method in (Method.SRT, Method.TRT):
        monos = M.default_monomials(st.name)
        groups = [[M.mono(*e)] for e in monos]
        if method == Method.SRT:
            per = [rates[0]] * len(monos)
        else:
            if len(rates) < 2:
                raise AssertionError("Not enough relaxation rates")
            per = [rates[0] if sum(e) % 2 == 0 else rates[1] for e in monos]
        kind = method.name.lower()
        if not lbm_config.delta_equilibrium:
            raise NotImplementedError("population-space SRT/TRT needs the delta equilibrium "
                                      "(lbmpy: 'Can only derive population-space equations for zero-centered "
                                      "storage if delta equilibrium is used.')")
    elif method == Method.MRT:
        if not lbm_config.weighted:
            raise NotImplementedError("only the weighted-orthogonal MRT basis is built")
        groups = M.mrt_orthogonal_groups(st.name)
        per = M.rates_for_groups(rates, groups, dim, lbm_config.conserved_moments) if all(
            _is_number(r) for r in rates) else _symbolic_rates_for_groups(rates, groups, dim,
                                                                           lbm_config.conserved_moments)
        kind = "mrt"
        if not lbm_config.delta_equilibrium:
            raise NotImplementedError("the MRT sweep uses the delta equilibrium of zero-centred storage")
    elif method == Method.CUMULANT:
        if st.name != "D3Q27":
            raise NotImplementedError("the cumulant sweep is built for D3Q27")
        if lbm_config.fourth_order_correction:
            # creationfunctions.py:696-707, :835-846: shear and bulk rate (bulk 1 by default), the
            # optimal third-order rates, 1 for orders 4-6 (the sweep limits the third-order rates
            # per cell and adds the fourth-order correction terms)
            assert len(rates) <= 2, ("Optimal parametrisation for fourth-order cumulants needs either one or two "
                                     "relaxation rates, associated with the shear (and bulk) viscosity. All other "
                                     "relaxation rates are automatically chosen optimally")
            w1 = rates[0]
            w2 = rates[1] if len(rates) > 1 else 1
            (w3, w4, w5), _ = M.fourth_order_rates(w1, w2)
            rates = [w1, w2, w3, w4, w5, 1, 1, 1, 1, 1]
        groups = M.cumulant_groups()
        per = M.rates_for_groups(rates, groups, dim, lbm_config.conserved_moments) if all(
            _is_number(r) for r in rates) else _symbolic_rates_for_groups(rates, groups, dim,
                                                                           lbm_config.conserved_moments)
        kind = "cumulant"
    elif method == Method.CENTRAL_MOMENT:
        # creationfunctions.py:818-822, methods/creationfunctions.py:336-381: the default D3Q27 central
        # moment groups (default_moment_sets.py:110-148) are the cumulant groups
        if st.name != "D3Q27":
            raise NotImplementedError("the central-moment sweep is built for D3Q27")
        if not lbm_config.compressible:
            raise NotImplementedError("the central-moment sweep is built for compressible methods")
        groups = M.cumulant_groups()
        per = M.rates_for_groups(rates, groups, dim, lbm_config.conserved_moments) if all(
            _is_number(r) for r in rates) else _symbolic_rates_for_groups(rates, groups, dim,
                                                                           lbm_config.conserved_moments)
        kind = "central_moment"
    else:
        raise NotImplementedError(f"method {method} is not built for the B200 sweep")
    fm = lbm_config.force_model
    if fm is not None and not isinstance(fm, (forcemodels.Simple, forcemodels.Luo, forcemodels.Guo,
                                              forcemodels.CentralMoment)):
        raise NotImplementedError(f"force model {fm} is not built")
    if kind == "cumulant" and fm is not None and not isinstance(fm, forcemodels.CentralMoment):
        raise NotImplementedError("the cumulant sweep supports the CentralMoment force model only")
    if kind != "cumulant" and isinstance(fm, forcemodels.CentralMoment):
        raise ValueError("This force model can only be combined with the Cumulant collision model")
    m = LbMethod(st, kind, groups, per, lbm_config.compressible, lbm_config.zero_centered,
                 lbm_config.delta_equilibrium, lbm_config.equilibrium_order, lbm_config.continuous_equilibrium,
                 fm, method)
    lbm_config.lb_method = m
    return m


def _symbolic_rates_for_groups(rates, groups, dim, conserved):
    """Same rule as methods.rates_for_groups, keeping symbolic rates symbolic."""
    numeric = [float(i + 1) * 1000.0 for i in range(len(rates))]   # unique placeholders
    per = M.rates_for_groups(numeric, groups, dim, conserved)
    back = {v: r for v, r in zip(numeric, rates)}
    return [back.get(v, v) for v in per]


# ------------------------------------------------------------------------- collision rule
@dataclass
class LbmCollisionRule:
    """What lbmpy's collision rule adds on top of the method: Galilean correction, SGS model and
    output quantities (creationfunctions.py:641-770)."""
    method: LbMethod
    galilean_correction: bool = False
    subgrid_scale_model: Any = None
    smagorinsky_constant: float = 0.12
    output: dict = field(default_factory=dict)
    closure: Any = None               # MLPClosure for SubgridScaleModel.LEARNED
    simplification_hints: dict = field(default_factory=dict)
    fourth_order_limiter: float = 0.0  # > 0: fourth-order cumulant correction with this limiter


def create_lb_collision_rule(lb_method=None, lbm_config=None, lbm_optimisation=None, config=None,
                             optimization=None, **kwargs):
    lbm_config, lbm_optimisation, config = update_with_default_parameters(kwargs, optimization, lbm_config,
                                                                          lbm_optimisation, config)
    if lbm_config.lb_method is not None:
        lb_method = lbm_config.lb_method
    if lb_method is None:
        lb_method = create_lb_method(lbm_config)
    if lbm_config.density_input is not None or lbm_config.velocity_input is not None:
        raise NotImplementedError("density/velocity input fields are not built")
    if lbm_config.galilean_correction and (lb_method.kind != "cumulant" or lb_method.stencil.name != "D3Q27"):
        raise ValueError("Galilean correction is only defined for D3Q27 cumulant methods.")
    sgs, c, closure = None, 0.12, None
    if lbm_config.subgrid_scale_model:
        sgs = lbm_config.subgrid_scale_model
        if isinstance(sgs, tuple):
            sgs, arg = sgs[0], sgs[1]
            if sgs == SubgridScaleModel.LEARNED:
                closure = arg
            else:
                c = float(arg)
        if sgs == SubgridScaleModel.LEARNED:
            if closure is None:
                raise ValueError("the learned closure needs its network: (SubgridScaleModel.LEARNED, MLPClosure)")
            if lb_method.kind != "cumulant" or lb_method.stencil.name != "D3Q27":
                raise NotImplementedError("the learned closure is built for the D3Q27 cumulant method")
        elif sgs != SubgridScaleModel.SMAGORINSKY:
            raise NotImplementedError("the Smagorinsky and learned subgrid-scale models are built")
    foc = 0.0
    if lbm_config.fourth_order_correction:
        # creationfunctions.py:696-707: True means limiters of 1e6 (practically none)
        if lb_method.kind != "cumulant" or lb_method.stencil.name != "D3Q27":
            raise ValueError("Fourth-order correction is only defined for D3Q27 cumulant methods.")
        if sgs is not None:
            raise NotImplementedError("the fourth-order correction is not built with subgrid-scale models")
        foc = 1e6 if lbm_config.fourth_order_correction is True else float(lbm_config.fourth_order_correction)
    rule = LbmCollisionRule(lb_method, bool(lbm_config.galilean_correction), sgs, c, dict(lbm_config.output),
                            closure=closure, fourth_order_limiter=foc)
    lbm_config.collision_rule = rule
    return rule


# ---------------------------------------------------------------------------- update rule
_DTYPES = {"float64": N.DTYPE_F64, "double": N.DTYPE_F64, "float32": N.DTYPE_F32, "float": N.DTYPE_F32,
           "float16": N.DTYPE_F16, "half": N.DTYPE_F16, "bfloat16": N.DTYPE_BF16, "e3m12": N.DTYPE_E3M12}


def _dtype_name(dt) -> str:
    s = str(dt)
    for k in ("bfloat16", "float16", "float32", "float64", "e3m12"):
        if k in s:
            return k
    if s in ("double",):
        return "float64"
    if s in ("float", "single"):
        return "float32"
    if s in ("half",):
        return "float16"
    raise ValueError(f"unsupported data type {dt}")


@dataclass
class LbmUpdateRule:
    """Collision rule bound to a streaming pattern and PDF fields (creationfunctions.py:585-638)."""
    collision_rule: LbmCollisionRule
    streaming_pattern: str
    timestep: Timestep
    field_name: str
    temporary_field_name: str
    data_type: str
    storage_dtype: str
    builtin_periodicity: Tuple[bool, bool, bool]

    @property
    def method(self):
        return self.collision_rule.method


def create_lb_update_rule(collision_rule=None, lbm_config=None, lbm_optimisation=None, config=None,
                          optimization=None, **kwargs):
    lbm_config, lbm_optimisation, config = update_with_default_parameters(kwargs, optimization, lbm_config,
                                                                          lbm_optimisation, config)
    if lbm_config.collision_rule is not None:
        collision_rule = lbm_config.collision_rule
    if collision_rule is None:
        collision_rule = create_lb_collision_rule(lbm_config.lb_method, lbm_config=lbm_config,
                                                  lbm_optimisation=lbm_optimisation, config=config)
    if lbm_config.kernel_type != "default_stream_collide":
        raise NotImplementedError(f"kernel_type {lbm_config.kernel_type!r} is not built; the fused "
                                  "stream-collide sweep is")
    pattern = lbm_config.streaming_pattern
    if pattern not in ("pull", "push", "aa", "esotwist", "esopull", "esopush"):
        raise NotImplementedError(f"streaming pattern {pattern!r} is not built (pull, push, aa, esotwist, "
                                  "esopull and esopush are)")
    if is_inplace(pattern) and lbm_config.timestep == Timestep.BOTH:
        raise ValueError(f"Invalid timestep for streaming pattern {pattern}: Both")
    if lbm_optimisation.field_layout not in ("fzyx", "f", "reverse_numpy", "SoA"):
        raise NotImplementedError("the sweep needs the fzyx (SoA, x fastest) layout")
    dt = config.data_type
    if isinstance(dt, dict):
        dt = dt.get(lbm_config.field_name, next(iter(dt.values())))
    data_type = _dtype_name(dt)
    storage = _dtype_name(lbm_optimisation.storage_dtype) if lbm_optimisation.storage_dtype else data_type
    if data_type not in ("float64", "float32"):
        raise ValueError("the arithmetic type (CreateKernelConfig.data_type) must be float64 or float32")
    if storage in ("float16", "bfloat16", "e3m12") and data_type != "float32":
        raise ValueError("16-bit PDF storage collides in float32: set data_type='float32'")
    if storage == "float64" and data_type != "float64" or storage == "float32" and data_type != "float32":
        raise ValueError("storage_dtype must match data_type unless it is a 16-bit type")
    if storage in ("float16", "bfloat16", "e3m12") and pattern in ("push", "esopull", "esopush"):
        raise NotImplementedError(f"streaming pattern {pattern!r} is built for float64 / float32 storage")
    rule = LbmUpdateRule(collision_rule, pattern, lbm_config.timestep, lbm_config.field_name,
                         lbm_config.temporary_field_name, data_type, storage,
                         tuple(bool(b) for b in (list(lbm_optimisation.builtin_periodicity) + [False] * 3)[:3]))
    lbm_config.update_rule = rule
    return rule


def create_lb_ast(update_rule=None, lbm_config=None, lbm_optimisation=None, config=None, optimization=None,
                  **kwargs):
    """There is no AST: returns the update rule the sweep is built from."""
    lbm_config, lbm_optimisation, config = update_with_default_parameters(kwargs, optimization, lbm_config,
                                                                          lbm_optimisation, config)
    if lbm_config.update_rule is not None:
        update_rule = lbm_config.update_rule
    if update_rule is None:
        update_rule = create_lb_update_rule(lbm_config.collision_rule, lbm_config=lbm_config,
                                            lbm_optimisation=lbm_optimisation, config=config)
    return update_rule


def create_lb_function(ast=None, lbm_config=None, lbm_optimisation=None, config=None, optimization=None,
                       **kwargs):
    """Returns a callable that runs one fused stream-collide sweep on the GPU:
    ``kernel(src=pdfs, dst=tmp, flags=None, **params)`` (in-place patterns: ``kernel(src=pdfs)``)."""
    lbm_config, lbm_optimisation, config = update_with_default_parameters(kwargs, optimization, lbm_config,
                                                                          lbm_optimisation, config)
    update_rule = ast
    if lbm_config.ast is not None:
        update_rule = lbm_config.ast
    if update_rule is None:
        update_rule = create_lb_update_rule(lbm_config.collision_rule, lbm_config=lbm_config,
                                            lbm_optimisation=lbm_optimisation, config=config)
    from .kernel import LbKernel
    k = LbKernel(update_rule)
    k.method = update_rule.method
    k.update_rule = update_rule
    k.ast = update_rule
    return k


def update_with_default_parameters(params, opt_params=None, lbm_config=None, lbm_optimisation=None, config=None):
    """creationfunctions.py:920-971: merges legacy ``optimization={...}`` dicts and kwargs."""
    pystencils_keys = ["target", "backend", "cpu_openmp", "double_precision", "gpu_indexing", "gpu_indexing_params",
                       "cpu_vectorize_info"]
    config_params = {k: v for k, v in (opt_params or {}).items() if k in pystencils_keys}
    if "double_precision" in config_params:
        config_params["data_type"] = "float64" if config_params.pop("double_precision") else "float32"
    config_params.pop("gpu_indexing", None)
    config_params.pop("cpu_vectorize_info", None)
    if "target" in config_params and isinstance(config_params["target"], str):
        config_params["target"] = Target[config_params["target"].upper()]
    if not config:
        config = CreateKernelConfig(**config_params)
    else:
        config = replace(config, **config_params)
    opt_keys = ["cse_pdfs", "cse_global", "simplification", "pre_simplification", "split", "field_size",
                "field_layout", "symbolic_field", "symbolic_temporary_field", "builtin_periodicity", "storage_dtype"]
    opt_dict = {k: v for k, v in (opt_params or {}).items() if k in opt_keys}
    if not lbm_optimisation:
        lbm_optimisation = LBMOptimisation(**opt_dict)
    else:
        lbm_optimisation = replace(lbm_optimisation, **opt_dict)
    params = dict(params or {})
    if not lbm_config:
        lbm_config = LBMConfig(**params)
    else:
        for k in params:
            if not hasattr(lbm_config, k):
                raise KeyError(f"{params[k]} is not a valid kwarg. Please look in LBMConfig for valid settings")
        if params:
            lbm_config = replace(lbm_config, **params)
    return lbm_config, lbm_optimisation, config
