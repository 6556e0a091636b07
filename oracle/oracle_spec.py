"""Method description for the CPU oracle -- TEST INFRASTRUCTURE ONLY.

This module is part of the oracle that the parity tests, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of ``bench.py`` use as the checker.  The product (``lbmpy_b200``) never
imports it.

It restates, with sympy, how lbmpy turns an ``LBMConfig`` into the numbers a sweep needs:
stencil order and weights, the moment basis, the relaxation rate of every moment, the
equilibrium moments and the force / subgrid-scale settings.  Each step cites the lbmpy source
it follows (paths relative to ``src/lbmpy`` of mabau/lbmpy).  The derivation is deliberately
independent from the product's own (``lbmpy_b200/methods.py``), so that a mistake in one of
them shows up as a parity failure.

Parity status: the restatement is checked against the reference's golden data
(``tests/reference_files/*.npz`` -> ``tests/golden``: direction order, getter arithmetic and
the force shift) and against the reference's structural known-answer tests (zero-centring
identity, streaming-pattern equivalence, set/get round trip, Poiseuille).  lbmpy itself cannot
be imported in this environment (its code generator pystencils is absent), so sweep-level
parity with lbmpy's own kernel is pinned only through those tests.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from fractions import Fraction
from typing import Dict, List, Optional, Sequence, Tuple

import sympy as sp

X, Y, Z = sp.symbols("x y z")
MOMENT_SYMBOLS = (X, Y, Z)

# --------------------------------------------------------------------------------------------
# Stencils: walberla ordering, stencils.py:132-134 (D2Q9), :193-199 (D3Q19), :220-227 (D3Q27)
# --------------------------------------------------------------------------------------------
_STENCILS = {
    "D2Q9": ((0, 0), (0, 1), (0, -1), (-1, 0), (1, 0), (-1, 1), (1, 1), (-1, -1), (1, -1)),
    "D3Q19": ((0, 0, 0), (0, 1, 0), (0, -1, 0), (-1, 0, 0), (1, 0, 0), (0, 0, 1), (0, 0, -1),
              (-1, 1, 0), (1, 1, 0), (-1, -1, 0), (1, -1, 0), (0, 1, 1), (0, -1, 1), (-1, 0, 1),
              (1, 0, 1), (0, 1, -1), (0, -1, -1), (-1, 0, -1), (1, 0, -1)),
    "D3Q27": ((0, 0, 0), (0, 1, 0), (0, -1, 0), (-1, 0, 0), (1, 0, 0), (0, 0, 1), (0, 0, -1),
              (-1, 1, 0), (1, 1, 0), (-1, -1, 0), (1, -1, 0), (0, 1, 1), (0, -1, 1), (-1, 0, 1),
              (1, 0, 1), (0, 1, -1), (0, -1, -1), (-1, 0, -1), (1, 0, -1), (1, 1, 1), (-1, 1, 1),
              (1, -1, 1), (-1, -1, 1), (1, 1, -1), (-1, 1, -1), (1, -1, -1), (-1, -1, -1)),
}

# lattice weights by |c|_1, maxwellian_equilibrium.py:24-61
_WEIGHTS = {
    9: {0: Fraction(4, 9), 1: Fraction(1, 9), 2: Fraction(1, 36)},
    19: {0: Fraction(1, 3), 1: Fraction(1, 18), 2: Fraction(1, 36)},
    27: {0: Fraction(8, 27), 1: Fraction(2, 27), 2: Fraction(1, 54), 3: Fraction(1, 216)},
}


def stencil_directions(name: str):
    return _STENCILS[name]


def stencil_weights(name: str):
    dirs = _STENCILS[name]
    return [_WEIGHTS[len(dirs)][sum(abs(c) for c in d)] for d in dirs]


# --------------------------------------------------------------------------------------------
# Moments, moments.py
# --------------------------------------------------------------------------------------------
def _poly_from_exponents(e):
    r = sp.Integer(1)
    for s, k in zip(MOMENT_SYMBOLS, e):
        r *= s ** k
    return r


def get_order(moment) -> int:
    """moments.py:248-266: degree of the leading monomial."""
    if isinstance(moment, tuple):
        return sum(moment)
    if len(moment.atoms(sp.Symbol)) == 0:
        return 0
    lm = sp.polys.polytools.LM(moment)
    return sum(sp.degree(lm, gen=m) for m in lm.atoms(sp.Symbol))


def moment_sort_key(moment):
    """moments.py:175-179."""
    s = str(moment)
    return get_order(moment), len(moment.atoms(sp.Symbol)), len(s), s


def default_moment_set(name: str):
    """moments.py:512-548 (``get_default_moment_set_for_stencil``) for D2Q9/D3Q19/D3Q27."""
    import itertools
    if name == "D2Q9":
        monos = list(itertools.product(range(3), repeat=2))
        return sorted((_poly_from_exponents(e + (0,)) for e in monos), key=moment_sort_key)
    all27 = list(itertools.product(range(3), repeat=3))
    if name == "D3Q27":
        return sorted((_poly_from_exponents(e) for e in all27), key=moment_sort_key)
    if name == "D3Q19":
        non_matched = [(1, 2, 2), (1, 1, 2), (2, 2, 2), (1, 1, 1)]
        removed = set()
        for t in non_matched:
            removed |= set(itertools.permutations(t))
        keep = [e for e in all27 if e not in removed]
        return sorted((_poly_from_exponents(e) for e in keep), key=moment_sort_key)
    raise ValueError(name)


def poly_terms(poly, dim=3) -> List[Tuple[Fraction, Tuple[int, int, int]]]:
    """Polynomial in x,y,z -> [(coefficient, exponent tuple)] (moments.py:143-172)."""
    poly = sp.expand(sp.sympify(poly))
    out = []
    for term in sp.Add.make_args(poly):
        coef, rest = term.as_coeff_Mul()
        e = [0, 0, 0]
        for f in sp.Mul.make_args(rest):
            if f == 1:
                continue
            b, k = f.as_base_exp()
            e[MOMENT_SYMBOLS.index(b)] += int(k)
        out.append((Fraction(int(sp.numer(coef)), int(sp.denom(coef))), tuple(e)))
    return out


def moment_matrix(moments, dirs):
    """moments.py:417-441: row = moment polynomial evaluated at every lattice velocity."""
    rows = []
    for m in moments:
        terms = poly_terms(m)
        row = []
        for d in dirs:
            d3 = tuple(d) + (0,) * (3 - len(d))
            v = Fraction(0)
            for coef, e in terms:
                v += coef * (d3[0] ** e[0]) * (d3[1] ** e[1]) * (d3[2] ** e[2])
            row.append(v)
        rows.append(row)
    return rows


def is_bulk_moment(moment, dim) -> bool:
    """moments.py:348-362."""
    found = [Fraction(0)] * dim
    quadratic = False
    for coef, e in poly_terms(moment):
        s = sum(e)
        if s == 2:
            quadratic = True
            for i in range(dim):
                if e[i] == 2:
                    found[i] += coef
        elif s > 2:
            return False
    return quadratic and found != [0] * dim and len(set(found)) == 1


def is_shear_moment(moment, dim) -> bool:
    """moments.py:365-380."""
    if is_bulk_moment(moment, dim):
        return False
    quadratic = False
    for coef, e in poly_terms(moment):
        s = sum(e)
        if s == 2:
            quadratic = True
        elif s > 2:
            return False
    return quadratic


def is_even(moment) -> bool:
    """moments.py:201-223: invariant under c -> -c."""
    opp = moment.subs({X: -X, Y: -Y, Z: -Z}, simultaneous=True)
    return sp.expand(moment - opp) == 0


def gram_schmidt(moments, dirs, weights):
    """moments.py:469-510, weighted scalar product <a,b> = sum a_i b_i w_i."""
    moments = list(moments)
    cols = [[Fraction(v) for v in row] for row in moment_matrix(moments, dirs)]
    ortho = []
    for i in range(len(cols)):
        cur = list(cols[i])
        for j in range(i):
            prev = ortho[j]
            den = sum(p * p * w for p, w in zip(prev, weights))
            ov = sum(c * p * w for c, p, w in zip(cur, prev, weights)) / den
            cur = [c - ov * p for c, p in zip(cur, prev)]
            moments[i] = moments[i] - sp.Rational(ov.numerator, ov.denominator) * moments[j]
        ortho.append(cur)
    return [sp.expand(m) for m in moments]


def _common_denominator(expr):
    """Least common multiple of the denominators of all coefficients."""
    dens = [c.denominator for c, _ in poly_terms(expr)]
    return math.lcm(*dens) if dens else 1


def mrt_orthogonal_nested_moments(name: str, weighted: bool = True):
    """methods/creationfunctions.py:464-516 (``create_mrt_orthogonal`` without nested_moments)."""
    dirs = stencil_directions(name)
    dim = len(dirs[0])
    moments = default_moment_set(name)
    if dim == 2:
        diag = [X ** 2 + Y ** 2, X ** 2]
    else:
        diag = [X ** 2 + Y ** 2 + Z ** 2, X ** 2, Y ** 2 - Z ** 2]
    for i, d in enumerate(MOMENT_SYMBOLS[:dim]):
        if d ** 2 in moments:
            moments[moments.index(d ** 2)] = diag[i]
    w = stencil_weights(name) if weighted else [Fraction(1)] * len(dirs)
    ortho = gram_schmidt(moments, dirs, w)
    scaled = [sp.expand(e * _common_denominator(e)) for e in ortho]
    groups: Dict[int, list] = {}
    for m in scaled:
        groups.setdefault(get_order(m), []).append(m)
    nested = [groups[k] for k in groups]
    second = nested[2]
    bulk = [m for m in second if is_bulk_moment(m, dim)]
    shear = [m for m in second if is_shear_moment(m, dim)]
    assert len(bulk) + len(shear) == len(second)
    nested[2] = shear
    nested.insert(3, bulk)
    return nested


def cumulant_groups_d3q27():
    """methods/default_moment_sets.py:110-148 (Geier et al. 2015 polynomial cumulants)."""
    x, y, z = X, Y, Z
    return [
        [sp.Integer(1)],
        [x, y, z],
        [x * y, x * z, y * z, x ** 2 - y ** 2, x ** 2 - z ** 2],
        [x ** 2 + y ** 2 + z ** 2],
        [x * y ** 2 + x * z ** 2, x ** 2 * y + y * z ** 2, x ** 2 * z + y ** 2 * z],
        [x * y ** 2 - x * z ** 2, x ** 2 * y - y * z ** 2, x ** 2 * z - y ** 2 * z],
        [x * y * z],
        [x ** 2 * y ** 2 - 2 * x ** 2 * z ** 2 + y ** 2 * z ** 2,
         x ** 2 * y ** 2 + x ** 2 * z ** 2 - 2 * y ** 2 * z ** 2],
        [x ** 2 * y ** 2 + x ** 2 * z ** 2 + y ** 2 * z ** 2],
        [x ** 2 * y * z, x * y ** 2 * z, x * y * z ** 2],
        [x ** 2 * y ** 2 * z, x ** 2 * y * z ** 2, x * y ** 2 * z ** 2],
        [x ** 2 * y ** 2 * z ** 2],
    ]


def relaxation_info(rates: Sequence[float], nested, dim, conserved_moments=True):
    """methods/creationfunctions.py:600-706 (``_get_relaxation_info_dict``)."""
    result = []  # list of (moment, rate) in nested order
    number = sum(len(g) for g in nested)
    n_shear = sum(1 for g in nested for m in g if is_shear_moment(m, dim))
    n_bulk = sum(1 for g in nested for m in g if is_bulk_moment(m, dim))
    if len(rates) == 1:
        for g in nested:
            for m in g:
                if conserved_moments:
                    if get_order(m) <= 1:
                        r = 0.0
                    elif is_shear_moment(m, dim):
                        r = rates[0]
                    else:
                        r = 1.0
                else:
                    r = rates[0] if (is_shear_moment(m, dim) or get_order(m) <= 1) else 1.0
                result.append((m, r))
        return result
    if len(rates) == number:
        it = iter(rates)
        return [(m, next(it)) for g in nested for m in g]
    it = iter(rates)
    try:
        shear_rr = next(it) if n_shear > 0 else None
        bulk_rr = next(it) if n_bulk > 0 else None
        next_rr = True
        rr = None
        for g in nested:
            if next_rr:
                rr = next(it)
            next_rr = False
            for m in g:
                if conserved_moments:
                    if get_order(m) <= 1:
                        r = 0.0
                    elif is_shear_moment(m, dim):
                        r = shear_rr
                    elif is_bulk_moment(m, dim):
                        r = bulk_rr
                    else:
                        next_rr = True
                        r = rr
                else:
                    if is_shear_moment(m, dim) or get_order(m) <= 1:
                        r = shear_rr
                    elif is_bulk_moment(m, dim):
                        r = bulk_rr
                    else:
                        next_rr = True
                        r = rr
                result.append((m, r))
    except StopIteration:
        raise ValueError("Not enough relaxation rates are specified.")
    return result


def magic_rate(omega, magic=Fraction(3, 16)):
    """relaxationrates.py:17-20."""
    return (4 - 2 * omega) / (4 * float(magic) * omega + 2 - omega)


# --------------------------------------------------------------------------------------------
# The resolved method that the C oracle consumes
# --------------------------------------------------------------------------------------------
KIND_MOMENT, KIND_CUMULANT, KIND_CENTRAL = 0, 1, 2
FORCE_NONE, FORCE_GUO, FORCE_CENTRAL_MOMENT, FORCE_SIMPLE, FORCE_LUO = 0, 1, 2, 3, 4
SGS_NONE, SGS_SMAGORINSKY, SGS_MLP = 0, 1, 2


@dataclass
class OracleMethod:
    stencil: str
    kind: int
    dirs: tuple
    weights: list
    moments: list                 # sympy polynomials (moments, or polynomial cumulants)
    rates: list                   # one per moment
    compressible: bool
    zero_centered: bool
    delta_equilibrium: bool
    equilibrium_order: int = 2
    force_model: int = FORCE_NONE
    force: tuple = (0.0, 0.0, 0.0)
    galilean_correction: bool = False
    sgs: int = SGS_NONE
    sgs_constant: float = 0.12
    shear_rate: float = 0.0
    mlp: object = None            # learned-closure parameters (float32 array) when sgs == SGS_MLP
    continuous_equilibrium: bool = True   # SRT/TRT/MRT: False = discrete Maxwellian
    fourth_order_limiter: float = 0.0     # > 0: fourth-order correction with this limiter

    @property
    def Q(self):
        return len(self.dirs)

    @property
    def D(self):
        return len(self.dirs[0])


def fourth_order_rates(w1: float, w2: float):
    """Optimal third-order rates (w3, w4, w5) before the limiters and the parameters (a, b) of the
    fourth-order correction for shear rate w1 and bulk rate w2 (Geier et al. 2017, eq. 111-116;
    methods/cumulantbased/fourth_order_correction.py:79-97 and :149-170)."""
    w11, w12, w22 = w1 * w1, w1 * w2, w2 * w2
    w3 = (8 * (w1 - 2) * (w2 * (3 * w1 - 1) - 5 * w1)) / (
        8 * (5 - 2 * w1) * w1 + w2 * (8 + w1 * (9 * w1 - 26)))
    w4 = (8 * (w1 - 2) * (w1 + w2 * (3 * w1 - 7))) / (w2 * (56 - 42 * w1 + 9 * w11) - 8 * w1)
    w5 = (24 * (w1 - 2) * (4 * w11 + w12 * (18 - 13 * w1) + w22 * (2 + w1 * (6 * w1 - 11)))) / (
        16 * w11 * (w1 - 6) - 2 * w12 * (216 + 5 * w1 * (9 * w1 - 46))
        + w22 * (w1 * (3 * w1 - 10) * (15 * w1 - 28) - 48))
    den = (w1 - w2) * (w2 * (2 + 3 * w1) - 8 * w1)
    a = (4 * w11 + 2 * w12 * (w1 - 6) + w22 * (w1 * (10 - 3 * w1) - 4)) / den
    b = (4 * w12 * (9 * w1 - 16) - 4 * w11 - 2 * w22 * (2 + 9 * w1 * (w1 - 2))) / (3 * den)
    return (w3, w4, w5), (a, b)


def resolve(stencil: str, method: str, relaxation_rate=None, relaxation_rates=None,
            compressible=False, zero_centered=True, delta_equilibrium=None,
            equilibrium_order=2, force=(0.0, 0.0, 0.0), force_model=None,
            galilean_correction=False, smagorinsky=None, mlp=None,
            continuous_equilibrium=True, fourth_order_correction=False) -> OracleMethod:
    """Follows ``LBMConfig.__post_init__`` (creationfunctions.py:347-484) and
    ``create_lb_method`` (creationfunctions.py:773-868) for SRT/TRT/MRT/CUMULANT."""
    method = method.lower()
    dirs = stencil_directions(stencil)
    dim = len(dirs[0])
    w = stencil_weights(stencil)
    if relaxation_rates is None:
        if relaxation_rate is None:
            raise ValueError("numeric relaxation rates are required by the oracle")
        if method == "trt":
            relaxation_rates = [relaxation_rate, magic_rate(relaxation_rate)]
        else:
            relaxation_rates = [relaxation_rate]
    relaxation_rates = list(relaxation_rates)
    foc_limiter = 0.0
    if fourth_order_correction:
        # creationfunctions.py:696-707 and :835-846: the method takes ten rates, the shear and bulk
        # rates (bulk 1 by default), the optimal third-order rates and 1 for every higher group
        if method != "cumulant" or stencil != "D3Q27":
            raise ValueError("Fourth-order correction can only be applied to D3Q27 cumulant methods.")
        if len(relaxation_rates) == 1:
            relaxation_rates.append(1.0)
        w1, w2 = float(relaxation_rates[0]), float(relaxation_rates[1])
        (w3, w4, w5), _ = fourth_order_rates(w1, w2)
        relaxation_rates = [w1, w2, w3, w4, w5, 1.0, 1.0, 1.0, 1.0, 1.0]
        foc_limiter = 1e6 if fourth_order_correction is True else float(fourth_order_correction)
    if method == "cumulant" and not compressible:
        raise ValueError("Incompressible cumulant-based methods are not supported (yet).")
    if delta_equilibrium is None:
        delta_equilibrium = bool(zero_centered) and method != "cumulant"
    force = tuple(float(f) for f in force) + (0.0,) * (3 - len(force))
    fm = FORCE_NONE
    if any(f != 0 for f in force):
        if force_model is None:
            force_model = "centralmoment" if method == "cumulant" else "guo"
        fm = {"guo": FORCE_GUO, "schiller": FORCE_GUO, "centralmoment": FORCE_CENTRAL_MOMENT,
              "simple": FORCE_SIMPLE, "luo": FORCE_LUO}[force_model.lower()]
    if method in ("srt", "trt"):
        moments = default_moment_set(stencil)
        if method == "srt":
            rates = [relaxation_rates[0]] * len(moments)
        else:
            rates = [relaxation_rates[0] if is_even(m) else relaxation_rates[1] for m in moments]
        kind = KIND_MOMENT
    elif method == "mrt":
        nested = mrt_orthogonal_nested_moments(stencil, weighted=True)
        info = relaxation_info(relaxation_rates, nested, dim)
        moments = [m for m, _ in info]
        rates = [float(r) for _, r in info]
        kind = KIND_MOMENT
    elif method == "cumulant":
        if stencil != "D3Q27":
            raise ValueError("oracle cumulant method: D3Q27 only")
        nested = cumulant_groups_d3q27()
        info = relaxation_info(relaxation_rates, nested, dim)
        moments = [m for m, _ in info]
        rates = [float(r) for _, r in info]
        kind = KIND_CUMULANT
        delta_equilibrium = False
    elif method in ("central_moment", "centralmoment"):
        # creationfunctions.py:818-822 -> methods/creationfunctions.py:336-381 with
        # default_moment_sets.cascaded_moment_sets_literature (the D3Q27 groups equal the cumulants')
        if stencil != "D3Q27":
            raise ValueError("oracle central-moment method: D3Q27 only")
        if not compressible:
            raise ValueError("oracle central-moment method: compressible only")
        nested = cumulant_groups_d3q27()
        info = relaxation_info(relaxation_rates, nested, dim)
        moments = [m for m, _ in info]
        rates = [float(r) for _, r in info]
        kind = KIND_CENTRAL
        delta_equilibrium = False
    else:
        raise ValueError(method)
    if galilean_correction and (method != "cumulant" or stencil != "D3Q27"):
        raise ValueError("Galilean correction is only defined for D3Q27 cumulant methods.")
    shear_rates = {r for m, r in zip(moments, rates) if is_shear_moment(m, dim)}
    shear = shear_rates.pop() if len(shear_rates) == 1 else 0.0
    sgs = SGS_NONE
    c_sgs = 0.12
    if smagorinsky is not None:
        sgs = SGS_SMAGORINSKY
        c_sgs = 0.12 if smagorinsky is True else float(smagorinsky)
    if mlp is not None:
        sgs = SGS_MLP
    return OracleMethod(stencil=stencil, kind=kind, dirs=dirs, weights=w, moments=moments,
                        rates=[float(r) for r in rates], compressible=bool(compressible),
                        zero_centered=bool(zero_centered), delta_equilibrium=bool(delta_equilibrium),
                        equilibrium_order=equilibrium_order, force_model=fm, force=force,
                        galilean_correction=bool(galilean_correction), sgs=sgs, sgs_constant=c_sgs,
                        shear_rate=float(shear), mlp=mlp,
                        continuous_equilibrium=bool(continuous_equilibrium) or kind != KIND_MOMENT,
                        fourth_order_limiter=foc_limiter)
