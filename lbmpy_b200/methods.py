"""Numeric description of lbmpy's lattice Boltzmann methods for the B200 sweep.

lbmpy derives every method symbolically (sympy) and hands the equations to a code generator.
Here the same definitions are evaluated with exact rational arithmetic and reduced to the
handful of tables the hand-written CUDA kernels need:

* the stencil in lbmpy's default ('walberla') direction order and its weights
  (lbmpy ``stencils.py:193-227``, ``maxwellian_equilibrium.py:24-61``);
* the equilibrium of the zero-centred, delta-equilibrium storage used by SRT/TRT/MRT
  (``equilibrium/continuous_hydro_maxwellian.py:19-235``; continuous Maxwellian moments truncated
  at second order in u, which differs from the textbook discrete equilibrium for D3Q19);
* the weighted-orthogonal MRT moment basis (``methods/creationfunctions.py:464-526``,
  ``moments.py:469-548``) and lbmpy's rule for assigning relaxation rates to moment groups
  (``methods/creationfunctions.py:600-706``);
* the D3Q27 polynomial cumulant groups of Geier et al. 2015
  (``methods/default_moment_sets.py:110-148``).

Polynomials are dicts ``{(a, b, c): Fraction}`` meaning ``sum coef * x^a y^b z^c``.
"""
from __future__ import annotations

import itertools
import math
from fractions import Fraction
from typing import Dict, List, Sequence, Tuple

Poly = Dict[Tuple[int, int, int], Fraction]

# ----------------------------------------------------------------------------- stencils
WALBERLA_ORDER = {
    "D2Q9": ((0, 0), (0, 1), (0, -1), (-1, 0), (1, 0), (-1, 1), (1, 1), (-1, -1), (1, -1)),
    "D3Q19": ((0, 0, 0), (0, 1, 0), (0, -1, 0), (-1, 0, 0), (1, 0, 0), (0, 0, 1), (0, 0, -1),
              (-1, 1, 0), (1, 1, 0), (-1, -1, 0), (1, -1, 0), (0, 1, 1), (0, -1, 1), (-1, 0, 1),
              (1, 0, 1), (0, 1, -1), (0, -1, -1), (-1, 0, -1), (1, 0, -1)),
}
WALBERLA_ORDER["D3Q27"] = WALBERLA_ORDER["D3Q19"] + (
    (1, 1, 1), (-1, 1, 1), (1, -1, 1), (-1, -1, 1), (1, 1, -1), (-1, 1, -1), (1, -1, -1), (-1, -1, -1))

_WEIGHT_BY_NORM = {
    9: (Fraction(4, 9), Fraction(1, 9), Fraction(1, 36)),
    19: (Fraction(1, 3), Fraction(1, 18), Fraction(1, 36)),
    27: (Fraction(8, 27), Fraction(2, 27), Fraction(1, 54), Fraction(1, 216)),
}


def directions(name: str):
    return WALBERLA_ORDER[name]


def weights(name: str) -> List[Fraction]:
    dirs = WALBERLA_ORDER[name]
    return [_WEIGHT_BY_NORM[len(dirs)][sum(abs(v) for v in d)] for d in dirs]


def inverse_index(name: str) -> List[int]:
    dirs = WALBERLA_ORDER[name]
    return [dirs.index(tuple(-v for v in d)) for d in dirs]


def _d3(d):
    return tuple(d) + (0,) * (3 - len(d))


# ----------------------------------------------------------------------------- polynomials
def mono(a=0, b=0, c=0) -> Poly:
    return {(a, b, c): Fraction(1)}


def padd(p: Poly, q: Poly, s=1) -> Poly:
    r = dict(p)
    for e, v in q.items():
        r[e] = r.get(e, Fraction(0)) + s * v
        if r[e] == 0:
            del r[e]
    return r


def pscale(p: Poly, s) -> Poly:
    return {e: v * s for e, v in p.items() if v * s != 0}


def peval(p: Poly, d) -> Fraction:
    d = _d3(d)
    return sum((v * d[0] ** e[0] * d[1] ** e[1] * d[2] ** e[2] for e, v in p.items()), Fraction(0))


def leading_exponent(p: Poly):
    """Leading monomial under lex order x > y > z (sympy's ``LM``)."""
    return max(p) if p else (0, 0, 0)


def order(p: Poly) -> int:
    """Degree of the leading monomial (lbmpy ``moments.get_order``)."""
    return sum(leading_exponent(p)) if any(sum(e) for e in p) else 0


def _mono_str(e) -> str:
    """The string sympy prints for a monomial in x, y, z (used by lbmpy's moment sort key)."""
    parts = []
    for s, k in zip("xyz", e):
        if k == 1:
            parts.append(s)
        elif k > 1:
            parts.append(f"{s}**{k}")
    return "*".join(parts) if parts else "1"


def _mono_sort_key(e):
    s = _mono_str(e)
    return sum(e), sum(1 for k in e if k), len(s), s


def is_bulk(p: Poly, dim: int) -> bool:
    found = [Fraction(0)] * dim
    quadratic = False
    for e, v in p.items():
        if sum(e) == 2:
            quadratic = True
            for i in range(dim):
                if e[i] == 2:
                    found[i] += v
        elif sum(e) > 2:
            return False
    return quadratic and any(found) and len(set(found)) == 1


def is_shear(p: Poly, dim: int) -> bool:
    if is_bulk(p, dim):
        return False
    quadratic = False
    for e in p:
        if sum(e) == 2:
            quadratic = True
        elif sum(e) > 2:
            return False
    return quadratic


def default_monomials(name: str) -> List[Tuple[int, int, int]]:
    """lbmpy ``get_default_moment_set_for_stencil`` (moments.py:512-548), sorted like lbmpy."""
    if name == "D2Q9":
        monos = [(a, b, 0) for a in range(3) for b in range(3)]
    else:
        monos = [(a, b, c) for a in range(3) for b in range(3) for c in range(3)]
        if name == "D3Q19":
            drop = set()
            for t in [(1, 2, 2), (1, 1, 2), (2, 2, 2), (1, 1, 1)]:
                drop |= set(itertools.permutations(t))
            monos = [m for m in monos if m not in drop]
    return sorted(monos, key=_mono_sort_key)


# ----------------------------------------------------------------------------- MRT basis
def _gram_schmidt(polys: List[Poly], dirs, w) -> List[Poly]:
    vecs, out = [], []
    for p in polys:
        v = [peval(p, d) for d in dirs]
        q = dict(p)
        for pv, pp in zip(vecs, out):
            den = sum(a * a * wi for a, wi in zip(pv, w))
            ov = sum(a * b * wi for a, b, wi in zip(v, pv, w)) / den
            v = [a - ov * b for a, b in zip(v, pv)]
            q = padd(q, pp, -ov)
        vecs.append(v)
        out.append(q)
    return out


def mrt_orthogonal_groups(name: str) -> List[List[Poly]]:
    """Weighted-orthogonal MRT moments grouped like lbmpy's ``create_mrt_orthogonal``:
    [density], [momentum], [shear], [bulk], then one group per higher order."""
    dirs = directions(name)
    dim = len(dirs[0])
    polys = [mono(*e) for e in default_monomials(name)]
    if dim == 2:
        diag = [padd(mono(2), mono(0, 2)), mono(2)]
    else:
        diag = [padd(padd(mono(2), mono(0, 2)), mono(0, 0, 2)), mono(2), padd(mono(0, 2), mono(0, 0, 2), -1)]
    for i in range(dim):
        e = [0, 0, 0]
        e[i] = 2
        sq = mono(*e)
        if sq in polys:
            polys[polys.index(sq)] = diag[i]
    ortho = _gram_schmidt(polys, dirs, weights(name))
    scaled = []
    for p in ortho:
        den = math.lcm(*[v.denominator for v in p.values()])
        scaled.append(pscale(p, den))
    groups: Dict[int, List[Poly]] = {}
    for p in scaled:
        groups.setdefault(order(p), []).append(p)
    nested = [groups[k] for k in groups]
    second = nested[2]
    nested[2] = [p for p in second if is_shear(p, dim)]
    nested.insert(3, [p for p in second if is_bulk(p, dim)])
    return nested


def cumulant_groups() -> List[List[Poly]]:
    """D3Q27 polynomial cumulant groups (Geier et al. 2015)."""
    m = mono
    return [
        [m()],
        [m(1), m(0, 1), m(0, 0, 1)],
        [m(1, 1), m(1, 0, 1), m(0, 1, 1), padd(m(2), m(0, 2), -1), padd(m(2), m(0, 0, 2), -1)],
        [padd(padd(m(2), m(0, 2)), m(0, 0, 2))],
        [padd(m(1, 2), m(1, 0, 2)), padd(m(2, 1), m(0, 1, 2)), padd(m(2, 0, 1), m(0, 2, 1))],
        [padd(m(1, 2), m(1, 0, 2), -1), padd(m(2, 1), m(0, 1, 2), -1), padd(m(2, 0, 1), m(0, 2, 1), -1)],
        [m(1, 1, 1)],
        [padd(padd(m(2, 2), pscale(m(2, 0, 2), -2)), m(0, 2, 2)),
         padd(padd(m(2, 2), m(2, 0, 2)), pscale(m(0, 2, 2), -2))],
        [padd(padd(m(2, 2), m(2, 0, 2)), m(0, 2, 2))],
        [m(2, 1, 1), m(1, 2, 1), m(1, 1, 2)],
        [m(2, 2, 1), m(2, 1, 2), m(1, 2, 2)],
        [m(2, 2, 2)],
    ]


def fourth_order_rates(w1, w2):
    """The third-order rates (w3, w4, w5) before the per-cell limiters, and the parameters (a, b), of
    the fourth-order cumulant correction for shear rate w1 and bulk rate w2 (Geier et al. 2017,
    eq. 111-116; methods/cumulantbased/fourth_order_correction.py:79-97, :149-170).  Works on numbers
    and on sympy expressions."""
    w11, w12, w22 = w1 * w1, w1 * w2, w2 * w2
    w3 = 8 * (w1 - 2) * (w2 * (3 * w1 - 1) - 5 * w1) / (8 * (5 - 2 * w1) * w1 + w2 * (8 + w1 * (9 * w1 - 26)))
    w4 = 8 * (w1 - 2) * (w1 + w2 * (3 * w1 - 7)) / (w2 * (56 - 42 * w1 + 9 * w11) - 8 * w1)
    w5 = 24 * (w1 - 2) * (4 * w11 + w12 * (18 - 13 * w1) + w22 * (2 + w1 * (6 * w1 - 11))) / (
        16 * w11 * (w1 - 6) - 2 * w12 * (216 + 5 * w1 * (9 * w1 - 46))
        + w22 * (w1 * (3 * w1 - 10) * (15 * w1 - 28) - 48))
    den = (w1 - w2) * (w2 * (2 + 3 * w1) - 8 * w1)
    a = (4 * w11 + 2 * w12 * (w1 - 6) + w22 * (w1 * (10 - 3 * w1) - 4)) / den
    b = (4 * w12 * (9 * w1 - 16) - 4 * w11 - 2 * w22 * (2 + 9 * w1 * (w1 - 2))) / (3 * den)
    return (w3, w4, w5), (a, b)


def rates_for_groups(rates: Sequence[float], groups: List[List[Poly]], dim: int,
                     conserved_moments: bool = True) -> List[float]:
    """Per-moment relaxation rates in group order, following lbmpy's rule
    (methods/creationfunctions.py:600-706): one rate -> shear = rate, conserved 0, rest 1;
    one rate per moment -> as given; otherwise [shear, bulk, one per higher group]."""
    flat = [p for g in groups for p in g]
    n_shear = sum(1 for p in flat if is_shear(p, dim))
    n_bulk = sum(1 for p in flat if is_bulk(p, dim))
    rates = [float(r) for r in rates]
    out: List[float] = []
    if len(rates) == 1:
        for p in flat:
            if conserved_moments and order(p) <= 1:
                out.append(0.0)
            elif is_shear(p, dim) or (not conserved_moments and order(p) <= 1):
                out.append(rates[0])
            else:
                out.append(1.0)
        return out
    if len(rates) == len(flat):
        return list(rates)
    it = iter(rates)
    try:
        shear = next(it) if n_shear else None
        bulk = next(it) if n_bulk else None
        take, rr = True, None
        for g in groups:
            if take:
                rr = next(it)
            take = False
            for p in g:
                if order(p) <= 1:
                    out.append(0.0 if conserved_moments else shear)
                elif is_shear(p, dim):
                    out.append(shear)
                elif is_bulk(p, dim):
                    out.append(bulk)
                else:
                    take = True
                    out.append(rr)
    except StopIteration:
        raise ValueError("Not enough relaxation rates are specified. You can either specify one relaxation "
                         "rate, which is used as the shear relaxation rate, one rate for shear, bulk and each "
                         "higher-order group, or one rate per moment.") from None
    return out


def relaxation_rate_from_magic_number(omega, magic_number=Fraction(3, 16)):
    """Second TRT rate from the magic number (relaxationrates.py:17-20)."""
    return (4 - 2 * omega) / (4 * float(magic_number) * omega + 2 - omega)


def relaxation_rate_from_lattice_viscosity(nu):
    return 2 / (6 * nu + 1)


def lattice_viscosity_from_relaxation_rate(omega):
    return (2 - omega) / (6 * omega)


# ----------------------------------------------------------------------------- equilibrium
def _gauss_1d(n: int) -> List[Fraction]:
    """<(u + c_s Z)^n> as polynomial coefficients in u (c_s^2 = 1/3)."""
    coef = [Fraction(0)] * (n + 1)
    for k in range(0, n + 1, 2):
        df = 1
        for j in range(k - 1, 0, -2):
            df *= j
        coef[n - k] += math.comb(n, k) * df * Fraction(1, 3) ** (k // 2)
    return coef


def maxwell_moment(e, max_order=2) -> Dict[Tuple[int, int, int], Fraction]:
    """Raw moment x^a y^b z^c of the unit-density continuous Maxwellian, as a polynomial in
    (ux, uy, uz) truncated at total degree ``max_order``."""
    g = [_gauss_1d(k) for k in e]
    out: Dict[Tuple[int, int, int], Fraction] = {}
    for p in range(len(g[0])):
        for q in range(len(g[1])):
            for r in range(len(g[2])):
                if p + q + r > max_order:
                    continue
                v = g[0][p] * g[1][q] * g[2][r]
                if v:
                    out[(p, q, r)] = out.get((p, q, r), Fraction(0)) + v
    return out


def moment_equilibrium(poly: Poly, max_order=2):
    """Equilibrium of a polynomial moment: (P(0), linear[3], quadratic[6]) so that the unit-density
    value is P0 + lin.u + sum quad_ab u_a u_b with ab in (xx, yy, zz, xy, xz, yz)."""
    acc: Dict[Tuple[int, int, int], Fraction] = {}
    for e, v in poly.items():
        for k, c in maxwell_moment(e, max_order).items():
            acc[k] = acc.get(k, Fraction(0)) + v * c
    p0 = acc.get((0, 0, 0), Fraction(0))
    lin = [acc.get((1, 0, 0), Fraction(0)), acc.get((0, 1, 0), Fraction(0)), acc.get((0, 0, 1), Fraction(0))]
    quad = [acc.get((2, 0, 0), Fraction(0)), acc.get((0, 2, 0), Fraction(0)), acc.get((0, 0, 2), Fraction(0)),
            acc.get((1, 1, 0), Fraction(0)), acc.get((1, 0, 1), Fraction(0)), acc.get((0, 1, 1), Fraction(0))]
    return p0, lin, quad


def _solve(rows: List[List[Fraction]]) -> List[List[Fraction]]:
    n = len(rows)
    a = [list(map(Fraction, r)) + [Fraction(int(i == j)) for j in range(n)] for i, r in enumerate(rows)]
    for col in range(n):
        piv = next(r for r in range(col, n) if a[r][col] != 0)
        a[col], a[piv] = a[piv], a[col]
        pv = a[col][col]
        a[col] = [v / pv for v in a[col]]
        for r in range(n):
            if r != col and a[r][col]:
                f = a[r][col]
                a[r] = [x - f * y for x, y in zip(a[r], a[col])]
    return [r[n:] for r in a]


def population_equilibrium(name: str, continuous: bool = True):
    """Per-direction equilibrium coefficients of the unit-density equilibrium:
    f_eq_i = w_i + lin_i.u + sum quad_i,ab u_a u_b  (quadratic order (xx, yy, zz, xy, xz, yz)).
    continuous=True: M^-1 of the truncated continuous Maxwellian moments (lbmpy's default);
    continuous=False: the discrete textbook equilibrium (maxwellian_equilibrium.py:85-122)."""
    dirs = directions(name)
    w = weights(name)
    if not continuous:
        lins, quads = [], []
        for d, wi in zip(dirs, w):
            c = _d3(d)
            lins.append([3 * wi * ci for ci in c])
            quads.append([wi * (Fraction(9, 2) * c[0] ** 2 - Fraction(3, 2)),
                          wi * (Fraction(9, 2) * c[1] ** 2 - Fraction(3, 2)),
                          wi * (Fraction(9, 2) * c[2] ** 2 - Fraction(3, 2)),
                          wi * 9 * c[0] * c[1], wi * 9 * c[0] * c[2], wi * 9 * c[1] * c[2]])
        return w, lins, quads
    polys = [mono(*e) for e in default_monomials(name)]
    M = [[peval(p, d) for d in dirs] for p in polys]
    Minv = _solve(M)
    eqs = [moment_equilibrium(p) for p in polys]
    Q = len(dirs)
    lins = [[sum(Minv[i][k] * eqs[k][1][a] for k in range(Q)) for a in range(3)] for i in range(Q)]
    quads = [[sum(Minv[i][k] * eqs[k][2][a] for k in range(Q)) for a in range(6)] for i in range(Q)]
    w0 = [sum(Minv[i][k] * eqs[k][0] for k in range(Q)) for i in range(Q)]
    assert w0 == w, "moment-matched background must reproduce the lattice weights"
    return w, lins, quads


def mrt_tables(name: str):
    """Moment matrix M (rows: moments in group order), its inverse and the equilibrium
    coefficients (P0, lin, quad) of every moment of the weighted-orthogonal MRT basis."""
    groups = mrt_orthogonal_groups(name)
    flat = [p for g in groups for p in g]
    dirs = directions(name)
    M = [[peval(p, d) for d in dirs] for p in flat]
    Minv = _solve(M)
    eq = [moment_equilibrium(p) for p in flat]
    return groups, M, Minv, eq
