"""Writes ``lbm_tables.h``: the compile-time lattice tables of the CUDA sweep.

Run ``python -m lbmpy_b200.csrc.gen_tables`` (the build does it).  The tables come from
``lbmpy_b200.methods`` (exact rationals) and are emitted as ``constexpr`` functions so that
fully unrolled kernel loops fold every coefficient into the instruction stream; zero
coefficients disappear at compile time.
"""
from __future__ import annotations

import os
from fractions import Fraction

from lbmpy_b200 import methods as M

HERE = os.path.dirname(os.path.abspath(__file__))


def _f(v) -> str:
    v = Fraction(v)
    if v.denominator == 1:
        return f"{v.numerator}.0"
    return repr(float(v))


def _array_fn(name, values, rettype="double", nidx=1, dims=None):
    flat = ", ".join(values)
    if nidx == 1:
        return (f"LBM_HD constexpr {rettype} {name}(int i) {{\n"
                f"    constexpr {rettype} t[{len(values)}] = {{{flat}}};\n    return t[i];\n}}\n")
    n0, n1 = dims
    return (f"LBM_HD constexpr {rettype} {name}(int i, int j) {{\n"
            f"    constexpr {rettype} t[{n0 * n1}] = {{{flat}}};\n    return t[i * {n1} + j];\n}}\n")


def generate() -> str:
    out = ["// Generated by gen_tables.py from lbmpy_b200/methods.py -- do not edit.",
           "// Lattice tables of lbmpy's D3Q19 / D3Q27 methods in walberla direction order.",
           "#pragma once", "",
           "#ifndef LBM_HD", "#if defined(__CUDACC__)", "#define LBM_HD __host__ __device__ __forceinline__",
           "#else", "#define LBM_HD inline", "#endif", "#endif", "",
           "namespace lbm_tables {", ""]
    for name in ("D3Q19", "D3Q27"):
        q = len(M.directions(name))
        dirs = M.directions(name)
        inv = M.inverse_index(name)
        w = M.weights(name)
        pre = f"q{q}_"
        out.append(f"// ---------------- {name}")
        for d, axis in enumerate("xyz"):
            out.append(_array_fn(pre + "c" + axis, [str(v[d]) for v in dirs], "int"))
        out.append(_array_fn(pre + "inv", [str(v) for v in inv], "int"))
        # one representative direction per pair of opposite directions (the lower index)
        out.append(_array_fn(pre + "pair", [str(i) for i in range(1, q) if i < inv[i]], "int"))
        out.append(_array_fn(pre + "w", [_f(v) for v in w]))
        for cont, tag in ((True, "cont"), (False, "disc")):
            _, lin, quad = M.population_equilibrium(name, cont)
            out.append(_array_fn(pre + "eqlin_" + tag, [_f(v) for r in lin for v in r], nidx=2, dims=(q, 3)))
            out.append(_array_fn(pre + "eqquad_" + tag, [_f(v) for r in quad for v in r], nidx=2, dims=(q, 6)))
        groups, Mm, Minv, eq = M.mrt_tables(name)
        # the sweep transforms sums and differences of opposite populations: every row of M must be
        # even or odd under c -> -c, and column k of M^-1 must share row k's parity
        for k in range(q):
            ev = all(Mm[k][i] == Mm[k][inv[i]] for i in range(q))
            od = all(Mm[k][i] == -Mm[k][inv[i]] for i in range(q))
            assert ev != od, f"{name} MRT row {k} has no definite parity"
            assert all(Minv[i][k] == (1 if ev else -1) * Minv[inv[i]][k] for i in range(q)), \
                f"{name} MRT inverse column {k} breaks the parity of row {k}"
        gid = [gi for gi, g in enumerate(groups) for _ in g]
        out.append(f"constexpr int {pre}mrt_ngroups = {len(groups)};")
        out.append(_array_fn(pre + "mrt_group", [str(v) for v in gid], "int"))
        even = [int(all(Mm[k][i] == Mm[k][inv[i]] for i in range(q))) for k in range(q)]
        out.append(_array_fn(pre + "mrt_even", [str(v) for v in even], "int"))
        out.append(_array_fn(pre + "mrt_M", [_f(v) for r in Mm for v in r], nidx=2, dims=(q, q)))
        out.append(_array_fn(pre + "mrt_Minv", [_f(v) for r in Minv for v in r], nidx=2, dims=(q, q)))
        out.append(_array_fn(pre + "mrt_p0", [_f(e[0]) for e in eq]))
        # moments of the Luo / Guo force populations w_i (9 (c.F)(c.u) + 3 c.F - 3 u.F): for an even
        # row, 9 sum_ab T_k,ab F_a u_b - 3 (u.F) S_k; for an odd row, 3 sum_a B_k,a F_a
        prs = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))
        T = [[sum(Mm[k][i] * w[i] * dirs[i][a] * dirs[i][b] for i in range(q)) for a, b in prs] for k in range(q)]
        B = [[sum(Mm[k][i] * w[i] * dirs[i][a] for i in range(q)) for a in range(3)] for k in range(q)]
        S = [sum(Mm[k][i] * w[i] for i in range(q)) for k in range(q)]
        out.append(_array_fn(pre + "mrt_fT", [_f(v) for r in T for v in r], nidx=2, dims=(q, 6)))
        out.append(_array_fn(pre + "mrt_fB", [_f(v) for r in B for v in r], nidx=2, dims=(q, 3)))
        out.append(_array_fn(pre + "mrt_fS", [_f(v) for v in S]))
        out.append(_array_fn(pre + "mrt_lin", [_f(v) for e in eq for v in e[1]], nidx=2, dims=(q, 3)))
        out.append(_array_fn(pre + "mrt_quad", [_f(v) for e in eq for v in e[2]], nidx=2, dims=(q, 6)))
        out.append("")
    out.append("}  // namespace lbm_tables")
    return "\n".join(out) + "\n"


def write(path=None):
    path = path or os.path.join(HERE, "lbm_tables.h")
    text = generate()
    old = open(path).read() if os.path.exists(path) else None
    if old != text:
        with open(path, "w") as f:
            f.write(text)
    return path


if __name__ == "__main__":
    print(write())
