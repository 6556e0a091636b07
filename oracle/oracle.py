"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loaded by tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` as
the checker; the product never imports it.  Arrays follow lbmpy's convention: shape
``(X+2, Y+2, Z+2, Q)`` (ghost layer included) with the fzyx memory layout (x fastest, PDF index
slowest), i.e. ``arr[x, y, z, q]`` with numpy strides ``(8, 8*(X+2), ..., ...)``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from fractions import Fraction

import numpy as np
import sympy as sp

from . import oracle_spec as spec

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

QMAX, TMAX = 27, 40
MLP_NPARAM = 10 * 32 + 32 + 32 * 32 + 32 + 32 + 1 + 1
PATTERNS = {"pull": 0, "push": 1, "aa": 2, "esotwist": 3, "esopull": 4, "esopush": 5}


class OmMethod(ctypes.Structure):
    _fields_ = [
        ("D", ctypes.c_int), ("Q", ctypes.c_int),
        ("c", (ctypes.c_int * 3) * QMAX),
        ("inv", ctypes.c_int * QMAX),
        ("w", ctypes.c_double * QMAX),
        ("kind", ctypes.c_int),
        ("compressible", ctypes.c_int), ("zero_centered", ctypes.c_int),
        ("delta_eq", ctypes.c_int), ("eq_order", ctypes.c_int),
        ("nterms", ctypes.c_int * QMAX),
        ("texp", ((ctypes.c_int * 3) * TMAX) * QMAX),
        ("tcoef", (ctypes.c_double * TMAX) * QMAX),
        ("M", (ctypes.c_double * QMAX) * QMAX),
        ("Minv", (ctypes.c_double * QMAX) * QMAX),
        ("rate", ctypes.c_double * QMAX),
        ("force_model", ctypes.c_int),
        ("F", ctypes.c_double * 3),
        ("galilean", ctypes.c_int),
        ("sgs", ctypes.c_int),
        ("sgs_c", ctypes.c_double),
        ("shear_rate", ctypes.c_double),
        ("mlp", ctypes.c_float * MLP_NPARAM),
        ("discrete_eq", ctypes.c_int),
        ("ubb_adapt", ctypes.c_int),
        ("ubb_density", ctypes.c_double),
        ("ubb_link", ctypes.c_void_p),
        ("fd_rho1", ctypes.c_double),
        ("link_code", ctypes.c_void_p),
        ("link_value", ctypes.c_void_p),
        ("foc_limiter", ctypes.c_double),
    ]


class OmGrid(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int * 3), ("g", ctypes.c_int * 3), ("s", ctypes.c_int64 * 4)]


def build():
    """Compile the oracle library in place (make in this directory)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liblbm_oracle.so")
        if not os.path.exists(path):
            build()
        _LIB = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        _LIB.om_sizeof_method.restype = ctypes.c_int
        assert _LIB.om_sizeof_method() == ctypes.sizeof(OmMethod), "oracle struct layout mismatch"
        _LIB.om_run.restype = ctypes.c_int
    return _LIB


def _exact_inverse(rows):
    n = len(rows)
    a = [[Fraction(v) for v in r] + [Fraction(int(i == j)) for j in range(n)] for i, r in enumerate(rows)]
    for col in range(n):
        piv = next(r for r in range(col, n) if a[r][col] != 0)
        a[col], a[piv] = a[piv], a[col]
        p = a[col][col]
        a[col] = [v / p for v in a[col]]
        for r in range(n):
            if r != col and a[r][col] != 0:
                fct = a[r][col]
                a[r] = [v - fct * pv for v, pv in zip(a[r], a[col])]
    return [row[n:] for row in a]


class Oracle:
    """A resolved lbmpy method on the CPU oracle."""

    def __init__(self, method: spec.OracleMethod):
        self.spec = method
        m = OmMethod()
        dirs = method.dirs
        D, Q = method.D, method.Q
        m.D, m.Q = D, Q
        for i, d in enumerate(dirs):
            d3 = tuple(d) + (0,) * (3 - D)
            for k in range(3):
                m.c[i][k] = d3[k]
            m.inv[i] = dirs.index(tuple(-v for v in d))
            m.w[i] = float(method.weights[i])
        m.kind = method.kind
        m.compressible = int(method.compressible)
        m.zero_centered = int(method.zero_centered)
        m.delta_eq = int(method.delta_equilibrium)
        m.eq_order = method.equilibrium_order
        for k, mom in enumerate(method.moments):
            terms = spec.poly_terms(mom)
            assert len(terms) <= TMAX
            m.nterms[k] = len(terms)
            for t, (coef, e) in enumerate(terms):
                m.tcoef[k][t] = float(coef)
                for j in range(3):
                    m.texp[k][t][j] = e[j]
            m.rate[k] = method.rates[k]
        if method.kind == spec.KIND_MOMENT:
            M = spec.moment_matrix(method.moments, dirs)
        else:
            monos = [(a, b, c) for a in range(3) for b in range(3) for c in range(3)]
            M = []
            for mom in method.moments:
                row = [Fraction(0)] * 27
                for coef, e in spec.poly_terms(mom):
                    row[monos.index(e)] += coef
                M.append(row)
        Minv = _exact_inverse(M)
        for k in range(Q):
            for i in range(Q):
                m.M[k][i] = float(M[k][i])
                m.Minv[k][i] = float(Minv[k][i])
        m.force_model = method.force_model
        for k in range(3):
            m.F[k] = method.force[k]
        m.galilean = int(method.galilean_correction)
        m.sgs = method.sgs
        m.sgs_c = method.sgs_constant
        m.shear_rate = method.shear_rate
        if method.mlp is not None:
            w = np.asarray(method.mlp, dtype=np.float32).reshape(-1)
            assert w.size == MLP_NPARAM, f"closure parameters: {w.size} != {MLP_NPARAM}"
            ctypes.memmove(ctypes.addressof(m.mlp), w.ctypes.data, w.nbytes)
        m.discrete_eq = int(not method.continuous_equilibrium)
        m.foc_limiter = float(method.fourth_order_limiter)
        self._m = m
        self.M = np.array([[float(v) for v in r] for r in M])
        self.Minv = np.array([[float(v) for v in r] for r in Minv])

    # -- helpers -------------------------------------------------------------------------------
    @property
    def Q(self):
        return self.spec.Q

    @property
    def D(self):
        return self.spec.D

    def new_field(self, shape):
        """Zeroed PDF array for an interior domain `shape` in lbmpy's fzyx layout."""
        shape = tuple(shape) + (1,) * (3 - len(shape))
        ext = [s + 2 for s in shape[:self.D]] + [1] * (3 - self.D)
        buf = np.zeros((self.Q, ext[2], ext[1], ext[0]), dtype=np.float64)
        return buf.transpose(3, 2, 1, 0)

    def _grid(self, arr):
        g = OmGrid()
        ext = arr.shape[:3]
        for d in range(3):
            gl = 1 if d < self.D else 0
            g.g[d] = gl
            g.n[d] = ext[d] - 2 * gl
        for d in range(4):
            g.s[d] = arr.strides[d] // 8
        return g

    @staticmethod
    def _ptr(a):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    # -- kernels -------------------------------------------------------------------------------
    def collide(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.zeros_like(f)
        om = ctypes.c_double(0.0)
        lib().om_collide(ctypes.byref(self._m), self._ptr(f), self._ptr(out), ctypes.byref(om))
        return out

    def equilibrium(self, rho, u):
        u3 = np.zeros(3)
        u3[:len(u)] = u
        out = np.zeros(self.Q)
        lib().om_equilibrium(ctypes.byref(self._m), ctypes.c_double(rho), self._ptr(u3), self._ptr(out))
        return out

    def set_equilibrium(self, f, rho, u, pattern="pull", prev_parity=0):
        """rho: interior shape; u: interior shape + (D,)."""
        g = self._grid(f)
        n = (g.n[0], g.n[1], g.n[2])
        rho_c = np.ascontiguousarray(np.broadcast_to(rho, n[:self.D]).reshape(n).transpose(2, 1, 0), np.float64)
        u3 = np.zeros((3,) + n[::-1])
        uu = np.asarray(u, np.float64).reshape(n + (self.D,))
        for d in range(self.D):
            u3[d] = uu[..., d].transpose(2, 1, 0)
        lib().om_set_equilibrium(ctypes.byref(self._m), ctypes.byref(g), PATTERNS[pattern], prev_parity,
                                 self._ptr(rho_c), self._ptr(u3), self._ptr(f))

    def get_macroscopic(self, f, pattern="pull", prev_parity=0):
        g = self._grid(f)
        n = (g.n[0], g.n[1], g.n[2])
        rho = np.zeros(n[::-1])
        u3 = np.zeros((3,) + n[::-1])
        lib().om_get_macroscopic(ctypes.byref(self._m), ctypes.byref(g), PATTERNS[pattern], prev_parity,
                                 self._ptr(f), self._ptr(rho), self._ptr(u3))
        rho = rho.transpose(2, 1, 0)[(slice(None),) * self.D + (0,) * (3 - self.D)]
        u = np.stack([u3[d].transpose(2, 1, 0) for d in range(self.D)], axis=-1)
        u = u[(slice(None),) * self.D + (0,) * (3 - self.D)]
        return rho, u

    def run(self, f, steps, pattern="pull", parity=0, periodic=(True, True, True), flags=None,
            ubb_velocity=(0.0, 0.0, 0.0), tmp=None, fixed_density=1.0, ubb_link=None, ubb_adapt=False,
            ubb_density=None, fixed_density1=1.0, link_code=None, link_value=None):
        """Runs `steps` time steps.  Returns (field holding the result, new parity).  Flags: 1 NoSlip,
        2 UBB (ubb_velocity, or per link ubb_link[x, y, z, q, 3] for the link from interior cell
        (x, y, z) in direction q; ubb_adapt shifts the wall velocity by -F/(2 rho_ref); ubb_density
        prescribes the wall density), 6 / 7 FixedDensity (fixed_density / fixed_density1), 8-11 FreeSlip,
        SimpleExtrapolationOutflow, ExtrapolationOutflow, NoSlipLinearBouzidi with the per-link
        link_code [x, y, z, Q] and link_value [x, y, z, Q, 2] (the outflow state is updated in a copy)."""
        g = self._grid(f)
        # small grids: the OpenMP fork per loop costs more than the loop
        lib().om_set_threads(1 if g.n[0] * g.n[1] * g.n[2] < 4096 else 0)
        link = None
        if ubb_link is not None:
            link = np.ascontiguousarray(np.asarray(ubb_link, np.float64).transpose(2, 1, 0, 3, 4))
        self._m.ubb_link = link.ctypes.data if link is not None else None
        self._m.ubb_adapt = int(bool(ubb_adapt))
        self._m.ubb_density = float(ubb_density) if ubb_density else 0.0
        self._m.fd_rho1 = float(fixed_density1)
        code = val = None
        if link_code is not None:
            code = np.ascontiguousarray(np.asarray(link_code, np.int32).transpose(2, 1, 0, 3))
        if link_value is not None:
            val = np.ascontiguousarray(np.asarray(link_value, np.float64).transpose(2, 1, 0, 3, 4))
        self._m.link_code = code.ctypes.data if code is not None else None
        self._m.link_value = val.ctypes.data if val is not None else None
        per = (ctypes.c_int * 3)(*[int(p) for p in periodic])
        par = ctypes.c_int(parity)
        ub = np.array(list(ubb_velocity) + [0.0] * (3 - len(ubb_velocity)), np.float64)
        fl = None
        if flags is not None:
            fl = np.ascontiguousarray(flags.transpose(2, 1, 0) if flags.ndim == 3 else flags.T, np.uint8)
        if pattern in ("pull", "push"):
            if tmp is None:
                tmp = np.zeros_like(f)
                tmp = self.new_field(tuple(s - 2 for s in f.shape[:self.D]))
                tmp[...] = f
            sw = lib().om_run(ctypes.byref(self._m), ctypes.byref(g), PATTERNS[pattern], ctypes.byref(par),
                              steps, per, fl.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)) if fl is not None
                              else None, self._ptr(ub), ctypes.c_double(fixed_density), self._ptr(f),
                              self._ptr(tmp))
            self._m.ubb_link = self._m.link_code = self._m.link_value = None
            return (tmp if sw else f), par.value
        lib().om_run(ctypes.byref(self._m), ctypes.byref(g), PATTERNS[pattern], ctypes.byref(par), steps, per,
                     fl.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)) if fl is not None else None,
                     self._ptr(ub), ctypes.c_double(fixed_density), self._ptr(f), self._ptr(f))
        self._m.ubb_link = self._m.link_code = self._m.link_value = None
        return f, par.value

    def periodic_sync(self, f, pattern="pull", prev_parity=0, periodic=(True, True, True)):
        """Moves values the previous step wrote into ghost cells to their periodic images and
        refreshes the periodic ghost layers (the oracle's communication step)."""
        g = self._grid(f)
        per = (ctypes.c_int * 3)(*[int(p) for p in periodic])
        lib().om_periodic_sync(ctypes.byref(self._m), ctypes.byref(g), PATTERNS[pattern], prev_parity, per,
                               self._ptr(f))

    def accessor_table(self, pattern, parity, rw):
        """Offsets [Q, 3] and slots [Q] where direction i is read (rw = 0) or written (rw = 1)."""
        q = self._m.Q
        off = np.zeros((q, 3), np.int32)
        slot = np.zeros(q, np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        lib().om_accessor_table(ctypes.byref(self._m), PATTERNS[pattern], parity, rw, off.ctypes.data_as(ip),
                                slot.ctypes.data_as(ip))
        return off, slot

    def reduce(self, f, pattern="pull", prev_parity=0, flags=None):
        g = self._grid(f)
        out = np.zeros(5)
        fl = None
        if flags is not None:
            fl = np.ascontiguousarray(flags.transpose(2, 1, 0) if flags.ndim == 3 else flags.T, np.uint8)
        lib().om_reduce(ctypes.byref(self._m), ctypes.byref(g), PATTERNS[pattern], prev_parity, self._ptr(f),
                        fl.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)) if fl is not None else None,
                        self._ptr(out))
        return out


    # -- sparse (list-based) domains --------------------------------------------------------
    def sparse_ubb(self, flat, n_cells, links, velocity):
        """lbmpy's UBB on a PDF list (the kernel SparseLbBoundaryMapper builds, sparse/mapping.py:157-247,
        with boundaries/boundaryconditions.py UBB): for every link (dir d, fluid cell c, boundary cell
        b), slot inv(d) of b receives f(c, d) - 6 w_d rho (c_d . u), rho the cell density when
        compressible (zero-centred PDFs: 1 + sum f), else 1."""
        dirs, w = self.spec.dirs, self.spec.weights
        u = np.zeros(3)
        u[:len(velocity)] = velocity
        for d, c, b in links:
            d, c, b = int(d), int(c), int(b)
            if not 1 <= d < self.Q:
                continue
            rho = 1.0
            if self.spec.compressible:
                rho = float(sum(flat[c + i * n_cells] for i in range(self.Q)))
                rho += 1.0 if self.spec.zero_centered else 0.0
            inv = dirs.index(tuple(-v for v in dirs[d]))
            cu = sum(dirs[d][k] * u[k] for k in range(self.D))
            flat[b + inv * n_cells] = flat[c + d * n_cells] - 6.0 * float(w[d]) * cu * rho

    def sparse_run(self, f, index, steps, ubb_links=None, ubb_velocity=(0.0, 0.0, 0.0)):
        """lbmpy's sparse stream-pull-collide (sparse/update_rule_sparse.py:22-52 and the
        substitutions of :115-125): f is a PDF list [n_cells, Q] (element (c, i) = PDF i of list cell
        c), index the [n_fluid, Q - 1] pull index (sparse/mapping.py:100-156); each step cell c < n_fluid
        gathers f(c, 0) and flat[index[c, i - 1]] for i >= 1, collides (om_collide) and writes its own
        slots of the new list.  ubb_links [(dir, fluid cell, boundary cell)] run sparse_ubb on the
        source list before each step.  Returns the new list (boundary cells keep their values)."""
        n_cells, q = f.shape
        n_fluid = index.shape[0]
        flat = np.ascontiguousarray(np.asarray(f, np.float64).T).reshape(-1)
        idx = np.asarray(index, np.int64)
        for _ in range(steps):
            if ubb_links is not None:
                self.sparse_ubb(flat, n_cells, ubb_links, ubb_velocity)
            gathered = np.empty((n_fluid, q))
            gathered[:, 0] = flat[:n_fluid]
            gathered[:, 1:] = flat[idx]
            out = flat.copy()
            for c in range(n_fluid):
                fo = self.collide(gathered[c])
                out[c + np.arange(q) * n_cells] = fo
            flat = out
        return flat.reshape(q, n_cells).T.copy()


def make(stencil, method, **kw) -> Oracle:
    return Oracle(spec.resolve(stencil, method, **kw))


def mlp_features(P6, rho, u):
    """Closure features of one cell from the C restatement (om_mlp_features)."""
    P6 = np.ascontiguousarray(P6, np.float64)
    uu = np.ascontiguousarray(u, np.float64)
    x = np.zeros(10)
    dp = ctypes.POINTER(ctypes.c_double)
    lib().om_mlp_features(P6.ctypes.data_as(dp), ctypes.c_double(float(rho)), uu.ctypes.data_as(dp),
                          x.ctypes.data_as(dp))
    return x


def mlp_nu_t(params, x):
    """nu_t of one feature vector from the C restatement (om_mlp_nu_t)."""
    w = np.ascontiguousarray(params, np.float32)
    xx = np.ascontiguousarray(x, np.float64)
    f = lib().om_mlp_nu_t
    f.restype = ctypes.c_double
    return f(w.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), xx.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
