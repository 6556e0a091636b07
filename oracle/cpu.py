"""ctypes front end of the closed-form CPU sweeps (``lbm_cpu.c``) -- TEST INFRASTRUCTURE ONLY.

These kernels restate lbmpy's generated OpenMP kernels for two methods (D3Q19/D3Q27 TRT with pull
streaming; D3Q27 cumulant with AA streaming, Galilean correction and CentralMoment force).  They
are the CPU baseline bench.py times and a fast checker for long runs; each is pinned to the
generic oracle (``oracle.py``) by tests/test_cpu_kernels.py.  Fields use the oracle's convention:
``arr[x, y, z, q]`` with ghost layers, fzyx memory layout, zero-centred values (f - w).
"""
from __future__ import annotations

import ctypes
import os
from fractions import Fraction

import numpy as np

from . import oracle as O
from . import oracle_spec as S

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class OcpuParams(ctypes.Structure):
    _fields_ = [
        ("q", ctypes.c_int),
        ("c", (ctypes.c_int * 3) * 27),
        ("inv", ctypes.c_int * 27),
        ("w", ctypes.c_double * 27),
        ("eq_lin", (ctypes.c_double * 3) * 27),
        ("eq_quad", (ctypes.c_double * 6) * 27),
        ("omega_even", ctypes.c_double), ("omega_odd", ctypes.c_double),
        ("compressible", ctypes.c_int),
        ("galilean", ctypes.c_int),
        ("force", ctypes.c_double * 3),
        ("ubb", ctypes.c_double * 3),
        ("n", ctypes.c_int * 3),
        ("sy", ctypes.c_int64), ("sz", ctypes.c_int64), ("sq", ctypes.c_int64),
        ("periodic", ctypes.c_int * 3),
    ]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liblbm_cpu.so")
        if not os.path.exists(path):
            O.build()
        _LIB = ctypes.CDLL(path)
        for sfx in ("f64", "f32"):
            assert getattr(_LIB, f"ocpu_sizeof_params_{sfx}")() == ctypes.sizeof(OcpuParams), "struct layout"
            getattr(_LIB, f"ocpu_run_trt_pull_{sfx}").restype = ctypes.c_int
            getattr(_LIB, f"ocpu_run_cum_aa_{sfx}").restype = ctypes.c_int
            getattr(_LIB, f"ocpu_tables_match_{sfx}").restype = ctypes.c_int
    return _LIB


def equilibrium_tables(orc: O.Oracle):
    """Coefficients of the delta-form equilibrium f_eq_i - w_i drho = rf (lin_i . u + quad_i . uu),
    uu = (uxx, uyy, uzz, uxy, uxz, uyz), read off the oracle's equilibrium at unit velocities
    (exact: the equilibrium is a quadratic polynomial with small rational coefficients)."""
    q = orc.Q
    f0 = orc.equilibrium(1.0, [0, 0, 0])
    lin = np.zeros((q, 3))
    quad = np.zeros((q, 6))
    e = np.eye(3)
    for a in range(3):
        fp, fm = orc.equilibrium(1.0, e[a]), orc.equilibrium(1.0, -e[a])
        lin[:, a] = (fp - fm) / 2
        quad[:, a] = (fp + fm) / 2 - f0
    for k, (a, b) in enumerate(((0, 1), (0, 2), (1, 2))):
        fab = orc.equilibrium(1.0, e[a] + e[b])
        quad[:, 3 + k] = fab - f0 - lin[:, a] - lin[:, b] - quad[:, a] - quad[:, b]

    def exact(v):
        return float(Fraction(float(v)).limit_denominator(10000))
    return np.vectorize(exact)(lin), np.vectorize(exact)(quad)


class FastCPU:
    """One resolved method on the closed-form CPU kernels."""

    def __init__(self, kind, orc: O.Oracle, dtype=np.float64, force=(0.0, 0.0, 0.0), galilean=False,
                 ubb=(0.0, 0.0, 0.0)):
        assert kind in ("trt", "cumulant")
        self.kind, self.orc, self.dtype = kind, orc, np.dtype(dtype)
        self.sfx = "f64" if self.dtype == np.float64 else "f32"
        sp = orc.spec
        p = OcpuParams()
        p.q = sp.Q
        for i, d in enumerate(sp.dirs):
            for k in range(3):
                p.c[i][k] = d[k]
            p.inv[i] = sp.dirs.index(tuple(-v for v in d))
            p.w[i] = float(sp.weights[i])
        if kind == "trt":
            rates = sorted({r for r in sp.rates if r != 0.0}, key=lambda r: -sp.rates.count(r))
            even = [r for m, r in zip(sp.moments, sp.rates) if S.is_even(m) and S.get_order(m) >= 2]
            odd = [r for m, r in zip(sp.moments, sp.rates) if not S.is_even(m) and S.get_order(m) >= 3]
            assert len(set(even)) == 1 and len(set(odd)) <= 1 and rates, "TRT rates"
            p.omega_even = even[0]
            p.omega_odd = odd[0] if odd else even[0]
            lin, quad = equilibrium_tables(orc)
            for i in range(sp.Q):
                for a in range(3):
                    p.eq_lin[i][a] = lin[i, a]
                for a in range(6):
                    p.eq_quad[i][a] = quad[i, a]
            assert sp.force_model == S.FORCE_NONE, "the TRT CPU kernel is force-free"
        else:
            assert sp.Q == 27 and sp.compressible
            shear = [r for m, r in zip(sp.moments, sp.rates) if S.is_shear_moment(m, 3)]
            bulk = [r for m, r in zip(sp.moments, sp.rates) if S.is_bulk_moment(m, 3)]
            higher = [r for m, r in zip(sp.moments, sp.rates) if S.get_order(m) >= 3]
            assert len(set(shear)) == 1 and all(r == 1.0 for r in higher), "cumulant rates"
            p.omega_even = shear[0]
            p.omega_odd = bulk[0]
            p.galilean = int(sp.galilean_correction)
            for k in range(3):
                p.force[k] = sp.force[k]
        p.compressible = int(sp.compressible)
        for k in range(3):
            p.ubb[k] = ubb[k]
        self._p = p
        assert getattr(lib(), f"ocpu_tables_match_{self.sfx}")(ctypes.byref(p)) == 1, "direction order"

    def new_field(self, n):
        buf = np.zeros((self.orc.Q, n[2] + 2, n[1] + 2, n[0] + 2), dtype=self.dtype)
        return buf.transpose(3, 2, 1, 0)

    def _bind(self, arr, periodic):
        p = self._p
        es = arr.dtype.itemsize
        assert arr.strides[0] == es, "x must be the fastest axis"
        for d in range(3):
            p.n[d] = arr.shape[d] - 2
            p.periodic[d] = int(bool(periodic[d]))
        p.sy, p.sz, p.sq = arr.strides[1] // es, arr.strides[2] // es, arr.strides[3] // es

    @staticmethod
    def _flags(flags):
        if flags is None:
            return None, None
        fl = np.ascontiguousarray(flags.transpose(2, 1, 0), np.uint8)
        return fl, fl.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))

    def _ptr(self, a):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double if self.sfx == "f64" else ctypes.c_float))

    def run(self, f, steps, parity=0, periodic=(True, True, True), flags=None, tmp=None):
        """TRT: pull, returns (field holding the result, 0).  Cumulant: AA in place from `parity`,
        returns (f, next parity).  Flags: 1 NoSlip, 2 UBB (TRT only)."""
        assert f.dtype == self.dtype
        self._bind(f, periodic)
        fl, flp = self._flags(flags)
        if self.kind == "trt":
            if tmp is None:
                tmp = self.new_field(tuple(s - 2 for s in f.shape[:3]))
                tmp[...] = f
            in_b = getattr(lib(), f"ocpu_run_trt_pull_{self.sfx}")(ctypes.byref(self._p), self._ptr(f),
                                                                     self._ptr(tmp), flp, int(steps))
            return (tmp if in_b else f), 0
        assert fl is None or not (fl == 2).any(), "the cumulant CPU kernel takes NoSlip walls only"
        par = getattr(lib(), f"ocpu_run_cum_aa_{self.sfx}")(ctypes.byref(self._p), self._ptr(f), flp, int(parity),
                                                            int(steps))
        return f, par
