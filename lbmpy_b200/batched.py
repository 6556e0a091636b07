"""Many independent lattice Boltzmann domains of uneven sizes, one persistent launch per step.

lbmpy has no batch object: a study of many small domains (a parameter sweep over cavities, an
ensemble) runs one ``LatticeBoltzmannStep`` per domain (``lbstep.py:18-450``), one kernel launch
per domain and step.  ``LatticeBoltzmannBatch`` keeps every domain's PDF field in two shared
device buffers (each domain in lbmpy's own ghost-layered fzyx layout at its own offset) and
updates all domains with one launch per time step: the blocks of a persistent grid walk a table
of tiles that spans every domain (``lbm_batch_create`` / ``lbm_batch_sweep`` in
``include/lbm_b200.h``).  The steps of ``run`` are captured once into a CUDA graph and replayed.

Per domain: its size, its periodicity, its boundaries (a ``LatticeBoltzmannBoundaryHandling``
each, NoSlip / UBB), and its kernel parameters (the values of the method's free symbols, e.g.
``omega_shear``).  Shared: stencil, method family, storage type, streaming pattern, force.

The tile shape (``tile_x`` x ``tile_y`` threads, ``cells_z`` cells per thread along z, blocks per
SM) is chosen by ``autotune``, which times each candidate on the batch itself.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from types import MappingProxyType
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _native as N
from .boundaries import LatticeBoltzmannBoundaryHandling
from .creationfunctions import create_lb_function, update_with_default_parameters
from .enums import Stencil, Timestep, is_inplace
from .fields import ALIGN_BYTES, torch_dtype
from .kernel import build_desc
from .macroscopic_value_kernels import _MacroPlanCache, get_macroscopic, set_equilibrium
from .stencils import LBStencil


@dataclass(frozen=True)
class Tiling:
    tile_x: int = 32
    tile_y: int = 8
    cells_z: int = 1
    blocks_per_sm: int = 0

    def native(self) -> N.LbmBatchTiling:
        t = N.LbmBatchTiling()
        t.tile_x, t.tile_y, t.cells_z, t.blocks_per_sm = self.tile_x, self.tile_y, self.cells_z, self.blocks_per_sm
        return t


DEFAULT_CANDIDATES: Tuple[Tiling, ...] = (
    Tiling(32, 8, 1, 0), Tiling(16, 16, 1, 0), Tiling(16, 8, 1, 0), Tiling(32, 4, 1, 0), Tiling(64, 4, 1, 0),
    Tiling(32, 8, 2, 0), Tiling(16, 8, 2, 0), Tiling(32, 8, 1, 8), Tiling(16, 16, 1, 8), Tiling(32, 8, 2, 8),
    Tiling(16, 8, 4, 16), Tiling(32, 4, 4, 16),
)


def _field_layout(size, q, itemsize):
    """Strides and extent of one ghost-layered fzyx field, rows padded so that element x=1 of every
    row starts on a 32-byte boundary when the field starts at a multiple of 32 bytes minus one
    element (as ``create_pdf_array``)."""
    a = max(1, ALIGN_BYTES // itemsize)
    ex, ey, ez = (int(s) + 2 for s in size)
    sy = -(-ex // a) * a
    sz = sy * ey
    sq = sz * ez
    return (1, sy, sz, sq), q * sq, a


class LatticeBoltzmannBatch:
    def __init__(self, domain_sizes: Sequence[Sequence[int]], kernel_params=MappingProxyType({}), periodicity=False,
                 lbm_config=None, lbm_optimisation=None, config=None, tiling="auto", use_cuda_graph=True,
                 device="cuda", **method_parameters):
        sizes = [tuple(int(s) for s in d) for d in domain_sizes]
        if not sizes:
            raise ValueError("a batch needs at least one domain")
        if any(len(s) != 3 or min(s) < 1 for s in sizes):
            raise ValueError("every domain size must have three positive entries")
        n = len(sizes)
        if isinstance(kernel_params, (list, tuple)):
            if len(kernel_params) != n:
                raise ValueError(f"kernel_params has {len(kernel_params)} entries for {n} domains")
            params = [dict(p) for p in kernel_params]
        else:
            params = [dict(kernel_params) for _ in range(n)]
        if isinstance(periodicity, bool) or (len(periodicity) == 3 and isinstance(periodicity[0], (bool, int))):
            per = periodicity if not isinstance(periodicity, bool) else (periodicity,) * 3
            periodic = [tuple(bool(p) for p in per)] * n
        else:
            periodic = [tuple(bool(p) for p in per) for per in periodicity]
            if len(periodic) != n:
                raise ValueError(f"periodicity has {len(periodic)} entries for {n} domains")
        if lbm_config is not None:
            method_parameters["stencil"] = lbm_config.stencil
        method_parameters.setdefault("stencil", LBStencil(Stencil.D3Q19))
        lbm_config, lbm_optimisation, config = update_with_default_parameters(method_parameters, {}, lbm_config,
                                                                              lbm_optimisation, config)
        self._lbm_config = lbm_config
        self.streaming_pattern = lbm_config.streaming_pattern
        if self.streaming_pattern not in ("pull", "aa"):
            raise NotImplementedError("batched sweeps are built for the pull and AA patterns")
        self._inplace = is_inplace(self.streaming_pattern)
        if self._inplace:
            # the batch launches both parities itself; the update rule only supplies the method
            from dataclasses import replace
            lbm_config = replace(lbm_config, timestep=Timestep.EVEN)
        self._kernel = create_lb_function(lbm_config=lbm_config, lbm_optimisation=lbm_optimisation, config=config)
        self.update_rule = self._kernel.update_rule
        self.method = self._kernel.method
        self.device = torch.device(device)
        self._storage = self.update_rule.storage_dtype
        self._dtype = torch_dtype(self._storage)
        self.domain_sizes = sizes
        self.kernel_params = params
        self.periodicity = periodic
        self.use_cuda_graph = bool(use_cuda_graph)
        q = self.method.stencil.Q
        itemsize = torch.tensor([], dtype=self._dtype).element_size()

        # one allocation per buffer; each field starts one element before a 32-byte boundary
        self._layout = []
        off = 0
        for s in sizes:
            strides, extent, a = _field_layout(s, q, itemsize)
            start = -(-off // a) * a + (a - 1)
            self._layout.append((start, strides, extent))
            off = start + extent
        self.buffer_elems = off
        self._buf = [torch.zeros(off, dtype=self._dtype, device=self.device)]
        self._buf.append(self._buf[0] if self._inplace else torch.zeros(off, dtype=self._dtype, device=self.device))
        self._handlings = [LatticeBoltzmannBoundaryHandling(self.method, s, p, name=f"domain{k}", device=device,
                                                            streaming_pattern=self.streaming_pattern)
                           for k, (s, p) in enumerate(zip(sizes, periodic))]
        self._macro = _MacroPlanCache(self.method, self.streaming_pattern, self.update_rule.collision_rule)
        self._current = 0                    # pull: which buffer holds the state
        self._prev = Timestep.ODD if self._inplace else Timestep.BOTH
        self.time_steps_run = 0
        self._tiling_request = tiling
        self.tiling: Optional[Tiling] = None
        self.tuning: List[Tuple[Tiling, float]] = []
        self._handle = None
        self._flags = None
        self._graphs: Dict[Tuple[int, int, int], torch.cuda.CUDAGraph] = {}
        self._stream = None
        for k in range(n):
            self.set_pdf_fields_from_macroscopic_values(k)

    # ------------------------------------------------------------------------------ domains
    @property
    def n_domains(self) -> int:
        return len(self.domain_sizes)

    @property
    def number_of_cells(self) -> int:
        return int(sum(int(np.prod(s)) for s in self.domain_sizes))

    def boundary_handling(self, k: int) -> LatticeBoltzmannBoundaryHandling:
        """Boundary handling of domain k; changing it invalidates the finalized batch."""
        self._release()
        return self._handlings[k]

    def _view(self, k: int, buf: torch.Tensor) -> torch.Tensor:
        start, strides, _ = self._layout[k]
        ex, ey, ez = (s + 2 for s in self.domain_sizes[k])
        return torch.as_strided(buf, (ex, ey, ez, self.method.stencil.Q), strides, start)

    def pdfs(self, k: int) -> torch.Tensor:
        """The current PDF field of domain k, shape (X+2, Y+2, Z+2, Q), a view into the batch."""
        return self._view(k, self._buf[self._current])

    def set_pdf_fields_from_macroscopic_values(self, k: int, density=1.0, velocity=(0.0, 0.0, 0.0)):
        """Equilibrium of domain k from a density and velocity (scalars or interior-shaped tensors)."""
        set_equilibrium(self._macro, self.pdfs(k), density, velocity, self._prev, self.kernel_params[k],
                        self.periodicity[k])

    def macroscopic_values(self, k: int):
        """(density, velocity) of domain k as device tensors of the compute type."""
        cd = torch.float64 if self._storage == "float64" else torch.float32
        size = self.domain_sizes[k]
        rho = torch.empty(size, dtype=cd, device=self.device)
        u = torch.empty(size + (3,), dtype=cd, device=self.device)
        get_macroscopic(self._macro, self.pdfs(k), rho, u, self._prev, self.kernel_params[k], self.periodicity[k])
        return rho, u

    @property
    def previous_timestep(self):
        return self._prev

    # ------------------------------------------------------------------------------ native batch
    def _descs(self):
        q = self.method.stencil.Q
        domains = (N.LbmDomainDesc * self.n_domains)()
        flag_sizes = [int(np.prod([s + 2 for s in size])) for size in self.domain_sizes]
        has_flags = [h.has_boundaries for h in self._handlings]
        flag_offsets, total = [], 0
        for k in range(self.n_domains):
            if has_flags[k]:
                flag_offsets.append(total)
                total += -(-flag_sizes[k] // 16) * 16
            else:
                flag_offsets.append(-1)
        common = None
        for k, size in enumerate(self.domain_sizes):
            if self._handlings[k].fixed_density is not None:
                raise NotImplementedError("FixedDensity boundaries are not built for batches")
            d = build_desc(self.update_rule, size, self.periodicity[k], self.kernel_params[k],
                           self._handlings[k].ubb_velocities)
            if common is None:
                common = d
            e = domains[k]
            for i in range(3):
                e.dims[i] = size[i]
                e.periodic[i] = int(self.periodicity[k][i])
            start, strides, _ = self._layout[k]
            for i in range(4):
                e.strides[i] = strides[i]
            e.offset = start
            e.flags_offset = flag_offsets[k]
            ctypes.memmove(ctypes.addressof(e.rates), ctypes.addressof(d.rates), ctypes.sizeof(e.rates))
            ctypes.memmove(ctypes.addressof(e.ubb_velocity), ctypes.addressof(d.ubb_velocity),
                           ctypes.sizeof(e.ubb_velocity))
        flags = None
        if total:
            host = np.zeros(total, dtype=np.uint8)
            for k, h in enumerate(self._handlings):
                if flag_offsets[k] >= 0:
                    host[flag_offsets[k]:flag_offsets[k] + flag_sizes[k]] = h._host.reshape(-1)
            flags = torch.from_numpy(host).to(self.device)
        assert q == common.stencil
        return common, domains, flags

    def _create(self, tiling: Tiling):
        common, domains, flags = self._descs()
        h = ctypes.c_void_p()
        fl_ptr = ctypes.c_void_p(flags.data_ptr() if flags is not None else None)
        fl_bytes = flags.numel() if flags is not None else 0
        N.check(N.lib().lbm_batch_create(ctypes.byref(common), domains, self.n_domains,
                                         ctypes.c_void_p(self._buf[0].data_ptr()),
                                         ctypes.c_void_p(self._buf[1].data_ptr()),
                                         self.buffer_elems, fl_ptr, fl_bytes, ctypes.byref(tiling.native()),
                                         ctypes.byref(h)), "lbm_batch_create")
        return h, flags

    def _release(self):
        self._graphs.clear()
        if self._handle is not None and self._handle.value:
            N.lib().lbm_batch_destroy(self._handle)
        self._handle = None
        self._flags = None

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass

    def info(self) -> Dict[str, int]:
        """Tiles, blocks, interior cells and thread slots of the finalized batch."""
        self.finalize()
        out = (ctypes.c_int64 * 4)()
        N.check(N.lib().lbm_batch_info(self._handle, out), "lbm_batch_info")
        return {"tiles": out[0], "blocks": out[1], "cells": out[2], "thread_slots": out[3]}

    def finalize(self):
        """Uploads boundaries and per-domain arguments; tunes the tiling on first use if asked."""
        if self._handle is not None:
            return
        if self._tiling_request == "auto" and self.tiling is None:
            self.autotune()
            return
        tiling = self.tiling or (self._tiling_request if isinstance(self._tiling_request, Tiling) else Tiling())
        self._handle, self._flags = self._create(tiling)
        self.tiling = tiling

    # ------------------------------------------------------------------------------ stepping
    def _launch(self, parity: int, stream_handle: int):
        rc = N.lib().lbm_batch_sweep(self._handle, parity, ctypes.c_void_p(stream_handle))
        if rc:
            N.check(rc, "lbm_batch_sweep")

    def _sweep_parities(self, steps: int):
        """Parity of each of the next `steps` sweeps, from the current state."""
        if self._inplace:
            first = int(self._prev.next().idx)
            return [(first + t) % 2 for t in range(steps)]
        return [(self._current + t) % 2 for t in range(steps)]

    def _advance(self, steps: int):
        if self._inplace:
            self._prev = Timestep((int(self._prev.next().idx) + steps - 1) % 2)
        else:
            self._current = (self._current + steps) % 2
        self.time_steps_run += steps

    def run_sweeps(self, steps: int):
        """`steps` time steps of every domain: replays a CUDA graph of the launches (captured on
        first use for this step count and start parity), or launches directly."""
        steps = int(steps)
        if steps <= 0:
            return
        self.finalize()
        parities = self._sweep_parities(steps)
        if not self.use_cuda_graph:
            s = torch.cuda.current_stream().cuda_stream
            for p in parities:
                self._launch(p, s)
        else:
            key = (steps, parities[0], torch.cuda.current_device())
            g = self._graphs.get(key)
            if g is None:
                torch.cuda.synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    s = torch.cuda.current_stream().cuda_stream
                    for p in parities:
                        self._launch(p, s)
                self._graphs[key] = g
            g.replay()
        self._advance(steps)

    def run(self, steps: int):
        self.run_sweeps(steps)

    def time_step(self):
        self.run_sweeps(1)

    # ------------------------------------------------------------------------------ tuning
    def _time_candidate(self, tiling: Tiling, sweeps: int, repeats: int) -> float:
        h, flags = self._create(tiling)
        try:
            s = torch.cuda.current_stream().cuda_stream
            lib = N.lib()
            # pull: repeated sweeps from the current buffer leave the state untouched
            parity = self._current if not self._inplace else 0
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            for _ in range(2):
                N.check(lib.lbm_batch_sweep(h, parity, ctypes.c_void_p(s)), "lbm_batch_sweep")
            best = float("inf")
            for _ in range(repeats):
                start.record()
                for t in range(sweeps):
                    p = parity if not self._inplace else t % 2
                    rc = lib.lbm_batch_sweep(h, p, ctypes.c_void_p(s))
                    if rc:
                        N.check(rc, "lbm_batch_sweep")
                stop.record()
                stop.synchronize()
                best = min(best, start.elapsed_time(stop) / sweeps)
            return best
        finally:
            lib.lbm_batch_destroy(h)
            del flags

    def autotune(self, candidates: Sequence[Tiling] = DEFAULT_CANDIDATES, sweeps: int = 5,
                 repeats: int = 3) -> Tiling:
        """Times every candidate tiling on this batch (ms per sweep, best of `repeats`) and keeps the
        fastest.  The state is unchanged: pull sweeps read the current buffer only, in-place runs
        are undone from a snapshot."""
        self._release()
        snapshot = self._buf[0].clone() if self._inplace else None
        try:
            results = []
            for c in candidates:
                results.append((c, self._time_candidate(c, sweeps, repeats)))
        finally:
            if snapshot is not None:
                self._buf[0].copy_(snapshot)
                torch.cuda.synchronize()
        self.tuning = sorted(results, key=lambda r: r[1])
        self.tiling = self.tuning[0][0]
        self._handle, self._flags = self._create(self.tiling)
        return self.tiling

    def benchmark_run(self, steps: int) -> float:
        """MLUPS over all domains for `steps` time steps (CUDA events around the replay)."""
        self.run_sweeps(steps)           # capture / warm the graph for this step count
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        self.run_sweeps(steps)
        stop.record()
        torch.cuda.synchronize()
        return self.number_of_cells * steps / (start.elapsed_time(stop) * 1e-3) * 1e-6


def lid_driven_cavity_batch(n_cavities: int, seed: int = 0, edges=tuple(range(16, 97, 8)), lid_velocity=0.05,
                            omega_range=(1.5, 1.95), storage_dtype="float32", cubic=True,
                            **kwargs) -> LatticeBoltzmannBatch:
    """A batch of independent lid-driven cavities (lbmpy ``create_lid_driven_cavity``,
    ``scenarios.py:72-101``: UBB lid on the N face moving in x, NoSlip on W, E, S, T, B) with the
    D3Q19 weighted-orthogonal MRT method.  Per cavity, seeded: the edge length drawn from `edges`
    (one edge per cube, or one per axis with cubic=False), shear and bulk rates drawn uniformly
    from `omega_range`; the higher moments relax with rate 1."""
    import sympy as sp
    from .boundaries import NoSlip, UBB, slice_from_direction
    from .creationfunctions import CreateKernelConfig, LBMConfig, LBMOptimisation
    from .enums import Method
    rng = np.random.default_rng(seed)
    sizes = [tuple(int(e) for e in rng.choice(edges, 1 if cubic else 3)) * (3 if cubic else 1)
             for _ in range(n_cavities)]
    rates = rng.uniform(omega_range[0], omega_range[1], size=(n_cavities, 2))
    w_s, w_b = sp.Symbol("omega_shear"), sp.Symbol("omega_bulk")
    cfg = LBMConfig(stencil=LBStencil(Stencil.D3Q19), method=Method.MRT, relaxation_rates=[w_s, w_b, 1, 1],
                    compressible=False)
    batch = LatticeBoltzmannBatch(sizes, kernel_params=[{"omega_shear": float(a), "omega_bulk": float(b)}
                                                        for a, b in rates],
                                  lbm_config=cfg, lbm_optimisation=LBMOptimisation(storage_dtype=storage_dtype),
                                  config=CreateKernelConfig(data_type="float64" if storage_dtype == "float64"
                                                            else "float32"), **kwargs)
    for k in range(n_cavities):
        bh = batch.boundary_handling(k)
        bh.set_boundary(UBB(velocity=(lid_velocity, 0, 0)), slice_from_direction("N", 3))
        for d in ("W", "E", "S", "T", "B"):
            bh.set_boundary(NoSlip(), slice_from_direction(d, 3))
    return batch
