"""``LatticeBoltzmannStep`` on one B200 (lbmpy ``lbstep.py:18-450``).

Fields live on the GPU as PyTorch tensors in lbmpy's fzyx layout.  A time step is one launch of
the fused sweep: periodicity (index wrap) and NoSlip/UBB bounce-back happen inside it, so
lbmpy's sync -> boundary -> sweep -> swap sequence (:271-282) becomes sweep -> swap.  As in
lbmpy, the velocity and density arrays the user sees are host (numpy) arrays that ``run`` fills
at the end (post_run, :311-314) and that ``set_pdf_fields_from_macroscopic_values`` reads.

Extension over lbmpy: ``streaming_pattern='aa'`` / ``'esotwist'`` / ``'esopull'`` / ``'esopush'``
run in place on one field (lbmpy's step supports two-field patterns only, :153-156 and :282);
``'push'`` runs on two fields like ``'pull'``.
"""
from __future__ import annotations

import time
from types import MappingProxyType

import numpy as np
import torch

from .boundaries import LatticeBoltzmannBoundaryHandling
from .creationfunctions import create_lb_function, update_with_default_parameters
from .enums import Stencil, Timestep, get_timesteps, is_inplace
from .fields import create_pdf_array
from .macroscopic_value_kernels import _MacroPlanCache, get_macroscopic, set_equilibrium
from .stencils import LBStencil


class SlicedGetter:
    def __init__(self, fn):
        self._fn = fn

    def __getitem__(self, item):
        return self._fn(item)


class LatticeBoltzmannStep:
    def __init__(self, domain_size=None, lbm_kernel=None, periodicity=False, kernel_params=MappingProxyType({}),
                 data_handling=None, name="lbm", optimization=None, velocity_data_name=None,
                 density_data_name=None, density_data_index=None, compute_velocity_in_every_step=False,
                 compute_density_in_every_step=False, velocity_input_array_name=None,
                 time_step_order="stream_collide", flag_interface=None, alignment_if_vectorized=64,
                 fixed_loop_sizes=True, timeloop_creation_function=None, lbm_config=None, lbm_optimisation=None,
                 config=None, device="cuda", **method_parameters):
        if data_handling is not None:
            raise NotImplementedError("pystencils data handlings are not used; pass domain_size")
        if domain_size is None:
            raise ValueError("Specify either domain_size or data_handling")
        if time_step_order != "stream_collide":
            raise NotImplementedError("only the fused stream-collide order is built")
        if velocity_input_array_name is not None:
            raise NotImplementedError("velocity input arrays are not built")
        domain_size = tuple(int(s) for s in domain_size)
        if len(domain_size) != 3:
            raise NotImplementedError("the B200 sweep is three-dimensional")
        if isinstance(periodicity, bool):
            periodicity = (periodicity,) * 3
        self.periodicity = tuple(bool(p) for p in periodicity)
        optimization = dict(optimization or {})
        if lbm_config is not None:
            method_parameters["stencil"] = lbm_config.stencil
        method_parameters.setdefault("stencil", LBStencil(Stencil.D3Q27))
        lbm_config, lbm_optimisation, config = update_with_default_parameters(method_parameters, optimization,
                                                                              lbm_config, lbm_optimisation, config)
        self.name = name
        self.device = device
        self._domain = domain_size
        self.kernel_params = dict(kernel_params)
        self._lbm_config = lbm_config
        self._lbm_optimisation = lbm_optimisation
        self._config = config
        self.streaming_pattern = lbm_config.streaming_pattern
        self._inplace = is_inplace(self.streaming_pattern)
        from dataclasses import replace
        if lbm_kernel is None:
            if self._inplace:
                self._kernels = [create_lb_function(lbm_config=replace(lbm_config, timestep=t),
                                                    lbm_optimisation=lbm_optimisation, config=config)
                                 for t in get_timesteps(self.streaming_pattern)]
            else:
                self._kernels = [create_lb_function(lbm_config=lbm_config, lbm_optimisation=lbm_optimisation,
                                                    config=config)]
        else:
            self._kernels = [lbm_kernel]
        self.method = self._kernels[0].method
        ur = self._kernels[0].update_rule
        self._storage = ur.storage_dtype
        self._compute = ur.data_type
        q = self.method.stencil.Q
        self._pdf_arr_name = name + "_pdfSrc"
        self._tmp_arr_name = name + "_pdfTmp"
        self.velocity_data_name = velocity_data_name or name + "_velocity"
        self.density_data_name = density_data_name or name + "_density"
        self.density_data_index = density_data_index
        self.pdfs = create_pdf_array(domain_size, q, dtype=self._storage, device=device)
        self.pdfs_tmp = None if self._inplace else create_pdf_array(domain_size, q, dtype=self._storage,
                                                                      device=device)
        # host density and velocity (lbmpy's CPU arrays of the step) live in page-locked memory, so
        # that the copies of set_pdf_fields_from_macroscopic_values() and post_run() go by DMA; the
        # numpy arrays are views of it
        td = torch.float64 if self._compute == "float64" else torch.float32
        pin = torch.cuda.is_available()
        self._velocity_t = torch.zeros(tuple(domain_size) + (3,), dtype=td, pin_memory=pin)
        self._density_t = torch.ones(tuple(domain_size), dtype=td, pin_memory=pin)
        self._velocity = self._velocity_t.numpy()
        self._density = self._density_t.numpy()
        self._boundary_handling = LatticeBoltzmannBoundaryHandling(self.method, domain_size, self.periodicity,
                                                                   name=name + "_boundary_handling", device=device,
                                                                   streaming_pattern=self.streaming_pattern)
        self._macro = _MacroPlanCache(self.method, self.streaming_pattern, self._kernels[0].update_rule.collision_rule)
        # parity of the last completed step: in-place patterns start as if an ODD step just ran
        self._prev = Timestep.ODD if self._inplace else Timestep.BOTH
        self._bound_sweep = None
        self.time_steps_run = 0
        self.set_pdf_fields_from_macroscopic_values()

    # ------------------------------------------------------------------------------ properties
    @property
    def boundary_handling(self):
        return self._boundary_handling

    @property
    def dim(self):
        return 3

    @property
    def domain_size(self):
        return self._domain

    @property
    def number_of_cells(self):
        n = 1
        for d in self._domain:
            n *= d
        return n

    @property
    def pdf_array_name(self):
        return self._pdf_arr_name

    @property
    def lbm_config(self):
        return self._lbm_config

    @property
    def lbm_optimisation(self):
        return self._lbm_optimisation

    @property
    def config(self):
        return self._config

    @property
    def velocity(self):
        return SlicedGetter(lambda sl: self._velocity[sl])

    @property
    def density(self):
        return SlicedGetter(lambda sl: self._density[sl])

    @property
    def velocity_array(self):
        """Host velocity field (interior, [x, y, z, 3]); writable before set_pdf_fields_from_macroscopic_values."""
        return self._velocity

    @property
    def density_array(self):
        return self._density

    def velocity_slice(self, slice_obj=None, masked=True):
        if slice_obj is None:
            slice_obj = (slice(None), slice(None), self._domain[2] // 2)
        return self._velocity[slice_obj]

    def density_slice(self, slice_obj=None, masked=True):
        if slice_obj is None:
            slice_obj = (slice(None), slice(None), self._domain[2] // 2)
        return self._density[slice_obj]

    @property
    def current_pdfs(self) -> torch.Tensor:
        return self.pdfs

    @property
    def previous_timestep(self):
        return self._prev

    def sweep_variant(self) -> str:
        """Name of the kernel the next sweep runs ("cell", "pair", "quad" or "staged")."""
        b = self._bound()
        if self._inplace:
            p = self.pdfs.data_ptr()
            return b.variant(p, p, int(self._prev.next().idx))
        return b.variant(self.pdfs.data_ptr(), self.pdfs_tmp.data_ptr(), 0)

    def sweep_status(self, clear: bool = True) -> int:
        """Device status of the sweeps run so far (synchronises): 0 when every sweep ran to
        completion, else the STATUS_* bits of lbmpy_b200._native (a staged sweep that gave up
        waiting for its data leaves its remaining cells un-updated and sets a bit)."""
        v = 0
        for k in self._kernels:
            v |= k.status(clear)
        return v

    # ------------------------------------------------------------------------------ running
    def _flags(self, kernel):
        if not self._boundary_handling.has_boundaries:
            return None
        bh = self._boundary_handling
        plan = kernel.plan([d for d in self._domain], self.periodicity, self.kernel_params, bh.ubb_velocities,
                           bh.fixed_density, bh.ubb_options)
        return bh.flags(plan)

    def _bound(self):
        """The sweep with plan, strides, flags and stream resolved; rebuilt when boundaries,
        kernel parameters or the current stream change."""
        bh = self._boundary_handling
        key = (id(bh._dev), bh._dev is None, tuple(sorted(self.kernel_params.items())),
               torch.cuda.current_stream().cuda_stream)
        if getattr(self, "_bound_key", None) != key or self._bound_sweep is None:
            k = self._kernels[0]
            flags = self._flags(k)
            self._bound_sweep = k.bind(self.pdfs, self.periodicity, flags, bh.ubb_velocities, self.kernel_params,
                                       fixed_density=bh.fixed_density, ubb_options=bh.ubb_options)
            if flags is not None:
                bh.attach_links(self._bound_sweep.plan, self.pdfs, self._prev.idx if self._inplace else 0)
            self._bound_key = (id(bh._dev), bh._dev is None, tuple(sorted(self.kernel_params.items())),
                               torch.cuda.current_stream().cuda_stream)
        closure = self._kernels[0].update_rule.collision_rule.closure
        if closure is not None:
            closure.ensure_uploaded()          # a retrained closure reaches the next sweep
        return self._bound_sweep

    def set_pdf_fields_from_macroscopic_values(self):
        rho = self._density_t.to(self.device)
        u = self._velocity_t.to(self.device)
        set_equilibrium(self._macro, self.pdfs, rho, u, self._prev, self.kernel_params, self.periodicity)

    def pre_run(self):
        pass

    def time_step(self):
        b = self._bound()
        if self._inplace:
            nxt = self._prev.next()
            p = self.pdfs.data_ptr()
            b.sweep(p, p, int(nxt.idx))
            self._prev = nxt
        else:
            b.sweep(self.pdfs.data_ptr(), self.pdfs_tmp.data_ptr(), 0)
            self.pdfs, self.pdfs_tmp = self.pdfs_tmp, self.pdfs
        self.time_steps_run += 1

    def run_sweeps(self, time_steps):
        """`time_steps` sweeps launched from one C call (no per-step Python), no getter."""
        n = int(time_steps)
        if n <= 0:
            return
        b = self._bound()
        if self._inplace:
            nxt = self._prev.next()
            p = self.pdfs.data_ptr()
            b.run(p, p, int(nxt.idx), n)
            self._prev = Timestep((int(nxt.idx) + n - 1) % 2)
        else:
            if b.run(self.pdfs.data_ptr(), self.pdfs_tmp.data_ptr(), 0, n):
                self.pdfs, self.pdfs_tmp = self.pdfs_tmp, self.pdfs
        self.time_steps_run += n

    def post_run(self):
        cd = torch.float64 if self._compute == "float64" else torch.float32
        rho = torch.empty(self._domain, dtype=cd, device=self.device)
        u = torch.empty(self._domain + (3,), dtype=cd, device=self.device)
        get_macroscopic(self._macro, self.pdfs, rho, u, self._prev, self.kernel_params, self.periodicity)
        self._density_t.copy_(rho)
        self._velocity_t.copy_(u)

    def run(self, time_steps):
        self.pre_run()
        self.run_sweeps(time_steps)
        self.post_run()

    def benchmark_run(self, time_steps, number_of_cells=None):
        """MLUPS of `time_steps` sweeps timed with CUDA events (lbstep.py:329-335)."""
        if number_of_cells is None:
            number_of_cells = self.number_of_cells
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        self.run_sweeps(time_steps)
        stop.record()
        torch.cuda.synchronize()
        seconds = start.elapsed_time(stop) * 1e-3 / max(int(time_steps), 1)
        return number_of_cells / seconds * 1e-6

    def benchmark(self, time_for_benchmark=5, init_time_steps=2, number_of_time_steps_for_estimation="auto"):
        for _ in range(init_time_steps):
            self.time_step()
        est = 20 if number_of_time_steps_for_estimation == "auto" else int(number_of_time_steps_for_estimation)
        mlups = self.benchmark_run(est)
        steps = max(1, int(time_for_benchmark * mlups * 1e6 / self.number_of_cells))
        return self.benchmark_run(steps)

    def reduce_conserved(self):
        """FP64 [mass, momentum x/y/z, kinetic energy] over fluid cells of the current state."""
        from .reductions import reduce_conserved
        return reduce_conserved(self)

    def run_iterative_initialization(self, *args, **kwargs):
        raise NotImplementedError("Mei's iterative initialisation is not built")

    def write_vtk(self):
        raise NotImplementedError("VTK output is not built")
