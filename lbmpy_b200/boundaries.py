"""NoSlip / UBB boundaries and the boundary handling of a PDF field.

lbmpy applies boundaries with a separate link kernel before every sweep
(``boundaries/boundaryhandling.py:15-199``, ``boundaries/boundaryconditions.py:104-139`` NoSlip,
``:724-841`` UBB).  Here the boundary handling only maintains a uint8 flag field over the
ghost-inclusive domain; the sweep performs the halfway bounce-back itself while it pulls, which
yields the same populations as lbmpy's link kernel followed by the sweep.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional

import numpy as np
import torch

from . import _native as N

FLUID, NOSLIP, UBB0, FIXED_DENSITY, FIXED_DENSITY1 = 0, 1, 2, 6, 7
MAX_UBB = 4
TYPE_MASK = 15          # low 4 bits of a flag: the cell type; bit 7: fluid cell next to a boundary


class LbBoundary:
    inner_or_boundary = True

    def __init__(self, name=None, calculate_force_on_boundary=False):
        if calculate_force_on_boundary:
            raise NotImplementedError("force evaluation on boundaries is not built")
        self._name = name

    @property
    def name(self):
        return self._name or type(self).__name__

    def __hash__(self):
        return hash(self.name)

    def __eq__(self, other):
        return type(self) is type(other) and self.__dict__ == other.__dict__


class NoSlip(LbBoundary):
    """Halfway bounce-back, f_inv(i)(x, t+1) = f*_i(x, t) (boundaryconditions.py:104-139)."""


class UBB(LbBoundary):
    """Velocity bounce-back f_inv(i) = f*_i - 2 w_i rho c_i.u_w / c_s^2 (boundaryconditions.py:724-841).

    - velocity: a constant vector, or a callback ``velocity(boundary_data)`` that sets one velocity
      per boundary link (``boundary_data['vel_0'] = ...``; positions from
      ``boundary_data.link_positions(coord)``), as lbmpy's UBB and ``add_pipe_inflow_boundary``
      (geometry.py:36-86) use it; the callback needs ``dim``.
    - density: compressible methods scale the wall term by this density instead of the fluid
      cell's (:824-830).
    - adapt_velocity_to_force: the wall velocity becomes the equilibrium velocity u - F / (2 rho_ref)
      of the method's force model (:790-794).
    """

    def __init__(self, velocity, density=None, adapt_velocity_to_force=False, dim=None, name=None,
                 data_type="double"):
        if callable(velocity) and not dim:
            raise ValueError("When using a velocity callback the dimension has to be specified with the dim parameter")
        self._callback = velocity if callable(velocity) else None
        self._velocity = (0.0,) * int(dim) if callable(velocity) else tuple(float(v) for v in velocity)
        self.dim = int(dim) if callable(velocity) else len(self._velocity)
        if density is not None and not float(density) > 0:
            raise ValueError("the UBB wall density must be positive")
        self._density = None if density is None else float(density)
        self._adapt = bool(adapt_velocity_to_force)
        super().__init__(name)

    @property
    def velocity(self):
        return self._velocity

    @property
    def velocity_is_callable(self):
        return self._callback is not None

    @property
    def density(self):
        return self._density

    @property
    def adapt_velocity_to_force(self):
        return self._adapt

    def same_as(self, other) -> bool:
        if self._callback is not None or other._callback is not None:
            return self is other
        return (self._velocity, self._density, self._adapt) == (other._velocity, other._density, other._adapt)


class BoundaryData:
    """The per-link view a UBB velocity callback receives (pystencils' ``BoundaryDataSetter``, the
    object lbmpy's callbacks are written against: ``geometry.py:58-86``,
    ``tests/test_free_slip.py:16-21``).  ``index_array`` is a record array with the fluid cell's
    ghost-inclusive ``x``, ``y``, ``z``, the link direction ``dir`` (index into the method's
    stencil, pointing from the fluid cell to the wall) and ``vel_0..2``."""

    def __init__(self, index_array, stencil_dirs):
        self.index_array = index_array
        self.dim = 3
        self._dirs = np.asarray(stencil_dirs, dtype=np.int64)
        self.boundary_data_names = {"vel_0", "vel_1", "vel_2"}

    def non_boundary_cell_positions(self, coord):
        """Cell-centre coordinate of the fluid cell (interior cells at 0.5 .. n - 0.5)."""
        return self.index_array["xyz"[coord]] - 1 + 0.5

    def link_offsets(self):
        return self._dirs[self.index_array["dir"]]

    def link_positions(self, coord):
        """Coordinate of the link's midpoint, where the halfway wall sits."""
        return self.non_boundary_cell_positions(coord) + 0.5 * self.link_offsets()[:, coord]

    def boundary_cell_positions(self, coord):
        return self.non_boundary_cell_positions(coord) + self.link_offsets()[:, coord]

    def __setitem__(self, key, value):
        if key not in self.boundary_data_names:
            raise KeyError(f"{key!r} is not boundary data; choose from {sorted(self.boundary_data_names)}")
        self.index_array[key] = value

    def __getitem__(self, item):
        return self.index_array[item]

    def __len__(self):
        return len(self.index_array)


class FixedDensity(LbBoundary):
    """Prescribed density (pressure p = rho / 3) at the wall (boundaryconditions.py:1044-1099):
    f_in(inv i) = 2 feq_even_i(rho_w, u) - f*_i, with feq_even the part of the method's equilibrium
    that is even in u and u the fluid cell's velocity from its outgoing populations at density
    rho_w.  Up to two densities per domain (an inlet and an outlet); force-free methods."""

    def __init__(self, density, name=None):
        if callable(density):
            raise NotImplementedError("density callbacks are not built; use a constant density")
        self.density = float(density)
        if not self.density > 0:
            raise ValueError("FixedDensity needs a positive density")
        super().__init__(name)


def slice_from_direction(direction_name: str, dim: int, normal_offset=0, tangential_offset=0):
    """pystencils' compass-direction slices over the ghost-inclusive array: 'N' is the last y
    layer (the ghost layer), 'S' the first, 'E'/'W' in x, 'T'/'B' in z."""
    if tangential_offset != 0:
        raise NotImplementedError("tangential offsets are not supported")
    axes = {"W": (0, 0), "E": (0, -1), "S": (1, 0), "N": (1, -1), "B": (2, 0), "T": (2, -1)}
    result = [slice(None)] * dim
    for ch in direction_name:
        ax, side = axes[ch]
        result[ax] = normal_offset if side == 0 else -1 - normal_offset
    return tuple(result)


class LatticeBoltzmannBoundaryHandling:
    """Flag field plus boundary objects for one PDF field.

    ``shape`` is the interior domain; flags cover the ghost-inclusive domain (x fastest, contiguous)."""

    def __init__(self, lb_method, shape, periodicity=(False, False, False), name="boundary_handling",
                 device="cuda", streaming_pattern="pull"):
        self.method = lb_method
        self.shape = tuple(int(s) for s in shape)
        self.periodicity = tuple(bool(p) for p in periodicity)
        self.name = name
        self.streaming_pattern = streaming_pattern
        self.device = device
        ex, ey, ez = (s + 2 for s in self.shape)
        self._host = np.zeros((ez, ey, ex), dtype=np.uint8)   # [z, y, x]
        self._ubbs: List[UBB] = []
        self._fixed_densities: List[float] = []
        self._dev: Optional[torch.Tensor] = None
        self._finalized_for = None
        self._links = None          # (cell block tensor, link velocity tensor, mask) for callable UBBs
        self._links_for = None

    # --------------------------------------------------------------------------- setup
    def _flag_for(self, boundary_obj) -> int:
        if boundary_obj is None or boundary_obj == "domain":
            return FLUID
        if isinstance(boundary_obj, NoSlip):
            return NOSLIP
        if isinstance(boundary_obj, UBB):
            for k, u in enumerate(self._ubbs):
                if u.same_as(boundary_obj):
                    return UBB0 + k
            if len(self._ubbs) >= MAX_UBB:
                raise ValueError(f"at most {MAX_UBB} different UBB boundaries are supported")
            self._ubbs.append(boundary_obj)
            return UBB0 + len(self._ubbs) - 1
        if isinstance(boundary_obj, FixedDensity):
            if boundary_obj.density in self._fixed_densities:
                return FIXED_DENSITY + self._fixed_densities.index(boundary_obj.density)
            if len(self._fixed_densities) >= 2:
                raise ValueError("at most two FixedDensity densities per domain are supported")
            self._fixed_densities.append(boundary_obj.density)
            return FIXED_DENSITY + len(self._fixed_densities) - 1
        raise NotImplementedError(f"boundary {type(boundary_obj).__name__} is not built (NoSlip, UBB and "
                                  "FixedDensity are)")

    def set_boundary(self, boundary_obj, slice_obj=None, mask_callback=None, ghost_layers=True,
                     inner_ghost_layers=True, replace=True, force_flag_value=None):
        """Marks cells (indexed over the ghost-inclusive domain) with a boundary; lbmpy's
        ``BoundaryHandling.set_boundary``.  ``mask_callback(x, y, z)`` receives cell-midpoint
        coordinates (interior cells at 0.5 .. n-0.5, ghost cells at -0.5 and n+0.5)."""
        flag = self._flag_for(boundary_obj)
        view = self._host.transpose(2, 1, 0)           # [x, y, z]
        if not ghost_layers:
            view = view[1:-1, 1:-1, 1:-1]
        sl = (slice(None),) * 3 if slice_obj is None else tuple(slice_obj) + (slice(None),) * (3 - len(slice_obj))
        region = view[sl]
        if mask_callback is not None:
            shift = -0.5 if ghost_layers else 0.5
            coords = np.meshgrid(*[np.arange(n) + shift for n in view.shape], indexing="ij")
            mask = np.asarray(mask_callback(*[c[sl] for c in coords]), dtype=bool)
        else:
            mask = np.ones(region.shape, dtype=bool)
        if replace:
            region[mask] = flag
        else:
            region[mask & (region == FLUID)] = flag
        self._dev = None
        self._links = None
        return flag

    def get_mask(self, slice_obj, boundary_obj, inverse=False):
        """Boolean mask (ghost-inclusive, [x, y, z]) of the cells that carry `boundary_obj`."""
        view = self._host.transpose(2, 1, 0)
        if boundary_obj == "domain":
            m = view == FLUID
        else:
            m = view == self._flag_for(boundary_obj)
        if slice_obj is not None:
            m = m[tuple(slice_obj)]
        return ~m if inverse else m

    @property
    def ubb_velocities(self):
        return [u.velocity for u in self._ubbs]

    @property
    def ubb_options(self):
        """Prescribed wall densities (0: none) and the adapt-to-force mask of the UBB numbers."""
        return {"densities": [u.density or 0.0 for u in self._ubbs],
                "adapt_mask": sum(1 << k for k, u in enumerate(self._ubbs) if u.adapt_velocity_to_force)}

    def ubb_links(self, periodicity=None):
        """Every link from a fluid cell into a cell of each callable UBB, with the velocities its
        callback set: {UBB number: record array (x, y, z ghost-inclusive fluid cell, dir, vel_0..2)}.
        Periodic axes wrap, as the sweep's neighbour lookup does."""
        periodicity = self.periodicity if periodicity is None else periodicity
        dirs = [tuple(int(v) for v in d) for d in self.method.stencil]
        flags = self._host.transpose(2, 1, 0) & TYPE_MASK    # [x, y, z], ghost-inclusive
        n = self.shape
        out = {}
        for k, u in enumerate(self._ubbs):
            if not u.velocity_is_callable:
                continue
            recs = []
            fluid = flags[1:-1, 1:-1, 1:-1] == FLUID
            for q, c in enumerate(dirs):
                if c == (0, 0, 0):
                    continue
                idx = []
                for a in range(3):
                    i = np.arange(n[a]) + c[a]
                    if periodicity[a]:
                        i = i % n[a]
                    idx.append(i + 1)
                nb = flags[np.ix_(*idx)]
                hit = fluid & (nb == UBB0 + k)
                xs, ys, zs = np.nonzero(hit)
                if len(xs):
                    recs.append((xs + 1, ys + 1, zs + 1, np.full(len(xs), q)))
            dt = np.dtype([("x", np.int32), ("y", np.int32), ("z", np.int32), ("dir", np.int32),
                           ("vel_0", np.float64), ("vel_1", np.float64), ("vel_2", np.float64)])
            arr = np.zeros(sum(len(r[0]) for r in recs), dtype=dt)
            pos = 0
            for xs, ys, zs, qs in recs:
                m = len(xs)
                arr["x"][pos:pos + m], arr["y"][pos:pos + m], arr["z"][pos:pos + m] = xs, ys, zs
                arr["dir"][pos:pos + m] = qs
                pos += m
            u._callback(BoundaryData(arr, dirs))
            out[k] = arr
        return out

    def ubb_link_velocities_dense(self):
        """[x, y, z, Q, 3] velocities of every callable-UBB link (zero elsewhere), for checkers that
        take a dense per-link array."""
        q = len(self.method.stencil)
        dense = np.zeros(self.shape + (q, 3))
        for arr in self.ubb_links().values():
            for k in range(3):
                dense[arr["x"] - 1, arr["y"] - 1, arr["z"] - 1, arr["dir"], k] = arr[f"vel_{k}"]
        return dense

    def attach_links(self, plan):
        """Builds (once per boundary set-up) the per-link velocity tables of the callable UBBs and
        hands them to `plan` (lbm_plan_set_ubb_links)."""
        if not any(u.velocity_is_callable for u in self._ubbs):
            return
        if self._links is None:
            links = self.ubb_links()
            q = len(self.method.stencil)
            n = self.shape
            block = np.full(n[0] * n[1] * n[2], -1, dtype=np.int32)      # x fastest
            allr = np.concatenate(list(links.values())) if links else np.zeros(0, dtype=np.int32)
            cell = (allr["x"] - 1) + n[0] * ((allr["y"] - 1) + n[1] * (allr["z"] - 1)) if len(allr) else allr
            uniq, inv = np.unique(cell, return_inverse=True)
            vel = np.zeros((max(len(uniq), 1), q, 3))
            for k in range(3):
                if len(allr):
                    vel[inv, allr["dir"], k] = allr[f"vel_{k}"]
            block[uniq] = np.arange(len(uniq), dtype=np.int32)
            mask = sum(1 << k for k, u in enumerate(self._ubbs) if u.velocity_is_callable)
            self._links = (torch.from_numpy(block).to(self.device), torch.from_numpy(vel).to(self.device), mask,
                           vel.shape[0])
        blk, vel, mask, nb = self._links
        N.check(N.lib().lbm_plan_set_ubb_links(plan.handle, ctypes.c_void_p(blk.data_ptr()),
                                               ctypes.c_void_p(vel.data_ptr()), nb, mask), "lbm_plan_set_ubb_links")

    @property
    def fixed_density(self):
        """Densities (first, second) of the FixedDensity cells, None if there are none."""
        types = self._host & TYPE_MASK
        used = [rho if bool((types == FIXED_DENSITY + k).any()) else 0.0 for k, rho in enumerate(self._fixed_densities)]
        return tuple(used) if any(used) else None

    @property
    def has_boundaries(self) -> bool:
        return bool((self._host & TYPE_MASK).any())

    @property
    def flag_array(self) -> np.ndarray:
        """Host copy of the cell types, [x, y, z] over the ghost-inclusive domain."""
        return self._host.transpose(2, 1, 0)

    def flags(self, plan) -> torch.Tensor:
        """Device flag field with the near-boundary bit computed for `plan`'s stencil/periodicity."""
        key = (int(plan.desc.stencil), tuple(plan.desc.periodic))
        if self._dev is None or self._finalized_for != key:
            t = torch.from_numpy(self._host.copy()).to(self.device).permute(2, 1, 0)
            N.check(N.lib().lbm_flags_finalize(plan.handle, ctypes.c_void_p(t.data_ptr()),
                                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
                    "lbm_flags_finalize")
            self._dev = t
            self._finalized_for = key
        return self._dev

    def __call__(self, *args, **kwargs):
        """Boundaries are applied inside the sweep; calling the handling is a no-op kept for
        lbmpy's time-loop structure (sync -> boundaries -> sweep)."""
        return None
