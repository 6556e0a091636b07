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

FLUID, NOSLIP, UBB0, FIXED_DENSITY = 0, 1, 2, 6
MAX_UBB = 4


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
    """Velocity bounce-back f_inv(i) = f*_i - 2 w_i rho c_i.u_w / c_s^2 (boundaryconditions.py:724-841);
    rho from the fluid cell for compressible methods, 1 otherwise."""

    def __init__(self, velocity, density=None, adapt_velocity_to_force=False, dim=None, name=None,
                 data_type="double"):
        if callable(velocity):
            raise NotImplementedError("velocity callbacks are not built; use a constant wall velocity")
        if density is not None:
            raise NotImplementedError("a prescribed wall density is not built")
        if adapt_velocity_to_force:
            raise NotImplementedError("adapt_velocity_to_force is not built")
        self._velocity = tuple(float(v) for v in velocity)
        self.dim = len(self._velocity)
        super().__init__(name)

    @property
    def velocity(self):
        return self._velocity


class FixedDensity(LbBoundary):
    """Prescribed density (pressure p = rho / 3) at the wall (boundaryconditions.py:1044-1099):
    f_in(inv i) = 2 feq_even_i(rho_w, u) - f*_i, with feq_even the part of the method's equilibrium
    that is even in u and u the fluid cell's velocity from its outgoing populations at density
    rho_w.  One density per domain; force-free methods."""

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
        self._fixed_density: Optional[float] = None
        self._dev: Optional[torch.Tensor] = None
        self._finalized_for = None

    # --------------------------------------------------------------------------- setup
    def _flag_for(self, boundary_obj) -> int:
        if boundary_obj is None or boundary_obj == "domain":
            return FLUID
        if isinstance(boundary_obj, NoSlip):
            return NOSLIP
        if isinstance(boundary_obj, UBB):
            for k, u in enumerate(self._ubbs):
                if u.velocity == boundary_obj.velocity:
                    return UBB0 + k
            if len(self._ubbs) >= MAX_UBB:
                raise ValueError(f"at most {MAX_UBB} different UBB velocities are supported")
            self._ubbs.append(boundary_obj)
            return UBB0 + len(self._ubbs) - 1
        if isinstance(boundary_obj, FixedDensity):
            if self._fixed_density is not None and self._fixed_density != boundary_obj.density:
                raise ValueError("one FixedDensity density per domain is supported")
            self._fixed_density = boundary_obj.density
            return FIXED_DENSITY
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
    def fixed_density(self):
        """Density of the FixedDensity cells, if any are set."""
        return self._fixed_density if bool(((self._host & 7) == FIXED_DENSITY).any()) else None

    @property
    def has_boundaries(self) -> bool:
        return bool((self._host & 7).any())

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
