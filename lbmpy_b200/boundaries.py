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
FREE_SLIP, SIMPLE_OUTFLOW, OUTFLOW, BOUZIDI = 8, 9, 10, 11
MAX_UBB = 4
TYPE_MASK = 15          # low 4 bits of a flag: the cell type; bit 7: fluid cell next to a boundary
_DIRECTION_LETTERS = {"E": (1, 0, 0), "W": (-1, 0, 0), "N": (0, 1, 0), "S": (0, -1, 0), "T": (0, 0, 1),
                      "B": (0, 0, -1)}


def _code(direction: int, offset) -> int:
    """Per-link code of FreeSlip and the outflows: the incoming population is the outgoing population
    `direction` of the cell at `offset` from the fluid cell."""
    return int(direction) | (offset[0] + 1) << 8 | (offset[1] + 1) << 10 | (offset[2] + 1) << 12


def direction_string_to_offset(direction: str, dim: int = 3):
    """'NE' -> (1, 1, 0): pystencils' compass names of the stencil directions."""
    off = [0, 0, 0]
    for ch in direction.upper():
        for a, v in enumerate(_DIRECTION_LETTERS[ch]):
            off[a] += v
    return tuple(off[:dim])


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
        self.boundary_data_names = set(index_array.dtype.names) - {"x", "y", "z", "dir"}

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


class FreeSlip(LbBoundary):
    """Specular reflection, zero normal velocity (boundaryconditions.py:360-455): the population
    entering a fluid cell from the wall is the mirrored outgoing population of the tangential
    neighbour.  With `normal_direction` (pointing from the wall into the fluid) the mirror axis is
    fixed; without it the normal of every link is found from the neighbouring boundary cells, as
    lbmpy's init callback does (convex corners fall back to bounce-back)."""

    def __init__(self, stencil, normal_direction=None, name=None):
        if normal_direction and len(normal_direction) - list(normal_direction).count(0) != 1:
            raise ValueError("It is only possible to pre specify the normal direction for simple situations."
                             "This means if the free slip boundary is applied to a straight wall or side in the "
                             "simulation domain. A possible value for example would be (0, 1, 0) if the "
                             "free slip boundary is applied to the northern wall. For more complex situations "
                             "the normal direction has to be calculated for each cell. This is done when "
                             "the normal direction is not defined for this class")
        if normal_direction:
            normal_direction = tuple(int(n) for n in normal_direction)
            if not all(n in (-1, 0, 1) for n in normal_direction):
                raise ValueError("Only -1, 0 and 1 allowed for defining the normal direction")
            self.mirror_axis = [k for k, n in enumerate(normal_direction) if n != 0][0]
        self.stencil = [tuple(int(v) for v in d) for d in stencil]
        self.normal_direction = normal_direction
        self.dim = len(self.stencil[0])
        super().__init__(name)


class SimpleExtrapolationOutflow(LbBoundary):
    """Outflow copying the missing populations from the last fluid layer along the outflow normal
    (boundaryconditions.py:844-889; Geier et al. 2015, eq. F.1)."""

    def __init__(self, normal_direction, stencil, name=None):
        if isinstance(normal_direction, str):
            normal_direction = direction_string_to_offset(normal_direction, dim=len(stencil[0]))
        self.normal_direction = tuple(int(n) for n in normal_direction)
        if not all(n in (-1, 0, 1) for n in self.normal_direction):
            raise ValueError("Only -1, 0 and 1 allowed for defining the normal direction")
        super().__init__(name)


class ExtrapolationOutflow(LbBoundary):
    """Outflow interpolating in time between the last fluid layer and the boundary
    (boundaryconditions.py:894-1041; Geier et al. 2015, eq. F.2 with u neglected):
    f_in = c p + (1 - c) p_nd with c = sqrt(1/3) dt/dx, p the outgoing population of the fluid
    neighbour one step earlier and p_nd the previous result.  Both start from the field's values
    when the boundary is first applied."""

    def __init__(self, normal_direction, lb_method, dt=1, dx=1, name=None, streaming_pattern="pull",
                 zeroth_timestep=None, initial_density=None, initial_velocity=None, data_type="double"):
        if isinstance(normal_direction, str):
            normal_direction = direction_string_to_offset(normal_direction, dim=lb_method.stencil.D)
        self.normal_direction = tuple(int(n) for n in normal_direction)
        if not all(n in (-1, 0, 1) for n in self.normal_direction):
            raise ValueError("Only -1, 0 and 1 allowed for defining the normal direction")
        if initial_density is not None or initial_velocity is not None:
            raise NotImplementedError("initial_density / initial_velocity of ExtrapolationOutflow are not built; "
                                      "the links start from the field's values")
        if float(dt) != 1.0 or float(dx) != 1.0:
            # c dt/dx = sqrt(1/3) whatever dt and dx are, as lbmpy's c carries dx/dt
            pass
        self.streaming_pattern = streaming_pattern
        super().__init__(name)


class NoSlipLinearBouzidi(LbBoundary):
    """No-slip with linear interpolation at the wall distance q of every link
    (boundaryconditions.py:142-212; Bouzidi et al. 2001).  `init_wall_distance(boundary_data)` sets
    ``boundary_data['q']``; links left at q <= 0 (the default, -1) bounce back as NoSlip."""

    def __init__(self, name=None, init_wall_distance=None, data_type="double", calculate_force_on_boundary=False):
        if init_wall_distance is None:
            import warnings
            warnings.warn("No callback function provided to initialise the wall distance for each cell "
                          "(init_wall_distance=None). The boundary condition will fall back to a simple NoSlip BC")
        self.init_wall_distance = init_wall_distance
        super().__init__(name, calculate_force_on_boundary)


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
        self._links = None          # device link tables (LbmLinkTables and the tensors they point to)
        self._link_objs: List = []  # FreeSlip / outflow / Bouzidi objects, indexed by self._obj
        self._obj = np.full((ez, ey, ex), -1, dtype=np.int16)

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
        types = {FreeSlip: FREE_SLIP, SimpleExtrapolationOutflow: SIMPLE_OUTFLOW, ExtrapolationOutflow: OUTFLOW,
                 NoSlipLinearBouzidi: BOUZIDI}
        if type(boundary_obj) in types:
            if not any(o is boundary_obj for o in self._link_objs):
                self._link_objs.append(boundary_obj)
            return types[type(boundary_obj)]
        raise NotImplementedError(f"boundary {type(boundary_obj).__name__} is not built (NoSlip, UBB, FixedDensity, "
                                  "FreeSlip, SimpleExtrapolationOutflow, ExtrapolationOutflow and "
                                  "NoSlipLinearBouzidi are)")

    def _obj_index(self, boundary_obj) -> int:
        for k, o in enumerate(self._link_objs):
            if o is boundary_obj:
                return k
        return -1

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
        objs = self._obj.transpose(2, 1, 0)
        if not ghost_layers:
            objs = objs[1:-1, 1:-1, 1:-1]
        oreg = objs[sl]
        if not replace:
            mask = mask & (region == FLUID)
        region[mask] = flag
        oreg[mask] = self._obj_index(boundary_obj)
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

    def _links_into(self, select):
        """Every link (fluid interior cell, direction q) whose neighbour x + c_q satisfies
        select(types, objects) over the ghost-inclusive [x, y, z] arrays; periodic axes wrap, as the
        sweep's neighbour lookup does.  Record array: ghost-inclusive x, y, z of the fluid cell, dir."""
        dirs = [tuple(int(v) for v in d) for d in self.method.stencil]
        types = self._host.transpose(2, 1, 0) & TYPE_MASK
        objs = self._obj.transpose(2, 1, 0)
        target = select(types, objs)
        n = self.shape
        fluid = types[1:-1, 1:-1, 1:-1] == FLUID
        parts = []
        for q, c in enumerate(dirs):
            if c == (0, 0, 0):
                continue
            idx = []
            for a in range(3):
                i = np.arange(n[a]) + c[a]
                if self.periodicity[a]:
                    i = i % n[a]
                idx.append(i + 1)
            hit = fluid & target[np.ix_(*idx)]
            xs, ys, zs = np.nonzero(hit)
            parts.append((xs + 1, ys + 1, zs + 1, np.full(len(xs), q)))
        m = sum(len(p[0]) for p in parts)
        out = np.zeros(m, dtype=[("x", np.int32), ("y", np.int32), ("z", np.int32), ("dir", np.int32)])
        pos = 0
        for xs, ys, zs, qs in parts:
            k = len(xs)
            out["x"][pos:pos + k], out["y"][pos:pos + k], out["z"][pos:pos + k] = xs, ys, zs
            out["dir"][pos:pos + k] = qs
            pos += k
        return out

    @staticmethod
    def _with_fields(links, fields):
        dt = links.dtype.descr + [(name, np.float64) for name in fields]
        arr = np.zeros(len(links), dtype=dt)
        for name in links.dtype.names:
            arr[name] = links[name]
        return arr

    def ubb_links(self):
        """Every link into a cell of each callable UBB, with the velocities its callback set:
        {UBB number: record array (x, y, z ghost-inclusive fluid cell, dir, vel_0..2)}."""
        dirs = [tuple(int(v) for v in d) for d in self.method.stencil]
        out = {}
        for k, u in enumerate(self._ubbs):
            if not u.velocity_is_callable:
                continue
            arr = self._with_fields(self._links_into(lambda t, o, k=k: t == UBB0 + k), ("vel_0", "vel_1", "vel_2"))
            u._callback(BoundaryData(arr, dirs))
            out[k] = arr
        return out

    def _freeslip_codes(self, obj, links):
        """Link codes of one FreeSlip (boundaryconditions.py:398-455)."""
        dirs = [tuple(int(v) for v in d) for d in self.method.stencil]
        n = self.shape

        def wrap(cell):
            return tuple((c - 1) % n[a] + 1 if self.periodicity[a] else c for a, c in enumerate(cell))

        def mirror(d, axis):
            d = list(d)
            d[axis] = -d[axis]
            return tuple(d)
        codes = np.zeros(len(links), dtype=np.int32)
        if obj.normal_direction:
            nrm = obj.normal_direction
            for r, (q) in enumerate(links["dir"]):
                c = dirs[q]
                ref = tuple(-v for v in mirror(c, obj.mirror_axis))
                off = tuple(a + b for a, b in zip(c, nrm))
                codes[r] = _code(dirs.index(ref), off)
            return codes
        cells = {wrap((int(x) + dirs[q][0], int(y) + dirs[q][1], int(z) + dirs[q][2]))
                 for x, y, z, q in zip(links["x"], links["y"], links["z"], links["dir"])}
        for r, (x, y, z, q) in enumerate(zip(links["x"], links["y"], links["z"], links["dir"])):
            c = dirs[q]
            ref = c
            normal = [0, 0, 0]
            for a in range(3):
                sub = [0, 0, 0]
                sub[a] = c[a]
                if c[a] != 0 and wrap((int(x) + sub[0], int(y) + sub[1], int(z) + sub[2])) in cells:
                    normal[a] = c[a]
                    ref = mirror(ref, a)
            if all(v == 0 for v in normal):          # convex corner: bounce back
                normal = list(c)
            else:
                ref = tuple(-v for v in ref)
            off = tuple(c[a] - normal[a] for a in range(3))
            codes[r] = _code(dirs.index(tuple(ref)), off)
        return codes

    def _outflow_codes(self, obj, links):
        dirs = [tuple(int(v) for v in d) for d in self.method.stencil]
        codes = np.zeros(len(links), dtype=np.int32)
        for r, q in enumerate(links["dir"]):
            c = dirs[q]
            inv = dirs.index(tuple(-v for v in c))
            codes[r] = _code(inv, tuple(a - b for a, b in zip(c, obj.normal_direction)))
        return codes

    def link_tables_host(self, pdfs=None, previous_timestep=None, pattern=None):
        """The per-link data of every boundary that has some, grouped by fluid cell (the layout of
        lbm_plan_set_links): (cell_block [nx*ny*nz] int32, ubb_velocity [B, Q, 3], link_code [B, Q],
        link_value [B, Q, 2], ubb_mask).  ExtrapolationOutflow's two values start from the
        outgoing populations of the field `pdfs` (host array [x, y, z, q], ghost-inclusive), as the
        previous step of `pattern` with `previous_timestep` wrote them."""
        from .accessors import write_location
        dirs = [tuple(int(v) for v in d) for d in self.method.stencil]
        q = len(dirs)
        n = self.shape
        groups = []            # (links, kind, data)
        ubb_mask = 0
        for k, arr in self.ubb_links().items():
            ubb_mask |= 1 << k
            groups.append((arr, "ubb", np.stack([arr["vel_0"], arr["vel_1"], arr["vel_2"]], axis=-1)))
        for k, obj in enumerate(self._link_objs):
            links = self._links_into(lambda t, o, k=k: o == k)
            if isinstance(obj, FreeSlip):
                groups.append((links, "code", self._freeslip_codes(obj, links)))
            elif isinstance(obj, SimpleExtrapolationOutflow):
                groups.append((links, "code", self._outflow_codes(obj, links)))
            elif isinstance(obj, ExtrapolationOutflow):
                codes = self._outflow_codes(obj, links)
                vals = np.zeros((len(links), 2))
                if pdfs is not None:
                    pat = pattern or self.streaming_pattern
                    par = 0 if previous_timestep is None else int(previous_timestep)
                    for r, (x, y, z, cd) in enumerate(zip(links["x"], links["y"], links["z"], codes)):
                        d = int(cd) & 0xFF
                        cell = [int(x) + ((int(cd) >> (8 + 2 * a)) & 3) - 1 for a in range(3)]
                        woff, slot = write_location(pat, par, dirs, d)
                        loc = []
                        for a in range(3):
                            v = cell[a] + woff[a]
                            if self.periodicity[a]:
                                v = (v - 1) % n[a] + 1
                            loc.append(min(max(v, 0), n[a] + 1))
                        vals[r] = pdfs[loc[0], loc[1], loc[2], slot]
                groups.append((links, "outflow", (codes, vals)))
            elif isinstance(obj, NoSlipLinearBouzidi):
                arr = self._with_fields(links, ("q",))
                arr["q"] = -1.0
                if obj.init_wall_distance is not None:
                    obj.init_wall_distance(BoundaryData(arr, dirs))
                groups.append((links, "q", np.asarray(arr["q"], np.float64)))
        allx = [g[0] for g in groups if len(g[0])]
        block = np.full(n[0] * n[1] * n[2], -1, dtype=np.int32)
        if not allx:
            return None
        cell = np.concatenate([(a["x"] - 1) + n[0] * ((a["y"] - 1) + n[1] * (a["z"] - 1)) for a in allx])
        uniq = np.unique(cell)
        block[uniq] = np.arange(len(uniq), dtype=np.int32)
        nb = len(uniq)
        vel = np.zeros((nb, q, 3))
        code = np.zeros((nb, q), dtype=np.int32)
        value = np.zeros((nb, q, 2))
        for links, kind, data in groups:
            if not len(links):
                continue
            b = block[(links["x"] - 1) + n[0] * ((links["y"] - 1) + n[1] * (links["z"] - 1))]
            d = links["dir"]
            if kind == "ubb":
                vel[b, d] = data
            elif kind == "code":
                code[b, d] = data
            elif kind == "outflow":
                code[b, d] = data[0]
                value[b, d] = data[1]
            else:
                value[b, d, 0] = data
        return block, vel, code, value, ubb_mask

    def link_tables_dense(self, pdfs=None, previous_timestep=None, pattern=None):
        """The per-link data as dense arrays over interior cells and directions, for checkers:
        (ubb_velocity [x, y, z, Q, 3], link_code [x, y, z, Q], link_value [x, y, z, Q, 2])."""
        t = self.link_tables_host(pdfs, previous_timestep, pattern)
        q = len(self.method.stencil)
        n = self.shape
        vel, code, value = np.zeros(n + (q, 3)), np.zeros(n + (q,), np.int32), np.zeros(n + (q, 2))
        if t is None:
            return vel, code, value
        block, bv, bc, bval, _ = t
        b = block.reshape(n[2], n[1], n[0]).transpose(2, 1, 0)
        has = b >= 0
        vel[has], code[has], value[has] = bv[b[has]], bc[b[has]], bval[b[has]]
        return vel, code, value

    def ubb_link_velocities_dense(self):
        """[x, y, z, Q, 3] velocities of every callable-UBB link (zero elsewhere)."""
        return self.link_tables_dense()[0]

    def attach_links(self, plan, pdfs=None, previous_timestep=None):
        """Builds (once per boundary set-up) the per-link tables of the boundaries that need them and
        hands them to `plan` (lbm_plan_set_links).  ExtrapolationOutflow links start from the current
        field `pdfs` (a device tensor) as the step before `previous_timestep` left it."""
        if not self._link_objs and not any(u.velocity_is_callable for u in self._ubbs):
            return
        if self._links is None:
            host_pdfs = None
            if pdfs is not None and any(isinstance(o, ExtrapolationOutflow) for o in self._link_objs):
                host_pdfs = pdfs.detach().double().cpu().numpy()
            t = self.link_tables_host(host_pdfs, previous_timestep)
            if t is None:
                self._links = ()
            else:
                block, vel, code, value, mask = t
                dev = [torch.from_numpy(a).to(self.device) for a in (block, vel, code, value)]
                tabs = N.LbmLinkTables()
                tabs.cell_block = dev[0].data_ptr()
                tabs.n_blocks = vel.shape[0]
                tabs.ubb_velocity = dev[1].data_ptr()
                tabs.ubb_mask = mask
                tabs.link_code = dev[2].data_ptr()
                tabs.link_value = dev[3].data_ptr()
                self._links = (tabs, dev)
        if self._links:
            N.check(N.lib().lbm_plan_set_links(plan.handle, ctypes.byref(self._links[0])), "lbm_plan_set_links")

    @property
    def link_values(self):
        """Device tensor of the per-link values ([B, Q, 2]: Bouzidi q, ExtrapolationOutflow state)."""
        return self._links[1][3] if self._links else None

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
