"""Sparse (list-based) LBM: lbmpy's ``lbmpy.sparse`` on the sm_100a sweep.

lbmpy stores only the cells that matter — fluid cells first, then the boundary cells their
stencils reach — as a list, PDF i of list cell c at element ``c + i * len(mapping)`` (a numpy array
of shape ``(len(mapping), Q)`` in Fortran order), and streams through an index list built once on
the host (sparse/mapping.py:13-156).  The pieces, with lbmpy's names:

- ``SparseLbMapper(stencil, flag_arr, fluid_flag, no_slip_flag, other_boundary_mask)``: the cell
  list and ``create_index_array()``, the ``(num_fluid_cells, Q - 1)`` uint32 pull index (NoSlip
  folded in as the cell's own inverse slot, periodic images at the ghost layer).  The numpy
  construction here yields lbmpy's array element for element.
- ``create_lb_update_rule_sparse(collision_rule, src, dst, idx, kernel_type)`` and
  ``create_lb_function_sparse(update_rule)``: the stream-pull-collide kernel, called as
  ``kernel(f=pdfs, d=pdfs_tmp, idx=index)`` with CUDA tensors (sparse/update_rule_sparse.py:22-52).
- ``create_macroscopic_value_setter_sparse`` / ``..._getter_sparse``: equilibrium initialisation
  and density / velocity output of the fluid cells (sparse/update_rule_sparse.py:55-85).
- ``SparseLbBoundaryMapper(UBB(...), method, pdf_field)``: velocity bounce-back into the boundary
  cells' slots before the sweep (sparse/mapping.py:157-247).

PDF lists are CUDA tensors whose element (c, i) lies at ``c + i * n_cells``: a ``(Q, n_cells)``
contiguous tensor, or its transpose ``(n_cells, Q)`` (the layout of lbmpy's Fortran-order array).
``pdf_list(n_cells, q, dtype)`` allocates one.  Storage is FP64 or FP32.
"""
from __future__ import annotations

import ctypes
from typing import Tuple

import numpy as np
import torch

from . import _native as N
from .kernel import _stream_handle, build_desc, free_parameters

_COORD_NAMES = ("x", "y", "z")
NOT_FOUND = np.uint32(0xFFFFFFFF)


def _dirs(stencil):
    return [tuple(int(v) for v in d) for d in stencil]


# ---------------------------------------------------------------------------- cell list
class SparseLbMapper:
    """Cell list and pull index of a sparse domain (sparse/mapping.py:13-156).

    Args:
        stencil: the method's stencil (sequence of direction tuples, centre first)
        flag_arr: integer array over the ghost-inclusive domain, one bit per cell type
        fluid_flag: bit of fluid cells
        no_slip_flag: bit of NoSlip cells (folded into the index array, not listed)
        other_boundary_mask: bits of boundary cells that stay in the list (their slots receive the
            values of boundary kernels, e.g. UBB)
    """

    def __init__(self, stencil, flag_arr, fluid_flag, no_slip_flag, other_boundary_mask):
        self._flag_arr = flag_arr
        self._coordinate_arr = None
        self._lookup = None
        self._dirty = True
        self.fluid_flag = fluid_flag
        self.no_slip_flag = no_slip_flag
        self.other_boundary_mask = other_boundary_mask
        self._num_fluid_cells = None
        self.stencil = stencil

    @property
    def coordinates(self):
        if self._dirty:
            self._assemble()
        return self._coordinate_arr

    @property
    def fluid_coordinates(self):
        if self._dirty:
            self._assemble()
        return self._coordinate_arr[:self.num_fluid_cells]

    @property
    def num_fluid_cells(self):
        if self._dirty:
            self._assemble()
        return self._num_fluid_cells

    @property
    def flag_array(self):
        return self._flag_arr

    def cell_idx(self, coordinate: Tuple[int, ...]) -> np.uint32:
        """List index of the cell at `coordinate`; IndexError if the cell is not listed."""
        if self._dirty:
            self._assemble()
        c = tuple(int(v) for v in coordinate)
        if any(v < 0 or v >= s for v, s in zip(c, self._flag_arr.shape)) or self._lookup[c] == NOT_FOUND:
            raise IndexError("Coordinate not found")
        return self._lookup[c]

    def cell_idx_bulk(self, coordinates):
        """List indices of a structured coordinate array (fields x, y[, z]); cells that are not
        listed map to 0xFFFFFFFF."""
        if self._dirty:
            self._assemble()
        dim = self._flag_arr.ndim
        idx = np.stack([np.asarray(coordinates[n]).astype(np.int64) for n in _COORD_NAMES[:dim]], axis=-1)
        inside = np.all((idx >= 0) & (idx < np.array(self._flag_arr.shape)), axis=-1)
        out = np.full(idx.shape[:-1], NOT_FOUND, dtype=np.uint32)
        sel = idx[inside]
        out[inside] = self._lookup[tuple(sel.T)]
        return out

    def coordinate(self, cell_idx: int):
        if self._dirty:
            self._assemble()
        return self._coordinate_arr[cell_idx]

    def __len__(self):
        if self._dirty:
            self._assemble()
        return len(self._coordinate_arr)

    def _assemble(self):
        dim = self._flag_arr.ndim
        struct_type = np.dtype([(name, np.uint32) for name in _COORD_NAMES[:dim]])
        fluid = np.argwhere(np.bitwise_and(self._flag_arr, self.fluid_flag)).astype(np.uint32)
        boundary = np.argwhere(np.bitwise_and(self._flag_arr, self.other_boundary_mask)).astype(np.uint32)
        self._num_fluid_cells = fluid.shape[0]
        coords = np.empty((fluid.shape[0] + boundary.shape[0],), dtype=struct_type)
        for d, name in enumerate(_COORD_NAMES[:dim]):
            coords[name][:self._num_fluid_cells] = fluid[:, d]
            coords[name][self._num_fluid_cells:] = boundary[:, d]
        lookup = np.full(self._flag_arr.shape, NOT_FOUND, dtype=np.uint32)
        all_idx = np.concatenate([fluid, boundary]).astype(np.int64)
        if len(all_idx):
            lookup[tuple(all_idx.T)] = np.arange(len(all_idx), dtype=np.uint32)
        self._coordinate_arr = coords
        self._lookup = lookup
        self._dirty = False

    def create_index_array(self, ghost_layers=1):
        """The ``(num_fluid_cells, Q - 1)`` uint32 pull index: entry (c, i - 1) is the list element
        fluid cell c reads population i from — the neighbour c - e_i if it is listed, else the
        cell's own inverse slot if that neighbour is NoSlip, else the periodic image of a ghost
        neighbour (ValueError if there is none).  The array is a transposed view of a
        direction-major buffer, as lbmpy returns it."""
        if self._dirty:
            self._assemble()
        dirs = _dirs(self.stencil)
        n_fluid = self._num_fluid_cells
        n = len(self)
        shape = np.array(self._flag_arr.shape)
        fluid = np.stack([self._coordinate_arr[name][:n_fluid].astype(np.int64)
                          for name in _COORD_NAMES[:self._flag_arr.ndim]], axis=-1)
        listed_mask = self.other_boundary_mask | self.fluid_flag
        own = np.arange(n_fluid, dtype=np.int64)
        rows = []
        for i, c in enumerate(dirs):
            if all(v == 0 for v in c):
                assert i == 0
                continue
            inv = dirs.index(tuple(-v for v in c))
            nb = fluid - np.array(c)
            fl = self._flag_arr[tuple(nb.T)]
            res = np.empty(n_fluid, dtype=np.int64)
            listed = (fl & listed_mask) != 0
            res[listed] = self._lookup[tuple(nb[listed].T)].astype(np.int64) + i * n
            wall = ~listed & ((fl & self.no_slip_flag) != 0)
            res[wall] = own[wall] + inv * n
            rest = ~listed & ~wall
            if rest.any():
                img = nb[rest].copy()
                border = np.zeros(len(img), dtype=bool)
                for a in range(img.shape[1]):
                    lo = img[:, a] == ghost_layers - 1
                    hi = img[:, a] == shape[a] - ghost_layers
                    img[lo, a] += shape[a] - 2 * ghost_layers
                    img[hi, a] -= shape[a] - 2 * ghost_layers
                    border |= lo | hi
                if not border.all():
                    k = np.flatnonzero(rest)[np.flatnonzero(~border)[0]]
                    raise ValueError(f"Could not find neighbor for {tuple(fluid[k])} direction {c}")
                if not np.all(self._flag_arr[tuple(img.T)] & listed_mask):
                    raise AssertionError("the periodic image of a ghost neighbour is not a listed cell")
                res[rest] = self._lookup[tuple(img.T)].astype(np.int64) + i * n
            rows.append(res)
        index = np.array(rows, dtype=np.uint32).reshape(len(dirs) - 1, n_fluid)
        return index.swapaxes(0, 1)


# ---------------------------------------------------------------------------- PDF lists
def pdf_list(n_cells: int, q: int, dtype=torch.float64, device="cuda") -> torch.Tensor:
    """An (n_cells, Q) PDF list with element (c, i) at c + i * n_cells."""
    return torch.zeros((q, n_cells), dtype=dtype, device=device).t()


def _check_list(t: torch.Tensor, q: int, name: str) -> int:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if t.dim() != 2:
        raise ValueError(f"{name} must be 2-D: (n_cells, Q) or (Q, n_cells)")
    if t.shape[1] == q and t.stride() == (1, t.shape[0]):
        return t.shape[0]
    if t.shape[0] == q and t.stride() == (t.shape[1], 1):
        return t.shape[1]
    raise ValueError(f"{name} must hold element (c, i) at c + i * n_cells (shape {tuple(t.shape)}, "
                     f"strides {t.stride()}); allocate it with pdf_list()")


def _store_name(dtype) -> str:
    if dtype == torch.float64:
        return "float64"
    if dtype == torch.float32:
        return "float32"
    raise ValueError("sparse PDF lists are FP64 or FP32")


def _field_name(f, default):
    if f is None:
        return default
    return f if isinstance(f, str) else getattr(f, "name", default)


class SymbolicList:
    """What ``create_symbolic_list`` describes: a named list of num_cells x values_per_cell values
    (sparse/update_rule_sparse.py:9-19).  ``allocate()`` creates the matching CUDA tensor: the SoA
    layout puts value i of cell c at c + i * num_cells (the layout the sparse kernels read)."""

    def __init__(self, name, num_cells, values_per_cell, dtype, layout):
        self.name, self.num_cells, self.values_per_cell = name, num_cells, values_per_cell
        self.dtype, self.layout = dtype, layout

    def allocate(self, device="cuda") -> torch.Tensor:
        if isinstance(self.dtype, torch.dtype):
            dt = self.dtype
        else:
            dt = {"float64": torch.float64, "float32": torch.float32, "uint32": torch.int32,
                  "int32": torch.int32}.get(str(np.dtype(self.dtype)))
            if dt is None:
                raise ValueError(f"unsupported list dtype {self.dtype}")
        if self.values_per_cell == 1:
            return torch.zeros(self.num_cells, dtype=dt, device=device)
        if self.layout == "SoA":
            return torch.zeros((self.values_per_cell, self.num_cells), dtype=dt, device=device).t()
        return torch.zeros((self.num_cells, self.values_per_cell), dtype=dt, device=device)


def create_symbolic_list(name, num_cells, values_per_cell, dtype, layout="AoS"):
    assert layout in ("AoS", "SoA")
    return SymbolicList(name, num_cells, values_per_cell, dtype, layout)


# ---------------------------------------------------------------------------- kernels
class SparseUpdateRule:
    """Collision rule bound to list fields (sparse/update_rule_sparse.py:22-52)."""

    streaming_pattern = "pull"

    def __init__(self, collision_rule, src, dst, idx, kernel_type):
        self.collision_rule = collision_rule
        self.src_name = _field_name(src, "f")
        self.dst_name = _field_name(dst, "d")
        self.idx_name = _field_name(idx, "idx")
        self.kernel_type = kernel_type
        self.storage_dtype = "float64"

    @property
    def method(self):
        return self.collision_rule.method


def create_lb_update_rule_sparse(collision_rule, src, dst, idx, kernel_type="stream_pull_collide"):
    """lbmpy's sparse update rule.  Built: 'stream_pull_collide' (the sweep); 'collide_only' and
    'stream_pull_only' raise NotImplementedError."""
    assert kernel_type in ("stream_pull_collide", "collide_only", "stream_pull_only")
    if kernel_type != "stream_pull_collide":
        raise NotImplementedError(f"the sparse sweep is built as 'stream_pull_collide', not {kernel_type!r}")
    m = collision_rule.method
    if m.stencil.name not in ("D3Q19", "D3Q27"):
        raise NotImplementedError("sparse sweeps are built for D3Q19 and D3Q27")
    if collision_rule.closure is not None:
        raise NotImplementedError("the learned closure is not built for sparse domains")
    return SparseUpdateRule(collision_rule, src, dst, idx, kernel_type)


class _SparsePlans:
    def __init__(self, rule, rates_needed=True):
        self.rule = rule
        self._plans = {}
        self.rates_needed = rates_needed

    def plan(self, storage: str, params) -> N.Plan:
        self.rule.storage_dtype = storage
        desc = build_desc(self.rule, (1, 1, 1), (False, False, False), params or {},
                          rates_needed=self.rates_needed)
        key = (storage, torch.cuda.current_device())
        p = self._plans.get(key)
        if p is None:
            p = N.Plan(desc)
            self._plans[key] = p
        elif bytes(p.desc) != bytes(desc):
            p.update(desc)
        return p


class SparseLbKernel:
    """``kernel(f=pdfs, d=pdfs_tmp, idx=index, <rate symbols>=..., stream=None)``: one
    stream-pull-collide sweep of the fluid cells from list f into list d.  `idx` is the index
    array of ``SparseLbMapper.create_index_array`` (numpy or a CUDA tensor, either orientation);
    the number of fluid cells is its length.  Boundary cells of d are not written."""

    def __init__(self, update_rule: SparseUpdateRule):
        self.update_rule = update_rule
        self.method = update_rule.method
        self.parameters = free_parameters(update_rule)
        self._plans = _SparsePlans(update_rule)
        self._idx_cache = (None, None)

    def _index(self, idx, q) -> Tuple[torch.Tensor, int]:
        if self._idx_cache[0] is idx:
            return self._idx_cache[1]
        if isinstance(idx, np.ndarray):
            a = np.asarray(idx)
            if a.ndim != 2 or q - 1 not in a.shape:
                raise ValueError(f"index array must be (n_fluid, {q - 1})")
            if a.shape[1] != q - 1:
                a = a.T
            soa = np.ascontiguousarray(a.T.astype(np.uint32))
            n_fluid = a.shape[0]
            t = torch.from_numpy(soa.view(np.int32)).cuda()
        else:
            t = idx
            if t.dim() != 2 or q - 1 not in t.shape:
                raise ValueError(f"index tensor must be (n_fluid, {q - 1})")
            if t.shape[1] == q - 1 and t.shape[0] != q - 1:
                n_fluid = t.shape[0]
                t = t.t()
            else:
                n_fluid = t.shape[1]
            t = t.contiguous()
            if t.dtype not in (torch.int32, torch.uint32):
                raise ValueError("index tensor must be 32-bit")
        res = (t, n_fluid)
        self._idx_cache = (idx, res)
        return res

    def __call__(self, **kwargs):
        ur = self.update_rule
        q = self.method.stencil.Q
        src = kwargs.pop(ur.src_name, None)
        dst = kwargs.pop(ur.dst_name, None)
        idx = kwargs.pop(ur.idx_name, None)
        if src is None or dst is None or idx is None:
            raise ValueError(f"the sparse kernel needs {ur.src_name}=, {ur.dst_name}= and {ur.idx_name}=")
        stream = kwargs.pop("stream", None)
        unknown = set(kwargs) - self.parameters
        if unknown:
            raise ValueError(f"unknown kernel arguments {sorted(unknown)}; parameters are {sorted(self.parameters)}")
        n_cells = _check_list(src, q, ur.src_name)
        if _check_list(dst, q, ur.dst_name) != n_cells or dst.dtype != src.dtype:
            raise ValueError("src and dst lists must match in length and dtype")
        index, n_fluid = self._index(idx, q)
        if index.device != src.device:
            raise ValueError("index and PDF lists must be on the same device")
        plan = self._plans.plan(_store_name(src.dtype), kwargs)
        N.check(N.lib().lbm_sparse_sweep(plan.handle, ctypes.c_void_p(src.data_ptr()),
                                         ctypes.c_void_p(dst.data_ptr()), ctypes.c_void_p(index.data_ptr()),
                                         int(n_fluid), int(n_cells), ctypes.c_void_p(_stream_handle(stream))),
                "lbm_sparse_sweep")


def create_lb_function_sparse(update_rule: SparseUpdateRule) -> SparseLbKernel:
    """The compiled kernel of a sparse update rule (lbmpy compiles it with pystencils)."""
    return SparseLbKernel(update_rule)


class _MacroRule:
    def __init__(self, method):
        from .creationfunctions import LbmCollisionRule
        self.collision_rule = LbmCollisionRule(method)
        self.storage_dtype = "float64"
        self.streaming_pattern = "pull"


class SparseSetter:
    """``setter(pdfs, density=..., velocity=..., num_fluid_cells=None)``: equilibrium of the
    fluid cells (the first num_fluid_cells list cells, by default all).  density: a number or a
    per-cell array; velocity: a 3-vector or a (num_fluid_cells, 3) array."""

    def __init__(self, method, pdfs, density, velocity):
        self.method = method
        self.pdfs_name = _field_name(pdfs, "f")
        self.density = density
        self.velocity = velocity
        self._plans = _SparsePlans(_MacroRule(method), rates_needed=False)

    def __call__(self, pdfs=None, density=None, velocity=None, num_fluid_cells=None, stream=None, **kwargs):
        pdfs = kwargs.pop(self.pdfs_name, pdfs)
        q = self.method.stencil.Q
        n_cells = _check_list(pdfs, q, self.pdfs_name)
        n = n_cells if num_fluid_cells is None else int(num_fluid_cells)
        dens = self.density if density is None else density
        vel = self.velocity if velocity is None else velocity
        dev = pdfs.device
        rho = torch.as_tensor(np.array(np.broadcast_to(np.asarray(1.0 if dens is True else dens, dtype=np.float64),
                                                       (n,))), device=dev)
        v = np.asarray((0.0, 0.0, 0.0) if vel is True else vel, dtype=np.float64)
        u = torch.as_tensor(np.ascontiguousarray(np.broadcast_to(v, (n, 3)).T), device=dev)
        plan = self._plans.plan(_store_name(pdfs.dtype), {})
        N.check(N.lib().lbm_sparse_set_equilibrium(plan.handle, ctypes.c_void_p(pdfs.data_ptr()),
                                                   ctypes.c_void_p(rho.data_ptr()), ctypes.c_void_p(u.data_ptr()),
                                                   n, n_cells, ctypes.c_void_p(_stream_handle(stream))),
                "lbm_sparse_set_equilibrium")
        if stream is not None:   # rho / u are freed on return: let a side-stream launch finish first
            torch.cuda.synchronize(dev)


def create_macroscopic_value_setter_sparse(method, pdfs, density, velocity) -> SparseSetter:
    return SparseSetter(method, pdfs, density, velocity)


class SparseGetter:
    """``getter(pdfs, num_fluid_cells=None)`` -> dict with 'density' (n,) and 'velocity' (n, 3)
    FP64 CUDA tensors for the quantities of the output descriptor; a tensor given in the descriptor
    (``{'velocity': u}``) is filled in place."""

    def __init__(self, method, pdfs, output_descriptor):
        self.method = method
        self.pdfs_name = _field_name(pdfs, "f")
        self.outputs = dict(output_descriptor)
        bad = set(self.outputs) - {"density", "velocity"}
        if bad:
            raise NotImplementedError(f"sparse getters are built for density and velocity, not {sorted(bad)}")
        self._plans = _SparsePlans(_MacroRule(method), rates_needed=False)

    def __call__(self, pdfs=None, num_fluid_cells=None, stream=None, **kwargs):
        pdfs = kwargs.pop(self.pdfs_name, pdfs)
        q = self.method.stencil.Q
        n_cells = _check_list(pdfs, q, self.pdfs_name)
        n = n_cells if num_fluid_cells is None else int(num_fluid_cells)
        dev = pdfs.device
        rho = torch.empty(n, dtype=torch.float64, device=dev) if "density" in self.outputs else None
        u = torch.empty((3, n), dtype=torch.float64, device=dev) if "velocity" in self.outputs else None
        plan = self._plans.plan(_store_name(pdfs.dtype), {})
        N.check(N.lib().lbm_sparse_get_macroscopic(plan.handle, ctypes.c_void_p(pdfs.data_ptr()),
                                                   ctypes.c_void_p(rho.data_ptr() if rho is not None else None),
                                                   ctypes.c_void_p(u.data_ptr() if u is not None else None),
                                                   n, n_cells, ctypes.c_void_p(_stream_handle(stream))),
                "lbm_sparse_get_macroscopic")
        out = {}
        for name, val in (("density", rho), ("velocity", None if u is None else u.t())):
            if val is None:
                continue
            tgt = self.outputs[name]
            if isinstance(tgt, torch.Tensor):
                tgt.copy_(val.reshape(tgt.shape))
                val = tgt
            elif isinstance(tgt, np.ndarray):
                tgt[...] = val.cpu().numpy().reshape(tgt.shape)
                val = tgt
            out[name] = val
        return out


def create_macroscopic_value_getter_sparse(method, pdfs, output_descriptor) -> SparseGetter:
    return SparseGetter(method, pdfs, output_descriptor)


# ---------------------------------------------------------------------------- boundaries
class SparseLbBoundaryMapper:
    """A boundary condition on a sparse list (sparse/mapping.py:157-247): ``create_index_arr``
    lists the links from fluid cells into cells flagged `boundary_mask` (fields 'dir', 'nidx0'
    the fluid cell, 'nidx1' the boundary cell, list indices), and calling the mapper with
    ``f=pdfs, indexField=links`` writes the boundary's incoming values into the boundary cells'
    slots, before the sweep pulls them.  Built for UBB with a constant velocity."""

    def __init__(self, boundary, method, pdf_field_sparse=None):
        from .boundaries import UBB
        if not isinstance(boundary, UBB) or boundary.velocity_is_callable:
            raise NotImplementedError("sparse boundary mappers are built for UBB with a constant velocity")
        if getattr(boundary, "density", None) or getattr(boundary, "adapt_velocity_to_force", False):
            raise NotImplementedError("sparse UBB takes neither a wall density nor the force adaptation")
        self.boundary = boundary
        self.method = method
        self.pdfs_name = _field_name(pdf_field_sparse, "f")
        self.index_field_dtype = np.dtype([("dir", np.uint32), ("nidx0", np.uint32), ("nidx1", np.uint32)])
        self._plans = _SparsePlans(_MacroRule(method), rates_needed=False)
        self._dev_links = (None, None)

    def create_index_arr(self, mapping: SparseLbMapper, boundary_mask, nr_of_ghost_layers=1):
        dirs = _dirs(self.method.stencil)
        len(mapping)                                   # assembles the cell list
        fl = mapping.flag_array
        g = nr_of_ghost_layers
        inner = tuple(slice(g, s - g) for s in fl.shape)
        fluid = (fl & mapping.fluid_flag) != 0
        out = []
        coords = np.argwhere(fluid[inner]) + g
        for d, c in enumerate(dirs):
            if d == 0:
                continue
            nb = coords + np.array(c)
            hit = (fl[tuple(nb.T)] & boundary_mask) != 0
            if not hit.any():
                continue
            rec = np.empty(int(hit.sum()), dtype=self.index_field_dtype)
            rec["dir"] = d
            cc = coords[hit]
            rec["nidx0"] = mapping._lookup[tuple(cc.T)]
            rec["nidx1"] = mapping._lookup[tuple(nb[hit].T)]
            out.append(rec)
        res = np.concatenate(out) if out else np.empty(0, dtype=self.index_field_dtype)
        if np.any(res["nidx0"] == NOT_FOUND) or np.any(res["nidx1"] == NOT_FOUND):
            raise ValueError("a boundary link reaches a cell that is not in the list")
        return res

    def __call__(self, f=None, indexField=None, stream=None, **kwargs):
        pdfs = kwargs.pop(self.pdfs_name, f)
        if pdfs is None or indexField is None:
            raise ValueError("the sparse boundary kernel needs the PDF list and indexField=")
        q = self.method.stencil.Q
        n_cells = _check_list(pdfs, q, self.pdfs_name)
        if self._dev_links[0] is indexField:
            links = self._dev_links[1]
        else:
            soa = np.stack([indexField["dir"], indexField["nidx0"], indexField["nidx1"]]).astype(np.uint32)
            links = torch.from_numpy(np.ascontiguousarray(soa).view(np.int32)).to(pdfs.device)
            self._dev_links = (indexField, links)
        plan = self._plans.plan(_store_name(pdfs.dtype), {})
        vel = (ctypes.c_double * 3)(*[float(v) for v in (list(self.boundary.velocity) + [0.0] * 3)[:3]])
        N.check(N.lib().lbm_sparse_ubb(plan.handle, ctypes.c_void_p(pdfs.data_ptr()),
                                       ctypes.c_void_p(links.data_ptr()), int(links.shape[1]), int(n_cells), vel,
                                       ctypes.c_void_p(_stream_handle(stream))), "lbm_sparse_ubb")


__all__ = ["SparseLbMapper", "SparseLbBoundaryMapper", "create_lb_update_rule_sparse", "create_lb_function_sparse",
           "create_macroscopic_value_setter_sparse", "create_macroscopic_value_getter_sparse",
           "create_symbolic_list", "pdf_list"]
