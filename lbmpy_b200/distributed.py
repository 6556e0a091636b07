"""Slab decomposition of one lattice Boltzmann domain along z over torch.distributed ranks.

lbmpy itself runs on one process; its multi-GPU runs go through waLBerla, whose ghost-layer
exchange lbmpy describes with ``get_communication_slices``
(``advanced_streaming/communication.py:122-183``): after every step, the populations that will
stream across a block face are copied into the neighbour's ghost layer.  Here every rank owns a
slab of z-planes (one process per GPU), sweeps it with the fused kernel (z non-periodic locally,
so the kernel pulls from the z ghost planes as they are), and then refreshes those ghost planes
from its neighbours: the plane below receives the populations with c_z = +1 of the neighbour's
top interior plane, the plane above those with c_z = -1 of the neighbour's bottom plane (5 of 19
slots for D3Q19, 9 of 27 for D3Q27).  The exchange is one batch of point-to-point sends and
receives (NCCL on GPUs; gloo through host memory); with a periodic z axis the first and the last
rank are neighbours.  The pull pattern exchanges after every step; the in-place AA pattern before
and after every odd step (its even step stays inside each cell), as lbmpy's AA communication
slices do (advanced_streaming/communication.py:21-121).
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch
import torch.distributed as dist


def slab_bounds(nz: int, world: int, rank: int) -> Tuple[int, int]:
    """[z0, z1) of rank's slab; slabs differ in size by at most one plane."""
    base, rem = divmod(nz, world)
    z0 = rank * base + min(rank, rem)
    return z0, z0 + base + (1 if rank < rem else 0)


def halo_slots(directions: Sequence[Sequence[int]], cz: int) -> List[int]:
    """Slots whose velocity has z component cz."""
    return [i for i, d in enumerate(directions) if d[2] == cz]


class HaloExchange:
    """Refreshes the z ghost planes of a slab field (shape (X+2, Y+2, Zl+2, Q), x fastest).

    CUDA fields pack and unpack with one launch each (``lbm_halo_copy``: every plane of an
    exchange in one grid) into cached device buffers; NCCL moves the buffers.  Under gloo the
    packed buffers travel through host memory.  CPU fields (the oracle-driven tests) pack with
    torch indexing.  Pull: ``exchange`` after every step.  AA: ``before_odd`` and ``after_odd``
    around every odd step (the even step stays inside each cell)."""

    def __init__(self, directions, periodic_z: bool, group=None):
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.up_slots = halo_slots(directions, +1)        # c_z = +1: stream into the plane above
        self.down_slots = halo_slots(directions, -1)
        self.q = len(directions)
        r, w = self.rank, self.world
        self.below = (r - 1) % w if (periodic_z or r > 0) else None
        self.above = (r + 1) % w if (periodic_z or r < w - 1) else None
        self._staged = dist.get_backend(group) != "nccl"
        self._bufs = {}

    # -- buffers and packing ---------------------------------------------------------------
    def _buf(self, key, shape, like: torch.Tensor, host=False):
        k = (key, tuple(shape), like.dtype, "cpu" if host else str(like.device))
        b = self._bufs.get(k)
        if b is None:
            b = torch.empty(shape, dtype=like.dtype, device="cpu" if host else like.device,
                            pin_memory=bool(host and like.is_cuda))
            self._bufs[k] = b
        return b

    def _copy(self, pdfs: torch.Tensor, jobs, unpack: bool):
        """jobs: [(z, slots, buffer)]; buffer element (k, y, x) <-> pdfs[x, y, z, slots[k]]."""
        if not jobs:
            return
        if not pdfs.is_cuda:
            for z, slots, buf in jobs:
                idx = torch.tensor(slots, dtype=torch.long)
                plane = pdfs[:, :, z]
                if unpack:
                    plane.index_copy_(-1, idx, buf.permute(2, 1, 0))
                else:
                    buf.copy_(plane.index_select(-1, idx).permute(2, 1, 0))
            return
        import ctypes
        from . import _native as N
        arr = (N.LbmHaloJob * len(jobs))()
        for k, (z, slots, buf) in enumerate(jobs):
            arr[k].z = int(z)
            arr[k].unpack = int(unpack)
            arr[k].n_slots = len(slots)
            for j, sl in enumerate(slots):
                arr[k].slots[j] = int(sl)
            arr[k].buffer = buf.data_ptr()
        st = pdfs.stride()
        N.check(N.lib().lbm_halo_copy(ctypes.c_void_p(pdfs.data_ptr()), N.i64_array(st), self.q, pdfs.shape[0],
                                      pdfs.shape[1], pdfs.shape[2], pdfs.element_size(), arr, len(jobs),
                                      ctypes.c_void_p(torch.cuda.current_stream(pdfs.device).cuda_stream)),
                "lbm_halo_copy")

    def _run(self, pdfs: torch.Tensor, sends, recvs):
        """sends: [(peer, z, slots, tag)] packed from pdfs; recvs: [(peer, z, slots, tag)]
        unpacked into pdfs.  Upward messages carry tag 0, downward tag 1: with two ranks (or a
        periodic pair) both go to the same peer, and NCCL pairs sends and receives between two
        ranks in the order they are posted, which is the same on both sides."""
        if not sends and not recvs:
            return
        shape = lambda slots: (len(slots), pdfs.shape[1], pdfs.shape[0])
        sbufs = [self._buf(("s", tag), shape(slots), pdfs) for _, _, slots, tag in sends]
        rbufs = [self._buf(("r", tag), shape(slots), pdfs) for _, _, slots, tag in recvs]
        self._copy(pdfs, [(z, slots, b) for (_, z, slots, _), b in zip(sends, sbufs)], unpack=False)
        glob = (lambda r: dist.get_global_rank(self.group, r)) if self.group is not None else (lambda r: r)
        stage = self._staged and pdfs.is_cuda
        if stage:
            hs = [self._buf(("hs", tag), b.shape, pdfs, host=True) for (_, _, _, tag), b in zip(sends, sbufs)]
            hr = [self._buf(("hr", tag), b.shape, pdfs, host=True) for (_, _, _, tag), b in zip(recvs, rbufs)]
            for h, b in zip(hs, sbufs):
                h.copy_(b)
            txs, rxs = hs, hr
        else:
            txs, rxs = sbufs, rbufs
        ops = []
        for tag in (0, 1):
            for (peer, _, _, t), b in zip(sends, txs):
                if t == tag:
                    ops.append(dist.P2POp(dist.isend, b, glob(peer), self.group, tag=tag))
            for (peer, _, _, t), b in zip(recvs, rxs):
                if t == tag:
                    ops.append(dist.P2POp(dist.irecv, b, glob(peer), self.group, tag=tag))
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        if stage:
            for b, h in zip(rbufs, hr):
                b.copy_(h, non_blocking=False)
        self._copy(pdfs, [(z, slots, b) for (_, z, slots, _), b in zip(recvs, rbufs)], unpack=True)

    # -- exchanges -------------------------------------------------------------------------
    def exchange(self, pdfs: torch.Tensor):
        """Pull, after a step: the top interior plane's c_z = +1 populations go to the plane
        below the upper neighbour, the bottom plane's c_z = -1 populations to the plane above the
        lower neighbour."""
        zl = pdfs.shape[2] - 2
        sends, recvs = [], []
        if self.above is not None:
            sends.append((self.above, zl, self.up_slots, 0))
            recvs.append((self.above, zl + 1, self.down_slots, 1))
        if self.below is not None:
            recvs.append((self.below, 0, self.up_slots, 0))
            sends.append((self.below, 1, self.down_slots, 1))
        self._run(pdfs, sends, recvs)

    def before_odd(self, pdfs: torch.Tensor):
        """AA, before an odd step: the odd step of a cell in the top plane reads the c_z = +1 slots
        of the cell above it, which the upper neighbour's bottom plane holds (and the bottom plane
        the c_z = -1 slots of the lower neighbour's top plane)."""
        zl = pdfs.shape[2] - 2
        sends, recvs = [], []
        if self.above is not None:
            sends.append((self.above, zl, self.down_slots, 0))
            recvs.append((self.above, zl + 1, self.up_slots, 1))
        if self.below is not None:
            recvs.append((self.below, 0, self.down_slots, 0))
            sends.append((self.below, 1, self.up_slots, 1))
        self._run(pdfs, sends, recvs)

    def after_odd(self, pdfs: torch.Tensor):
        """AA, after an odd step (and after the setter, which writes as an odd step does): the top
        plane's cells wrote their c_z = +1 populations into the ghost plane above; they belong to
        the upper neighbour's bottom plane (and the ghost plane below's c_z = -1 slots to the
        lower neighbour's top plane)."""
        zl = pdfs.shape[2] - 2
        sends, recvs = [], []
        if self.above is not None:
            sends.append((self.above, zl + 1, self.up_slots, 0))
            recvs.append((self.above, zl, self.down_slots, 1))
        if self.below is not None:
            recvs.append((self.below, 1, self.up_slots, 0))
            sends.append((self.below, 0, self.down_slots, 1))
        self._run(pdfs, sends, recvs)

    def bytes_per_exchange(self, pdfs: torch.Tensor) -> int:
        """Bytes this rank sends per exchange."""
        per = pdfs.shape[0] * pdfs.shape[1] * pdfs.element_size()
        return per * ((len(self.up_slots) if self.above is not None else 0) +
                      (len(self.down_slots) if self.below is not None else 0))


class DistributedLatticeBoltzmannStep:
    """A LatticeBoltzmannStep over a z-slab of a global domain, one rank per GPU.

    Takes LatticeBoltzmannStep's method arguments; `domain_size` and `periodicity` are global.
    Boundaries may be set on the local step's handling (`local.boundary_handling`) with slices of
    the local slab; global z walls belong to the first ('B') and last ('T') rank.  With the pull
    pattern on CUDA fields (`overlap=True`) each step sweeps the two boundary planes first and
    exchanges their values on a second stream while the interior planes sweep."""

    def __init__(self, domain_size, periodicity=False, group=None, device=None, overlap=True, **kwargs):
        from .lbstep import LatticeBoltzmannStep
        if isinstance(periodicity, bool):
            periodicity = (periodicity,) * 3
        self.global_size = tuple(int(s) for s in domain_size)
        self.periodicity = tuple(bool(p) for p in periodicity)
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        nz = self.global_size[2]
        if nz < self.world:
            raise ValueError(f"{nz} z-planes cannot be split over {self.world} ranks")
        self.z0, self.z1 = slab_bounds(nz, self.world, self.rank)
        local_size = (self.global_size[0], self.global_size[1], self.z1 - self.z0)
        local_periodic = (self.periodicity[0], self.periodicity[1], self.periodicity[2] and self.world == 1)
        self.local = LatticeBoltzmannStep(domain_size=local_size, periodicity=local_periodic,
                                          device=device or "cuda", **kwargs)
        if self.local.streaming_pattern not in ("pull", "aa"):
            raise NotImplementedError("the slab decomposition supports the pull and AA patterns")
        self._aa = self.local.streaming_pattern == "aa"
        self.halo = HaloExchange(self.local.method.stencil.stencil_entries, self.periodicity[2], group) \
            if self.world > 1 else None
        self.time_steps_run = 0
        self.overlap = bool(overlap)
        self._split = None          # (key, [(byte offset, BoundSweep) of bottom, top, interior])
        self._comm = None

    def slab(self, a):
        """This rank's z-range of a global interior-shaped array."""
        return a[:, :, self.z0:self.z1]

    def set_pdf_fields_from_macroscopic_values(self, density=None, velocity=None):
        """Equilibrium from global density / velocity arrays (numpy, interior shape)."""
        if velocity is not None:
            self.local.velocity_array[...] = self.slab(np.asarray(velocity))
        if density is not None:
            self.local.density_array[...] = self.slab(np.asarray(density))
        self.local.set_pdf_fields_from_macroscopic_values()
        self._exchange()

    def _exchange(self):
        if self.halo is None:
            return
        if self._aa:
            # the setter and every odd step leave populations in the z ghost planes
            if self.local.previous_timestep.idx == 1:
                self.halo.after_odd(self.local.pdfs)
        else:
            self.halo.exchange(self.local.pdfs)

    def _overlap_sweeps(self):
        """Pull with the exchange overlapped: sweeps of the bottom plane, the top plane and the
        interior planes of the slab, each bound to a view of the field whose ghost planes are the
        neighbouring planes (None where the split does not apply: AA, one rank, slabs thinner
        than three planes, CPU fields, per-link boundary tables)."""
        loc = self.local
        zl = loc.pdfs.shape[2] - 2
        bh = loc.boundary_handling
        if (not self.overlap or self._aa or self.halo is None or zl < 3 or not loc.pdfs.is_cuda
                or getattr(bh, "_link_objs", None) or any(u.velocity_is_callable for u in getattr(bh, "_ubbs", []))):
            return None
        whole = loc._bound()
        if self._split is not None and self._split[0] is whole:
            return self._split[1]
        k = loc._kernels[0]
        flags = loc._flags(k)
        per = (loc.periodicity[0], loc.periodicity[1], False)
        parts = []
        for z0, nz in ((0, 1), (zl - 1, 1), (1, zl - 2)):    # interior planes [z0, z0 + nz)
            view = loc.pdfs[:, :, z0:z0 + nz + 2]
            fl = flags[:, :, z0:z0 + nz + 2] if flags is not None else None
            b = k.bind(view, per, fl, bh.ubb_velocities, loc.kernel_params, fixed_density=bh.fixed_density,
                       ubb_options=bh.ubb_options)
            parts.append((z0 * view.stride(2) * view.element_size(), b))
        self._split = (whole, parts)
        return parts

    def time_step(self):
        parts = self._overlap_sweeps()
        if parts is not None:
            # the two boundary planes first; the exchange of their new values runs on a second
            # stream while the interior planes sweep (disjoint planes of the destination field)
            loc = self.local
            src, dst = loc.pdfs, loc.pdfs_tmp
            main = torch.cuda.current_stream(src.device)
            if self._comm is None:
                self._comm = torch.cuda.Stream(device=src.device)
            for off, b in parts[:2]:
                b.sweep(src.data_ptr() + off, dst.data_ptr() + off, 0)
            ready = torch.cuda.Event()
            ready.record(main)
            off, b = parts[2]
            b.sweep(src.data_ptr() + off, dst.data_ptr() + off, 0)
            with torch.cuda.stream(self._comm):
                self._comm.wait_event(ready)
                self.halo.exchange(dst)
                done = torch.cuda.Event()
                done.record(self._comm)
            main.wait_event(done)
            loc.pdfs, loc.pdfs_tmp = dst, src
            loc.time_steps_run += 1
            self.time_steps_run += 1
            return
        odd = self._aa and self.local.previous_timestep.next().idx == 1
        if odd and self.halo is not None:
            self.halo.before_odd(self.local.pdfs)
        self.local.time_step()
        self._exchange()
        self.time_steps_run += 1

    def run(self, steps: int):
        for _ in range(int(steps)):
            self.time_step()
        self.local.post_run()

    def reduce_conserved(self) -> np.ndarray:
        """Global FP64 [mass, momentum x/y/z, kinetic energy] (an all-reduce over ranks)."""
        red = torch.tensor(self.local.reduce_conserved(), dtype=torch.float64,
                           device=self.local.pdfs.device if dist.get_backend(self.group) == "nccl" else "cpu")
        if self.world > 1:
            dist.all_reduce(red, group=self.group)
        return red.cpu().numpy()
