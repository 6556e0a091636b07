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
receives (NCCL on GPUs, gloo on CPU tensors); with a periodic z axis the first and the last rank
are neighbours.  The pull pattern is supported.
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
    """Refreshes the z ghost planes of a slab field (shape (X+2, Y+2, Zl+2, Q), x fastest)."""

    def __init__(self, directions, periodic_z: bool, group=None):
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.up_slots = halo_slots(directions, +1)        # stream upwards: needed in the plane above
        self.down_slots = halo_slots(directions, -1)
        r, w = self.rank, self.world
        self.below = (r - 1) % w if (periodic_z or r > 0) else None
        self.above = (r + 1) % w if (periodic_z or r < w - 1) else None
        self._idx = {}

    def _index(self, slots, device):
        key = (tuple(slots), str(device))
        t = self._idx.get(key)
        if t is None:
            t = torch.tensor(slots, dtype=torch.long, device=device)
            self._idx[key] = t
        return t

    def exchange(self, pdfs: torch.Tensor):
        """Sends the top interior plane's c_z = +1 populations up and the bottom interior plane's
        c_z = -1 populations down; receives the neighbours' into the ghost planes."""
        zl = pdfs.shape[2] - 2
        up = self._index(self.up_slots, pdfs.device)
        down = self._index(self.down_slots, pdfs.device)
        ops, recv = [], []
        glob = (lambda r: dist.get_global_rank(self.group, r)) if self.group is not None else (lambda r: r)
        # Upward traffic first, then downward, with a tag per direction: with two ranks (or a
        # periodic pair) both messages go to the same peer, and NCCL pairs the sends and receives
        # between two ranks in the order they are posted.
        if self.above is not None:
            send_up = pdfs[:, :, zl].index_select(-1, up).contiguous()
            ops.append(dist.P2POp(dist.isend, send_up, glob(self.above), self.group, tag=0))
        if self.below is not None:
            buf = torch.empty((pdfs.shape[0], pdfs.shape[1], len(self.up_slots)), dtype=pdfs.dtype,
                              device=pdfs.device)
            ops.append(dist.P2POp(dist.irecv, buf, glob(self.below), self.group, tag=0))
            recv.append((0, up, buf))
        if self.below is not None:
            send_down = pdfs[:, :, 1].index_select(-1, down).contiguous()
            ops.append(dist.P2POp(dist.isend, send_down, glob(self.below), self.group, tag=1))
        if self.above is not None:
            buf = torch.empty((pdfs.shape[0], pdfs.shape[1], len(self.down_slots)), dtype=pdfs.dtype,
                              device=pdfs.device)
            ops.append(dist.P2POp(dist.irecv, buf, glob(self.above), self.group, tag=1))
            recv.append((zl + 1, down, buf))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for z, idx, buf in recv:
            plane = pdfs[:, :, z]
            plane.index_copy_(-1, idx, buf)

    def bytes_per_exchange(self, pdfs: torch.Tensor) -> int:
        """Bytes this rank sends per exchange."""
        per = pdfs.shape[0] * pdfs.shape[1] * pdfs.element_size()
        return per * ((len(self.up_slots) if self.above is not None else 0) +
                      (len(self.down_slots) if self.below is not None else 0))


class DistributedLatticeBoltzmannStep:
    """A LatticeBoltzmannStep over a z-slab of a global domain, one rank per GPU.

    Takes LatticeBoltzmannStep's method arguments; `domain_size` and `periodicity` are global.
    Boundaries may be set on the local step's handling (`local.boundary_handling`) with slices of
    the local slab; global z walls belong to the first ('B') and last ('T') rank."""

    def __init__(self, domain_size, periodicity=False, group=None, device=None, **kwargs):
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
        if self.local.streaming_pattern != "pull":
            raise NotImplementedError("the slab decomposition supports the pull pattern")
        self.halo = HaloExchange(self.local.method.stencil.stencil_entries, self.periodicity[2], group) \
            if self.world > 1 else None
        self.time_steps_run = 0

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
        if self.halo is not None:
            self.halo.exchange(self.local.pdfs)

    def time_step(self):
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
