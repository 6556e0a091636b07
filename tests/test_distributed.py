"""Slab decomposition along z on CPU ranks (gloo): the halo exchange of lbmpy_b200.distributed
around the oracle's sweep must reproduce a single-domain run exactly, for periodic and walled z
and for 2 and 3 ranks.  (The GPU path runs the same exchange around the CUDA sweep with NCCL.)"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import oracle as O
from tests.helpers import random_velocity

N = (8, 6, 12)
STEPS = 12


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _initial():
    u = random_velocity(N, 0.03, seed=4)
    rho = 1 + 1e-3 * np.random.default_rng(5).uniform(-1, 1, N)
    return rho, u


def _walls(flags, bottom, top):
    if bottom:
        flags[:, :, 0] = 1
    if top:
        flags[:, :, -1] = 1


def _fold_ghost_planes(f, dirs):
    """The oracle leaves values an AA odd step (or the AA setter) writes across a periodic x / y face
    in the x / y ghost cells; in the z ghost planes of a slab its periodic sync does not move them
    (z is not periodic there).  Fold them onto their x / y images, as the CUDA sweep writes them
    in the first place, before the planes are sent."""
    nx, ny = f.shape[0] - 2, f.shape[1] - 2
    for z in (0, f.shape[2] - 1):
        for q, c in enumerate(dirs):
            if c[2] == 0:
                continue
            pl = f[:, :, z, q]
            if c[0] == -1:
                pl[nx, :] = pl[0, :]
            elif c[0] == 1:
                pl[1, :] = pl[nx + 1, :]
            if c[1] == -1:
                pl[:, ny] = pl[:, 0]
            elif c[1] == 1:
                pl[:, 1] = pl[:, ny + 1]


def _worker_aa(rank, world, port, periodic_z, queue):
    """AA in place: the exchange before and after every odd step (and after the setter)."""
    import torch.distributed as dist
    from lbmpy_b200.distributed import HaloExchange, slab_bounds
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        orc = O.make("D3Q27", "cumulant", relaxation_rate=1.9, compressible=True, galilean_correction=True,
                     force=(1e-5, 0, 0))
        rho, u = _initial()
        z0, z1 = slab_bounds(N[2], world, rank)
        local = (N[0], N[1], z1 - z0)
        f = orc.new_field(local)
        orc.set_equilibrium(f, rho[:, :, z0:z1], u[:, :, z0:z1], "aa", 1)
        flags = None
        if not periodic_z:
            flags = np.zeros((local[0] + 2, local[1] + 2, local[2] + 2), np.uint8)
            _walls(flags, rank == 0, rank == world - 1)
        halo = HaloExchange(orc.spec.dirs, periodic_z)
        xy = (1, 1, 0)
        orc.periodic_sync(f, "aa", 1, xy)
        _fold_ghost_planes(f, orc.spec.dirs)
        halo.after_odd(torch.from_numpy(f))
        prev = 1
        for _ in range(STEPS):
            if prev == 0:                        # the next step is odd
                halo.before_odd(torch.from_numpy(f))
            f, prev = orc.run(f, 1, "aa", prev, periodic=xy, flags=flags)
            orc.periodic_sync(f, "aa", prev, xy)
            if prev == 1:
                _fold_ghost_planes(f, orc.spec.dirs)
                halo.after_odd(torch.from_numpy(f))
        queue.put((rank, np.ascontiguousarray(f[1:-1, 1:-1, 1:-1])))
    finally:
        dist.destroy_process_group()


def _worker(rank, world, port, periodic_z, queue):
    import torch.distributed as dist
    from lbmpy_b200.distributed import HaloExchange, slab_bounds
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        orc = O.make("D3Q19", "trt", relaxation_rate=1.8, compressible=True, force=(1e-5, 0, 0))
        rho, u = _initial()
        z0, z1 = slab_bounds(N[2], world, rank)
        local = (N[0], N[1], z1 - z0)
        f = orc.new_field(local)
        orc.set_equilibrium(f, rho[:, :, z0:z1], u[:, :, z0:z1])
        flags = None
        if not periodic_z:
            flags = np.zeros((local[0] + 2, local[1] + 2, local[2] + 2), np.uint8)
            _walls(flags, rank == 0, rank == world - 1)
        halo = HaloExchange(orc.spec.dirs, periodic_z)
        # the oracle reads the x/y ghost cells of the z ghost planes (the CUDA sweep wraps its
        # indices instead): refresh the sender's x/y ghosts before each exchange of whole planes
        orc.periodic_sync(f, "pull", 0, (1, 1, 0))
        halo.exchange(torch.from_numpy(f))
        for _ in range(STEPS):
            f, _ = orc.run(f, 1, "pull", 0, periodic=(1, 1, 0), flags=flags)
            orc.periodic_sync(f, "pull", 0, (1, 1, 0))
            halo.exchange(torch.from_numpy(f))
        queue.put((rank, np.ascontiguousarray(f[1:-1, 1:-1, 1:-1])))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("periodic_z", [True, False])
def test_slab_decomposition_reproduces_single_domain(world, periodic_z):
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, periodic_z, queue)) for r in range(world)]
    for p in procs:
        p.start()
    parts = dict(queue.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    orc = O.make("D3Q19", "trt", relaxation_rate=1.8, compressible=True, force=(1e-5, 0, 0))
    rho, u = _initial()
    f = orc.new_field(N)
    orc.set_equilibrium(f, rho, u)
    flags = None
    if not periodic_z:
        flags = np.zeros(tuple(n + 2 for n in N), np.uint8)
        _walls(flags, True, True)
    f, _ = orc.run(f, STEPS, "pull", 0, periodic=(1, 1, periodic_z), flags=flags)
    ref = f[1:-1, 1:-1, 1:-1]
    got = np.concatenate([parts[r] for r in range(world)], axis=2)
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("periodic_z", [True, False])
def test_slab_decomposition_aa_reproduces_single_domain(world, periodic_z):
    """The in-place AA pattern across slabs (D3Q27 cumulant with force): the exchanges around the
    odd steps reproduce the single-domain run bit for bit."""
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_aa, args=(r, world, port, periodic_z, queue)) for r in range(world)]
    for p in procs:
        p.start()
    parts = dict(queue.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    orc = O.make("D3Q27", "cumulant", relaxation_rate=1.9, compressible=True, galilean_correction=True,
                 force=(1e-5, 0, 0))
    rho, u = _initial()
    f = orc.new_field(N)
    orc.set_equilibrium(f, rho, u, "aa", 1)
    per = (1, 1, int(periodic_z))
    orc.periodic_sync(f, "aa", 1, per)
    flags = None
    if not periodic_z:
        flags = np.zeros(tuple(n + 2 for n in N), np.uint8)
        _walls(flags, True, True)
    f, par = orc.run(f, STEPS, "aa", 1, periodic=per, flags=flags)
    orc.periodic_sync(f, "aa", par, per)      # the last (odd) step's writes across periodic faces
    ref = f[1:-1, 1:-1, 1:-1]
    got = np.concatenate([parts[r] for r in range(world)], axis=2)
    np.testing.assert_array_equal(got, ref)


def test_slab_bounds_cover_the_domain():
    from lbmpy_b200.distributed import halo_slots, slab_bounds
    for nz, world in ((12, 2), (13, 3), (5, 5), (100, 7)):
        b = [slab_bounds(nz, world, r) for r in range(world)]
        assert b[0][0] == 0 and b[-1][1] == nz
        assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
        assert max(z1 - z0 for z0, z1 in b) - min(z1 - z0 for z0, z1 in b) <= 1
    from lbmpy_b200 import methods as M
    assert len(halo_slots(M.WALBERLA_ORDER["D3Q19"], 1)) == 5
    assert len(halo_slots(M.WALBERLA_ORDER["D3Q27"], -1)) == 9
