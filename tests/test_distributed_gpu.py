"""DistributedLatticeBoltzmannStep driving the CUDA sweep: two ranks as two processes on one GPU
(gloo, the packed ghost planes staged through host memory; the sweeps of the two processes never
wait on one another, the exchange is host-side), pull and AA, periodic and walled z.  The slabs
reproduce one LatticeBoltzmannStep over the whole domain."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

N = (16, 12, 20)
STEPS = 14
KW = dict(relaxation_rate=1.9, compressible=True, galilean_correction=True, force=(1e-5, 0, 0))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _initial():
    rng = np.random.default_rng(4)
    return 1 + 1e-3 * rng.uniform(-1, 1, N), 0.03 * rng.uniform(-1, 1, N + (3,))


def _step_kwargs(pattern):
    import lbmpy_b200 as L
    return dict(stencil=L.Stencil.D3Q27, method=L.Method.CUMULANT, streaming_pattern=pattern,
                config=L.CreateKernelConfig(data_type="float64"), **KW)


def _worker(rank, world, port, pattern, periodic_z, overlap, queue):
    os.environ["LBM_B200_PAIR"] = "0"
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from lbmpy_b200.boundaries import NoSlip, slice_from_direction
        from lbmpy_b200.distributed import DistributedLatticeBoltzmannStep
        step = DistributedLatticeBoltzmannStep(N, periodicity=(True, True, periodic_z), overlap=overlap,
                                               **_step_kwargs(pattern))
        if not periodic_z:
            if rank == 0:
                step.local.boundary_handling.set_boundary(NoSlip(), slice_from_direction("B", 3))
            if rank == world - 1:
                step.local.boundary_handling.set_boundary(NoSlip(), slice_from_direction("T", 3))
        rho, u = _initial()
        step.set_pdf_fields_from_macroscopic_values(rho, u)
        step.run(STEPS)
        assert step.local.sweep_status() == 0
        assert (step._split is not None) == (overlap and pattern == "pull")
        queue.put((rank, step.local.velocity_array.copy(), step.local.density_array.copy(),
                   step.reduce_conserved()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("pattern,overlap", [("pull", True), ("pull", False), ("aa", True)])
@pytest.mark.parametrize("periodic_z", [True, False])
def test_slabs_on_the_cuda_sweep_reproduce_one_domain(cuda, pattern, overlap, periodic_z, monkeypatch):
    """overlap: the pull step sweeps the boundary planes, exchanges them on a second stream and
    sweeps the interior planes meanwhile (AA ignores it)."""
    world = 2
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, pattern, periodic_z, overlap, queue))
             for r in range(world)]
    for p in procs:
        p.start()
    parts = {}
    for _ in range(world):
        r, u, rho, red = queue.get(timeout=300)
        parts[r] = (u, rho, red)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    monkeypatch.setenv("LBM_B200_PAIR", "0")
    import lbmpy_b200 as L
    from lbmpy_b200.boundaries import NoSlip, slice_from_direction
    ref = L.LatticeBoltzmannStep(domain_size=N, periodicity=(True, True, periodic_z), **_step_kwargs(pattern))
    if not periodic_z:
        ref.boundary_handling.set_boundary(NoSlip(), slice_from_direction("B", 3))
        ref.boundary_handling.set_boundary(NoSlip(), slice_from_direction("T", 3))
    rho, u = _initial()
    ref.density_array[...] = rho
    ref.velocity_array[...] = u
    ref.set_pdf_fields_from_macroscopic_values()
    ref.run(STEPS)
    got_u = np.concatenate([parts[r][0] for r in range(world)], axis=2)
    got_rho = np.concatenate([parts[r][1] for r in range(world)], axis=2)
    assert np.abs(got_u - ref.velocity_array).max() < 1e-14
    assert np.abs(got_rho - ref.density_array).max() < 1e-13
    red = ref.reduce_conserved()
    np.testing.assert_allclose(parts[0][2], red, rtol=1e-12, atol=1e-15)
