"""Benchmark of the fused stream-collide sweep on B200.

Workload (default, one GPU): D3Q27 cumulant (Galilean-corrected, compressible), FP32, AA in-place
streaming, 256 x 128 x 128 channel with NoSlip walls on the y and z faces, periodic in x, body
force 1e-7 in x, omega = 1.95, rho = 1, velocity seeded uniform in +-1e-4.  A step is one sweep
over the whole channel.  Metric: GLUPS (giga lattice-cell updates per second).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

With torchrun (N > 1) every rank updates its own channel (replicas; the sweep has no data-path
collective), and `value` is the sum over ranks divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SHAPE = (256, 128, 128)
Q = 27
OMEGA = 1.95
FORCE = 1e-7
E2E_SWEEPS = 100          # sweeps per end-to-end call (one LatticeBoltzmannStep.run() in lbmpy terms)
FALLBACK_HBM_GBS = 6650.0
METRIC = "D3Q19/D3Q27 GLUPS and % of HBM roofline; FP16-store vs FP32 at equal L2 error"

# DRAM bytes (read + write) per sweep launch from one ncu capture of the same workload, averaged
# over the launches captured; summaries with their commands are under profiles/.
NCU_TRAFFIC_BYTES = {
    "d3q27-cumulant-aa-channel-256x128x128": 872_550_000,   # k_sweep_d3q27_cumulant_aa_channel_256x128x128.md
    "d3q19-trt-pull-float32-256": 2_548_790_000,            # k_sweep_d3q19_fp32_fp16_256.md
    "d3q19-mrt-pull-float32-256": 2_555_021_000,
    "d3q19-trt-pull-float16-256": 1_276_317_824,             # k_sweep_quad_d3q19_trt_pull_fp16_256.md
    "d3q19-trt-pull-e3m12-256": 1_273_168_384,               # k_sweep_quad_d3q19_trt_pull_e3m12_256.md
    "sparse-porous-192-d3q19-trt-float32": 996_429_312,      # k_sweep_sparse_porous_192_d3q19_trt_fp32.md
}


def algorithmic_bytes_per_sweep(cells: int, q: int = Q, itemsize: int = 4) -> int:
    """2 * Q * sizeof(PDF) per lattice update: every population read once and written once."""
    return 2 * q * itemsize * cells


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while the timed region runs."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap"}

    def __init__(self, device_index: int):
        self.idx = device_index
        self.samples = []
        self.reasons = set()
        self._stop = threading.Event()
        self._thread = None
        self.max_mhz = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:   # NVML unavailable: report no samples
            self._nv = None

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                for bit, name in self.REASONS.items():
                    if mask & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.01)

    def __enter__(self):
        if self._nv is not None:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread is not None:
            self._thread.join()

    def summary(self):
        return {"sm_mhz": float(statistics.median(self.samples)) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": len(self.samples)}


def make_d3q19_tgv(device, n, storage, seed=0, method="trt", pattern="pull"):
    """D3Q19 periodic box, Taylor-Green vortex u0 = 0.04 plus Gaussian noise 1e-3 (seeded)."""
    import lbmpy_b200 as L
    compute = "float64" if storage == "float64" else "float32"
    kw = dict(relaxation_rate=1.8) if method == "trt" else dict(relaxation_rates=[1.8, 1.6, 1.0, 1.0])
    step = L.LatticeBoltzmannStep(domain_size=(n, n, n), periodicity=True, stencil=L.Stencil.D3Q19,
                                  method=getattr(L.Method, method.upper()), compressible=True,
                                  streaming_pattern=pattern, config=L.CreateKernelConfig(data_type=compute),
                                  optimization={"storage_dtype": storage}, device=device, **kw)
    x = np.arange(n)
    k = 2 * np.pi / n
    u = np.zeros((n, n, n, 3))
    u[..., 0] = (0.04 * np.sin(k * x)[:, None] * np.cos(k * x)[None, :])[:, :, None]
    u[..., 1] = (-0.04 * np.cos(k * x)[:, None] * np.sin(k * x)[None, :])[:, :, None]
    u += 1e-3 * np.random.default_rng(seed).standard_normal(u.shape, dtype=np.float32)
    step.velocity_array[...] = u
    step.set_pdf_fields_from_macroscopic_values()
    return step


# name -> (factory(device), cells per sweep, populations per cell, bytes per stored population)
WORKLOADS = {
    "d3q27-cumulant-aa-channel-256x128x128": (lambda dev: make_channel(dev), SHAPE[0] * SHAPE[1] * SHAPE[2], 27, 4),
}
for _n in (64, 256, 512):
    for _st, _isz in (("float64", 8), ("float32", 4), ("float16", 2), ("bfloat16", 2), ("e3m12", 2)):
        WORKLOADS[f"d3q19-trt-pull-{_st}-{_n}"] = (
            (lambda dev, n=_n, st=_st: make_d3q19_tgv(dev, n, st)), _n ** 3, 19, _isz)
    WORKLOADS[f"d3q19-mrt-pull-float32-{_n}"] = (
        (lambda dev, n=_n: make_d3q19_tgv(dev, n, "float32", method="mrt")), _n ** 3, 19, 4)
    WORKLOADS[f"d3q19-trt-aa-float32-{_n}"] = (
        (lambda dev, n=_n: make_d3q19_tgv(dev, n, "float32", pattern="aa")), _n ** 3, 19, 4)


def make_cavity_batch(device, n_cavities=512, seed=0):
    """512 independent cubic lid-driven cavities (D3Q19 MRT, FP32, pull), edge seeded from
    {16, 24, ..., 96}, shear/bulk rates seeded uniform in [1.5, 1.95], lid 0.05; one
    persistent launch per step over all cavities, tiling autotuned, steps replayed from a CUDA
    graph."""
    from lbmpy_b200.batched import lid_driven_cavity_batch
    b = lid_driven_cavity_batch(n_cavities, seed=seed, device=device)
    b.finalize()
    return b


WORKLOADS["batched-ldc-512-d3q19-mrt-float32"] = (lambda dev: make_cavity_batch(dev), None, 19, 4)
WORKLOADS["batched-ldc-64-d3q19-mrt-float32"] = (lambda dev: make_cavity_batch(dev, 64), None, 19, 4)


class SparsePorousMedium:
    """A periodic n^3 box filled with seeded random spheres (radius 3-7 cells, about a third of the
    cells solid; the ghost layers mirror the solid cells of their periodic images), stored as a fluid-cell list with lbmpy's sparse layout (SparseLbMapper: NoSlip in
    the index array), D3Q19 TRT FP32, force driven; one stream-pull-collide sweep of the list per
    step (lbmpy_b200.sparse).  number_of_cells counts fluid cells."""

    def __init__(self, device, n=192, seed=0):
        import torch
        import lbmpy_b200 as L
        from lbmpy_b200 import sparse as S
        rng = np.random.default_rng(seed)
        ext = n + 2
        solid = np.zeros((ext, ext, ext), bool)
        ax = np.arange(ext)
        centres = rng.uniform(1, n + 1, (int(0.02 * n ** 3 / 27), 3))
        radii = rng.uniform(3, 7, len(centres))
        for c, r in zip(centres, radii):
            lo = np.maximum(np.floor(c - r).astype(int), 1)
            hi = np.minimum(np.ceil(c + r).astype(int) + 1, n + 1)
            X, Y, Z = np.meshgrid(ax[lo[0]:hi[0]], ax[lo[1]:hi[1]], ax[lo[2]:hi[2]], indexing="ij")
            solid[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] |= (X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 < r * r
        for a in range(3):      # ghost layers mirror their periodic images (a solid image bounces back)
            sl = [slice(None)] * 3
            src, dst = list(sl), list(sl)
            src[a], dst[a] = n, 0
            solid[tuple(dst)] = solid[tuple(src)]
            src[a], dst[a] = 1, n + 1
            solid[tuple(dst)] = solid[tuple(src)]
        flags = np.zeros((ext, ext, ext), np.uint8)
        flags[1:-1, 1:-1, 1:-1] = 1
        flags[solid] = 2
        kw = dict(relaxation_rate=1.8, compressible=False, force=(1e-6, 0, 0))
        rule = L.create_lb_collision_rule(lbm_config=L.LBMConfig(stencil=L.Stencil.D3Q19, method=L.Method.TRT, **kw))
        self.mapper = S.SparseLbMapper([tuple(d) for d in rule.method.stencil], flags, 1, 2, 0)
        idx = self.mapper.create_index_array(1)
        self.number_of_cells = self.mapper.num_fluid_cells
        self.solid_fraction = float(solid[1:-1, 1:-1, 1:-1].mean())
        self.kernel = S.create_lb_function_sparse(S.create_lb_update_rule_sparse(rule, "f", "d", "idx"))
        self.f = S.pdf_list(len(self.mapper), 19, torch.float32, device)
        self.d = S.pdf_list(len(self.mapper), 19, torch.float32, device)
        S.create_macroscopic_value_setter_sparse(rule.method, "f", 1.0, (0.0, 0.0, 0.0))(self.f)
        self.idx_host = idx

    def time_step(self):
        self.kernel(f=self.f, d=self.d, idx=self.idx_host)
        self.f, self.d = self.d, self.f


WORKLOADS["sparse-porous-192-d3q19-trt-float32"] = (lambda dev: SparsePorousMedium(dev), None, 19, 4)


def make_closure_box(device, shape=(256, 128, 128), closure=True):
    """D3Q27 cumulant (omega 1.99) with the learned closure, FP32, AA, periodic box; the network
    is a seeded untrained one (its cost does not depend on the parameter values).  closure=False:
    the same box with the plain method, the closure's cost reference."""
    import lbmpy_b200 as L
    from lbmpy_b200.closure import MLPClosure
    kw = {}
    if closure:
        kw["subgrid_scale_model"] = (L.SubgridScaleModel.LEARNED, MLPClosure(seed=0, nu_scale=3e-4, device=device))
    step = L.LatticeBoltzmannStep(domain_size=shape, periodicity=True, stencil=L.Stencil.D3Q27,
                                  method=L.Method.CUMULANT, relaxation_rate=1.99, compressible=True,
                                  streaming_pattern="aa", config=L.CreateKernelConfig(data_type="float32"),
                                  device=device, **kw)
    rng = np.random.default_rng(0)
    step.velocity_array[...] = rng.uniform(-0.02, 0.02, shape + (3,)).astype(np.float32)
    step.set_pdf_fields_from_macroscopic_values()
    return step


WORKLOADS["d3q27-cumulant-closure-aa-periodic-256x128x128"] = (lambda dev: make_closure_box(dev), None, 27, 4)
WORKLOADS["d3q27-cumulant-aa-periodic-256x128x128"] = (lambda dev: make_closure_box(dev, closure=False), None, 27, 4)
WORKLOADS["d3q27-trt-aa-channel-256x128x128"] = (lambda dev: make_channel(dev, method="trt"), SHAPE[0] * SHAPE[1] * SHAPE[2],
                                                 27, 4)


def make_channel(device, shape=SHAPE, seed=0, method="cumulant"):
    """The channel through the lbmpy-compatible API (create_channel-style set-up, AA in place).
    method "trt": the same channel with the D3Q27 TRT method instead of the cumulant one."""
    import lbmpy_b200 as L
    kw = dict(galilean_correction=True) if method == "cumulant" else {}
    step = L.LatticeBoltzmannStep(domain_size=shape, periodicity=(True, False, False), stencil=L.Stencil.D3Q27,
                                  method=getattr(L.Method, method.upper()), relaxation_rate=OMEGA, compressible=True,
                                  force=(FORCE, 0, 0), streaming_pattern="aa",
                                  config=L.CreateKernelConfig(data_type="float32"), device=device, **kw)
    for d in ("N", "S", "T", "B"):
        step.boundary_handling.set_boundary(L.NoSlip(), L.slice_from_direction(d, 3))
    rng = np.random.default_rng(seed)
    step.velocity_array[...] = rng.uniform(-1e-4, 1e-4, shape + (3,)).astype(np.float32)
    step.set_pdf_fields_from_macroscopic_values()
    return step


def _cpu_channel(dtype=np.float32):
    """The headline channel on the closed-form CPU kernel (oracle/lbm_cpu.c, lbmpy's generated-kernel
    style: fzyx, one cell per inner iteration vectorised over x, OpenMP over rows), same shape,
    method, storage type and initial state as the GPU run."""
    from oracle import cpu as C
    from oracle import oracle as O
    orc = O.make("D3Q27", "cumulant", relaxation_rate=OMEGA, compressible=True, galilean_correction=True,
                 force=(FORCE, 0, 0))
    fc = C.FastCPU("cumulant", orc, dtype=dtype)
    n = SHAPE
    f = orc.new_field(n)
    rng = np.random.default_rng(0)
    orc.set_equilibrium(f, np.ones(n), rng.uniform(-1e-4, 1e-4, n + (3,)), "aa", 0)
    g = fc.new_field(n)
    g[...] = f
    del f
    flags = np.zeros((n[0] + 2, n[1] + 2, n[2] + 2), np.uint8)
    flags[:, 0, :] = flags[:, -1, :] = flags[:, :, 0] = flags[:, :, -1] = 1
    return fc, g, flags


def _cpu_info():
    model = None
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return threads, model


def cpu_baseline_sample(seconds_budget=15.0):
    """The full 256 x 128 x 128 channel (D3Q27 cumulant AA, FP32) on the closed-form CPU kernel,
    OpenMP on every host thread: sweeps timed until about a third of the budget has passed."""
    fc, g, flags = _cpu_channel()
    par = fc.run(g, 2, 1, periodic=(1, 0, 0), flags=flags)[1]      # warm-up
    steps, t0 = 0, time.perf_counter()
    while True:
        par = fc.run(g, 2, par, periodic=(1, 0, 0), flags=flags)[1]
        steps += 2
        if time.perf_counter() - t0 > seconds_budget / 3 or steps >= 200:
            break
    dt = time.perf_counter() - t0
    cells = SHAPE[0] * SHAPE[1] * SHAPE[2]
    threads, model = _cpu_info()
    return {"value": cells * steps / dt / 1e9, "unit": "GLUPS", "cores": threads, "kind": "port",
            "cpu_model": model,
            "sample": f"{steps} sweeps of the full 256x128x128 channel (D3Q27 cumulant AA, FP32, closed-form "
                      f"OpenMP kernel vectorised over x, oracle/lbm_cpu.c)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    O.build()
    fc, g, flags = _cpu_channel()
    par = 1
    for _ in range(args.warmup):
        par = fc.run(g, 1, par, periodic=(1, 0, 0), flags=flags)[1]
    t0 = time.perf_counter()
    for _ in range(args.steps):
        par = fc.run(g, 1, par, periodic=(1, 0, 0), flags=flags)[1]
    dt = time.perf_counter() - t0
    cells = SHAPE[0] * SHAPE[1] * SHAPE[2]
    value = cells * args.steps / dt / 1e9
    threads, model = _cpu_info()
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "GLUPS",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "d3q27-cumulant-aa-channel-256x128x128", "shape": list(SHAPE),
                       "omega": OMEGA, "force": FORCE, "pattern": "aa", "galilean_correction": True,
                       "storage": "float32 zero-centred"},
            "cpu_baseline": {"value": value, "unit": "GLUPS", "cores": threads, "kind": "port",
                             "cpu_model": model,
                             "sample": "one sweep of the full 256x128x128 channel per step (closed-form "
                                       "OpenMP kernel in lbmpy's generated-kernel style, FP32, all host "
                                       "threads; lbmpy itself cannot be imported here)"},
            "e2e": {"value": value, "unit": "GLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--accuracy-steps", type=int, default=5000,
                    help="sweeps of the FP16/BF16/FP32-vs-FP64 accuracy run in `secondary` (0: skip)")
    ap.add_argument("--workload", default="d3q27-cumulant-aa-channel-256x128x128", choices=sorted(WORKLOADS))
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=device)

    from lbmpy_b200 import _native
    _native.lib()
    factory, cells, q_pop, itemsize = WORKLOADS[args.workload]
    step = factory(device)
    cells = step.number_of_cells
    headline = args.workload == "d3q27-cumulant-aa-channel-256x128x128"
    batched = args.workload.startswith("batched")
    warm = max(args.warmup, 3)
    for _ in range(warm):
        step.time_step()
    if batched:
        step.run_sweeps(args.steps)          # captures the graph of K launches that is timed below
    torch.cuda.synchronize()

    stream = torch.cuda.current_stream()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        start.record(stream)
        if batched:
            step.run_sweeps(args.steps)      # one graph replay: K persistent launches
        else:
            for _ in range(args.steps):
                step.time_step()
        stop.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = start.elapsed_time(stop)
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    ms_per_step = ms_max / args.steps
    glups = world * cells * args.steps / (ms_max * 1e-3) / 1e9

    # roofline of the sweep kernel (the only kernel in the timed region)
    peak, peak_kind = measured_peak()
    bytes_per_sweep = algorithmic_bytes_per_sweep(cells, q_pop, itemsize)
    if args.workload.startswith("sparse"):
        bytes_per_sweep += 4 * (q_pop - 1) * cells          # the pull index of every fluid cell
    achieved = bytes_per_sweep / (ms / args.steps * 1e-3) / 1e9
    traffic = NCU_TRAFFIC_BYTES.get(args.workload)

    # end to end through the public API, as an lbmpy user runs a simulation: macroscopic fields in
    # host memory -> set_pdf_fields_from_macroscopic_values() (host->device copy and the setter),
    # run(K) (K sweeps, the getter and the device->host copy of density and velocity)
    e2e = None
    if not args.no_e2e and headline:
        # the user's input: density and velocity in the step's host arrays
        step.density_array[...] = 1.0
        step.velocity_array[...] = np.random.default_rng(1).uniform(-1e-4, 1e-4, SHAPE + (3,))
        calls = 2
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(calls):
            step.set_pdf_fields_from_macroscopic_values()
            step.run(E2E_SWEEPS)
        e1.record(stream)
        torch.cuda.synchronize()
        ems = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=device)
        if world > 1:
            dist.all_reduce(ems, op=dist.ReduceOp.MAX)
        e_glups = world * cells * E2E_SWEEPS * calls / (float(ems.item()) * 1e-3) / 1e9
        fld = step.density_array.itemsize                   # the step's host fields (compute dtype)
        h2d = cells * 4 * fld                               # density and velocity in
        d2h = cells * 4 * fld                               # density and velocity out
        e2e = {"value": e_glups, "unit": "GLUPS",
               "h2d_bytes_per_step": int(h2d / E2E_SWEEPS), "d2h_bytes_per_step": int(d2h / E2E_SWEEPS),
               "sweeps_per_call": E2E_SWEEPS,
               "call": "density/velocity host arrays -> set_pdf_fields_from_macroscopic_values() -> "
                       "run(100): sweeps, getter, density/velocity device->host"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and headline:
        cpu = cpu_baseline_sample()

    secondary = None
    if headline and rank == 0 and world == 1 and not args.no_secondary:
        # FP16 / BF16 storage against FP32 on the 512^3 D3Q19 TRT periodic box (same kernel family)
        del step
        torch.cuda.empty_cache()
        secondary = {}
        for name in ("d3q19-trt-pull-float32-512", "d3q19-trt-pull-float16-512", "d3q19-trt-pull-bfloat16-512",
                     "d3q19-trt-pull-e3m12-512"):
            f2, c2, q2, i2 = WORKLOADS[name]
            st2 = f2(device)
            for _ in range(4):
                st2.time_step()
            a2, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a2.record(stream)
            st2.run_sweeps(20)
            b2.record(stream)
            torch.cuda.synchronize()
            ms2 = a2.elapsed_time(b2) / 20
            g2 = c2 / (ms2 * 1e-3) / 1e9
            secondary[name] = {"GLUPS": g2, "GB/s": g2 * 2 * q2 * i2, "frac": g2 * 2 * q2 * i2 / peak}
            del st2
            torch.cuda.empty_cache()
        secondary["fp16_over_fp32"] = (secondary["d3q19-trt-pull-float16-512"]["GLUPS"] /
                                       secondary["d3q19-trt-pull-float32-512"]["GLUPS"])
        secondary["e3m12_over_fp32"] = (secondary["d3q19-trt-pull-e3m12-512"]["GLUPS"] /
                                        secondary["d3q19-trt-pull-float32-512"]["GLUPS"])
        # other sweeps of the same family: weighted-orthogonal MRT (even/odd-paired transforms),
        # and the sparse list sweep on a porous medium (bytes per fluid cell: Q reads, Q writes,
        # Q - 1 four-byte indices)
        for name, bpc in (("d3q19-mrt-pull-float32-256", 2 * 19 * 4), ("sparse-porous-192-d3q19-trt-float32",
                                                                        2 * 19 * 4 + 18 * 4)):
            st2 = WORKLOADS[name][0](device)
            for _ in range(4):
                st2.time_step()
            a2, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a2.record(stream)
            for _ in range(20):
                st2.time_step()
            b2.record(stream)
            torch.cuda.synchronize()
            g2 = st2.number_of_cells / (a2.elapsed_time(b2) / 20 * 1e-3) / 1e9
            secondary[name] = {"GLUPS": g2, "GB/s": g2 * bpc, "frac": g2 * bpc / peak, "bytes_per_cell": bpc}
            if name.startswith("sparse"):
                secondary[name].update({"fluid_cells": st2.number_of_cells, "solid_fraction": st2.solid_fraction})
            del st2
            torch.cuda.empty_cache()
        if args.accuracy_steps > 0:
            # the same box from the same seeded state, stored in each type and in FP64 for the
            # reference: relative L2 velocity error after accuracy_steps sweeps (config c3: 5000)
            from lbmpy_b200.precision import precision_study
            acc = precision_study(512, args.accuracy_steps, args.accuracy_steps,
                                  storages=("float32", "float16", "bfloat16", "e3m12"), device=device,
                                  log=lambda *_: None)
            for st in ("float32", "float16", "bfloat16", "e3m12"):
                secondary[f"d3q19-trt-pull-{st}-512"]["l2_vs_fp64"] = acc[st]["final_l2_velocity_error"]
                secondary[f"d3q19-trt-pull-{st}-512"]["max_ke_rel_error"] = acc[st]["max_ke_rel_error"]
            secondary["accuracy_steps"] = args.accuracy_steps
            torch.cuda.empty_cache()

    if rank == 0:
        line = {"metric": METRIC,
                "value": glups, "unit": "GLUPS", "n_gpus": world,
                "steps": args.steps, "warmup": warm, "ms_per_step": ms_per_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": {8: "f64", 4: "f32", 2: "f32 (16-bit storage)"}[itemsize], "data": "synthetic",
                "config": {"workload": args.workload, "cells": cells, "populations": q_pop,
                           "bytes_per_population": itemsize, "parallelism": f"replicas{world}",
                           "l2": "inputs larger than L2" if cells * q_pop * itemsize > 126e6
                           else "inputs fit in L2 (no flush)"},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                             "bytes_per_lu": bytes_per_sweep / cells},
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": args.steps,
                "clocks": clocks.summary(), "secondary": secondary}
        if batched:
            line["config"].update({"domains": step.n_domains, "tiling": vars(step.tiling), **step.info(),
                                   "graph": "K launches captured in one CUDA graph, replayed once"})
        if headline:
            line["config"].update({"shape": list(SHAPE), "omega": OMEGA, "force": FORCE, "pattern": "aa",
                                   "galilean_correction": True, "storage": "float32 zero-centred"})
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
