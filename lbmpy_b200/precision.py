"""Storage-precision study: the same Taylor-Green run stored in FP64, FP32, FP16, BF16 and e3m12.

The D3Q19 TRT periodic box (relaxation rate 1.8, magic-number odd rate, compressible) starts
from a Taylor-Green vortex u0 = 0.04 in x/y plus seeded Gaussian noise (sigma 1e-3); every run
uses the same initial field.  FP16 / BF16 / e3m12 store zero-centred PDFs (f - w_i, lbmpy's
zero-centring) and collide in FP32 registers.  Reported per storage type, against the FP64 run:
the relative L2 velocity error at the end and along the way, and the kinetic-energy history
(FP64 reduction on the GPU), with GLUPS.

    python -m lbmpy_b200.precision [--n 512 --steps 5000 --every 500]
"""
from __future__ import annotations

import json
import time

import numpy as np
import torch


def tgv_field(n: int, u0: float = 0.04, noise: float = 1e-3, seed: int = 0, device="cuda") -> torch.Tensor:
    x = torch.arange(n, dtype=torch.float64, device=device)
    k = 2 * np.pi / n
    u = torch.zeros((n, n, n, 3), dtype=torch.float64, device=device)
    u[..., 0] = (u0 * torch.sin(k * x)[:, None] * torch.cos(k * x)[None, :])[:, :, None]
    u[..., 1] = (-u0 * torch.cos(k * x)[:, None] * torch.sin(k * x)[None, :])[:, :, None]
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    u += noise * torch.randn(u.shape, dtype=torch.float64, device=device, generator=g)
    return u


def _run(n, storage, steps, every, u_init, device):
    import lbmpy_b200 as L
    from .macroscopic_value_kernels import get_macroscopic, set_equilibrium
    compute = "float64" if storage == "float64" else "float32"
    step = L.LatticeBoltzmannStep(domain_size=(n, n, n), periodicity=True, stencil=L.Stencil.D3Q19,
                                  method=L.Method.TRT, relaxation_rate=1.8, compressible=True,
                                  config=L.CreateKernelConfig(data_type=compute),
                                  optimization={"storage_dtype": storage}, device=device)
    set_equilibrium(step._macro, step.pdfs, 1.0, u_init, step.previous_timestep, step.kernel_params,
                    step.periodicity)
    out = {"ke": [], "u": []}
    ms = 0.0
    done = 0
    while done < steps:
        k = min(every, steps - done)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        step.run_sweeps(k)
        b.record()
        torch.cuda.synchronize()
        ms += a.elapsed_time(b)
        done += k
        red = step.reduce_conserved()
        out["ke"].append((done, float(red[4])))
        u = torch.empty((n, n, n, 3), dtype=torch.float64 if compute == "float64" else torch.float32, device=device)
        get_macroscopic(step._macro, step.pdfs, None, u, step.previous_timestep, step.kernel_params, step.periodicity)
        out["u"].append(u)
    out["glups"] = n ** 3 * steps / (ms * 1e-3) / 1e9
    del step
    torch.cuda.empty_cache()
    return out


def precision_study(n: int = 512, steps: int = 5000, every: int = 500, seed: int = 0,
                    storages=("float32", "float16", "bfloat16", "e3m12"), device="cuda", log=print):
    t0 = time.time()
    u0 = tgv_field(n, seed=seed, device=device)
    ref = _run(n, "float64", steps, every, u0, device)
    log(f"float64: {ref['glups']:.2f} GLUPS ({time.time() - t0:.0f} s)")
    res = {"n": n, "steps": steps, "every": every, "ke_float64": ref["ke"], "glups_float64": ref["glups"]}
    # keep only the reference velocities on the device, in FP64
    ref_u = ref.pop("u")
    for st in storages:
        r = _run(n, st, steps, every, u0, device)
        errs = []
        for (t, _), u, ur in zip(r["ke"], r["u"], ref_u):
            e = float(torch.linalg.vector_norm(u.double() - ur) / torch.linalg.vector_norm(ur))
            errs.append((t, e))
        ke_rel = [(t, abs(a - b) / b) for (t, a), (_, b) in zip(r["ke"], ref["ke"])]
        res[st] = {"glups": r["glups"], "l2_velocity_error": errs, "final_l2_velocity_error": errs[-1][1],
                   "ke": r["ke"], "ke_rel_error": ke_rel, "max_ke_rel_error": max(e for _, e in ke_rel)}
        log(f"{st}: {r['glups']:.2f} GLUPS, final L2 velocity error {errs[-1][1]:.3e}, "
            f"max KE relative error {res[st]['max_ke_rel_error']:.3e}")
        del r
        torch.cuda.empty_cache()
    res["seconds"] = time.time() - t0
    return res


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description="FP16/BF16/FP32 storage against FP64 on a Taylor-Green box")
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--every", type=int, default=500)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    res = precision_study(a.n, a.steps, a.every)
    print(json.dumps({k: (v if not isinstance(v, dict) else {kk: vv for kk, vv in v.items() if kk in
                                                               ("glups", "final_l2_velocity_error",
                                                                "max_ke_rel_error")})
                      for k, v in res.items() if not k.startswith("ke_")}))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh)


if __name__ == "__main__":
    main()
