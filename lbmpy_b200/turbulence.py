"""Decaying homogeneous turbulence: initial fields, spectra, filtered training data for the
learned closure, and the closure study.

The scenario follows lbmpy's decaying-turbulence and Kida-vortex set-ups
(``tests/full_scenarios/kida_vortex_flow/scenario_kida_vortex_flow.py:56-82`` computes an energy
spectrum with numpy's FFT; restated here on the GPU with torch's FFT): a periodic box, a seeded
divergence-free velocity field with E(k) ~ k^4 exp(-2 (k/k0)^2), unit density, and the D3Q27
cumulant method.  Resolutions are related by acoustic scaling: a box r times finer runs r times
more steps with r times the lattice viscosity, and the same initial field (generated on a common
base grid and spectrally interpolated).

Training data for the closure (``closure.MLPClosure``): a fine run's velocity is box-filtered by
r onto the coarse grid; the subgrid stress tau = filter(u u) - filter(u) filter(u) and the
filtered strain rate S (central differences on the coarse grid) give the eddy viscosity that
best explains tau, nu* = max(0, -dev(tau):S / (2 S:S)).  The coarse cell would carry the
non-equilibrium stress Pi = -(2/3) rho (tau0 + 3 nu*) S (Chapman-Enskog, the relation lbmpy's
Smagorinsky model inverts), from which the sweep's features follow.
"""
from __future__ import annotations

import math
import time
from typing import Dict, Optional

import numpy as np
import torch

from . import closure as C


# ------------------------------------------------------------------------------ fields
def solenoidal_velocity(n: int, k0: float = 4.0, u_rms: float = 0.03, seed: int = 0, base: int = 32,
                        device="cuda") -> torch.Tensor:
    """Divergence-free periodic velocity [n, n, n, 3] (float64) with E(k) ~ k^4 exp(-2 (k/k0)^2),
    RMS velocity per component u_rms; the same field for every n >= base (modes |k_i| < base/2,
    generated from the seed on the base grid; with k0 = 4 the spectrum beyond |k| = 16 holds less
    than 1e-9 of the energy)."""
    if n < base:
        raise ValueError(f"the field is defined on a {base}^3 base grid; n = {n} is coarser")
    rng = np.random.default_rng(seed)
    shape = (base, base, base, 3)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    k1 = np.fft.fftfreq(base, 1.0 / base)
    kx, ky, kz = np.meshgrid(k1, k1, k1, indexing="ij")
    kk = np.stack([kx, ky, kz], -1)
    k2 = (kk ** 2).sum(-1)
    kmag = np.sqrt(k2)
    k2s = np.where(k2 == 0, 1.0, k2)
    a = a - kk * ((a * kk).sum(-1) / k2s)[..., None]              # project out the k component
    amp = kmag * np.exp(-(kmag / k0) ** 2)                        # |u_k| ~ sqrt(E(k) / k^2)
    nyq = (np.abs(kx) >= base // 2) | (np.abs(ky) >= base // 2) | (np.abs(kz) >= base // 2)
    amp[nyq] = 0.0
    a *= amp[..., None]
    ub = np.real(np.fft.ifftn(a, axes=(0, 1, 2)))
    ub *= u_rms / np.sqrt((ub ** 2).mean(axis=(0, 1, 2)).mean())
    uh = np.fft.fftn(ub, axes=(0, 1, 2))                          # Hermitian, zero at the Nyquist planes
    if n == base:
        return torch.from_numpy(ub).to(device)
    uh_t = torch.from_numpy(uh).to(device)
    full = torch.zeros((n, n, n, 3), dtype=torch.complex128, device=device)
    h = base // 2
    idx = torch.cat([torch.arange(0, h), torch.arange(n - h, n)]).to(device)
    src = torch.cat([torch.arange(0, h), torch.arange(base - h, base)]).to(device)
    full[idx[:, None, None], idx[None, :, None], idx[None, None, :]] = \
        uh_t[src[:, None, None], src[None, :, None], src[None, None, :]]
    u = torch.fft.ifftn(full, dim=(0, 1, 2)).real * (n / base) ** 3
    return u


def energy_spectrum(u: torch.Tensor):
    """Shell-summed kinetic energy spectrum E(k), k = 0 .. n/2 (integer shells), of a periodic
    velocity [n, n, n, 3]; sum_k E(k) = mean(|u|^2) / 2."""
    n = u.shape[0]
    uh = torch.fft.fftn(u.to(torch.float64), dim=(0, 1, 2)) / n ** 3
    e = 0.5 * (uh.real ** 2 + uh.imag ** 2).sum(-1)
    k1 = torch.fft.fftfreq(n, 1.0 / n, device=u.device, dtype=torch.float64)
    kmag = torch.sqrt(k1[:, None, None] ** 2 + k1[None, :, None] ** 2 + k1[None, None, :] ** 2)
    shell = torch.round(kmag).long().clamp_max(n)
    E = torch.zeros(n + 1, dtype=torch.float64, device=u.device).index_add_(0, shell.reshape(-1), e.reshape(-1))
    return E[: n // 2 + 1].cpu().numpy()


def box_filter(a: torch.Tensor, r: int) -> torch.Tensor:
    """Mean over r x r x r blocks of the first three axes."""
    n = a.shape[0]
    m = n // r
    rest = a.shape[3:]
    return a.reshape(m, r, m, r, m, r, *rest).mean(dim=(1, 3, 5))


def strain_rate(u: torch.Tensor) -> torch.Tensor:
    """Periodic central-difference strain rate S_ab = (d_a u_b + d_b u_a) / 2, [n, n, n, 3, 3]."""
    g = torch.stack([(torch.roll(u, -1, a) - torch.roll(u, 1, a)) * 0.5 for a in range(3)], -2)  # g[..., a, b] = d_a u_b
    return 0.5 * (g + g.transpose(-1, -2))


def training_samples(u_fine: torch.Tensor, rho_fine: torch.Tensor, r: int, tau0: float):
    """(state [10, m], nu* [m], weight [m]) for the coarse cells of a fine velocity field filtered
    by r (see the module docstring); weight = S:S / mean(S:S)."""
    u = u_fine.to(torch.float64)
    ub = box_filter(u, r)
    rb = box_filter(rho_fine.to(torch.float64), r)
    uu = box_filter(u[..., :, None] * u[..., None, :], r)
    tau = uu - ub[..., :, None] * ub[..., None, :]
    S = strain_rate(ub)
    eye = torch.eye(3, dtype=torch.float64, device=u.device)
    tdev = tau - (tau.diagonal(dim1=-2, dim2=-1).sum(-1) / 3.0)[..., None, None] * eye
    ss = (S * S).sum((-1, -2))
    num = -(tdev * S).sum((-1, -2))
    nu = torch.clamp(num / (2.0 * ss.clamp_min(1e-30)), min=0.0)
    Pi = -(2.0 / 3.0) * rb[..., None, None] * (tau0 + 3.0 * nu)[..., None, None] * S
    state = torch.stack([Pi[..., 0, 0], Pi[..., 1, 1], Pi[..., 2, 2], Pi[..., 0, 1], Pi[..., 0, 2], Pi[..., 1, 2],
                         rb, ub[..., 0], ub[..., 1], ub[..., 2]], 0).reshape(10, -1)
    w = (ss / ss.mean()).reshape(-1)
    return state.to(torch.float32), nu.reshape(-1).to(torch.float32), w.to(torch.float32)


# ------------------------------------------------------------------------------ runs
def omega_for(omega_coarse: float, r: int) -> float:
    """Relaxation rate of a box r times finer with the same physical viscosity (acoustic scaling)."""
    nu = (1.0 / omega_coarse - 0.5) / 3.0
    return 1.0 / (3.0 * r * nu + 0.5)


def decaying_turbulence(n: int, omega: float, seed: int = 0, k0: float = 4.0, u_rms: float = 0.03,
                        sgs=None, storage="float32", device="cuda", base: int = 32):
    """A LatticeBoltzmannStep: D3Q27 cumulant, compressible, AA, periodic n^3 box, initial field
    from solenoidal_velocity.  sgs: None, ("smagorinsky", C) or an MLPClosure."""
    import lbmpy_b200 as L
    kw = {}
    if isinstance(sgs, tuple) and sgs[0] == "smagorinsky":
        kw["subgrid_scale_model"] = (L.SubgridScaleModel.SMAGORINSKY, float(sgs[1]))
    elif sgs is not None:
        kw["subgrid_scale_model"] = (L.SubgridScaleModel.LEARNED, sgs)
    step = L.LatticeBoltzmannStep(domain_size=(n, n, n), periodicity=True, stencil=L.Stencil.D3Q27,
                                  method=L.Method.CUMULANT, relaxation_rate=omega, compressible=True,
                                  streaming_pattern="aa", config=L.CreateKernelConfig(data_type="float32"),
                                  optimization={"storage_dtype": storage}, device=device, **kw)
    u = solenoidal_velocity(n, k0, u_rms, seed, base=base, device=device)
    from .macroscopic_value_kernels import set_equilibrium
    set_equilibrium(step._macro, step.pdfs, 1.0, u, step.previous_timestep, step.kernel_params, step.periodicity)
    return step


def velocity_field(step) -> torch.Tensor:
    """Device velocity [n, n, n, 3] and density of the current state (FP32)."""
    from .macroscopic_value_kernels import get_macroscopic
    n = step.domain_size
    rho = torch.empty(n, dtype=torch.float32, device=step.pdfs.device)
    u = torch.empty(n + (3,), dtype=torch.float32, device=step.pdfs.device)
    get_macroscopic(step._macro, step.pdfs, rho, u, step.previous_timestep, step.kernel_params, step.periodicity)
    return u, rho


def spectral_error(E: np.ndarray, E_ref: np.ndarray, kmax: int) -> float:
    """Mean |log10(E / E_ref)| over shells 1 .. kmax."""
    k = np.arange(1, kmax + 1)
    return float(np.mean(np.abs(np.log10(np.maximum(E[k], 1e-300) / np.maximum(E_ref[k], 1e-300)))))


def closure_study(n: int = 128, omega: float = 1.99, steps: int = 1000, r_train: int = 4, r_ref: int = 2,
                  snapshots: int = 4, smagorinsky: float = 0.1, seed: int = 0, train_steps: int = 3000,
                  batch: int = 65536, device="cuda", log=print) -> Dict:
    """Trains the closure on box-filtered runs r_train times finer and compares energy spectra of
    the n^3 runs (plain cumulant, Smagorinsky, learned closure) at the same physical time with an
    r_ref times finer plain run and with the box-filtered fine run (the field an LES on n^3
    approximates).  Returns spectra, errors, timings and the trained closure."""
    t_start = time.time()
    res: Dict = {"n": n, "omega": omega, "steps": steps, "r_train": r_train, "r_ref": r_ref}
    tau0 = 1.0 / omega
    base = min(32, n)              # one initial field for every resolution
    res["base"] = base
    # 1. training data from the fine run
    nf = n * r_train
    fine = decaying_turbulence(nf, omega_for(omega, r_train), seed=seed, device=device, base=base)
    states, targets, weights = [], [], []
    every = steps * r_train // snapshots
    for s in range(snapshots):
        fine.run_sweeps(every)
        u, rho = velocity_field(fine)
        st, nu, w = training_samples(u, rho, r_train, tau0)
        states.append(st), targets.append(nu), weights.append(w)
        if s == snapshots - 1:          # the filtered fine field at the end: the LES target
            E_filt = energy_spectrum(box_filter(u.to(torch.float64), r_train))
        del u, rho
    del fine
    torch.cuda.empty_cache()
    state = torch.cat(states, 1)
    target = torch.cat(targets)
    weight = torch.cat(weights)
    feats = C.closure_features(state)
    res["samples"] = int(target.numel())
    res["nu_target_mean"] = float(target.mean())
    log(f"training data: {res['samples']} samples, mean nu* {res['nu_target_mean']:.3e} "
        f"({time.time() - t_start:.1f} s)")
    # 2. training (scale: the output unit is about the mean target)
    closure = C.MLPClosure(seed=seed, nu_scale=max(float(target.mean()), 1e-6), device=device)
    t0 = time.time()
    closure.fit(feats, target, weight, steps=train_steps, batch=batch, seed=seed)
    torch.cuda.synchronize()
    res["train_seconds"] = time.time() - t0
    res["train_history"] = closure.history
    pred = closure.predict(feats)
    wsum = float(weight.double().sum())
    res["train_loss_learned"] = float((weight.double() * (pred.double() - target.double()) ** 2).sum() / wsum)
    res["train_loss_zero"] = float((weight.double() * target.double() ** 2).sum() / wsum)
    # Smagorinsky on the same cells, from the same stress (lbmpy's closed form inverted for nu_t)
    P = state[:6].double()
    pim = torch.sqrt(2.0 * (P[0] ** 2 + P[1] ** 2 + P[2] ** 2 + 2.0 * (P[3] ** 2 + P[4] ** 2 + P[5] ** 2))) / \
        state[6].double()
    om_s = 2.0 / (tau0 + torch.sqrt(18.0 * smagorinsky ** 2 * pim + tau0 ** 2))
    nu_s = (1.0 / om_s - tau0) / 3.0
    res["train_loss_smagorinsky"] = float((weight.double() * (nu_s - target.double()) ** 2).sum() / wsum)
    log(f"trained in {res['train_seconds']:.1f} s: weighted MSE {res['train_loss_learned']:.3e} "
        f"(no closure {res['train_loss_zero']:.3e}, Smagorinsky {res['train_loss_smagorinsky']:.3e})")
    # 3. reference and the three coarse runs
    ref = decaying_turbulence(n * r_ref, omega_for(omega, r_ref), seed=seed, device=device, base=base)
    ref.run_sweeps(steps * r_ref)
    E_ref = energy_spectrum(velocity_field(ref)[0])
    del ref
    torch.cuda.empty_cache()
    runs = {"plain": None, "smagorinsky": ("smagorinsky", smagorinsky), "learned": closure}
    kmax = n // 3
    res["kmax"] = kmax
    res["E_ref"] = E_ref.tolist()
    res["E_filtered_fine"] = E_filt.tolist()
    for name, sgs in runs.items():
        st = decaying_turbulence(n, omega, seed=seed, sgs=sgs, device=device, base=base)
        st.run_sweeps(3)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        st.run_sweeps(steps - 3)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / (steps - 3)
        E = energy_spectrum(velocity_field(st)[0])
        res[f"E_{name}"] = E.tolist()
        res[f"err_{name}"] = spectral_error(E, E_ref, kmax)
        res[f"err_filtered_{name}"] = spectral_error(E, E_filt, kmax)
        res[f"ms_per_step_{name}"] = ms
        res[f"glups_{name}"] = n ** 3 / (ms * 1e-3) / 1e9
        log(f"{name:12s} spectral error vs {n * r_ref}^3 plain {res[f'err_{name}']:.4f}, vs filtered "
            f"{nf}^3 {res[f'err_filtered_{name}']:.4f}  {ms:.3f} ms/step")
        del st
    res["closure"] = closure
    res["seconds"] = time.time() - t_start
    return res


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train the learned closure and compare energy spectra")
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--omega", type=float, default=1.99)
    ap.add_argument("--r-train", type=int, default=4)
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--out", default=None, help="write the results (JSON) here")
    a = ap.parse_args(argv)
    res = closure_study(n=a.n, omega=a.omega, steps=a.steps, r_train=a.r_train, train_steps=a.train_steps)
    closure = res.pop("closure")
    summary = {k: v for k, v in res.items() if not k.startswith("E_") and k != "train_history"}
    print(json.dumps(summary))
    if a.out:
        res["closure_params"] = closure.params.cpu().numpy().tolist()
        with open(a.out, "w") as fh:
            json.dump(res, fh)


if __name__ == "__main__":
    main()
