"""Learned eddy-viscosity closure for the D3Q27 cumulant sweep.

lbmpy's Smagorinsky model (``turbulence_models.py:25-84``) sets the shear relaxation rate of each
cell from the magnitude of its non-equilibrium stress, omega = 2 / (tau0 + sqrt(18 C^2 Pi +
tau0^2)).  The closure here keeps that hook and replaces the closed form by a small network:

    features(Pi_neq, rho, u)  ->  10 -> 32 -> 32 -> 1 perceptron (SiLU)  ->  nu_t = s * softplus(y)
    omega = 1 / (tau0 + 3 nu_t)

evaluated per cell inside the sweep (``lbm_closure.cuh``), with FP32 parameters in constant
memory.  Training runs on the GPU through the library's own forward / backward / Adam kernels
(``lbm_mlp_loss_grad``, ``lbm_mlp_adam``); the training data come from box-filtered fine-grid runs
of the same method (``turbulence.py``).

Use::

    closure = MLPClosure(seed=0)
    closure.fit(features, targets)                      # device tensors [10, n], [n]
    cfg = LBMConfig(stencil=Stencil.D3Q27, method=Method.CUMULANT, relaxation_rate=1.99,
                    compressible=True, subgrid_scale_model=(SubgridScaleModel.LEARNED, closure))

The parameters live once per device and process: the last closure uploaded is the one every
closure sweep on that device uses.
"""
from __future__ import annotations

import ctypes
import math
from typing import Optional

import numpy as np
import torch

from . import _native as N

NIN, NH = 10, 32
W1, B1 = 0, NIN * NH
W2 = B1 + NH
B2 = W2 + NH * NH
W3 = B2 + NH
B3 = W3 + NH
SCALE = B3 + 1
NPARAM = SCALE + 1
assert NPARAM == N.MLP_PARAMS

_uploaded = {}          # device index -> (id(closure), version)


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: Optional[torch.Tensor]):
    return ctypes.c_void_p(t.data_ptr() if t is not None else None)


def closure_features(state: torch.Tensor) -> torch.Tensor:
    """Features [10, n] of cells given their state [10, n] (Pi_xx, Pi_yy, Pi_zz, Pi_xy, Pi_xz,
    Pi_yz, rho, ux, uy, uz), FP32 on the GPU; the sweep computes the same features in place."""
    if state.dim() != 2 or state.shape[0] != 10:
        raise ValueError("state must have shape [10, n]")
    state = state.to(torch.float32).contiguous()
    if not state.is_cuda:
        raise ValueError("state must be a CUDA tensor")
    out = torch.empty_like(state)
    N.check(N.lib().lbm_closure_features(_ptr(state), state.shape[1], _ptr(out), _stream()), "lbm_closure_features")
    return out


class MLPClosure:
    """Parameters of the closure network (FP32, on the GPU) with its training loop."""

    def __init__(self, params: Optional[torch.Tensor] = None, seed: int = 0, nu_scale: float = 1e-3,
                 device="cuda"):
        self.device = torch.device(device)
        if params is None:
            rng = np.random.default_rng(seed)
            p = np.zeros(NPARAM, dtype=np.float32)
            p[W1:B1] = rng.normal(0, math.sqrt(1.0 / NIN), NIN * NH)
            p[W2:B2] = rng.normal(0, math.sqrt(1.0 / NH), NH * NH)
            p[W3:B3] = rng.normal(0, math.sqrt(1.0 / NH), NH)
            p[B3] = -2.0
            p[SCALE] = nu_scale
            params = torch.from_numpy(p)
        params = torch.as_tensor(params, dtype=torch.float32)
        if params.numel() != NPARAM:
            raise ValueError(f"the closure has {NPARAM} parameters, got {params.numel()}")
        self.params = params.reshape(-1).to(self.device).contiguous()
        self.version = 0
        self.history = []

    # ---------------------------------------------------------------------------- parameters
    @property
    def nu_scale(self) -> float:
        return float(self.params[SCALE])

    def normalise_inputs(self, mean: torch.Tensor, std: torch.Tensor):
        """Folds x -> (x - mean) / std into the first layer, so that the network sees standardised
        features while the sweep feeds it raw ones."""
        mean = mean.to(self.device, torch.float32).reshape(NIN)
        std = std.to(self.device, torch.float32).reshape(NIN).clamp_min(1e-12)
        w1 = self.params[W1:B1].view(NIN, NH)
        b1 = self.params[B1:W2]
        b1 -= ((mean / std)[:, None] * w1).sum(0)
        w1 /= std[:, None]
        self.version += 1

    def upload(self):
        """Makes these parameters the ones the closure sweep reads on the current device."""
        host = self.params.detach().to("cpu", torch.float32).contiguous()
        N.check(N.lib().lbm_closure_set_weights(ctypes.c_void_p(host.data_ptr()), NPARAM, _stream()),
                "lbm_closure_set_weights")
        torch.cuda.current_stream().synchronize()
        _uploaded[torch.cuda.current_device()] = (id(self), self.version)

    def ensure_uploaded(self):
        if _uploaded.get(torch.cuda.current_device()) != (id(self), self.version):
            self.upload()

    # ---------------------------------------------------------------------------- evaluation
    def predict(self, feats: torch.Tensor) -> torch.Tensor:
        """nu_t of samples feats [10, n]."""
        feats = feats.to(self.device, torch.float32).contiguous()
        out = torch.empty(feats.shape[1], dtype=torch.float32, device=self.device)
        N.check(N.lib().lbm_mlp_forward(_ptr(self.params), _ptr(feats), feats.shape[1], _ptr(out), _stream()),
                "lbm_mlp_forward")
        return out

    def loss_and_grad(self, feats, target, weight=None, trainer=None):
        """(loss, gradient [1442]) of the weighted mean squared nu_t error, from the GPU kernels."""
        feats = feats.to(self.device, torch.float32).contiguous()
        target = target.to(self.device, torch.float32).contiguous()
        n = feats.shape[1]
        if weight is not None:
            weight = weight.to(self.device, torch.float32).contiguous()
            inv = 1.0 / float(weight.double().sum())
        else:
            inv = 1.0 / n
        own = trainer is None
        if own:
            trainer = _Trainer()
        grad = torch.empty(NPARAM, dtype=torch.float32, device=self.device)
        loss = torch.empty(1, dtype=torch.float64, device=self.device)
        N.check(N.lib().lbm_mlp_loss_grad(trainer.handle, _ptr(self.params), _ptr(feats), _ptr(target), _ptr(weight),
                                          n, inv, _ptr(grad), _ptr(loss), _stream()), "lbm_mlp_loss_grad")
        return loss, grad

    def fit(self, feats: torch.Tensor, target: torch.Tensor, weight: Optional[torch.Tensor] = None,
            steps: int = 2000, batch: int = 65536, lr: float = 3e-3, lr_final: float = 3e-4, seed: int = 0,
            standardise: bool = True, log_every: int = 100):
        """Adam on minibatches drawn (seeded) from the samples.  With `standardise`, training sees
        standardised features and the standardisation is folded into the first layer at the end,
        so the trained parameters take raw features (as the sweep computes them).  Keeps (step,
        loss) pairs in `history`."""
        feats = feats.to(self.device, torch.float32).contiguous()
        target = target.to(self.device, torch.float32).contiguous()
        n = feats.shape[1]
        if standardise:
            mean, std = feats.mean(1), feats.std(1).clamp_min(1e-12)
            feats = ((feats - mean[:, None]) / std[:, None]).contiguous()
        gen = torch.Generator(device=self.device)
        gen.manual_seed(seed)
        trainer = _Trainer()
        m1 = torch.zeros(NPARAM, dtype=torch.float32, device=self.device)
        m2 = torch.zeros_like(m1)
        lib = N.lib()
        b = min(batch, n)
        fb = torch.empty(NIN, b, dtype=torch.float32, device=self.device)
        for t in range(1, steps + 1):
            idx = torch.randint(0, n, (b,), device=self.device, generator=gen)
            torch.index_select(feats, 1, idx, out=fb)
            tb = target.index_select(0, idx)
            wb = weight.index_select(0, idx).contiguous() if weight is not None else None
            loss, grad = self.loss_and_grad(fb, tb, wb, trainer)
            frac = (t - 1) / max(steps - 1, 1)
            rate = lr * (lr_final / lr) ** frac
            N.check(lib.lbm_mlp_adam(_ptr(grad), _ptr(self.params), _ptr(m1), _ptr(m2), rate, 0.9, 0.999, 1e-8, t,
                                     _stream()), "lbm_mlp_adam")
            if log_every and (t % log_every == 0 or t == steps):
                self.history.append((t, float(loss.item())))
        if standardise:
            self.normalise_inputs(mean, std)
        self.version += 1
        return self

    def state_dict(self):
        return {"params": self.params.detach().cpu().numpy().copy()}

    @classmethod
    def from_state_dict(cls, state, device="cuda"):
        return cls(params=torch.from_numpy(np.asarray(state["params"], np.float32)), device=device)


class _Trainer:
    def __init__(self, max_blocks: int = 0):
        if max_blocks <= 0:
            max_blocks = 4 * torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        h = ctypes.c_void_p()
        N.check(N.lib().lbm_mlp_create(int(max_blocks), ctypes.byref(h)), "lbm_mlp_create")
        self.handle = h

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and N._lib is not None:
            N._lib.lbm_mlp_destroy(h)
            self.handle = None
