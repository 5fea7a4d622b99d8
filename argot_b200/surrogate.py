"""Training and validation of the frequency-integral surrogate (driver of
the hand-written CUDA kernels in csrc/mlp.cu; PyTorch only allocates).

The network predicts t_j = ln(1 - ln(I_j / I_j0)) for the six integrals
of the rate stage (Gamma and heating of HI, HeI, HeII) from
x = (log10 tau_HI, log10 tau_HeI, log10 tau_HeII, log10 T).  Training data:
seeded samples of the exact 256-bin quadrature, generated on the device.

`error_envelope` measures, on held-out samples, the largest error of
ln(I/I0) in bins of the predicted t; the rate kernel uses that envelope
as the per-ray error bound that decides between the surrogate and the
exact quadrature.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import time

import numpy as np
import torch

from . import _lib as L

NT = 256            # temperature grid of the training spectra
NPARAM = 9030
ENV_BINS = 64       # error-envelope bins over predicted t in [0, T_MAX]
T_MAX = 6.0
DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
WEIGHTS = os.path.join(DATA, "surrogate.npz")


def _lib():
    lib = L.load()
    assert lib.argot_b200_mlp_num_params() == NPARAM
    return lib


class Surrogate:
    """Inference weights of a trained network on the current device."""

    def __init__(self, params, env, tol: float = 5e-4):
        self.lib = _lib()
        p = np.ascontiguousarray(params, np.float32)
        e = np.ascontiguousarray(env, np.float32)
        assert p.size == NPARAM and e.shape == (6, ENV_BINS)
        self.handle = C.c_void_p()
        L.check(self.lib.argot_b200_surrogate_create(p.ctypes.data, e.ctypes.data, float(tol),
                                                     C.byref(self.handle)), "surrogate_create")
        self.tol = tol

    def eval(self, X):
        """t_j predictions (n, 6) with the tensor-core inference numerics
        (X: device float32 tensor (n, 4) of raw inputs)."""
        n = X.shape[0]
        T = torch.empty((n, 6), dtype=torch.float32, device=X.device)
        L.check(self.lib.argot_b200_surrogate_eval(self.handle, X.data_ptr(), n, T.data_ptr(),
                                                   torch.cuda.current_stream(X.device).cuda_stream),
                "surrogate_eval")
        return T

    @classmethod
    def from_file(cls, path: str = WEIGHTS, tol: float = 5e-4):
        p, e = load(path)
        return cls(p, e, tol)

    def close(self):
        if self.handle:
            self.lib.argot_b200_surrogate_free(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def spectra_grid(nT: int = NT):
    spec = np.zeros((nT, 256), np.float64)
    i0 = np.zeros((nT, 6), np.float64)
    L.check(_lib().argot_b200_mlp_spectra(nT, spec.ctypes.data, i0.ctypes.data), "mlp_spectra")
    return spec, i0


def init_params(seed: int = 0):
    """Kaiming-uniform weights, zero biases."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float32)
    off = 0
    for fan_in, fan_out in ((4, 64), (64, 64), (64, 64), (64, 6)):
        lim = math.sqrt(6.0 / fan_in) if fan_out != 6 else math.sqrt(1.0 / fan_in)
        p[off:off + fan_in * fan_out] = rng.uniform(-lim, lim, fan_in * fan_out)
        off += fan_in * fan_out + fan_out
    return p


class Trainer:
    def __init__(self, device="cuda", nT: int = NT, seed: int = 0):
        self.lib = _lib()
        self.dev = torch.device(device)
        spec, i0 = spectra_grid(nT)
        self.nT = nT
        self.spec_np, self.i0_np = spec, i0
        self.spec = torch.from_numpy(spec).to(self.dev)
        self.i0 = torch.from_numpy(i0).to(self.dev)
        self.params = torch.from_numpy(init_params(seed)).to(self.dev)
        self.m = torch.zeros(NPARAM, dtype=torch.float32, device=self.dev)
        self.v = torch.zeros_like(self.m)
        self.step = 0
        self.work = None
        self.work_nb = 0

    @property
    def sp(self):
        return torch.cuda.current_stream(self.dev).cuda_stream

    def samples(self, n: int, seed: int):
        X = torch.empty((n, 4), dtype=torch.float32, device=self.dev)
        Y = torch.empty((n, 6), dtype=torch.float32, device=self.dev)
        L.check(self.lib.argot_b200_mlp_samples(self.spec.data_ptr(), self.i0.data_ptr(), self.nT, n,
                                                seed, X.data_ptr(), Y.data_ptr(), self.sp), "mlp_samples")
        return X, Y

    def _ensure_work(self, nb):
        if self.work is None or self.work_nb < nb:
            self.work = torch.empty(int(self.lib.argot_b200_mlp_workspace(nb)), dtype=torch.float32,
                                    device=self.dev)
            self.work_nb = nb

    def gradient(self, X, Y):
        """Loss gradient of one batch (no update), for checking."""
        nb = X.shape[0]
        self._ensure_work(nb)
        g = torch.zeros(NPARAM, dtype=torch.float32, device=self.dev)
        loss = torch.zeros(1, dtype=torch.float64, device=self.dev)
        L.check(self.lib.argot_b200_mlp_train_step(self.params.data_ptr(), self.m.data_ptr(),
                                                   self.v.data_ptr(), X.data_ptr(), Y.data_ptr(), nb,
                                                   0.0, 1, self.work.data_ptr(), g.data_ptr(),
                                                   loss.data_ptr(), self.sp), "mlp_train_step")
        return g, float(loss.item()) / (nb * 6)

    def train(self, X, Y, epochs: int, batch: int = 8192, lr: float = 2e-3, lr_min: float = 2e-5,
              seed: int = 0, log=None):
        n = X.shape[0]
        self._ensure_work(batch)
        g = torch.Generator(device="cpu").manual_seed(seed)
        steps_per_epoch = n // batch
        total = epochs * steps_per_epoch
        loss = torch.zeros(1, dtype=torch.float64, device=self.dev)
        t0 = time.time()
        hist = []
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g).to(self.dev)
            acc = 0.0
            for s in range(steps_per_epoch):
                idx = perm[s * batch:(s + 1) * batch]
                xb = X.index_select(0, idx).contiguous()
                yb = Y.index_select(0, idx).contiguous()
                k = self.step
                cur = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * min(k, total) / total))
                self.step += 1
                L.check(self.lib.argot_b200_mlp_train_step(self.params.data_ptr(), self.m.data_ptr(),
                                                           self.v.data_ptr(), xb.data_ptr(),
                                                           yb.data_ptr(), batch, cur, self.step,
                                                           self.work.data_ptr(), None,
                                                           loss.data_ptr(), self.sp), "mlp_train_step")
                if s == steps_per_epoch - 1:
                    acc = float(loss.item()) / (batch * 6)
            hist.append(acc)
            if log:
                log(f"epoch {ep + 1}/{epochs} loss {acc:.3e} ({time.time() - t0:.1f} s)")
        return hist

    def predict(self, X):
        """t_j predictions (n, 6) with the training forward (CUDA cores)."""
        n = X.shape[0]
        O = torch.empty((6, n), dtype=torch.float32, device=self.dev)
        L.check(self.lib.argot_b200_mlp_forward(self.params.data_ptr(), X.data_ptr(), n,
                                                O.data_ptr(), self.sp), "mlp_forward")
        return (O * 2.75 + 2.75).t()


def ln_ratio(t):
    """ln(I/I0) from t = ln(1 - ln(I/I0))."""
    return 1.0 - np.exp(np.asarray(t, np.float64))


def error_envelope(t_pred, t_true, bins: int = ENV_BINS, t_max: float = T_MAX, safety: float = 1.5):
    """Largest |error of ln(I/I0)| per output and bin of predicted t, times
    `safety`; empty bins inherit the largest error of their output."""
    t_pred = np.asarray(t_pred, np.float64)
    err = np.abs(ln_ratio(t_pred) - ln_ratio(t_true))
    env = np.zeros((6, bins))
    b = np.clip((t_pred / t_max * bins).astype(int), 0, bins - 1)
    for j in range(6):
        mx = np.zeros(bins)
        np.maximum.at(mx, b[:, j], err[:, j])
        seen = np.bincount(b[:, j], minlength=bins) > 0
        mx[~seen] = err[:, j].max()
        # monotone envelope: an error bound may only grow with t
        env[j] = np.maximum.accumulate(mx) * safety
    return env


def save(params, env, path: str = WEIGHTS, meta=None):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, params=np.asarray(params, np.float32), envelope=np.asarray(env, np.float32),
             t_max=T_MAX, **(meta or {}))


def load(path: str = WEIGHTS):
    d = np.load(path)
    return d["params"], d["envelope"]
