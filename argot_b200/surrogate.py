"""Training and validation of the frequency-integral surrogate (driver of
the hand-written CUDA kernels in csrc/mlp.cu; PyTorch only allocates).

The network predicts q_j = ln(y_j / ylin_j) for the six integrals of the
rate stage (Gamma and heating of HI, HeI, HeII), y_j = ln(I_j / I_j0) and
ylin_j = -sum_s tau_s m_js its exact thin limit (m_js: first moments of the
normalised cross sections under the emitter's spectrum), from
x = (log10 tau_HI, log10 tau_HeI, log10 tau_HeII, log10 T).  Training data:
seeded samples of the exact 256-bin quadrature, generated on the device.

`error_envelope` measures, on held-out samples, the largest error of q in
bins of the predicted q; the rate kernels turn it into a per-ray relative
error bound |y| dq of each contribution and keep, per cell, the
predictions whose bounds fit the cell's error budget.
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
ENV_BINS = 64       # error-envelope bins over predicted q in [Q_LO, 0]
Q_LO = -7.0
OUT_SCALE, OUT_SHIFT = 3.5, -3.5  # q = 3.5 o - 3.5
DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
WEIGHTS = os.path.join(DATA, "surrogate.npz")


def _lib():
    lib = L.load()
    assert lib.argot_b200_mlp_num_params() == NPARAM
    return lib


class Surrogate:
    """Inference weights of a trained network on the current device."""

    def __init__(self, params, env, tol: float = 5e-4):
        """tol: per-cell relative error budget of the surrogate's
        contributions (the rest of a 1e-3 target is left to float rounding
        and the exact rays)."""
        self.lib = _lib()
        p = np.ascontiguousarray(params, np.float32)
        e = np.ascontiguousarray(env, np.float32)
        assert p.size == NPARAM and e.shape == (6, ENV_BINS)
        self.handle = C.c_void_p()
        L.check(self.lib.argot_b200_surrogate_create(p.ctypes.data, e.ctypes.data, float(tol),
                                                     C.byref(self.handle)), "surrogate_create")
        self.tol = tol

    def eval(self, X):
        """q_j predictions (n, 6) with the tensor-core inference numerics
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
        """q_j predictions (n, 6) with the training forward (CUDA cores)."""
        n = X.shape[0]
        O = torch.empty((6, n), dtype=torch.float32, device=self.dev)
        L.check(self.lib.argot_b200_mlp_forward(self.params.data_ptr(), X.data_ptr(), n,
                                                O.data_ptr(), self.sp), "mlp_forward")
        return (O * OUT_SCALE + OUT_SHIFT).t()

    def thin_limit(self, X):
        """ylin_j = -sum_s tau_s m_js(T) of samples X (host arrays)."""
        X = np.asarray(X, np.float64)
        it = np.rint((X[:, 3] - 4.0) / 1.5 * (self.nT - 1)).astype(int)
        m = moments_grid(self.spec_np, self.i0_np)
        return -np.einsum("ns,njs->nj", 10.0 ** X[:, :3], m[it])


def rate_weights():
    """w_j(nu) of the six integrals (256 x 6), the cross sections (256 x 3)
    and sigma_s at each species' first absorbing bin."""
    from .pipeline import tables
    nu, cs = tables()
    cs = cs.astype(np.float64)
    nuf = nu.astype(np.float32).astype(np.float64)
    thr = np.array([1.0, 1.8125, 4.0])
    w6 = np.concatenate([cs, cs * np.maximum(nuf[:, None] - thr[None, :], 0.0)], 1)
    sig0 = np.array([cs[cs[:, s] > 0, s][0] for s in range(3)])
    return w6, cs, sig0


def moments_grid(spec, i0):
    """m[t, j, s] = sum_nu w_j s_nu(T_t) sigma_s / sigma_s0 / I_j0(T_t)."""
    w6, cs, sig0 = rate_weights()
    return np.einsum("tv,vj,vs->tjs", spec, w6, cs / sig0) / i0[:, :, None]


def error_envelope(q_pred, q_true, bins: int = ENV_BINS, q_lo: float = Q_LO, safety: float = 1.5):
    """Largest |error of q| per output and bin of predicted q (over the bin
    and its two neighbours), times `safety`; empty bins take the largest
    error of their output."""
    q_pred = np.asarray(q_pred, np.float64)
    err = np.abs(q_pred - np.asarray(q_true, np.float64))
    env = np.zeros((6, bins))
    b = np.clip(((q_pred - q_lo) / -q_lo * bins).astype(int), 0, bins - 1)
    for j in range(6):
        mx = np.zeros(bins)
        np.maximum.at(mx, b[:, j], err[:, j])
        seen = np.bincount(b[:, j], minlength=bins) > 0
        mx[~seen] = err[:, j].max()
        nb = np.maximum(mx, np.maximum(np.r_[mx[1:], mx[-1]], np.r_[mx[0], mx[:-1]]))
        env[j] = nb * safety
    return env


def save(params, env, path: str = WEIGHTS, meta=None):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(path, params=np.asarray(params, np.float32), envelope=np.asarray(env, np.float32),
             q_lo=Q_LO, **(meta or {}))


def load(path: str = WEIGHTS):
    d = np.load(path)
    return d["params"], d["envelope"]
