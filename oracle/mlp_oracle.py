"""FP64 CPU restatement of the surrogate network and of its training
gradient (test infrastructure only): the checker for the hand-written CUDA
forward / backward kernels in argot_b200/csrc/mlp.cu.

Same architecture and numerics contract as the device code:
4 -> 64 -> 64 -> 64 -> 6, SiLU; weights rounded to BF16 (biases not);
inputs and activations unrounded (the tensor-core inference carries each
as a BF16 pair hi + lo, 16 mantissa bits); loss = mean over samples and
outputs of the squared error of the normalised output, gradients straight
through the weight rounding.
"""
from __future__ import annotations

import numpy as np

H, NIN, NOUT = 64, 4, 6
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * NIN
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H * H
OFF_W4 = OFF_B3 + H
OFF_B4 = OFF_W4 + NOUT * H
NPARAM = OFF_B4 + NOUT

TAU_LO, TAU_HI, T_LO, T_HI = -6.0, 3.0, 4.0, 5.5
OUT_SHIFT, OUT_SCALE = -3.5, 3.5


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even)."""
    a = np.ascontiguousarray(x, np.float32).view(np.uint32)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, NIN), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3].reshape(H, H), p[OFF_B3:OFF_W4],
            p[OFF_W4:OFF_B4].reshape(NOUT, H), p[OFF_B4:])


def norm_in(X):
    X = np.asarray(X, np.float64)
    out = np.empty_like(X)
    out[:, :3] = (X[:, :3] - 0.5 * (TAU_LO + TAU_HI)) * (2.0 / (TAU_HI - TAU_LO))
    out[:, 3] = (X[:, 3] - 0.5 * (T_LO + T_HI)) * (2.0 / (T_HI - T_LO))
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, X):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p)
    W1, W2, W3, W4 = (bf16(w.astype(np.float32)) for w in (W1, W2, W3, W4))
    x = norm_in(X)
    z1 = x @ W1.T + b1
    a1 = silu(z1)
    z2 = a1 @ W2.T + b2
    a2 = silu(z2)
    z3 = a2 @ W3.T + b3
    a3 = silu(z3)
    o = a3 @ W4.T + b4
    return o, (x, z1, a1, z2, a2, z3, a3, W1, W2, W3, W4)


def loss_and_grad(p, X, Y):
    """Mean squared error of the normalised outputs and its gradient."""
    o, (x, z1, a1, z2, a2, z3, a3, W1, W2, W3, W4) = forward(p, X)
    tgt = (np.asarray(Y, np.float64) - OUT_SHIFT) / OUT_SCALE
    n = len(X)
    e = o - tgt
    loss = float((e * e).sum() / (n * NOUT))
    d4 = 2.0 * e / (n * NOUT)
    d3 = (d4 @ W4) * silu_grad(z3)
    d2 = (d3 @ W3) * silu_grad(z2)
    d1 = (d2 @ W2) * silu_grad(z1)
    g = np.zeros(NPARAM)
    g[OFF_W1:OFF_B1] = (d1.T @ x).ravel()
    g[OFF_B1:OFF_W2] = d1.sum(0)
    g[OFF_W2:OFF_B2] = (d2.T @ a1).ravel()
    g[OFF_B2:OFF_W3] = d2.sum(0)
    g[OFF_W3:OFF_B3] = (d3.T @ a2).ravel()
    g[OFF_B3:OFF_W4] = d3.sum(0)
    g[OFF_W4:OFF_B4] = (d4.T @ a3).ravel()
    g[OFF_B4:] = d4.sum(0)
    return loss, g


def moments(spec, i0, cs, sig0, w6):
    """m[t, j, s]: first moment of sigma_s / sigma_s0 under the weight
    w_j(nu) s_nu(T_t), normalised by I_j0."""
    shat = cs / sig0
    return np.einsum("tv,vj,vs->tjs", spec, w6, shat) / i0[:, :, None]


def exact_targets(X, spec, i0, cs, sig0, w6, with_y=False):
    """q_j = ln(y_j / ylin_j), y_j = ln(I_j / I_j0), ylin_j = -sum_s tau_s m_js,
    by the exact 256-bin sums (FP64); spec rows indexed by the temperature
    grid position encoded in X[:, 3]."""
    nT = len(spec)
    it = np.rint((X[:, 3] - T_LO) / (T_HI - T_LO) * (nT - 1)).astype(int)
    tau = 10.0 ** np.asarray(X[:, :3], np.float64)
    shat = cs / sig0
    att = np.exp(-(tau @ shat.T)) * spec[it]
    I = att @ w6
    y = np.log(I / i0[it])
    ylin = -np.einsum("ns,njs->nj", tau, moments(spec, i0, cs, sig0, w6)[it])
    q = np.log(y / ylin)
    return (q, y) if with_y else q
