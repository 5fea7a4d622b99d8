"""Polynomial fits used by the FP32 rate kernel (argot_b200/csrc/photoion.cuh).

phi(x) = (1 - e^-x) / x is the photon-conserving cell factor of the rate
integral (calc_photoion_rate.c:327-386 forms it as (1 - e^-dtau) / dtau).
For small x the difference 1 - e^-x cancels, so the kernel evaluates phi
on [0, 1) as a polynomial and above 1 from the SFU exponential.  The
polynomial is a near-minimax fit of relative error (least squares on
Chebyshev-distributed points, reweighted by Lawson's iteration toward
equal ripple), with coefficients rounded to FP32.

    python -m argot_b200.fits     # prints the coefficients and the errors
"""
from __future__ import annotations

import numpy as np

PHI_X_MAX = 1.0
PHI_DEGREE = 6
# the kernel evaluates the polynomial in u = x / ln 2 (the log2-scaled
# cell optical depth it forms anyway), on [0, PHI_X_MAX / ln 2)
LN2 = 0.69314718055994531


def phi(x):
    """(1 - e^-x) / x in float64 (series near 0)."""
    x = np.asarray(x, np.float64)
    small = x < 1e-3
    xs = np.where(small, 1.0, x)
    return np.where(small, 1 - x / 2 + x * x / 6 - x ** 3 / 24 + x ** 4 / 120, -np.expm1(-xs) / xs)


def fit_phi(x_max: float = PHI_X_MAX, degree: int = PHI_DEGREE, points: int = 4000, iters: int = 200,
            scale: float = 1.0):
    """Power-basis coefficients c[0..degree] (FP32) of the fit of
    u -> phi(scale u) on [0, x_max / scale]."""
    t = np.cos(np.pi * (np.arange(points) + 0.5) / points) * 0.5 + 0.5
    x = t * (x_max / scale)
    V = np.vander(x, degree + 1, increasing=True)
    f = phi(scale * x)
    w = 1.0 / f
    wt = np.full_like(x, 1.0 / points)
    c = None
    for _ in range(iters):
        s = w * np.sqrt(wt)
        c, *_ = np.linalg.lstsq(V * s[:, None], f * s, rcond=None)
        err = np.abs(V @ c - f) / f
        wt = wt * (err / err.max() + 1e-3)
        wt /= wt.sum()
    return c.astype(np.float32)


def horner_f32(c, x):
    """The kernel's evaluation: Horner with one FP32 rounding per FMA."""
    x = np.asarray(x, np.float32).astype(np.float64)
    p = np.full(x.shape, np.float32(c[-1]), np.float32)
    for k in range(len(c) - 2, -1, -1):
        p = (x * p.astype(np.float64) + np.float64(c[k])).astype(np.float32)
    return p


def phi_error(c, x_max: float = PHI_X_MAX, n: int = 200001, scale: float = 1.0):
    """Largest relative error of the FP32 evaluation of u -> phi(scale u) on
    [0, x_max / scale]."""
    u = np.linspace(0.0, x_max / scale, n).astype(np.float32)
    ref = phi(scale * u.astype(np.float64))
    return float(np.max(np.abs(horner_f32(c, u).astype(np.float64) - ref) / ref))


if __name__ == "__main__":
    c = fit_phi(scale=LN2)
    print("coefficients (in u = x / ln 2):", ", ".join(f"{float(v):.9g}f" for v in c))
    print("max relative error of the FP32 evaluation on [0, %g / ln 2): %.3g"
          % (PHI_X_MAX, phi_error(c, scale=LN2)))
