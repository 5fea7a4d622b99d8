"""Polynomial fit used by the FP32 rate kernel (argot_b200/csrc/photoion.cuh).

phi(x) = (1 - e^-x) / x is the photon-conserving cell factor of the rate
integral (calc_photoion_rate.c:327-386 forms it as (1 - e^-dtau) / dtau);
every bin weighs its photons by e^-tau phi(x), tau the optical depth to the
cell and x the cell's own.  For small x the difference 1 - e^-x cancels, so
below x = PHI_X_MAX the kernel uses the identity

    e^-tau phi(x) = e^-(tau + x/2) sinh(y) / y,   y = x / 2:

the attenuation to the middle of the cell (one exponential, its exponent
folded into the ray's columns) times an even function of x, evaluated as a
polynomial of degree SINHC_DEGREE in v = u^2, u = x / ln 2 (the log2-scaled
cell optical depth the kernel forms anyway).  The polynomial is a
near-minimax fit of relative error (least squares on Chebyshev-distributed
points, reweighted by Lawson's iteration toward equal ripple), with
coefficients rounded to FP32.  Above PHI_X_MAX the kernel takes
(1 - e^-x) / x from the SFU exponential.

    python -m argot_b200.fits     # prints the coefficients and the error
"""
from __future__ import annotations

import numpy as np

PHI_X_MAX = 1.0
SINHC_DEGREE = 3
LN2 = 0.69314718055994531


def phi(x):
    """(1 - e^-x) / x in float64 (series near 0)."""
    x = np.asarray(x, np.float64)
    small = x < 1e-3
    xs = np.where(small, 1.0, x)
    return np.where(small, 1 - x / 2 + x * x / 6 - x ** 3 / 24 + x ** 4 / 120, -np.expm1(-xs) / xs)


def sinhc_half(u):
    """sinh(y) / y, y = u ln2 / 2 (float64)."""
    y = np.asarray(u, np.float64) * (LN2 / 2)
    small = y < 1e-4
    ys = np.where(small, 1.0, y)
    return np.where(small, 1 + y * y / 6, np.sinh(ys) / ys)


def _lawson(V, f, iters):
    """Near-minimax relative-error fit: least squares reweighted toward
    equal ripple (Lawson)."""
    w = 1.0 / f
    wt = np.full(len(f), 1.0 / len(f))
    c = None
    for _ in range(iters):
        s = w * np.sqrt(wt)
        c, *_ = np.linalg.lstsq(V * s[:, None], f * s, rcond=None)
        err = np.abs(V @ c - f) / f
        wt = wt * (err / err.max() + 1e-3)
        wt /= wt.sum()
    return c


def fit_sinhc(x_max: float = PHI_X_MAX, degree: int = SINHC_DEGREE, points: int = 4000, iters: int = 200):
    """Power-basis coefficients c[0..degree] (FP32) of the fit of
    v -> sinh(y) / y, v = u^2, y = u ln2 / 2, for u in [0, x_max / ln2]."""
    t = np.cos(np.pi * (np.arange(points) + 0.5) / points) * 0.5 + 0.5
    u = t * (x_max / LN2)
    c = _lawson(np.vander(u * u, degree + 1, increasing=True), sinhc_half(u), iters)
    return c.astype(np.float32)


def horner_f32(c, x):
    """The kernel's evaluation: Horner with one FP32 rounding per FMA."""
    x = np.asarray(x, np.float32).astype(np.float64)
    p = np.full(x.shape, np.float32(c[-1]), np.float32)
    for k in range(len(c) - 2, -1, -1):
        p = (x * p.astype(np.float64) + np.float64(c[k])).astype(np.float32)
    return p


def mid_cell_error(c, x_max: float = PHI_X_MAX, n: int = 200001):
    """Largest relative error of the kernel's FP32 evaluation of
    2^(-u/2) p(u^2) against phi(u ln2) on [0, x_max / ln2] (the factor
    2^(-u/2) rounded once to FP32, as the SFU's exponential of the
    mid-cell optical depth delivers it to about that accuracy)."""
    u = np.linspace(0.0, x_max / LN2, n).astype(np.float32)
    v = (u.astype(np.float64) ** 2).astype(np.float32)
    p = horner_f32(c, v).astype(np.float64)
    e = np.exp2(-u.astype(np.float64) / 2).astype(np.float32).astype(np.float64)
    w = (e * p).astype(np.float32).astype(np.float64)
    ref = phi(LN2 * u.astype(np.float64))
    return float(np.max(np.abs(w - ref) / ref))


if __name__ == "__main__":
    h = fit_sinhc()
    print("sinh(y)/y in v = u^2:", ", ".join(f"{float(v):.9g}f" for v in h))
    print("max relative error of 2^(-u/2) p(u^2) against phi on [0, %g / ln 2]: %.3g"
          % (PHI_X_MAX, mid_cell_error(h)))
