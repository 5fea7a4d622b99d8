"""Seeded synthetic workloads of the ARGOT point-source RT benchmark configs.

No public dataset is involved: every field and source list is drawn here
from fixed seeds, in the shapes, sizes and value distributions the benchmark
configurations specify.  Units follow ARGOT's Iliev-test initial conditions
(src/test_IC/cmpproj_test2_IC.c:51-75): unit box [0,1)^3 of 6.6 kpc,
code density 1 = n_H 1e-3 cm^-3.

Fields are float32, flattened with z fastest (cell index iz + N*(iy + N*ix),
the reference's MESH macro).  He fractions are relative to n_He =
HELIUM_FACT n_H.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

MPC = 3.086e24
MPROTON = 1.672623e-24
XHYDROGEN = 0.755  # helium build (prim_chem/chemistry.h:23)


def units(nH: float = 1.0e-3, lunit_mpc: float = 6.6e-3):
    """(lunit, denstonh) computed in the reference's operation order."""
    lunit = lunit_mpc * MPC
    cube = lunit * lunit * lunit
    munit = nH * cube * MPROTON / XHYDROGEN
    denstonh = munit / cube * XHYDROGEN / MPROTON
    return lunit, denstonh


@dataclasses.dataclass
class Workload:
    name: str
    edge: int
    dens: np.ndarray
    fHI: np.ndarray
    fHeI: np.ndarray
    fHeII: np.ndarray
    src_pos: np.ndarray        # (nsrc, 3) float32
    src_rate: np.ndarray       # (nsrc,) float64 total photon rate [s^-1]
    src_type: np.ndarray       # (nsrc,) int32: 0 blackbody
    src_param: np.ndarray      # (nsrc,) float32: T [K]
    theta: float = 0.5
    lunit: float = 0.0
    denstonh: float = 0.0
    notes: str = ""
    # optional explicit photon rates per bin (nsrc, 256), e.g. read from a
    # source file; otherwise formed from type, param and rate
    src_spectra: np.ndarray | None = None

    @property
    def nsrc(self) -> int:
        return len(self.src_rate)

    @property
    def ncell(self) -> int:
        return self.edge ** 3

    def fields(self):
        return (self.dens, self.fHI, self.fHeI, self.fHeII)


# --------------------------------------------------------------- spectra
def photon_rates(photon_counts, src_type, src_param, src_rate):
    """Per-source photon rate per bin, counts * (total / norm), formed exactly
    as setup_photon_rate does (source.c:135: one division, one product per
    bin), with the bin counts evaluated once per distinct spectral shape.
    ``photon_counts(type, param) -> (counts[256], norm)``."""
    out = np.zeros((len(src_rate), 256), np.float64)
    cache = {}
    for i, (t, p, tot) in enumerate(zip(src_type, src_param, src_rate)):
        key = (int(t), float(np.float32(p)))
        if key not in cache:
            cache[key] = photon_counts(*key)
        counts, norm = cache[key]
        out[i] = counts * (float(tot) / norm)
    return out


# ------------------------------------------------------------ random fields
def _gaussian_field(edge: int, slope: float, rng: np.random.Generator) -> np.ndarray:
    """Unit-variance Gaussian random field with P(k) ~ k^slope (k > 0)."""
    white = rng.standard_normal((edge, edge, edge)).astype(np.float64)
    fk = np.fft.rfftn(white)
    kx = np.fft.fftfreq(edge)[:, None, None]
    ky = np.fft.fftfreq(edge)[None, :, None]
    kz = np.fft.rfftfreq(edge)[None, None, :]
    k = np.sqrt(kx * kx + ky * ky + kz * kz)
    amp = np.zeros_like(k)
    amp[k > 0] = k[k > 0] ** (slope / 2.0)
    g = np.fft.irfftn(fk * amp, s=(edge, edge, edge), axes=(0, 1, 2))
    g -= g.mean()
    g /= g.std()
    return g


def lognormal_density(edge: int, sigma_ln: float, rng, slope: float = -3.0) -> np.ndarray:
    g = _gaussian_field(edge, slope, rng)
    rho = np.exp(sigma_ln * g - 0.5 * sigma_ln * sigma_ln)
    rho /= rho.mean()
    return rho.astype(np.float32).ravel()


def tanh_ionization(edge: int, pos: np.ndarray, rate: np.ndarray, lo=1.0e-5, hi=0.99,
                    r0=0.02, width_frac=0.25, device=None) -> np.ndarray:
    """x_HII = max over sources of 0.5*(1 - tanh((r - R_s)/w_s)), clipped to
    [lo, hi]; R_s = r0 (Ndot/1e49)^(1/3) box units (a Stromgren-like scaling),
    w_s = width_frac * R_s.  Each source only touches cells within R_s + 6 w_s,
    beyond which its profile is below the floor.  Evaluated with torch in
    float64 (on `device`, default: a GPU when present, else the CPU)."""
    import torch
    if device is None:
        device = "cuda" if torch.cuda.is_available() else "cpu"
    x = torch.zeros((edge, edge, edge), dtype=torch.float64, device=device)
    c = (torch.arange(edge, dtype=torch.float64, device=device) + 0.5) / edge
    for p, n in zip(pos.astype(np.float64), rate):
        R = r0 * (n / 1.0e49) ** (1.0 / 3.0)
        w = width_frac * R
        reach = R + 6.0 * w
        sl = []
        for a in range(3):
            i0 = max(0, int(math.floor((p[a] - reach) * edge)))
            i1 = min(edge, int(math.ceil((p[a] + reach) * edge)) + 1)
            sl.append(slice(i0, i1))
        if any(s.start >= s.stop for s in sl):
            continue
        dx = (c[sl[0]] - p[0])[:, None, None]
        dy = (c[sl[1]] - p[1])[None, :, None]
        dz = (c[sl[2]] - p[2])[None, None, :]
        r = torch.sqrt(dx * dx + dy * dy + dz * dz)
        prof = 0.5 * (1.0 - torch.tanh((r - R) / w))
        sub = x[sl[0], sl[1], sl[2]]
        torch.maximum(sub, prof, out=sub)
    return np.clip(x.cpu().numpy().astype(np.float32), lo, hi).ravel()


# ------------------------------------------------------------------ configs
def _rates_loguniform(rng, n, lo, hi):
    return 10.0 ** rng.uniform(math.log10(lo), math.log10(hi), n)


def _finish(name, edge, dens, xHII, fHeII, pos, rate, theta, notes, T=1.0e5):
    lunit, denstonh = units()
    fHI = (1.0 - xHII).astype(np.float32)
    fHeII = fHeII.astype(np.float32)
    fHeI = (1.0 - fHeII).astype(np.float32)
    n = len(rate)
    return Workload(name=name, edge=edge, dens=dens.astype(np.float32), fHI=fHI, fHeI=fHeI,
                    fHeII=fHeII, src_pos=np.ascontiguousarray(pos, np.float32),
                    src_rate=np.asarray(rate, np.float64),
                    src_type=np.zeros(n, np.int32), src_param=np.full(n, T, np.float32),
                    theta=theta, lunit=lunit, denstonh=denstonh, notes=notes)


def plain(edge: int = 64, nsrc: int = 16, seed: int = 1):
    """64^3 uniform mesh, n_H = 1e-3, x_HII and x_HeII ~ U[1e-4, 1e-2],
    16 sources uniform in the box, Ndot log-uniform in [1e48, 1e50], 1e5 K
    blackbody, theta = 0.5."""
    rng = np.random.default_rng(seed)
    n = edge ** 3
    dens = np.ones(n, np.float32)
    xHII = rng.uniform(1e-4, 1e-2, n).astype(np.float32)
    xHeII = rng.uniform(1e-4, 1e-2, n).astype(np.float32)
    pos = rng.uniform(0.0, 1.0, (nsrc, 3)).astype(np.float32)
    rate = _rates_loguniform(rng, nsrc, 1e48, 1e50)
    return _finish(f"plain{edge}_src{nsrc}", edge, dens, xHII, xHeII, pos, rate, 0.5,
                   "uniform density, x_HII, x_HeII ~ U[1e-4,1e-2]")


def _lognormal_ionized(name, edge, nsrc, sigma_ln, rate_lo, rate_hi, seed, pos=None, theta=0.5):
    rng = np.random.default_rng(seed)
    dens = lognormal_density(edge, sigma_ln, rng)
    if pos is None:
        pos = rng.uniform(0.0, 1.0, (nsrc, 3)).astype(np.float32)
    rate = _rates_loguniform(rng, nsrc, rate_lo, rate_hi)
    xHII = tanh_ionization(edge, pos, rate)
    return _finish(name, edge, dens, xHII, xHII, pos, rate, theta,
                   f"lognormal sigma_ln={sigma_ln}, P(k)~k^-3; tanh HII profiles; He tracks H")


def precision(edge: int = 128, nsrc: int = 256, seed: int = 2):
    return _lognormal_ionized(f"precision{edge}_src{nsrc}", edge, nsrc, 1.0, 1e49, 1e51, seed)


def learned(edge: int = 192, nsrc: int = 1024, seed: int = 4):
    return _lognormal_ionized(f"learned{edge}_src{nsrc}", edge, nsrc, 1.0, 1e49, 1e51, seed)


def clustered_positions(rng, nsrc, nclusters=32, sigma=0.05):
    centres = rng.uniform(0.1, 0.9, (nclusters, 3))
    which = rng.integers(0, nclusters, nsrc)
    pos = centres[which] + rng.normal(0.0, sigma, (nsrc, 3))
    return np.clip(pos, 1.0e-4, 1.0 - 1.0e-4).astype(np.float32)


def largest(edge: int = 256, nsrc: int = 4096, seed: int = 5):
    """256^3 lognormal (sigma_ln = 1.2) with 4096 sources in 32 Gaussian
    clusters (sigma = 0.05 box), Ndot log-uniform in [1e49, 1e52]."""
    rng = np.random.default_rng(seed)
    pos = clustered_positions(rng, nsrc)
    return _lognormal_ionized(f"largest{edge}_src{nsrc}", edge, nsrc, 1.2, 1e49, 1e52, seed + 100,
                              pos=pos)


def batched(nprob: int = 48, seed: int = 3, edges=(32, 48, 64, 96, 128)):
    """48 problems: edge from {32,48,64,96,128}, 4-512 sources, sigma_ln in
    [0.5, 1.5]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nprob):
        e = int(rng.choice(edges))
        ns = int(rng.integers(4, 513))
        s = float(rng.uniform(0.5, 1.5))
        out.append(_lognormal_ionized(f"batch{i}_n{e}_src{ns}", e, ns, s, 1e49, 1e51,
                                      seed * 1000 + i))
    return out


def ionized(edge: int = 64, nsrc: int = 64, seed: int = 9, sigma_ln: float = 1.0,
            neutral: float = 1e-4):
    """A fully ionised volume (H II and He III, as inside a merged ionised
    region late in reionisation): lognormal density, residual fractions
    fHI, fHeI, fHeII log-uniform within a factor 10 around `neutral`, so
    that most rays are optically thin."""
    rng = np.random.default_rng(seed)
    dens = lognormal_density(edge, sigma_ln, rng)
    pos = rng.uniform(0.0, 1.0, (nsrc, 3)).astype(np.float32)
    rate = _rates_loguniform(rng, nsrc, 1e49, 1e51)
    n = edge ** 3
    frac = lambda: (neutral * 10.0 ** rng.uniform(-0.5, 0.5, n)).astype(np.float32)
    w = _finish(f"ionized{edge}_src{nsrc}", edge, dens, 1.0 - frac(), np.zeros(n), pos, rate, 0.5,
                f"lognormal sigma_ln={sigma_ln}; H II + He III, neutral fractions ~{neutral}")
    w.fHeI = frac()
    w.fHeII = frac()
    return w


def tiny(edge: int = 16, nsrc: int = 4, seed: int = 7, sigma_ln: float = 1.0):
    """Small lognormal problem for unit tests."""
    return _lognormal_ionized(f"tiny{edge}_src{nsrc}", edge, nsrc, sigma_ln, 1e49, 1e51, seed)
