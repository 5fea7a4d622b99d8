// photoion.cuh -- per-ray photo-ionisation / heating rates
// (calc_photoion_rate, photon-conserving branch, H + He, not cosmological).
#pragma once
#include <algorithm>
#include <mutex>

#include "march.cuh"

namespace argot {

constexpr double kHNuL = kHPlanck * kNuL;  // hplanck*nuL, double

// Frequency tables of the rate kernels.  Every translation unit that
// includes this header has its own copy in its constant bank, filled by its
// own ensure_rate_tables().
__constant__ RateTables c_tab;

static int ensure_rate_tables(int device) {
  static std::mutex mu;
  static bool done[64] = {false};
  std::lock_guard<std::mutex> lock(mu);
  if (device < 0 || device >= 64) return ARGOT_B200_EINVAL;
  if (done[device]) return 0;
  double nu[kNu];
  float cs3[3 * kNu];
  host_tables(nu, cs3);
  RateTables t;
  const double thr[3] = {kThrHI, kThrHeI, kThrHeII};
  const double l2e = 1.4426950408889634074;
  for (int i = 0; i < kNu; i++) {
    const float nf = (float)nu[i];
    t.nu_f[i] = nf;
    for (int s = 0; s < 3; s++) {
      const float c = cs3[3 * i + s];
      t.cs[s][i] = c;
      t.cs_l2e[s][i] = (float)((double)c * l2e);
      const double w = ((double)nf > thr[s]) ? ((double)nf - thr[s]) : 0.0;
      t.hw[s][i] = (float)((double)c * w);
    }
  }
  // suffix maxima of the cross sections per 16-bin iteration (sfu_iters)
  // and the iterations below the helium thresholds (sigma_s is 0 below
  // nu_s in the fits of prim_chem/cross_section.c)
  int first[3];
  for (int s = 0; s < 3; s++) {
    float m = 0.f;
    first[s] = kNu / 16;
    for (int k = kNu - 1; k >= 0; k--) {
      m = fmaxf(m, t.cs[s][k]);
      if (k % 16 == 0) t.smax16[s][k / 16] = m;
      if (t.cs[s][k] != 0.f) first[s] = k / 16;
    }
  }
  t.iter_heii = first[2];
  t.iter_he = std::min(first[1], first[2]);
  ARGOT_CUDA_TRY(cudaMemcpyToSymbol(c_tab, &t, sizeof(t)));
  done[device] = true;
  return 0;
}

// Per-species quantities of the target cell for one ray (double):
// the column to the cell's entry face N_s [cm^-2], the cell's own column
// dN_s, and 1/(n_s V_shell + TINY).
struct RayCols {
  double N[3], dN[3], rN[3];
};

__device__ __forceinline__ RayCols ray_columns(const GridDev &g, float t_hi, float t_hei, float t_heii,
                                               float4 raw, RayGeom geo) {
  RayCols c;
  const double cd = __dmul_rn(g.lunit, g.denstonh);
  const double nH = __dmul_rn((double)raw.x, g.denstonh);
  const double nHe = __dmul_rn(nH, kHeliumFact);
  const double n[3] = {__dmul_rn(nH, (double)raw.y), __dmul_rn(nHe, (double)raw.z), __dmul_rn(nHe, (double)raw.w)};
  const float tt[3] = {t_hi, t_hei, t_heii};
  const double a = __dadd_rn((double)geo.dist, __dmul_rn(0.5, (double)geo.delta));
  const double b = __dsub_rn((double)geo.dist, __dmul_rn(0.5, (double)geo.delta));
  const double l3 = __dmul_rn(__dmul_rn(g.lunit, g.lunit), g.lunit);
  const double vsh = __dmul_rn(__dmul_rn(4.0 * kPi / 3.0, __dsub_rn(__dmul_rn(__dmul_rn(a, a), a), __dmul_rn(__dmul_rn(b, b), b))), l3);
#pragma unroll
  for (int s = 0; s < 3; s++) {
    c.dN[s] = __dmul_rn(__dmul_rn(n[s], (double)geo.delta), g.lunit);
    c.N[s] = __dsub_rn(__dmul_rn((double)tt[s], cd), __dmul_rn(0.5, c.dN[s]));
    c.rN[s] = __ddiv_rn(1.0, __dadd_rn(__dmul_rn(n[s], vsh), kTiny));
  }
  return c;
}

// The reference's 256-bin loop in FP64 with its operation order
// (calc_photoion_rate.c:285-387); out[0..2] Gamma, out[3..5] Heat*h*nu_L.
static __device__ __noinline__ void rate_bins_f64(const RayCols &c, const double *__restrict__ spec, double out[6]) {
  double G0 = 0, G1 = 0, G2 = 0, H0 = 0, H1 = 0, H2 = 0;
  for (int k = 0; k < kNu; k++) {
    const float v = c_tab.nu_f[k];
    const double s0 = (double)c_tab.cs[0][k], s1 = (double)c_tab.cs[1][k], s2 = (double)c_tab.cs[2][k];
    double tau = __dmul_rn(c.N[0], s0);
    double d0 = __dmul_rn(c.dN[0], s0);
    double dtot = d0;
    tau = __dadd_rn(tau, __dmul_rn(c.N[1], s1));
    tau = __dadd_rn(tau, __dmul_rn(c.N[2], s2));
    double d1 = __dmul_rn(c.dN[1], s1);
    double d2 = __dmul_rn(c.dN[2], s2);
    dtot = __dadd_rn(dtot, __dadd_rn(d1, d2));
    const double pabs = __dmul_rn(__dmul_rn(__ldg(spec + k), exp(-tau)), __dsub_rn(1.0, exp(-dtot)));
    const double den = __dadd_rn(dtot, kTiny);
    d0 = __ddiv_rn(d0, den);
    G0 = __dadd_rn(G0, __dmul_rn(__dmul_rn(d0, pabs), c.rN[0]));
    if ((double)v > kThrHI) H0 = __dadd_rn(H0, __dmul_rn(__dmul_rn(__dmul_rn(d0, pabs), __dsub_rn((double)v, kThrHI)), c.rN[0]));
    d1 = __ddiv_rn(d1, den);
    d2 = __ddiv_rn(d2, den);
    G1 = __dadd_rn(G1, __dmul_rn(__dmul_rn(d1, pabs), c.rN[1]));
    G2 = __dadd_rn(G2, __dmul_rn(__dmul_rn(d2, pabs), c.rN[2]));
    if ((double)v > kThrHeI) H1 = __dadd_rn(H1, __dmul_rn(__dmul_rn(__dmul_rn(d1, pabs), __dsub_rn((double)v, kThrHeI)), c.rN[1]));
    if ((double)v > kThrHeII) H2 = __dadd_rn(H2, __dmul_rn(__dmul_rn(__dmul_rn(d2, pabs), __dsub_rn((double)v, kThrHeII)), c.rN[2]));
  }
  out[0] = G0; out[1] = G1; out[2] = G2;
  out[3] = __dmul_rn(H0, kHNuL);
  out[4] = __dmul_rn(H1, kHNuL);
  out[5] = __dmul_rn(H2, kHNuL);
}

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// ---------------------------------------------------------------------------
// FP32 rates.  Per ray: the columns to the target cell's entry face N_s and
// of the cell D_s [cm^-2] and the prefactor P_s = total dN_s / (n_s V_shell)
// (calc_photoion_rate.c:159-246), all in FP32.  With dN_s = n_s delta lunit
// and V_shell = 4 pi / 3 ((r + delta/2)^3 - (r - delta/2)^3) lunit^3 =
// 4 pi (r^2 + delta^2 / 12) delta lunit^3 (the cube difference expanded,
// which has no cancellation), the density cancels:
// P_s = total / (4 pi lunit^2 (r^2 + delta^2 / 12)) for n_s > 0 and 0 for
// n_s = 0 (the reference's TINY only keeps 0/0 away; its n_s V_shell is
// above 1e40 whenever n_s is a positive float).  total (1e48-1e52 photons/s)
// and 1/(4 pi lunit^2) (1e-46) are outside the FP32 range, so their powers
// of two are added as integers and P_s (1e4-1e13) is formed in range.
struct RayParams {
  float N[3], D[3], P[3];
};

// v = m * 2^e for a positive double, m in [1, 2) from the leading 24
// significant bits (integer operations on the bit pattern)
__device__ __forceinline__ float mant_exp2(double v, int &e) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  e = (int)((b >> 52) & 0x7ffu) - 1023;
  return __uint_as_float(0x3f800000u | (unsigned)((b >> 29) & 0x7fffffu));
}

constexpr float kHeliumFactF = (float)kHeliumFact;
constexpr float kHNuLf = (float)kHNuL;

// The FP32 parameters of a ray from emitter (sx, sy, sz) to the centre of
// target cell (gix, giy, giz) (global indices) with code-unit columns t_s;
// raw = {dens, fHI, fHeI, fHeII} of the target cell.  A ray that starts at
// its target's centre (r = 0) contributes nothing, as in the reference,
// whose shell volume then diverges.
__device__ __forceinline__ RayParams ray_params_f32(const GridDev &g, int gix, int giy, int giz, float sx,
                                                    float sy, float sz, float t0, float t1, float t2, float4 raw,
                                                    double total) {
  RayParams p;
  const float x = fmaf((float)gix + 0.5f, g.dx, g.xmin);
  const float y = fmaf((float)giy + 0.5f, g.dy, g.ymin);
  const float z = fmaf((float)giz + 0.5f, g.dz, g.zmin);
  const float dx = x - sx, dy = y - sy, dz = z - sz;
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  // delta_length (calc_photoion_rate.c:52-90): the cell's chord along the
  // ray, min over the axes of the cell side over |cosine|
  const float delta = sqrtf(r2) * fminf(__fdividef(g.dx, fabsf(dx)),
                                        fminf(__fdividef(g.dy, fabsf(dy)), __fdividef(g.dz, fabsf(dz))));
  const float n[3] = {raw.x * raw.y, (raw.x * kHeliumFactF) * raw.z, (raw.x * kHeliumFactF) * raw.w};
  const float tt[3] = {t0, t1, t2};
  const float dc = delta * g.cdf;
  int et;
  const float mt = mant_exp2(total, et);
  const float pv = ldexpf(__fdividef(mt * g.pcm, fmaf(delta * delta, 1.f / 12.f, r2)), et + g.pce);
  const bool ok = r2 > 0.f;
#pragma unroll
  for (int s = 0; s < 3; s++) {
    p.D[s] = ok ? n[s] * dc : 0.f;
    p.N[s] = ok ? fmaf(tt[s], g.cdf, -0.5f * p.D[s]) : 0.f;
    p.P[s] = (ok && n[s] > 0.f) ? pv : 0.f;
  }
  return p;
}

// The six rates of one ray from its quadrature sums a_s = sum (sigma_s
// log2 e) w and b_s = sum (sigma_s log2 e) nu w (ray_bins_packed):
// Gamma_s = P_s ln2 a_s, Heat_s = P_s ln2 (b_s - nu_s a_s) h nu_L.
__device__ __forceinline__ void ray_rates6(const float (&P)[3], float a0, float a1, float a2, float b0, float b1,
                                           float b2, float (&out)[6]) {
  const float kLn2 = 0.69314718055994531f;
  const float a[3] = {a0, a1, a2}, bb[3] = {b0, b1, b2};
  const float thr[3] = {(float)kThrHI, (float)kThrHeI, (float)kThrHeII};
#pragma unroll
  for (int s = 0; s < 3; s++) {
    out[s] = P[s] * (kLn2 * a[s]);
    out[3 + s] = P[s] * (kLn2 * fmaf(-thr[s], a[s], bb[s])) * kHNuLf;
  }
}

// ---- packed FP32 bin loop: two bins per instruction with the f32x2 FMA
// and multiply of sm_100.  An 8-lane group integrates one ray (or two,
// ray_bins_packed2); lane j owns the bin pairs (j + 16 i, j + 16 i + 8),
// i = 0..15 (the bins j + 8 m), and keeps one partial sum per output, pair
// member and ray.
// The pair table holds, for the three species and the two bins,
// sigma_s log2(e) and sigma_s log2(e) nu, 48 bytes, three 16-byte shared
// loads per pair, each serving the two rays of the lane.  The sums run on
// these entries: sum sigma_s w = ln2 sum (sigma_s log2 e) w, and, because
// sigma_s vanishes below the species' threshold nu_s (the fits of
// prim_chem/cross_section.c are 0 there), the heating sum
// sum sigma_s (nu - nu_s)^+ w = ln2 (sum (sigma_s log2 e) nu w - nu_s
// sum (sigma_s log2 e) w).  A shared load delivers 128 bytes per wavefront
// whatever the broadcast (the four groups of a warp read the same
// entries), so the table's bytes per ray set the kernel's shared-memory
// traffic, which shares the L1 data path with the spectrum loads.
// Measured at 256^3 / 4096 sources: with one ray per lane, an 80-byte
// entry (sigma log2 e, sigma and sigma (nu - nu_s)^+ per species) kept the
// shared-memory pipe at 79% of its peak, and a 24-byte entry without the
// nu products (nu formed from the lane's first pair and the grid ratio,
// two packed multiplies per pair and ray) ran the rates in 0.93 s against
// 1.02 s for 32 bytes; with two rays per lane this 48-byte entry, which
// saves those multiplies, runs them in 0.78 s against 0.81 s for 24 bytes.
struct alignas(16) BinPair {
  float2 l2e[3];    // sigma_s log2(e) of the two bins
  float2 l2enu[3];  // sigma_s log2(e) nu
};
constexpr int kBinPairs = kNu / 2;

// Fills the pair table from the constant tables (all threads of the block
// take part; the caller synchronises).
__device__ __forceinline__ void load_bin_pairs(BinPair *tab) {
  for (int p = threadIdx.x; p < kBinPairs; p += blockDim.x) {
    const int j = p & 7, i = p >> 3;
    const int k0 = j + 16 * i, k1 = k0 + 8;
    BinPair b;
#pragma unroll
    for (int s = 0; s < 3; s++) {
      b.l2e[s] = make_float2(c_tab.cs_l2e[s][k0], c_tab.cs_l2e[s][k1]);
      b.l2enu[s] = make_float2(c_tab.cs_l2e[s][k0] * c_tab.nu_f[k0], c_tab.cs_l2e[s][k1] * c_tab.nu_f[k1]);
    }
    tab[p] = b;
  }
}

// The photon-conserving cell factor phi(x) = (1 - e^-x)/x (x the cell's
// optical depth in the bin) enters every bin as e^-tau phi(x), tau the
// optical depth to the cell.  Below x = kPhiXMax the difference 1 - e^-x
// cancels, so the loop forms e^-tau phi(x) = e^-(tau + x/2) sinh(y)/y,
// y = x / 2, with sinh(y)/y a polynomial (sinhc_half2); above, it takes
// e^-tau (1 - e^-x) / x from the SFU (~2e-7).  Only the leading iterations
// of a ray can hold a bin above kPhiXMax (sfu_iters); the SFU form is
// predicated, not branched, so where it is compiled in every pair pays its
// exponentials and reciprocal (ncu, 256^3 / 16 sources: three MUFU
// operations per bin instead of one, 60 warp instructions per iteration
// instead of ~40), and it is compiled only into those iterations.
constexpr float kPhiXMax = 1.0f;
constexpr float kPhiUMax = 1.44269504088896341f;  // kPhiXMax / ln 2

// sinh(y) / y, y = x / 2 = dl ln2 / 2, of the two bins of a pair from
// v = dl^2: a near-minimax fit of degree 3 in v made by argot_b200/fits.py
// (fit_sinhc; times the FP32 mid-cell attenuation 2^(-dl/2) it is within
// 1.5e-7 of phi(x) on [0, 1], checked by the CPU tests).  With it
// e^-tau phi(x) = e^-(tau + x/2) sinh(y) / y: the attenuation to the middle
// of the cell, whose exponent folds into the ray's columns, times an even
// polynomial, one packed multiply and three packed FMAs where the
// polynomial of phi(x) in x took six FMAs.
__device__ __forceinline__ float2 sinhc_half2(float2 dl) {
  constexpr float kShc[4] = {1.f, 0.0200188775f, 0.000120223514f, 3.4621803e-07f};
  const float2 v = __fmul2_rn(dl, dl);
  float2 p = __ffma2_rn(v, make_float2(kShc[3], kShc[3]), make_float2(kShc[2], kShc[2]));
  p = __ffma2_rn(v, p, make_float2(kShc[1], kShc[1]));
  return __ffma2_rn(v, p, make_float2(kShc[0], kShc[0]));
}

// Iterations of ray_bins_packed that may hold a bin with x = sum_s D_s
// sigma_s(nu) >= kPhiXMax: iteration i covers the bins 16 i .. 16 i + 15,
// whose x is at most sum_s D_s max_{k >= 16 i} sigma_s (smax16).  That bound
// does not grow with i, so the iterations that need the SFU path are the
// leading ones; the rest take the polynomial alone.  (A bin whose x lies
// within rounding of 1 may take the polynomial, 1e-7 accurate there.)
__device__ __forceinline__ int sfu_iters(float D0, float D1, float D2) {
  int n = 0;
#pragma unroll
  for (int i = 0; i < kNu / 16; i++)
    n += fmaf(D0, c_tab.smax16[0][i], fmaf(D1, c_tab.smax16[1][i], D2 * c_tab.smax16[2][i])) >= kPhiXMax;
  return n;
}

// A ray's columns as the bin loop uses them, each value in both halves of
// a float2: n = the negated mid-cell columns -(N_s + D_s / 2), d = the
// cell's columns D_s [cm^-2].
struct RayCols2 {
  float2 n[3], d[3];
};
__device__ __forceinline__ RayCols2 ray_cols2(float N0, float N1, float N2, float D0, float D1, float D2) {
  const float N[3] = {N0, N1, N2}, D[3] = {D0, D1, D2};
  RayCols2 c;
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const float m = -fmaf(0.5f, D[q], N[q]);
    c.n[q] = make_float2(m, m);
    c.d[q] = make_float2(D[q], D[q]);
  }
  return c;
}

// One iteration of the bin loop: the bin pair of the lane for one ray.
// ntm = -(tau + x / 2) log2(e) and w = s 2^ntm sinh(x/2)/(x/2).  With kSfu
// and `sfu` (an iteration below the ray's own sfu_iters count) a bin with
// x >= kPhiXMax takes w = s 2^(ntm + dl/2) (1 - 2^-dl) / x instead.  A
// bin's value depends on its own ray alone, whichever other rays share the
// loop's round.  kNS: the species whose cross sections can be non-zero in
// the iteration (1: HI, 2: HI and HeI, 3: all; the others are 0 there and
// their terms would add exact zeros, so the sums are the same bit for bit).
template <bool kSfu, int kNS>
__device__ __forceinline__ void bin_pair(const BinPair &b, float2 s, const RayCols2 &c, float2 (&acc)[6],
                                         bool sfu = false) {
  float2 ntm = __fmul2_rn(c.n[kNS - 1], b.l2e[kNS - 1]);
  float2 dl = __fmul2_rn(c.d[kNS - 1], b.l2e[kNS - 1]);
#pragma unroll
  for (int q = kNS - 2; q >= 0; q--) {
    ntm = __ffma2_rn(c.n[q], b.l2e[q], ntm);
    dl = __ffma2_rn(c.d[q], b.l2e[q], dl);
  }
  const float2 e = make_float2(ex2_approx(ntm.x), ex2_approx(ntm.y));
  float2 w = __fmul2_rn(__fmul2_rn(s, e), sinhc_half2(dl));
  if (kSfu) {
    const bool t0 = !sfu || dl.x < kPhiUMax, t1 = !sfu || dl.y < kPhiUMax;
    if (!(t0 && t1)) {
      const float kLn2 = 0.69314718055994531f;
      const float2 ntl = __ffma2_rn(dl, make_float2(0.5f, 0.5f), ntm);
      const float q0 = s.x * ex2_approx(ntl.x) * __fdividef(1.0f - ex2_approx(-dl.x), dl.x * kLn2);
      const float q1 = s.y * ex2_approx(ntl.y) * __fdividef(1.0f - ex2_approx(-dl.y), dl.y * kLn2);
      w.x = t0 ? w.x : q0;
      w.y = t1 ? w.y : q1;
    }
  }
#pragma unroll
  for (int q = 0; q < kNS; q++) {
    acc[q] = __ffma2_rn(b.l2e[q], w, acc[q]);
    acc[3 + q] = __ffma2_rn(b.l2enu[q], w, acc[3 + q]);
  }
}

// Unroll factor of the polynomial-only iterations (measured at 256^3 / 4096
// sources with two rays per lane: at 8 warps x 2 CTAs, 4 runs the rates 2%
// faster than 2, at 128 registers without spills; at the 96 registers of
// 5 CTAs of 4 warps, 4 spills and 2 does not).
#ifndef ARGOT_RATE_UNROLL
#define ARGOT_RATE_UNROLL 2
#endif
constexpr int kRateUnroll = ARGOT_RATE_UNROLL;

// Iterations [i0, i1) of the bin loop for kR rays (1 or 2) of the lane;
// one load of a table entry serves the kR rays.
template <int kR, bool kSfu, int kNS>
__device__ __forceinline__ void bin_iters(const BinPair *__restrict__ tab, const float2 *const (&sp)[kR], int j,
                                          int i0, int i1, const int (&own)[kR], const RayCols2 (&c)[kR],
                                          float2 (&acc)[kR][6]) {
#pragma unroll(kSfu ? 1 : kRateUnroll)
  for (int i = i0; i < i1; i++) {
    const BinPair b = tab[j + 8 * i];
#pragma unroll
    for (int r = 0; r < kR; r++) bin_pair<kSfu, kNS>(b, __ldg(sp[r] + 8 * i), c[r], acc[r], i < own[r]);
  }
}

// The lane's six partial sums of kR rays (1 or 2) from the columns c; sp:
// the emitters' normalised spectra as bin pairs, offset to the lane; j: the
// lane in the rays' 8-lane group; the first nsfu iterations are compiled
// with the SFU form (the caller passes the same count, the round's largest
// sfu_iters, to the four groups of the warp, so that their loops stay
// converged), which a ray takes in its own first own[r] (its sfu_iters);
// the loop runs in three stretches by the species present (iter_he,
// iter_heii of the tables), in increasing iteration order:
// out[r][s] = sum (sigma_s log2 e) w, out[r][3 + s] = sum (sigma_s log2 e)
// nu w over the lane's bins, w = s_nu e^-tau phi(dtau).  The caller adds the
// eight lanes and forms the rates (ray_rates6).
template <int kR>
__device__ __forceinline__ void ray_bins(const BinPair *__restrict__ tab, const float2 *const (&sp)[kR], int j,
                                         int nsfu, const int (&own)[kR], const RayCols2 (&c)[kR],
                                         float (&out)[kR][6]) {
  float2 acc[kR][6];
#pragma unroll
  for (int r = 0; r < kR; r++)
#pragma unroll
    for (int q = 0; q < 6; q++) acc[r][q] = make_float2(0.f, 0.f);
  constexpr int kIters = kBinPairs / 8;
  const int h1 = c_tab.iter_he, h2 = c_tab.iter_heii;
  const int s1 = min(nsfu, h1), s2 = min(max(nsfu, h1), h2), s3 = max(nsfu, h2);
  bin_iters<kR, true, 1>(tab, sp, j, 0, s1, own, c, acc);
  bin_iters<kR, false, 1>(tab, sp, j, s1, h1, own, c, acc);
  bin_iters<kR, true, 2>(tab, sp, j, h1, s2, own, c, acc);
  bin_iters<kR, false, 2>(tab, sp, j, s2, h2, own, c, acc);
  bin_iters<kR, true, 3>(tab, sp, j, h2, min(s3, kIters), own, c, acc);
  bin_iters<kR, false, 3>(tab, sp, j, s3, kIters, own, c, acc);
#pragma unroll
  for (int r = 0; r < kR; r++)
#pragma unroll
    for (int q = 0; q < 6; q++) out[r][q] = acc[r][q].x + acc[r][q].y;
}

// One ray: columns N (to the cell) and D (of the cell) in cm^-2, sp the
// emitter's normalised spectrum.
__device__ __forceinline__ void ray_bins_packed(const BinPair *__restrict__ tab, const float *__restrict__ sp,
                                                int j, int nsfu, int own, float N0, float N1, float N2, float D0,
                                                float D1, float D2, float (&out)[6]) {
  // the pair's two spectrum bins in one 8-byte load (pair order)
  const float2 *const sp2[1] = {reinterpret_cast<const float2 *>(sp) + j};
  const int own1[1] = {own};
  const RayCols2 c[1] = {ray_cols2(N0, N1, N2, D0, D1, D2)};
  float o[1][6];
  ray_bins<1>(tab, sp2, j, nsfu, own1, c, o);
#pragma unroll
  for (int q = 0; q < 6; q++) out[q] = o[0][q];
}

// Two rays (columns nd = N0, N1, N2, D0, D1, D2 of each, own SFU counts
// owna, ownb): one load of each bin pair of the table serves both rays,
// which halves the shared-memory traffic per ray; nsfu covers both.
__device__ __forceinline__ void ray_bins_packed2(const BinPair *__restrict__ tab, const float *__restrict__ spa,
                                                 const float *__restrict__ spb, int j, int nsfu, int owna,
                                                 int ownb, const float *nda, const float *ndb, float (&outa)[6],
                                                 float (&outb)[6]) {
  const float2 *const sp2[2] = {reinterpret_cast<const float2 *>(spa) + j, reinterpret_cast<const float2 *>(spb) + j};
  const int own[2] = {owna, ownb};
  const RayCols2 c[2] = {ray_cols2(nda[0], nda[1], nda[2], nda[3], nda[4], nda[5]),
                         ray_cols2(ndb[0], ndb[1], ndb[2], ndb[3], ndb[4], ndb[5])};
  float o[2][6];
  ray_bins<2>(tab, sp2, j, nsfu, own, c, o);
#pragma unroll
  for (int q = 0; q < 6; q++) {
    outa[q] = o[0][q];
    outb[q] = o[1][q];
  }
}

// Per-warp scratch of rate_block_f32.
struct RateWarpSmem {
  float nd[32][6];   // N_s, D_s of the chunk's rays (cm^-2)
  float p[32][3];    // prefactors P_s
  float out[32][6];  // per-ray rates
  int e[32], t[32];  // emitter, target lane
  int nsfu[32];      // iterations of the bin loop that may need the SFU path (sfu_iters)
  float acc[12][32]; // per target lane: Kahan sums and compensations (CellSum6Smem)
  int q[32];         // lanes of the chunk's rays that take the quadrature
  int cnt[32], src[32];  // per target lane: rays of the chunk, ray of the round
};

// A cell's six rates summed over its rays in ray order, FP32 with Kahan
// compensation (a cell receives up to a few hundred rays).  CellSum6 keeps
// the sums in registers; CellSum6Smem in the warp's shared memory (word
// [q][lane], conflict-free), which frees twelve registers across the bin
// loop of the rate kernel.
struct CellSum6Smem {
  float (*a)[32];
  int lane;
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int q = 0; q < 12; q++) a[q][lane] = 0.f;
  }
  __device__ __forceinline__ void add(const float *v) {
#pragma unroll
    for (int q = 0; q < 6; q++) {
      float s = a[q][lane], c = a[6 + q][lane];
      kahan_add(s, c, v[q]);
      a[q][lane] = s;
      a[6 + q][lane] = c;
    }
  }
  __device__ __forceinline__ float sum(int q) const { return a[q][lane]; }
};
struct CellSum6 {
  float s[6], c[6];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int q = 0; q < 6; q++) s[q] = c[q] = 0.f;
  }
  __device__ __forceinline__ void add(const float *v) {
#pragma unroll
    for (int q = 0; q < 6; q++) kahan_add(s[q], c[q], v[q]);
  }
  __device__ __forceinline__ float sum(int q) const { return s[q]; }
};

// Phase C of the block-rate kernels: lane k holds ray k of a chunk (its six
// values in out[k], its target lane t, -1 for none); every lane adds the
// rays that end in its cell, in ray order.  __match_any_sync ranks each ray
// among the chunk's rays with the same target; round r hands every cell
// its rank-r ray through `src`, so a chunk whose rays end in distinct cells
// takes one round (instead of every lane scanning the chunk's 32 rays).
template <class Acc>
__device__ __forceinline__ void add_chunk_in_order(Acc &acc, int lane, int t, const float (*out)[6], int *cnt,
                                                   int *src) {
  const unsigned same = __match_any_sync(0xffffffffu, t);
  const int rank = __popc(same & ((1u << lane) - 1u));
  cnt[lane] = 0;
  __syncwarp();
  if (t >= 0 && rank == 0) cnt[t] = __popc(same);
  const int rounds = __reduce_max_sync(0xffffffffu, t >= 0 ? rank + 1 : 0);
  __syncwarp();
  const int mine = cnt[lane];
  for (int r = 0; r < rounds; r++) {
    if (t >= 0 && rank == r) src[t] = lane;
    __syncwarp();
    if (r < mine) acc.add(out[src[lane]]);
    __syncwarp();
  }
}

// The FP32 rates of one target block b whose rays are [r0, r1) of `rays`
// (columns in three planes of nray), written to its cells in rates6; one
// warp.  Phase A: per-ray parameters (ray_params_f32), one lane per ray, 32
// rays at a time.  Phase B: four 8-lane groups, one ray each, over the bin
// pairs (ray_bins_packed; with kRaysPerLane 2, two rays per group,
// ray_bins_packed2), three butterfly steps.  Phase C: lane j adds the
// rays of cell j of the block in ray order (add_chunk_in_order).
// kServed: `pred` holds 7 planes of nray floats, six per-ray contributions
// and a flag; a ray whose flag is non-zero contributes those six values
// and skips the quadrature, which runs over the remaining rays of the
// chunk only (the surrogate's fallback).
template <bool kServed = false, int kRaysPerLane = 1>
__device__ __forceinline__ void rate_block_f32(const GridDev &g, const float4 *__restrict__ raw,
                                               const float4 *__restrict__ emit_pos, const float *__restrict__ specn,
                                               const double *__restrict__ total, const BinPair *__restrict__ pairs,
                                               uint64_t b, uint64_t r0, uint64_t r1,
                                               const uint32_t *__restrict__ rays, uint64_t nray,
                                               const float *__restrict__ tau, float *__restrict__ rates6,
                                               RateWarpSmem &S, int lane, const float *__restrict__ pred = nullptr) {
  const int grp = lane >> 3, j = lane & 7;
  const unsigned gmask = 0xffu << (8 * grp);
  const uint64_t ncell = (uint64_t)g.nx * g.ny * g.nz;
  int ix, iy, iz;
  const bool own_valid = block_cell(g, b, lane, &ix, &iy, &iz);
  const uint64_t own = own_valid ? cell_index(g, ix, iy, iz) : 0;
  CellSum6Smem acc{S.acc, lane};
  acc.zero();
  int bix, biy, biz;
  block_cell(g, b, 0, &bix, &biy, &biz);
  for (uint64_t rc = r0; rc < r1; rc += 32) {
    const uint64_t r = rc + lane;
    int t = -1;
    bool quad = false;
    if (r < r1) {
      const uint32_t w = __ldg(rays + r);
      const uint32_t e = w >> 5;
      t = (int)(w & 31u);
      if (kServed && __ldg(pred + 6 * nray + r) != 0.f) {
#pragma unroll
        for (int s = 0; s < 6; s++) S.out[lane][s] = __ldg(pred + s * nray + r);
      } else {
        quad = true;
        const int lx = bix + (t >> 4), ly = biy + ((t >> 2) & 3), lz = biz + (t & 3);
        const float4 ep = __ldg(emit_pos + e);
        const float4 rw = __ldg(raw + cell_index(g, lx, ly, lz));
        const RayParams p = ray_params_f32(g, g.ix0 + lx, g.iy0 + ly, g.iz0 + lz, ep.x, ep.y, ep.z, __ldg(tau + r),
                                           __ldg(tau + nray + r), __ldg(tau + 2 * nray + r), rw, __ldg(total + e));
#pragma unroll
        for (int s = 0; s < 3; s++) {
          S.nd[lane][s] = p.N[s];
          S.nd[lane][3 + s] = p.D[s];
          S.p[lane][s] = p.P[s];
        }
        S.e[lane] = (int)e;
        S.nsfu[lane] = sfu_iters(p.D[0], p.D[1], p.D[2]);
      }
    }
    S.t[lane] = t;
    const int nk = (int)min((uint64_t)32, r1 - rc);
    int nq = nk;
    if (kServed) {
      const unsigned m = __ballot_sync(0xffffffffu, quad);
      if (quad) S.q[__popc(m & ((1u << lane) - 1u))] = lane;
      nq = __popc(m);
    }
    __syncwarp();
    // rounds of four (eight) rays, one (two) per group; the groups of a
    // round run the same bin loop (the largest SFU count of the round), so
    // that the warp stays converged; a group without a ray in the last
    // round repeats the round's first ray and discards it
    static_assert(kRaysPerLane == 1 || kRaysPerLane == 2, "one or two rays per lane");
    if constexpr (kRaysPerLane == 2) {
      for (int i0 = 0; i0 < nq; i0 += 8) {
        const int ia = i0 + grp < nq ? i0 + grp : i0, ib = i0 + 4 + grp < nq ? i0 + 4 + grp : i0;
        const int qa = kServed ? S.q[ia] : ia, qb = kServed ? S.q[ib] : ib;
        int nsfu = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) nsfu = max(nsfu, i0 + k < nq ? S.nsfu[kServed ? S.q[i0 + k] : i0 + k] : 0);
        float pa[6], pb[6];
        ray_bins_packed2(pairs, specn + (size_t)S.e[qa] * kNu, specn + (size_t)S.e[qb] * kNu, j, nsfu, S.nsfu[qa],
                         S.nsfu[qb], S.nd[qa], S.nd[qb], pa, pb);
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
#pragma unroll
          for (int s = 0; s < 6; s++) {
            pa[s] += __shfl_xor_sync(gmask, pa[s], o);
            pb[s] += __shfl_xor_sync(gmask, pb[s], o);
          }
        }
        if (j == 0) {
          float out[6];
          if (i0 + grp < nq) {
            const float P[3] = {S.p[qa][0], S.p[qa][1], S.p[qa][2]};
            ray_rates6(P, pa[0], pa[1], pa[2], pa[3], pa[4], pa[5], out);
#pragma unroll
            for (int s = 0; s < 6; s++) S.out[qa][s] = out[s];
          }
          if (i0 + 4 + grp < nq) {
            const float P[3] = {S.p[qb][0], S.p[qb][1], S.p[qb][2]};
            ray_rates6(P, pb[0], pb[1], pb[2], pb[3], pb[4], pb[5], out);
#pragma unroll
            for (int s = 0; s < 6; s++) S.out[qb][s] = out[s];
          }
        }
      }
    } else {
      for (int i0 = 0; i0 < nq; i0 += 4) {
        const int i = i0 + grp < nq ? i0 + grp : i0;
        const int q = kServed ? S.q[i] : i;
        int nsfu = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) nsfu = max(nsfu, i0 + k < nq ? S.nsfu[kServed ? S.q[i0 + k] : i0 + k] : 0);
        float part[6];
        ray_bins_packed(pairs, specn + (size_t)S.e[q] * kNu, j, nsfu, S.nsfu[q], S.nd[q][0], S.nd[q][1], S.nd[q][2],
                        S.nd[q][3], S.nd[q][4], S.nd[q][5], part);
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
#pragma unroll
          for (int s = 0; s < 6; s++) part[s] += __shfl_xor_sync(gmask, part[s], o);
        }
        if (j == 0 && i0 + grp < nq) {
          const float P[3] = {S.p[q][0], S.p[q][1], S.p[q][2]};
          float out[6];
          ray_rates6(P, part[0], part[1], part[2], part[3], part[4], part[5], out);
#pragma unroll
          for (int s = 0; s < 6; s++) S.out[q][s] = out[s];
        }
      }
    }
    __syncwarp();
    add_chunk_in_order(acc, lane, t, S.out, S.cnt, S.src);
  }
  if (own_valid) {
#pragma unroll
    for (int s = 0; s < 6; s++) rates6[s * ncell + own] = acc.sum(s);
  }
}

}  // namespace argot
