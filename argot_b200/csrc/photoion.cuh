// photoion.cuh -- per-ray photo-ionisation / heating rates
// (calc_photoion_rate, photon-conserving branch, H + He, not cosmological).
#pragma once
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
  ARGOT_CUDA_TRY(cudaMemcpyToSymbol(c_tab, &t, sizeof(t)));
  done[device] = true;
  return 0;
}

// Geometry shared by both precisions (calc_photoion_rate.c:176-246, FP32
// where the reference uses float): target centre, distance, and the cell
// chord `delta` along the ray (delta_length, :52-90).
struct RayGeom {
  float dist, delta;
};

__device__ __forceinline__ RayGeom ray_geometry(const GridDev &g, int gix, int giy, int giz, float sx,
                                                float sy, float sz) {
  // x = delta_x*((float)ix + 0.5) + xmin, in double, stored as float
  const float x = __double2float_rn(__dadd_rn(__dmul_rn((double)g.dx, __dadd_rn((double)__int2float_rn(gix), 0.5)), (double)g.xmin));
  const float y = __double2float_rn(__dadd_rn(__dmul_rn((double)g.dy, __dadd_rn((double)__int2float_rn(giy), 0.5)), (double)g.ymin));
  const float z = __double2float_rn(__dadd_rn(__dmul_rn((double)g.dz, __dadd_rn((double)__int2float_rn(giz), 0.5)), (double)g.zmin));
  const float dx = __fsub_rn(x, sx), dy = __fsub_rn(y, sy), dz = __fsub_rn(z, sz);
  const float sxy = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
  const float s3 = __fadd_rn(sxy, __fmul_rn(dz, dz));
  const float dl = __double2float_rn(__dsqrt_rn(__dadd_rn((double)s3, kTiny)));
  const float dxy = __double2float_rn(__dsqrt_rn(__dadd_rn((double)sxy, kTiny)));
  const float ct = __fdiv_rn(dz, dl), st = __fdiv_rn(dxy, dl);
  const float cp = __fdiv_rn(dx, dxy), sp = __fdiv_rn(dy, dxy);
  const float xo = cosine_guard(__fmul_rn(cp, st));
  const float yo = cosine_guard(__fmul_rn(sp, st));
  const float zo = cosine_guard(ct);
  const float rx = fabsf(__fdiv_rn(g.dx, xo)), ry = fabsf(__fdiv_rn(g.dy, yo)), rz = fabsf(__fdiv_rn(g.dz, zo));
  RayGeom r;
  r.delta = fminf(rx, fminf(ry, rz));
  r.dist = __double2float_rn(__dsqrt_rn((double)s3));
  return r;
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

// (1 - e^-x)/x.  Below x = 0.1 the difference 1 - e^-x cancels, so the
// value is taken in FP64 from its Taylor series (error < x^6/5040 < 2e-10);
// above, FP32 with the hardware exponential is accurate to ~3e-6.
__device__ __forceinline__ float phi_pc(float x, float e_minus_x) {
  if (x < 0.1f) {
    const double d = (double)x;
    double p = fma(d, -1.0 / 720.0, 1.0 / 120.0);
    p = fma(d, p, -1.0 / 24.0);
    p = fma(d, p, 1.0 / 6.0);
    p = fma(d, p, -0.5);
    p = fma(d, p, 1.0);
    return (float)p;
  }
  return __fdividef(1.0f - e_minus_x, x);
}

// Per-ray parameters of the FP32 bin loop: columns to the cell's entry face
// and of the cell [cm^-2] as floats, and the FP64 prefactors
// total * dN_s / (n_s V_shell) of the three species.
struct RayParams {
  float N[3], D[3];
  double P[3];
};

__device__ __forceinline__ RayParams ray_params(const RayCols &c, double total) {
  RayParams p;
#pragma unroll
  for (int s = 0; s < 3; s++) {
    p.N[s] = (float)c.N[s];
    p.D[s] = (float)c.dN[s];
    p.P[s] = total * c.dN[s] * c.rN[s];
  }
  return p;
}

// FP32 rates: the same integral with the spectrum normalised by its total
// (FP32 cannot hold photon rates of 1e50 or rates of 1e-58) and the FP64
// per-ray prefactor total * dN_s * rN_s applied once.  Sums run in FP32 over
// 32 bins and are carried in FP64 across blocks of bins.
static __device__ __noinline__ void rate_bins_f32(const RayCols &c, const float *__restrict__ specn, double total,
                                           double out[6]) {
  const float N0 = (float)c.N[0], N1 = (float)c.N[1], N2 = (float)c.N[2];
  const float D0 = (float)c.dN[0], D1 = (float)c.dN[1], D2 = (float)c.dN[2];
  const float ln2 = 0.69314718055994531f;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int k0 = 0; k0 < kNu; k0 += 32) {
    float g0 = 0.f, g1 = 0.f, g2 = 0.f, h0 = 0.f, h1 = 0.f, h2 = 0.f;
#pragma unroll 8
    for (int k = k0; k < k0 + 32; k++) {
      const float a0 = c_tab.cs_l2e[0][k], a1 = c_tab.cs_l2e[1][k], a2 = c_tab.cs_l2e[2][k];
      const float tl2 = fmaf(N0, a0, fmaf(N1, a1, N2 * a2));
      const float dl2 = fmaf(D0, a0, fmaf(D1, a1, D2 * a2));
      const float e = ex2_approx(-tl2);
      const float ed = ex2_approx(-dl2);
      const float w = __ldg(specn + spec_pair_index(k)) * e * phi_pc(dl2 * ln2, ed);
      g0 = fmaf(c_tab.cs[0][k], w, g0);
      g1 = fmaf(c_tab.cs[1][k], w, g1);
      g2 = fmaf(c_tab.cs[2][k], w, g2);
      h0 = fmaf(c_tab.hw[0][k], w, h0);
      h1 = fmaf(c_tab.hw[1][k], w, h1);
      h2 = fmaf(c_tab.hw[2][k], w, h2);
    }
    acc[0] += g0; acc[1] += g1; acc[2] += g2;
    acc[3] += h0; acc[4] += h1; acc[5] += h2;
  }
#pragma unroll
  for (int s = 0; s < 3; s++) {
    const double p = total * c.dN[s] * c.rN[s];
    out[s] = p * acc[s];
    out[3 + s] = p * acc[3 + s] * kHNuL;
  }
}

// ---- packed FP32 bin loop: two bins per instruction with the f32x2 FMA
// and multiply of sm_100.  An 8-lane group integrates one ray; lane j owns
// the bin pairs (j + 16 i, j + 16 i + 8), i = 0..15 (the bins j + 8 m), and
// keeps one partial sum per output and pair member.  Aligned to 16 bytes so
// that a lane reads its pair with five 16-byte shared loads (measured: rates
// 2% faster than with the 8-byte alignment of float2).
struct alignas(16) BinPair {
  float2 l2e[3];  // sigma_s log2(e) of the two bins
  float2 cs[3];   // sigma_s
  float2 hw[3];   // sigma_s ((float) nu - nu_s)^+
  float2 pad;     // 80 B: the eight lanes of a group hit distinct banks
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
      b.cs[s] = make_float2(c_tab.cs[s][k0], c_tab.cs[s][k1]);
      b.hw[s] = make_float2(c_tab.hw[s][k0], c_tab.hw[s][k1]);
    }
    b.pad = make_float2(0.f, 0.f);
    tab[p] = b;
  }
}

// phi_pc of dl2 = dtau log2(e), with e^-dtau evaluated only where it is
// used (dtau >= 0.1): same values as phi_pc, one exponential fewer in the
// thin bins.
__device__ __forceinline__ float phi_pc_lazy(float dl2) {
  const float x = dl2 * 0.69314718055994531f;
  if (x < 0.1f) return phi_pc(x, 0.f);
  return phi_pc(x, ex2_approx(-dl2));
}

// The lane's six partial sums (Gamma then heating of HI, HeI, HeII) of one
// ray with columns N (to the cell) and D (of the cell) in cm^-2; sp: the
// emitter's normalised spectrum.  The caller adds the eight lanes.
__device__ __forceinline__ void ray_bins_packed(const BinPair *__restrict__ tab, const float *__restrict__ sp,
                                                int j, float N0, float N1, float N2, float D0, float D1, float D2,
                                                float (&out)[6]) {
  const float2 n0 = make_float2(N0, N0), n1 = make_float2(N1, N1), n2 = make_float2(N2, N2);
  const float2 d0 = make_float2(D0, D0), d1 = make_float2(D1, D1), d2 = make_float2(D2, D2);
  float2 acc[6];
#pragma unroll
  for (int q = 0; q < 6; q++) acc[q] = make_float2(0.f, 0.f);
#pragma unroll 4
  for (int i = 0; i < kBinPairs / 8; i++) {
    const BinPair &b = tab[j + 8 * i];
    const float2 l0 = b.l2e[0], l1 = b.l2e[1], l2 = b.l2e[2];
    const float2 c0 = b.cs[0], c1 = b.cs[1], c2 = b.cs[2];
    const float2 w0 = b.hw[0], w1 = b.hw[1], w2 = b.hw[2];
    const float2 tl = __ffma2_rn(n0, l0, __ffma2_rn(n1, l1, __fmul2_rn(n2, l2)));
    const float2 dl = __ffma2_rn(d0, l0, __ffma2_rn(d1, l1, __fmul2_rn(d2, l2)));
    // the pair's two spectrum bins in one 8-byte load (pair order)
    const float2 s = __ldg(reinterpret_cast<const float2 *>(sp) + j + 8 * i);
    const float2 e = make_float2(ex2_approx(-tl.x), ex2_approx(-tl.y));
    const float2 ph = make_float2(phi_pc_lazy(dl.x), phi_pc_lazy(dl.y));
    const float2 w = __fmul2_rn(__fmul2_rn(s, e), ph);
    acc[0] = __ffma2_rn(c0, w, acc[0]);
    acc[1] = __ffma2_rn(c1, w, acc[1]);
    acc[2] = __ffma2_rn(c2, w, acc[2]);
    acc[3] = __ffma2_rn(w0, w, acc[3]);
    acc[4] = __ffma2_rn(w1, w, acc[4]);
    acc[5] = __ffma2_rn(w2, w, acc[5]);
  }
#pragma unroll
  for (int q = 0; q < 6; q++) out[q] = acc[q].x + acc[q].y;
}

// Per-warp scratch of rate_block_f32.
struct RateWarpSmem {
  float nd[32][6];    // N_s, dN_s of the chunk's rays (cm^-2)
  double p[32][3];    // prefactors
  double out[32][6];  // per-ray rates
  int e[32], t[32];   // emitter, target lane
  int q[32];          // lanes of the chunk's rays that take the quadrature
};

// The FP32 rates of one target block b whose rays are [r0, r1) of `rays`
// (columns in three planes of nray), written to its cells in rates6; one
// warp.  Phase A: per-ray parameters, one lane per ray, 32 rays at a time.
// Phase B: four 8-lane groups, one ray each, over the bin pairs
// (ray_bins_packed), three butterfly steps.  Phase C: lane j adds the rays
// of cell j of the block in ray order.
// kServed: `pred` holds 7 planes of nray floats, six per-ray contributions
// and a flag; a ray whose flag is non-zero contributes those six values
// and skips the quadrature, which runs over the remaining rays of the
// chunk only (the surrogate's fallback).
template <bool kServed = false>
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
  double acc[6] = {0, 0, 0, 0, 0, 0};
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
        for (int s = 0; s < 6; s++) S.out[lane][s] = (double)__ldg(pred + s * nray + r);
      } else {
        quad = true;
        const int lx = bix + (t >> 4), ly = biy + ((t >> 2) & 3), lz = biz + (t & 3);
        const float4 ep = __ldg(emit_pos + e);
        const RayGeom geo = ray_geometry(g, g.ix0 + lx, g.iy0 + ly, g.iz0 + lz, ep.x, ep.y, ep.z);
        const float4 rw = __ldg(raw + cell_index(g, lx, ly, lz));
        const RayCols cols = ray_columns(g, __ldg(tau + r), __ldg(tau + nray + r), __ldg(tau + 2 * nray + r), rw, geo);
        const RayParams p = ray_params(cols, __ldg(total + e));
#pragma unroll
        for (int s = 0; s < 3; s++) {
          S.nd[lane][s] = p.N[s];
          S.nd[lane][3 + s] = p.D[s];
          S.p[lane][s] = p.P[s];
        }
        S.e[lane] = (int)e;
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
    for (int i = grp; i < nq; i += 4) {
      const int q = kServed ? S.q[i] : i;
      float part[6];
      ray_bins_packed(pairs, specn + (size_t)S.e[q] * kNu, j, S.nd[q][0], S.nd[q][1], S.nd[q][2], S.nd[q][3],
                      S.nd[q][4], S.nd[q][5], part);
      float g0 = part[0], g1 = part[1], g2 = part[2], h0 = part[3], h1 = part[4], h2 = part[5];
#pragma unroll
      for (int o = 1; o < 8; o <<= 1) {
        g0 += __shfl_xor_sync(gmask, g0, o);
        g1 += __shfl_xor_sync(gmask, g1, o);
        g2 += __shfl_xor_sync(gmask, g2, o);
        h0 += __shfl_xor_sync(gmask, h0, o);
        h1 += __shfl_xor_sync(gmask, h1, o);
        h2 += __shfl_xor_sync(gmask, h2, o);
      }
      if (j == 0) {
        const double p0 = S.p[q][0], p1 = S.p[q][1], p2 = S.p[q][2];
        S.out[q][0] = p0 * g0;
        S.out[q][1] = p1 * g1;
        S.out[q][2] = p2 * g2;
        S.out[q][3] = p0 * h0 * kHNuL;
        S.out[q][4] = p1 * h1 * kHNuL;
        S.out[q][5] = p2 * h2 * kHNuL;
      }
    }
    __syncwarp();
    for (int k = 0; k < nk; k++) {
      if (S.t[k] == lane) {
#pragma unroll
        for (int s = 0; s < 6; s++) acc[s] += S.out[k][s];
      }
    }
    __syncwarp();
  }
  if (own_valid) {
#pragma unroll
    for (int s = 0; s < 6; s++) rates6[s * ncell + own] = (float)acc[s];
  }
}

}  // namespace argot
