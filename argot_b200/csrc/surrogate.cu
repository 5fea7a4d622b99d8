// surrogate.cu -- per-cell rates with the BF16 MLP surrogate of the
// frequency integral, evaluated on the tensor cores, and the exact FP32
// quadrature as fallback.
//
// Photon-conserving cell factor.  For every frequency
//   e^{-tau} (1 - e^{-dtau}) / dtau = int_0^1 e^{-(tau + u dtau)} du,
// so the reference's sum over bins (calc_photoion_rate.c:327-386) equals
//   Gamma_s = P_s int_0^1 I_s(N + u dN) du,  P_s = Ndot dN_s / (n_s V_shell),
// with I_j(M) the thin-cell integral of mlp.cuh at column M.  The integral
// over u is taken by Gauss-Legendre quadrature with 1, 2 or 3 nodes chosen
// from the cell's largest optical depth dtau_max (relative error below
// dtau^2/24, dtau^4/4320 and dtau^6/2016000: < 4e-5 at the switch points);
// the network gives I_j / I_j0 at each node and the emitter's exact thin
// integrals I_j0 restore the scale.
//
// Error control per cell.  Kernel 1 predicts every ray's six contributions
// c_j with a relative error bound eps (from the validated envelope of the
// network's error, measured on held-out samples) and a lower bound S_j of
// each cell's total (each ray's true sum is at least I^ e^-x per node).
// Kernel 2 keeps the predictions of the rays with the smallest shares
// beta = eps max_j c_j / S_j while their sum stays within the cell's budget
// tol, so that the surrogate's error is at most tol S_j per cell and
// output; kernel 3 (the FP32 rate kernel) runs the exact quadrature for the
// other rays and sums the cells.  A ray always
// takes the exact quadrature when its emitter is not a single-temperature
// blackbody in [1e4, 10^5.5] K, when dtau_max > 2, or when a node's
// log10 tau lies above 3.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "mlp.cuh"
#include "photoion.cuh"

namespace argot {

int grid_blocks_for_rates(uint64_t n, int threads);
int launch_rate_f32_served(const GridDev &g, const float4 *raw, const float4 *emit_pos, const float *specn,
                           const double *total, uint64_t b0, uint64_t b1, const uint64_t *blk_off, uint64_t base,
                           const uint32_t *rays, uint64_t nray, const float *tau, float *rates6, const float *pred,
                           int *err, cudaStream_t st);
int *err_flag(int dev);

constexpr int kEnvBins = 64;        // error envelope bins over predicted q
constexpr float kEnvQLo = -7.0f;     // ... in [-7, 0]
constexpr int kHistBins = 64;        // half-octave bins of a ray's budget share
constexpr float kGLErr = 4e-5f;      // relative error of the Gauss-Legendre cell factor
constexpr int kWorkPlanes = 7;       // c_0..c_5, eps per ray
constexpr int kSurWarps = 4;
constexpr int kMaxEval = 96;  // 32 rays x 3 quadrature nodes

// B-fragments of the four layers (mma.m16n8k16, BF16), biases, envelope.
struct SurWeights {
  uint2 f1[8][32];        // layer 1: 8 N-tiles x 1 K-step (input hi|lo in k 0..7)
  uint2 f2[8][4][32];     // layer 2: 8 N-tiles x 4 K-steps
  uint2 f3[8][4][32];     // layer 3
  uint2 f4[8][32];        // layer 4: 1 N-tile x 8 K-steps (hidden hi | lo)
  float b1[64], b2[64], b3[64], b4[8];
  float env[6][kEnvBins]; // e^dq - 1, dq the bound of |error of q| per output and bin of q^
  float sig0[3];
  float tol;              // per-cell relative error budget
};

struct PredSmem {
  SurWeights w;
  // per warp
  float x[kSurWarps][kMaxEval][4];     // normalised network inputs
  float tout[kSurWarps][kMaxEval][6];  // network outputs q_j
  float c[kSurWarps][32][6];           // predicted per-ray contributions
  int t[kSurWarps][32];
};

struct SelSmem {
  // per warp
  float Sc[kSurWarps][32][6];                // lower bounds of the cell totals
  unsigned hist[kSurWarps][32][kHistBins];   // budget-share histogram per cell
  int thr[kSurWarps][32];                    // last accepted bin per cell
};

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint2 b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

// x -> BF16 pair (hi, lo) with hi + lo = x to 16 mantissa bits, packed two
// values per register as the mma fragments want them.
__device__ __forceinline__ void split_bf16x2(float x0, float x1, uint32_t *hi, uint32_t *lo) {
  const float h0 = bf16_round(x0), h1 = bf16_round(x1);
  *hi = pack_bf16x2(h0, h1);
  *lo = pack_bf16x2(x0 - h0, x1 - h1);
}

// SiLU of the 8 accumulator values of two N-tiles, in fragment order (the
// single-precision hardware tanh: a packed half-precision tanh was measured
// no faster here and less accurate).
__device__ __forceinline__ void silu8(const float (&a)[4], const float (&b)[4], float (&s)[8]) {
#pragma unroll
  for (int i = 0; i < 4; i++) {
    s[i] = silu_acc(a[i]);
    s[4 + i] = silu_acc(b[i]);
  }
}

// The network on 16 evaluations (rows r0..r0+15 of the warp's list).  The
// m16n8 accumulator of one layer is, register for register, the A fragment
// of the next (N-tiles 2kk, 2kk+1 -> K-step kk), so activations never leave
// the registers.
__device__ __forceinline__ void mlp_tile16(const SurWeights &W, const float (*x)[4], float (*tout)[6],
                                           int r0, int lane) {
  const int g = lane >> 2, tq = lane & 3;
  // layer 1: A = [hi(x) | lo(x) | 0] (k = 0..3 | 4..7 | 8..15)
  uint32_t a[4];
  {
    const int c0 = (2 * tq) & 3;  // columns 2tq, 2tq+1 of the 8 used
    const bool lo = tq >= 2;
    float v[4];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const float *xr = x[r0 + g + 8 * h];
      const float x0 = xr[c0], x1 = xr[c0 + 1];
      const float h0 = bf16_round(x0), h1 = bf16_round(x1);
      v[2 * h + 0] = lo ? x0 - h0 : h0;
      v[2 * h + 1] = lo ? x1 - h1 : h1;
    }
    a[0] = pack_bf16x2(v[0], v[1]);
    a[1] = pack_bf16x2(v[2], v[3]);
    a[2] = 0u;
    a[3] = 0u;
  }
  float acc[8][4];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const float bb0 = W.b1[8 * j + 2 * tq], bb1 = W.b1[8 * j + 2 * tq + 1];
    acc[j][0] = bb0; acc[j][1] = bb1; acc[j][2] = bb0; acc[j][3] = bb1;
    mma_bf16(acc[j], a, W.f1[j][lane]);
  }
  // layers 2 and 3: each activation as a BF16 pair hi + lo, both against
  // the same weight fragment
#pragma unroll
  for (int layer = 0; layer < 2; layer++) {
    uint32_t Ah[4][4], Al[4][4];
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
      float s[8];
      silu8(acc[2 * kk], acc[2 * kk + 1], s);
#pragma unroll
      for (int q = 0; q < 4; q++) split_bf16x2(s[2 * q], s[2 * q + 1], &Ah[kk][q], &Al[kk][q]);
    }
    const float *bias = layer == 0 ? W.b2 : W.b3;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const float bb0 = bias[8 * j + 2 * tq], bb1 = bias[8 * j + 2 * tq + 1];
      acc[j][0] = bb0; acc[j][1] = bb1; acc[j][2] = bb0; acc[j][3] = bb1;
#pragma unroll
      for (int kk = 0; kk < 4; kk++) {
        const uint2 bf = layer == 0 ? W.f2[j][kk][lane] : W.f3[j][kk][lane];
        mma_bf16(acc[j], Ah[kk], bf);
        mma_bf16(acc[j], Al[kk], bf);
      }
    }
  }
  // layer 4 on the last hidden layer split as hi | lo
  float o[4] = {W.b4[2 * tq], W.b4[2 * tq + 1], W.b4[2 * tq], W.b4[2 * tq + 1]};
#pragma unroll
  for (int kk = 0; kk < 4; kk++) {
    float s[8];
    silu8(acc[2 * kk], acc[2 * kk + 1], s);
    uint32_t hi[4], lo[4];
#pragma unroll
    for (int q = 0; q < 4; q++) split_bf16x2(s[2 * q], s[2 * q + 1], &hi[q], &lo[q]);
    mma_bf16(o, hi, W.f4[kk][lane]);
    mma_bf16(o, lo, W.f4[4 + kk][lane]);
  }
  if (tq < 3) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      tout[r0 + g + 8 * h][2 * tq] = fmaf(o[2 * h], kOutScale, kOutShift);
      tout[r0 + g + 8 * h][2 * tq + 1] = fmaf(o[2 * h + 1], kOutScale, kOutShift);
    }
  }
}

// Gauss-Legendre nodes and weights on [0, 1]
__device__ __forceinline__ void gl_node(int n, int i, float *u, float *w) {
  if (n == 1) { *u = 0.5f; *w = 1.f; return; }
  if (n == 2) { *u = i ? 0.78867513459481287f : 0.21132486540518713f; *w = 0.5f; return; }
  const float uu[3] = {0.11270166537925831f, 0.5f, 0.88729833462074169f};
  const float ww[3] = {5.f / 18.f, 8.f / 18.f, 5.f / 18.f};
  *u = uu[i];
  *w = ww[i];
}

// Phase A of both kernels: the ray's target lane, emitter and rate
// parameters (columns at cell entry N_s, cell columns D_s, prefactors P_s).
struct RayTask {
  int tl, e;
  RayParams p;
};
__device__ __forceinline__ RayTask ray_task(const GridDev &g, const float4 *__restrict__ raw,
                                            const float4 *__restrict__ emit_pos, const double *__restrict__ total,
                                            const uint32_t *__restrict__ rays, const float *__restrict__ tau,
                                            uint64_t nray, uint64_t r, int bix, int biy, int biz) {
  RayTask t;
  const uint32_t w = __ldg(rays + r);
  t.e = (int)(w >> 5);
  t.tl = (int)(w & 31u);
  const int lx = bix + (t.tl >> 4), ly = biy + ((t.tl >> 2) & 3), lz = biz + (t.tl & 3);
  const float4 ep = __ldg(emit_pos + t.e);
  const float4 rw = __ldg(raw + cell_index(g, lx, ly, lz));
  t.p = ray_params_f32(g, g.ix0 + lx, g.iy0 + ly, g.iz0 + lz, ep.x, ep.y, ep.z, __ldg(tau + r), __ldg(tau + nray + r),
                       __ldg(tau + 2 * nray + r), rw, __ldg(total + t.e));
  return t;
}

// Kernel 1 of the surrogate rates: for every ray of blocks [b0, b1) the
// network's prediction of its six contributions c_j and a relative error
// bound eps (work planes 0..5 and 6; eps = +inf for a ray that must take
// the exact quadrature), and per cell a lower bound S_j of the true total
// of its surrogate-capable rays (written to rates6, which kernel 2
// overwrites).
//
// Error bound of one ray: at quadrature node i the network's q has the
// validated error bound dq = env_j(q^) (largest error on held-out samples in
// bins of predicted q, times a safety factor), so with y^ = ylin e^q^,
// |y - y^| <= |y^| (e^dq - 1) = x and |I - I^| <= I^ (e^x - 1) <= I^ x e^x;
// the node bounds add up over the nodes.
// Launch shapes: kSurWarps warps per CTA, at least ARGOT_SUR_PREDICT_MIN_CTAS
// and ARGOT_SUR_FINISH_MIN_CTAS CTAs resident per SM (register caps).
#ifndef ARGOT_SUR_PREDICT_MIN_CTAS
#define ARGOT_SUR_PREDICT_MIN_CTAS 4
#endif
#ifndef ARGOT_SUR_FINISH_MIN_CTAS
#define ARGOT_SUR_FINISH_MIN_CTAS 1
#endif
__global__ void __launch_bounds__(32 * kSurWarps, ARGOT_SUR_PREDICT_MIN_CTAS)
    k_sur_predict(GridDev g, const float4 *__restrict__ raw, const float4 *__restrict__ emit_pos,
                  const double *__restrict__ total, const float *__restrict__ emit_logT,
                  const double *__restrict__ emit_i0, const float *__restrict__ emit_m,
                  const SurWeights *__restrict__ wts, uint64_t b0, uint64_t b1, const uint64_t *__restrict__ blk_off,
                  uint64_t base, const uint32_t *__restrict__ rays, uint64_t nray, const float *__restrict__ tau,
                  float *__restrict__ rates6, float *__restrict__ work, int *__restrict__ err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PredSmem &S = *reinterpret_cast<PredSmem *>(smem_raw);
  {
    const uint32_t *src = reinterpret_cast<const uint32_t *>(wts);
    uint32_t *dst = reinterpret_cast<uint32_t *>(&S.w);
    for (int i = threadIdx.x; i < (int)(sizeof(SurWeights) / 4); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const float s00 = c_tab.cs[0][0];
  const float s0a = c_tab.cs[0][44], s1a = c_tab.cs[1][44];
  const float s0b = c_tab.cs[0][103], s1b = c_tab.cs[1][103], s2b = c_tab.cs[2][103];
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarp = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t ncell = (uint64_t)g.nx * g.ny * g.nz;
  const float kInf = __int_as_float(0x7f800000);
  for (uint64_t b = b0 + warp; b < b1; b += nwarp) {
    int ix, iy, iz;
    const bool own_valid = block_cell(g, b, lane, &ix, &iy, &iz);
    const uint64_t own = own_valid ? cell_index(g, ix, iy, iz) : 0;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    int bix, biy, biz;
    block_cell(g, b, 0, &bix, &biy, &biz);
    uint64_t r0, r1;
    if (!block_rays(blk_off, b, base, nray, &r0, &r1)) {
      if (lane == 0) atomicExch(err, 1);
      continue;
    }
    for (uint64_t rc = r0; rc < r1; rc += 32) {
      // ---- phase A: per-ray parameters and quadrature nodes
      const uint64_t r = rc + lane;
      int tl = -1, nq = 0, e = 0;
      RayParams p;
      float xin[3][4];
      if (r < r1) {
        const RayTask t = ray_task(g, raw, emit_pos, total, rays, tau, nray, r, bix, biy, biz);
        tl = t.tl;
        e = t.e;
        p = t.p;
        const float lT = __ldg(emit_logT + e);
        const float dt0 = p.D[0] * s00;
        const float dt1 = fmaf(p.D[0], s0a, p.D[1] * s1a);
        const float dt2 = fmaf(p.D[0], s0b, fmaf(p.D[1], s1b, p.D[2] * s2b));
        const float dtm = fmaxf(dt0, fmaxf(dt1, dt2));
        nq = (lT >= kTLo && lT <= kTHi) ? (dtm <= 0.02f ? 1 : dtm <= 0.5f ? 2 : dtm <= 2.f ? 3 : 0) : 0;
        for (int i = 0; i < nq; i++) {
          float u, wq;
          gl_node(nq, i, &u, &wq);
#pragma unroll
          for (int s = 0; s < 3; s++) {
            const float m = fmaf(u, p.D[s], p.N[s]);
            float lt = log10f(fmaxf(m * S.w.sig0[s], 1e-30f));
            // beyond the trained range, or a negative entry column (a ray
            // that starts inside its target cell): exact quadrature
            if (lt > kTauHi || m < 0.f) nq = 0;
            lt = fmaxf(lt, kTauLo);
            xin[i][s] = (lt - 0.5f * (kTauLo + kTauHi)) * (2.f / (kTauHi - kTauLo));
          }
          xin[i][3] = (lT - 0.5f * (kTLo + kTHi)) * (2.f / (kTHi - kTLo));
        }
      }
      // exclusive scan of the node counts -> positions in the evaluation list
      int pos = nq;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, pos, o);
        if (lane >= o) pos += v;
      }
      const int nev = __shfl_sync(0xffffffffu, pos, 31);
      pos -= nq;
      for (int i = 0; i < nq; i++)
#pragma unroll
        for (int c = 0; c < 4; c++) S.x[wib][pos + i][c] = xin[i][c];
      S.t[wib][lane] = tl;
      // pad the last tile with valid inputs
      for (int q = nev + lane; q < ((nev + 15) & ~15); q += 32)
#pragma unroll
        for (int c = 0; c < 4; c++) S.x[wib][q][c] = 0.f;
      __syncwarp();
      // ---- phase B: the network on the tensor cores
      for (int r16 = 0; r16 < nev; r16 += 16) mlp_tile16(S.w, S.x[wib], S.tout[wib], r16, lane);
      __syncwarp();
      // ---- phase C: predicted contributions and their error bound
      if (tl >= 0) {
        float cj[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        float low[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // lower-bound factor of each c_j
        float eps = kInf;
        if (nq > 0) {
          float mj[18];
#pragma unroll
          for (int k = 0; k < 18; k++) mj[k] = __ldg(emit_m + 18 * (size_t)e + k);
          // G: predicted node sum; dG: bound of its error; Gl: lower bound
          // of the true sum (I >= I^ e^-x >= I^ (1 - x) at every node)
          float G[6] = {0, 0, 0, 0, 0, 0}, dG[6] = {0, 0, 0, 0, 0, 0}, Gl[6] = {0, 0, 0, 0, 0, 0};
          for (int i = 0; i < nq; i++) {
            float u, wq;
            gl_node(nq, i, &u, &wq);
            float ts[3];
#pragma unroll
            for (int s = 0; s < 3; s++) ts[s] = fmaxf(fmaf(u, p.D[s], p.N[s]), 0.f) * S.w.sig0[s];
#pragma unroll
            for (int j = 0; j < 6; j++) {
              const float qh = S.tout[wib][pos + i][j];
              const float ylin = -fmaf(ts[0], mj[3 * j], fmaf(ts[1], mj[3 * j + 1], ts[2] * mj[3 * j + 2]));
              const float yh = ylin * __expf(fminf(qh, 0.f));
              const int bin = min(kEnvBins - 1, max(0, (int)((qh - kEnvQLo) * (kEnvBins / -kEnvQLo))));
              const float x = -yh * S.w.env[j][bin];
              const float a = wq * __expf(yh);
              G[j] += a;
              // e^x <= 1 + x + x^2 (0 <= x <= 1) and e^-x >= 1 - x
              const float ex = x <= 1.f ? fmaf(x, x + 1.f, 1.f) : __expf(x);
              dG[j] = fmaf(a, x * ex, dG[j]);
              Gl[j] = fmaf(a, fmaxf(0.f, 1.f - x), Gl[j]);
            }
          }
          eps = 0.f;
#pragma unroll
          for (int j = 0; j < 6; j++) {
            eps = fmaxf(eps, G[j] > 0.f ? dG[j] / G[j] : (dG[j] > 0.f ? kInf : 0.f));
            low[j] = G[j] > 0.f ? (Gl[j] / G[j]) * (1.f - kGLErr) : 0.f;
          }
          // plus the Gauss-Legendre quadrature error of the cell factor
          eps += kGLErr;
#pragma unroll
          for (int s = 0; s < 3; s++) {
            cj[s] = (float)((double)p.P[s] * (double)G[s] * __ldg(emit_i0 + 6 * (size_t)e + s));
            cj[3 + s] = (float)((double)p.P[s] * (double)G[3 + s] * __ldg(emit_i0 + 6 * (size_t)e + 3 + s) * kHNuL);
          }
        }
        // the cell budget is taken from a lower bound of the true total:
        // c_true >= c (Gl / G) (1 - GL error)
#pragma unroll
        for (int j = 0; j < 6; j++) {
          work[j * nray + r] = cj[j];
          S.c[wib][lane][j] = cj[j] * low[j];
        }
        work[6 * nray + r] = eps;
      }
      __syncwarp();
      // ---- phase E: per-cell predicted totals in ray order
      const int nk = (int)min((uint64_t)32, r1 - rc);
      for (int k = 0; k < nk; k++) {
        if (S.t[wib][k] == lane) {
#pragma unroll
          for (int s = 0; s < 6; s++) acc[s] += S.c[wib][k][s];
        }
      }
      __syncwarp();
    }
    if (own_valid) {
#pragma unroll
      for (int s = 0; s < 6; s++) rates6[s * ncell + own] = (float)acc[s];
    }
  }
}

// Histogram bin of a ray's share of its cell's error budget,
//   beta = eps * max_j c_j / S_j,
// in half-octaves: bin 64 + k holds beta in [2^(k/2), 2^((k+1)/2)), bin 0
// everything below 2^-31.5; -1 = the ray takes the exact quadrature.  Exact
// in float (frexpf), so both passes of kernel 2 agree bit for bit.
__device__ __forceinline__ int beta_bin(const float *c, float eps, const float *Sc) {
  if (!(eps < 1.f)) return -1;
  float mx = 0.f;
#pragma unroll
  for (int j = 0; j < 6; j++) {
    if (c[j] > 0.f) {
      if (!(Sc[j] > 0.f)) return -1;
      mx = fmaxf(mx, c[j] / Sc[j]);
    }
  }
  const float beta = eps * mx;
  if (!(beta < 1.f)) return -1;
  if (beta <= 0.f) return 0;
  int E;
  const float f = frexpf(beta, &E);  // beta = f 2^E, f in [0.5, 1)
  const int k = 2 * (E - 1) + (f >= 0.70710678f ? 1 : 0);
  return max(0, k + kHistBins);
}
// upper edge of bin b
__device__ __forceinline__ double beta_edge(int b) { return exp2(0.5 * (double)(b - kHistBins + 1)); }

// Kernel 2: per cell, the rays whose error bounds fit the budget
// tol * S_j (the smallest bounds first, by the histogram of beta; the sum
// of a bin is bounded by its count times its upper edge) keep the
// network's contributions: their flag (work plane 6, which held eps) is set
// to 1, every other ray's to 0.  Kernel 3, the FP32 rate kernel
// (rate_block_f32<true>), then runs the exact quadrature for the flagged-0
// rays only, at its own occupancy, and sums every cell in ray order.
__global__ void __launch_bounds__(32 * kSurWarps)
    k_sur_select(GridDev g, float tol, uint64_t b0, uint64_t b1, const uint64_t *__restrict__ blk_off, uint64_t base,
                 const uint32_t *__restrict__ rays, uint64_t nray, const float *__restrict__ rates6,
                 float *__restrict__ work, unsigned long long *__restrict__ counters, int *__restrict__ err) {
  __shared__ SelSmem S;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarp = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t ncell = (uint64_t)g.nx * g.ny * g.nz;
  unsigned long long n_sur = 0, n_exact = 0;
  for (uint64_t b = b0 + warp; b < b1; b += nwarp) {
    uint64_t r0, r1;
    if (!block_rays(blk_off, b, base, nray, &r0, &r1)) {
      if (lane == 0) atomicExch(err, 1);
      continue;
    }
    int ix, iy, iz;
    const bool own_valid = block_cell(g, b, lane, &ix, &iy, &iz);
    const uint64_t own = own_valid ? cell_index(g, ix, iy, iz) : 0;
#pragma unroll
    for (int s = 0; s < 6; s++) S.Sc[wib][lane][s] = own_valid ? rates6[s * ncell + own] : 0.f;
    for (int k = 0; k < kHistBins; k++) S.hist[wib][lane][k] = 0u;
    __syncwarp();
    // ---- pass 1: histogram of beta per cell
    for (uint64_t r = r0 + lane; r < r1; r += 32) {
      const int tl = (int)(__ldg(rays + r) & 31u);
      float c[6];
#pragma unroll
      for (int j = 0; j < 6; j++) c[j] = work[j * nray + r];
      const int bin = beta_bin(c, work[6 * nray + r], S.Sc[wib][tl]);
      if (bin >= 0) atomicAdd(&S.hist[wib][tl][bin], 1u);
    }
    __syncwarp();
    {
      double cum = 0.0;
      int thr = -1;
      for (int k = 0; k < kHistBins; k++) {
        const unsigned n = S.hist[wib][lane][k];
        if (n) {
          cum += (double)n * beta_edge(k);
          if (cum > (double)tol) break;
        }
        thr = k;
      }
      S.thr[wib][lane] = thr;
    }
    __syncwarp();
    // ---- pass 2: the flags
    for (uint64_t r = r0 + lane; r < r1; r += 32) {
      const int tl = (int)(__ldg(rays + r) & 31u);
      float c[6];
#pragma unroll
      for (int j = 0; j < 6; j++) c[j] = work[j * nray + r];
      const int bin = beta_bin(c, work[6 * nray + r], S.Sc[wib][tl]);
      const bool served = bin >= 0 && bin <= S.thr[wib][tl];
      work[6 * nray + r] = served ? 1.f : 0.f;
      n_sur += served;
      n_exact += !served;
    }
    __syncwarp();
  }
  if (counters) {
    for (int o = 16; o; o >>= 1) {
      n_sur += __shfl_xor_sync(0xffffffffu, n_sur, o);
      n_exact += __shfl_xor_sync(0xffffffffu, n_exact, o);
    }
    if (lane == 0) {
      atomicAdd(counters + 0, n_sur);
      atomicAdd(counters + 1, n_exact);
    }
  }
}

// The network on a list of raw inputs (log10 tau x3, log10 T), one warp per
// 16 evaluations, with the inference numerics of k_rate_sur.
__global__ void __launch_bounds__(128) k_sur_eval(const SurWeights *__restrict__ wts, const float *__restrict__ X,
                                                  int n, float *__restrict__ T) {
  __shared__ SurWeights W;
  __shared__ float xs[4][16][4];
  __shared__ float ts[4][16][6];
  {
    const uint32_t *src = reinterpret_cast<const uint32_t *>(wts);
    uint32_t *dst = reinterpret_cast<uint32_t *>(&W);
    for (int i = threadIdx.x; i < (int)(sizeof(SurWeights) / 4); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nt = (n + 15) / 16;
  for (int tile = blockIdx.x * 4 + wib; tile < nt; tile += gridDim.x * 4) {
    if (lane < 16) {
      const int i = tile * 16 + lane;
#pragma unroll
      for (int c = 0; c < 4; c++) {
        float v = i < n ? X[4 * (size_t)i + c] : 0.f;
        if (c < 3) {
          v = fminf(fmaxf(v, kTauLo), kTauHi);
          v = (v - 0.5f * (kTauLo + kTauHi)) * (2.f / (kTauHi - kTauLo));
        } else {
          v = (v - 0.5f * (kTLo + kTHi)) * (2.f / (kTHi - kTLo));
        }
        xs[wib][lane][c] = v;
      }
    }
    __syncwarp();
    mlp_tile16(W, xs[wib], ts[wib], 0, lane);
    __syncwarp();
    for (int q = lane; q < 16 * 6; q += 32) {
      const int i = tile * 16 + q / 6;
      if (i < n) T[6 * (size_t)i + q % 6] = ts[wib][q / 6][q % 6];
    }
    __syncwarp();
  }
}

}  // namespace argot

using namespace argot;

// ------------------------------------------------------------- host side
struct argot_b200_surrogate {
  int device;
  SurWeights *dev;
  float tol;  // host copy of the per-cell budget (kernel 2 argument)
};

namespace {

uint16_t bf16_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  const uint32_t r = u + 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(r >> 16);
}
uint32_t pack2(float lo, float hi) { return (uint32_t)bf16_bits(lo) | ((uint32_t)bf16_bits(hi) << 16); }

// B fragment of N-tile j, K-step kk for W[n][k] (rows n, cols k, getter)
template <class F>
uint2 frag(F w, int j, int kk, int lane) {
  const int gq = lane >> 2, tq = lane & 3;
  const int n = 8 * j + gq, k = 16 * kk + 2 * tq;
  uint2 r;
  r.x = pack2(w(n, k), w(n, k + 1));
  r.y = pack2(w(n, k + 8), w(n, k + 9));
  return r;
}

}  // namespace

extern "C" {

// params: the 9030 FP32 network parameters (host); env: 6 x 64 bound of
// |error of q| in bins of predicted q over [-7, 0] (host); tol: per-cell
// relative error budget of the surrogate's contributions.
int argot_b200_surrogate_create(const float *params, const float *env, float tol, argot_b200_surrogate **out) {
  if (!params || !env || !out || !(tol > 0.f)) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  auto *h = new (std::nothrow) SurWeights();
  if (!h) { set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  const float *W1 = params + kOffW1, *W2 = params + kOffW2, *W3 = params + kOffW3, *W4 = params + kOffW4;
  for (int j = 0; j < 8; j++)
    for (int l = 0; l < 32; l++) {
      h->f1[j][l] = frag([&](int n, int k) { return k < 8 ? W1[n * kMlpIn + (k & 3)] : 0.f; }, j, 0, l);
      for (int kk = 0; kk < 4; kk++) {
        h->f2[j][kk][l] = frag([&](int n, int k) { return W2[n * kMlpH + k]; }, j, kk, l);
        h->f3[j][kk][l] = frag([&](int n, int k) { return W3[n * kMlpH + k]; }, j, kk, l);
      }
    }
  for (int kk = 0; kk < 8; kk++)
    for (int l = 0; l < 32; l++)
      h->f4[kk][l] = frag([&](int n, int k) { return n < kMlpOut ? W4[n * kMlpH + (k & 63)] : 0.f; }, 0, kk, l);
  std::memcpy(h->b1, params + kOffB1, sizeof(float) * 64);
  std::memcpy(h->b2, params + kOffB2, sizeof(float) * 64);
  std::memcpy(h->b3, params + kOffB3, sizeof(float) * 64);
  for (int j = 0; j < 8; j++) h->b4[j] = j < kMlpOut ? params[kOffB4 + j] : 0.f;
  // kernel 1 uses e^dq - 1: |q - q^| <= dq gives |y - y^| <= |y^| (e^dq - 1)
  for (int j = 0; j < 6; j++)
    for (int b = 0; b < kEnvBins; b++) h->env[j][b] = (float)std::expm1((double)env[j * kEnvBins + b]);
  double w6[6 * kNu];
  host_rate_weights(w6);
  for (int s = 0; s < 3; s++) {
    h->sig0[s] = 0.f;
    for (int k = 0; k < kNu && h->sig0[s] == 0.f; k++) h->sig0[s] = (float)w6[s * kNu + k];
  }
  h->tol = tol;
  auto *s = new (std::nothrow) argot_b200_surrogate();
  if (!s) { delete h; set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  s->tol = tol;
  cudaError_t e = cudaGetDevice(&s->device);
  if (e == cudaSuccess) e = cudaMalloc(&s->dev, sizeof(SurWeights));
  if (e == cudaSuccess) e = cudaMemcpy(s->dev, h, sizeof(SurWeights), cudaMemcpyHostToDevice);
  delete h;
  if (e != cudaSuccess) { delete s; return status_from_cuda(e); }
  *out = s;
  set_status(0);
  return 0;
}

void argot_b200_surrogate_free(argot_b200_surrogate *s) {
  if (!s) return;
  cudaFree(s->dev);
  delete s;
}

// q_j predictions (n x 6) for raw inputs X (n x 4: log10 tau_HI, tau_HeI,
// tau_HeII, log10 T) with the tensor-core inference numerics.
int argot_b200_surrogate_eval(const argot_b200_surrogate *s, const float *X, int n, float *T, void *stream) {
  if (!s || (n && (!X || !T))) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  if (n) {
    const int tiles = (n + 15) / 16;
    const int blocks = (tiles + 3) / 4 < 4096 ? (tiles + 3) / 4 : 4096;
    k_sur_eval<<<blocks, 128, 0, (cudaStream_t)stream>>>(s->dev, X, n, T);
    ARGOT_CUDA_TRY(cudaGetLastError());
  }
  set_status(0);
  return 0;
}

uint64_t argot_b200_surrogate_workspace(uint64_t nray_group) { return (uint64_t)kWorkPlanes * 4u * nray_group; }

// Rates of blocks [b0, b1) with the surrogate (see argot_b200_photoion_rays;
// work: device workspace of argot_b200_surrogate_workspace(nray) bytes;
// counters, optional device uint64[2], receive the numbers of rays taken by
// the surrogate and by the exact quadrature).
int argot_b200_photoion_rays_surrogate(const argot_b200_grid *gp, const void *packed, const argot_b200_dev_tree *t,
                                       const argot_b200_surrogate *sur, uint64_t b0, uint64_t b1,
                                       const uint64_t *blk_off, uint64_t base, const uint32_t *rays, uint64_t nray,
                                       const float *tau, float *work, float *rates6, unsigned long long *counters,
                                       void *stream) {
  uint64_t nb = 0;
  if (!grid_valid(gp) || !packed || !t || !sur || !blk_off || !rates6 || (nray && (!rays || !tau || !work)) ||
      !t->emit_logT || !t->emit_i0 || !t->emit_m || argot_b200_num_blocks(gp, &nb) || b0 > b1 || b1 > nb) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  if (b0 == b1) { set_status(0); return 0; }
  int dev = 0;
  ARGOT_CUDA_TRY(cudaGetDevice(&dev));
  int rc = ensure_rate_tables(dev);
  if (rc) return rc;
  int *err = err_flag(dev);
  if (!err) { set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  static std::mutex mu;
  static bool attr[64] = {false};
  {
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 0 || dev >= 64) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
    if (!attr[dev]) {
      ARGOT_CUDA_TRY(cudaFuncSetAttribute(k_sur_predict, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)sizeof(PredSmem)));
      attr[dev] = true;
    }
  }
  GridDev g = make_grid(*gp);
  const uint64_t ncell = (uint64_t)gp->nx * gp->ny * gp->nz;
  const float4 *raw = (const float4 *)packed + ncell;
  const int threads = 32 * kSurWarps;
  const int blocks = grid_blocks_for_rates((b1 - b0) * 32, threads);
  cudaStream_t st = (cudaStream_t)stream;
  k_sur_predict<<<blocks, threads, sizeof(PredSmem), st>>>(g, raw, t->emit_pos, t->emit_total, t->emit_logT,
                                                            t->emit_i0, t->emit_m, sur->dev, b0, b1, blk_off,
                                                            base, rays, nray, tau, rates6, work, err);
  ARGOT_CUDA_TRY(cudaGetLastError());
  k_sur_select<<<blocks, threads, 0, st>>>(g, sur->tol, b0, b1, blk_off, base, rays, nray, rates6, work,
                                            counters, err);
  ARGOT_CUDA_TRY(cudaGetLastError());
  rc = launch_rate_f32_served(g, raw, t->emit_pos, t->emit_specn, t->emit_total, b0, b1, blk_off, base, rays, nray,
                              tau, rates6, work, err, st);
  if (rc) return rc;
  set_status(0);
  return 0;
}

}  // extern "C"
