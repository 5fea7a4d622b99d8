// surrogate.cu -- per-cell rates with the BF16 MLP surrogate of the
// frequency integral, evaluated on the fifth-generation tensor cores
// (tcgen05: operands in shared memory, fp32 accumulators in TMEM), and the
// exact FP32 quadrature as fallback.
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
#include "umma.cuh"

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
constexpr int kSurWarps = 8;   // warps of the predict kernel: a tile's 128 rows x two column halves
constexpr int kSelWarps = 4;   // warps of the select kernel
constexpr int kMaxEval = 96;   // 32 rays x 3 quadrature nodes
constexpr int kTile = 128;     // network evaluations per tensor-core tile (MMA M)

// The network in the operand layout of the tensor cores (umma.cuh: BF16,
// K-major, no swizzle), built on the host, copied to shared memory as it is:
//   layer 1: N = 64, K = 16 (k 0..3 the inputs' BF16 high parts, 4..7 their
//            low parts, both against W1, 8..15 zero);
//   layers 2, 3: N = 64, K = 64 (the activations enter as a BF16 pair
//            hi + lo: two MMA chains against the same weights);
//   layer 4: N = 16 (outputs 0..5, the rest zero), K = 64, hi and lo.
// Every activation therefore carries 16 mantissa bits into the tensor
// cores; the weights are single BF16 values (the network is trained with
// them rounded).
struct TcNet {
  uint16_t b1[64 * 16];
  uint16_t b2[64 * 64];
  uint16_t b3[64 * 64];
  uint16_t b4[16 * 64];
  float bias1[64], bias2[64], bias3[64], bias4[16];
  float env[6][kEnvBins];  // e^dq - 1, dq the bound of |error of q| per output and bin of q^
  float sig0[3];
  float tol;               // per-cell relative error budget
};
static_assert(sizeof(TcNet) % 16 == 0, "TcNet copies in 16-byte words");

// Operand tiles of one 128-row tile and the tensor-core bookkeeping.
struct TcTile {
  uint16_t a1[kTile * 16];   // layer-1 inputs
  uint16_t ahi[kTile * 64];  // activations, BF16 high parts
  uint16_t alo[kTile * 64];  // ... and low parts
  uint64_t bar;              // MMA completion
  uint32_t tmem;             // TMEM base of the fp32 accumulator (64 columns)
  uint32_t phase;            // parity of the next completion of bar
};

constexpr uint32_t kWaitPolls = 1u << 22;  // bound of one MMA wait (far above a microsecond MMA)

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}

// The tensor-core thread of the CTA issues one layer and everyone waits for
// it: A rows from `a` (row stride of a K-major tile of 128 rows), `ksteps`
// K-steps of 16 over `a`, then (if `a2`) the same over `a2`, against B with
// its own LBO; fp32 result in TMEM columns [0, n).  Returns false (for the
// whole CTA) when the completion did not arrive in time; then nothing more
// is issued.
__device__ __forceinline__ bool tc_layer(TcTile &T, const uint16_t *a, const uint16_t *a2, const uint16_t *b,
                                         int ksteps, uint32_t b_lbo, int n, bool ok) {
  if (ok && threadIdx.x == 0) {
    umma::fence_after_sync();
    const uint32_t id = umma::idesc_bf16(kTile, n);
    const uint32_t a_lbo = (kTile / 8) * 128;
    int step = 0;
    for (int pass = 0; pass < (a2 ? 2 : 1); pass++) {
      const uint32_t ab = umma::smem_addr(pass ? a2 : a), bb = umma::smem_addr(b);
      for (int s = 0; s < ksteps; s++, step++)
        umma::mma_bf16(T.tmem, umma::smem_desc(ab + 2 * s * a_lbo, a_lbo, 128),
                       umma::smem_desc(bb + 2 * s * b_lbo, b_lbo, 128), id, step > 0);
    }
    umma::commit(&T.bar);
  }
  bool done = true;
  if (ok) {
    done = umma::mbar_wait(&T.bar, T.phase, kWaitPolls);
    umma::fence_after_sync();
  }
  ok = __syncthreads_and(ok && done);
  if (threadIdx.x == 0) T.phase ^= 1u;
  return ok;
}

// Epilogue of a hidden layer: thread (warp w, lane) takes row 32 (w % 4) +
// lane and columns [32 h, 32 h + 32), h = w / 4: the accumulator plus
// bias, SiLU, split into BF16 hi + lo, stored as the next layer's A.
__device__ __forceinline__ void tc_hidden_epilogue(TcTile &T, const float *__restrict__ bias, bool ok) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = 32 * (w & 3) + lane, h = w >> 2;
  if (ok) {
#pragma unroll
    for (int cc = 0; cc < 2; cc++) {
      const int k0 = 32 * h + 16 * cc;
      float v[16];
      umma::tmem_ld16(T.tmem + ((uint32_t)(32 * (w & 3)) << 16) + (uint32_t)k0, v);
      uint32_t hi[8], lo[8];
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const float s0 = silu_acc(v[2 * i] + bias[k0 + 2 * i]);
        const float s1 = silu_acc(v[2 * i + 1] + bias[k0 + 2 * i + 1]);
        const float h0 = bf16_round(s0), h1 = bf16_round(s1);
        hi[i] = pack_bf16x2(h0, h1);
        lo[i] = pack_bf16x2(s0 - h0, s1 - h1);
      }
      // two 8-element K chunks per 16 columns
      *reinterpret_cast<uint4 *>(reinterpret_cast<char *>(T.ahi) + umma::kmajor_offset(kTile, row, k0)) =
          make_uint4(hi[0], hi[1], hi[2], hi[3]);
      *reinterpret_cast<uint4 *>(reinterpret_cast<char *>(T.ahi) + umma::kmajor_offset(kTile, row, k0 + 8)) =
          make_uint4(hi[4], hi[5], hi[6], hi[7]);
      *reinterpret_cast<uint4 *>(reinterpret_cast<char *>(T.alo) + umma::kmajor_offset(kTile, row, k0)) =
          make_uint4(lo[0], lo[1], lo[2], lo[3]);
      *reinterpret_cast<uint4 *>(reinterpret_cast<char *>(T.alo) + umma::kmajor_offset(kTile, row, k0 + 8)) =
          make_uint4(lo[4], lo[5], lo[6], lo[7]);
    }
  }
  // the TMEM reads complete before the next MMA overwrites the columns,
  // the shared-memory writes are visible to the tensor cores
  umma::fence_before_sync();
  umma::fence_smem_to_async();
  __syncthreads();
}

// The network on one tile of up to 128 evaluations.  load(row, x[4]) gives
// the normalised inputs of tile row `row` (called for row < nrows by the
// threads of warps 0..3, thread = row); put(row, q[6]) receives the outputs
// q_j (same threads).  All threads of the CTA call it; `ok` is CTA-uniform.
template <class Load, class Put>
__device__ __forceinline__ bool mlp_tile_tc(const TcNet &W, TcTile &T, int nrows, Load load, Put put, bool ok) {
  const int tid = threadIdx.x, w = tid >> 5;
  if (w < 4) {
    const int row = tid;
    float x[4] = {0.f, 0.f, 0.f, 0.f};
    if (row < nrows) load(row, x);
    float h[4], l[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
      h[c] = bf16_round(x[c]);
      l[c] = x[c] - h[c];
    }
    // K chunk 0: hi | lo; chunk 1 stays zero (written once)
    *reinterpret_cast<uint4 *>(reinterpret_cast<char *>(T.a1) + umma::kmajor_offset(kTile, row, 0)) =
        make_uint4(pack_bf16x2(h[0], h[1]), pack_bf16x2(h[2], h[3]), pack_bf16x2(l[0], l[1]),
                   pack_bf16x2(l[2], l[3]));
  }
  umma::fence_before_sync();
  umma::fence_smem_to_async();
  __syncthreads();
  ok = tc_layer(T, T.a1, nullptr, W.b1, 1, (64 / 8) * 128, 64, ok);
  tc_hidden_epilogue(T, W.bias1, ok);
  ok = tc_layer(T, T.ahi, T.alo, W.b2, 4, (64 / 8) * 128, 64, ok);
  tc_hidden_epilogue(T, W.bias2, ok);
  ok = tc_layer(T, T.ahi, T.alo, W.b3, 4, (64 / 8) * 128, 64, ok);
  tc_hidden_epilogue(T, W.bias3, ok);
  ok = tc_layer(T, T.ahi, T.alo, W.b4, 4, (16 / 8) * 128, 16, ok);
  if (ok && w < 4) {
    float v[16];
    umma::tmem_ld16(T.tmem + ((uint32_t)(32 * w) << 16), v);
    if (tid < nrows) {
      float q[6];
#pragma unroll
      for (int j = 0; j < 6; j++) q[j] = fmaf(v[j] + W.bias4[j], kOutScale, kOutShift);
      put(tid, q);
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  return ok;
}

// Set-up of the tensor-core state of a CTA: the network image into shared
// memory, TMEM (warp 0), the mbarrier, the constant zero chunk of layer 1.
__device__ __forceinline__ void tc_setup(const TcNet *__restrict__ g_net, TcNet &W, TcTile &T) {
  {
    const uint4 *src = reinterpret_cast<const uint4 *>(g_net);
    uint4 *dst = reinterpret_cast<uint4 *>(&W);
    for (int i = threadIdx.x; i < (int)(sizeof(TcNet) / 16); i += blockDim.x) dst[i] = src[i];
  }
  for (int r = threadIdx.x; r < kTile; r += blockDim.x)
    *reinterpret_cast<uint4 *>(reinterpret_cast<char *>(T.a1) + umma::kmajor_offset(kTile, r, 8)) =
        make_uint4(0u, 0u, 0u, 0u);
  if (threadIdx.x < 32) umma::tmem_alloc(&T.tmem, 64);
  if (threadIdx.x == 0) {
    umma::mbar_init(&T.bar, 1);
    T.phase = 0;
  }
  umma::fence_before_sync();
  umma::fence_smem_to_async();
  __syncthreads();
  umma::fence_after_sync();
}

__device__ __forceinline__ void tc_teardown(TcTile &T) {
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  if (threadIdx.x < 32) umma::tmem_dealloc(T.tmem, 64);
}

struct PredSmem {
  TcNet w;
  TcTile tile;
  // per warp
  float x[kSurWarps][kMaxEval][4];     // normalised network inputs
  float tout[kSurWarps][kMaxEval][6];  // network outputs q_j
  float c[kSurWarps][32][6];           // predicted per-ray contributions
  int t[kSurWarps][32];
  int nev[kSurWarps];                  // evaluations of the warp's chunk this round
};

struct SelSmem {
  // per warp
  float Sc[kSelWarps][32][6];                // lower bounds of the cell totals
  unsigned hist[kSelWarps][32][kHistBins];   // budget-share histogram per cell
  int thr[kSelWarps][32];                    // last accepted bin per cell
};

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
// The kernel runs in rounds: in each round every warp of the CTA takes the
// next chunk of 32 rays of its target blocks (blocks b0 + warp, + nwarp,
// ...), forms their quadrature nodes' network inputs, and the CTA's tensor
// cores evaluate all the round's evaluations in tiles of 128 (the 8 warps'
// lists concatenated); then every warp turns its outputs into contributions,
// bounds and per-cell lower bounds.  A warp without work left takes part in
// the CTA's barriers only.
// Launch shape: kSurWarps warps per CTA, at least ARGOT_SUR_PREDICT_MIN_CTAS
// CTAs resident per SM.
#ifndef ARGOT_SUR_PREDICT_MIN_CTAS
#define ARGOT_SUR_PREDICT_MIN_CTAS 2
#endif
__global__ void __launch_bounds__(32 * kSurWarps, ARGOT_SUR_PREDICT_MIN_CTAS)
    k_sur_predict(GridDev g, const float4 *__restrict__ raw, const float4 *__restrict__ emit_pos,
                  const double *__restrict__ total, const float *__restrict__ emit_logT,
                  const double *__restrict__ emit_i0, const float *__restrict__ emit_m,
                  const TcNet *__restrict__ net, uint64_t b0, uint64_t b1, const uint64_t *__restrict__ blk_off,
                  uint64_t base, const uint32_t *__restrict__ rays, uint64_t nray, const float *__restrict__ tau,
                  float *__restrict__ rates6, float *__restrict__ work, int *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  PredSmem &S = *reinterpret_cast<PredSmem *>(smem_raw);
  tc_setup(net, S.w, S.tile);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const float s00 = c_tab.cs[0][0];
  const float s0a = c_tab.cs[0][44], s1a = c_tab.cs[1][44];
  const float s0b = c_tab.cs[0][103], s1b = c_tab.cs[1][103], s2b = c_tab.cs[2][103];
  const uint64_t nwarp = (uint64_t)gridDim.x * kSurWarps;
  const uint64_t ncell = (uint64_t)g.nx * g.ny * g.nz;
  const float kInf = __int_as_float(0x7f800000);
  // this warp's position: block b, chunk start rc in [r0, r1)
  uint64_t b = b0 + (uint64_t)blockIdx.x * kSurWarps + wib;
  uint64_t r0 = 0, r1 = 0, rc = 0;
  int bix = 0, biy = 0, biz = 0;
  bool own_valid = false;
  uint64_t own = 0;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  // the first block with rays at or after b (blocks with bad offsets are
  // reported and skipped; blocks without rays get a zero lower bound)
  auto open_block = [&]() {
    for (; b < b1; b += nwarp) {
      int ix, iy, iz;
      own_valid = block_cell(g, b, lane, &ix, &iy, &iz);
      own = own_valid ? cell_index(g, ix, iy, iz) : 0;
      block_cell(g, b, 0, &bix, &biy, &biz);
      if (!block_rays(blk_off, b, base, nray, &r0, &r1)) {
        if (lane == 0) atomicExch(err, 1);
        continue;
      }
      if (r0 < r1) break;
      if (own_valid) {
#pragma unroll
        for (int s = 0; s < 6; s++) rates6[s * ncell + own] = 0.f;
      }
    }
    rc = r0;
#pragma unroll
    for (int s = 0; s < 6; s++) acc[s] = 0.0;
  };
  open_block();
  bool ok = true;
  for (;;) {
    const bool active = b < b1;
    if (!__syncthreads_or(active)) break;
    // ---- phase A: per-ray parameters and quadrature nodes of the chunk
    const uint64_t r = rc + lane;
    int tl = -1, nq = 0, e = 0, pos = 0;
    RayParams p;
    if (active) {
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
      // exclusive scan of the node counts -> positions in the warp's list
      pos = nq;
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
      if (lane == 0) S.nev[wib] = nev;
    } else if (lane == 0) {
      S.nev[wib] = 0;
    }
    __syncthreads();
    // ---- phase B: the round's evaluations on the tensor cores
    int start[kSurWarps + 1];
    start[0] = 0;
#pragma unroll
    for (int k = 0; k < kSurWarps; k++) start[k + 1] = start[k] + S.nev[k];
    const int total_ev = start[kSurWarps];
    for (int t0 = 0; t0 < total_ev; t0 += kTile) {
      // tile row -> (warp, index in its list)
      auto where = [&](int row, int &wk, int &ik) {
        const int gi = t0 + row;
        wk = 0;
#pragma unroll
        for (int k = 1; k < kSurWarps; k++) wk += gi >= start[k];
        ik = gi - start[wk];
      };
      ok = mlp_tile_tc(
          S.w, S.tile, min(kTile, total_ev - t0),
          [&](int row, float(&x)[4]) {
            int wk, ik;
            where(row, wk, ik);
#pragma unroll
            for (int c = 0; c < 4; c++) x[c] = S.x[wk][ik][c];
          },
          [&](int row, const float(&q)[6]) {
            int wk, ik;
            where(row, wk, ik);
#pragma unroll
            for (int j = 0; j < 6; j++) S.tout[wk][ik][j] = q[j];
          },
          ok);
    }
    // (the tile's last barrier orders the outputs before their readers)
    if (active) {
      // ---- phase C: predicted contributions and their error bound
      if (tl >= 0) {
        float cj[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        float low[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // lower-bound factor of each c_j
        float eps = kInf;
        if (nq > 0 && ok) {
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
      // next chunk, or the block's lower bounds and the next block
      rc += 32;
      if (rc >= r1) {
        if (own_valid) {
#pragma unroll
          for (int s = 0; s < 6; s++) rates6[s * ncell + own] = (float)acc[s];
        }
        b += nwarp;
        open_block();
      }
    }
  }
  if (!ok && threadIdx.x == 0) atomicExch(err, 1);
  tc_teardown(S.tile);
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
__global__ void __launch_bounds__(32 * kSelWarps)
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

// The network on a list of raw inputs (log10 tau x3, log10 T) with the
// inference numerics of k_sur_predict: one CTA of 8 warps per tile of 128
// evaluations on the tensor cores (the inputs normalised as there).
struct EvalSmem {
  TcNet w;
  TcTile tile;
};
__global__ void __launch_bounds__(32 * kSurWarps) k_sur_eval(const TcNet *__restrict__ net,
                                                           const float *__restrict__ X, int n,
                                                           float *__restrict__ T, int *__restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  EvalSmem &S = *reinterpret_cast<EvalSmem *>(smem_raw);
  tc_setup(net, S.w, S.tile);
  bool ok = true;
  for (int t0 = blockIdx.x * kTile; t0 < n; t0 += gridDim.x * kTile) {
    ok = mlp_tile_tc(
        S.w, S.tile, min(kTile, n - t0),
        [&](int row, float(&x)[4]) {
          const size_t i = (size_t)(t0 + row);
#pragma unroll
          for (int c = 0; c < 4; c++) {
            float v = X[4 * i + c];
            if (c < 3) {
              v = fminf(fmaxf(v, kTauLo), kTauHi);
              v = (v - 0.5f * (kTauLo + kTauHi)) * (2.f / (kTauHi - kTauLo));
            } else {
              v = (v - 0.5f * (kTLo + kTHi)) * (2.f / (kTHi - kTLo));
            }
            x[c] = v;
          }
        },
        [&](int row, const float(&q)[6]) {
          const size_t i = (size_t)(t0 + row);
#pragma unroll
          for (int j = 0; j < 6; j++) T[6 * i + j] = q[j];
        },
        ok);
  }
  if (!ok && threadIdx.x == 0) atomicExch(err, 1);
  tc_teardown(S.tile);
}

}  // namespace argot

using namespace argot;

// ------------------------------------------------------------- host side
struct argot_b200_surrogate {
  int device;
  TcNet *dev;
  float tol;  // host copy of the per-cell budget (kernel 2 argument)
};

namespace {

uint16_t bf16_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  const uint32_t r = u + 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(r >> 16);
}

// W[n][k] (getter) into a K-major tile of R rows (umma.cuh layout)
template <class F>
void put_kmajor(uint16_t *tile, int R, int K, F w) {
  for (int n = 0; n < R; n++)
    for (int k = 0; k < K; k++) tile[umma::kmajor_offset(R, n, k) / 2] = bf16_bits(w(n, k));
}

// shared-memory bytes of the predict / eval kernels
size_t pred_smem() { return sizeof(PredSmem); }
size_t eval_smem() { return sizeof(EvalSmem); }

int kernel_attrs(int dev) {
  static std::mutex mu;
  static bool done[64] = {false};
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 0 || dev >= 64) return ARGOT_B200_EINVAL;
  if (!done[dev]) {
    ARGOT_CUDA_TRY(cudaFuncSetAttribute(k_sur_predict, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pred_smem()));
    ARGOT_CUDA_TRY(cudaFuncSetAttribute(k_sur_eval, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)eval_smem()));
    done[dev] = true;
  }
  return 0;
}

}  // namespace

extern "C" {

// params: the 9030 FP32 network parameters (host); env: 6 x 64 bound of
// |error of q| in bins of predicted q over [-7, 0] (host); tol: per-cell
// relative error budget of the surrogate's contributions.
int argot_b200_surrogate_create(const float *params, const float *env, float tol, argot_b200_surrogate **out) {
  if (!params || !env || !out || !(tol > 0.f)) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  auto *h = new (std::nothrow) TcNet();
  if (!h) { set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  const float *W1 = params + kOffW1, *W2 = params + kOffW2, *W3 = params + kOffW3, *W4 = params + kOffW4;
  // layer 1: k 0..3 against the inputs' high parts, 4..7 against their low parts
  put_kmajor(h->b1, 64, 16, [&](int n, int k) { return k < 8 ? W1[n * kMlpIn + (k & 3)] : 0.f; });
  put_kmajor(h->b2, 64, 64, [&](int n, int k) { return W2[n * kMlpH + k]; });
  put_kmajor(h->b3, 64, 64, [&](int n, int k) { return W3[n * kMlpH + k]; });
  put_kmajor(h->b4, 16, 64, [&](int n, int k) { return n < kMlpOut ? W4[n * kMlpH + k] : 0.f; });
  std::memcpy(h->bias1, params + kOffB1, sizeof(float) * 64);
  std::memcpy(h->bias2, params + kOffB2, sizeof(float) * 64);
  std::memcpy(h->bias3, params + kOffB3, sizeof(float) * 64);
  for (int j = 0; j < 16; j++) h->bias4[j] = j < kMlpOut ? params[kOffB4 + j] : 0.f;
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
  if (e == cudaSuccess) e = cudaMalloc(&s->dev, sizeof(TcNet));
  if (e == cudaSuccess) e = cudaMemcpy(s->dev, h, sizeof(TcNet), cudaMemcpyHostToDevice);
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
  if (!s || n < 0 || (n && (!X || !T))) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  if (n) {
    int dev = 0;
    ARGOT_CUDA_TRY(cudaGetDevice(&dev));
    int rc = kernel_attrs(dev);
    if (rc) { set_status(rc); return rc; }
    int *err = err_flag(dev);
    if (!err) { set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
    const int tiles = (n + kTile - 1) / kTile;
    const int blocks = tiles < 592 ? tiles : 592;
    k_sur_eval<<<blocks, 32 * kSurWarps, eval_smem(), (cudaStream_t)stream>>>(s->dev, X, n, T, err);
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
  if ((rc = kernel_attrs(dev))) { set_status(rc); return rc; }
  GridDev g = make_grid(*gp);
  const uint64_t ncell = (uint64_t)gp->nx * gp->ny * gp->nz;
  const float4 *raw = (const float4 *)packed + ncell;
  cudaStream_t st = (cudaStream_t)stream;
  const int pthreads = 32 * kSurWarps;
  k_sur_predict<<<grid_blocks_for_rates((b1 - b0) * 32, pthreads), pthreads, pred_smem(), st>>>(
      g, raw, t->emit_pos, t->emit_total, t->emit_logT, t->emit_i0, t->emit_m, sur->dev, b0, b1, blk_off, base, rays,
      nray, tau, rates6, work, err);
  ARGOT_CUDA_TRY(cudaGetLastError());
  const int sthreads = 32 * kSelWarps;
  k_sur_select<<<grid_blocks_for_rates((b1 - b0) * 32, sthreads), sthreads, 0, st>>>(
      g, sur->tol, b0, b1, blk_off, base, rays, nray, rates6, work, counters, err);
  ARGOT_CUDA_TRY(cudaGetLastError());
  rc = launch_rate_f32_served(g, raw, t->emit_pos, t->emit_specn, t->emit_total, b0, b1, blk_off, base, rays, nray,
                              tau, rates6, work, err, st);
  if (rc) return rc;
  set_status(0);
  return 0;
}

}  // extern "C"
