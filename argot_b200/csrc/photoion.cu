// photoion.cu -- per-cell photo-ionisation and heating rates from the rays
// of each target block (calc_photoion_rate on the device-resident layout).
#include "photoion.cuh"

namespace argot {

int grid_blocks_for_rates(uint64_t n, int threads);
int *err_flag(int dev);

// the tables of this translation unit's rate kernels
int ensure_tables(int device) { return ensure_rate_tables(device); }

constexpr int kRateWarps = 4;  // warps per CTA in the block-rate kernel

// One warp per target block.  Lanes compute the rates of 32 rays at a time
// into shared memory; then lane j, which owns cell j of the block, adds the
// contributions of the rays that end in its cell in ray order.  No atomics:
// the result does not depend on scheduling.  Each ray's rates are added to
// the existing float value with the reference's float += double rounding
// (calc_photoion_rate.c:403-425).
__global__ void __launch_bounds__(32 * kRateWarps)
    k_rate_blocks(GridDev g, const float4 *__restrict__ raw, const float4 *__restrict__ emit_pos,
                  const double *__restrict__ spec64, uint64_t b0, uint64_t b1,
                  const uint64_t *__restrict__ blk_off, uint64_t base, const uint32_t *__restrict__ rays,
                  uint64_t nray, const float *__restrict__ tau, float *__restrict__ rates6,
                  int *__restrict__ err) {
  __shared__ double buf[kRateWarps][32][7];
  __shared__ int tl[kRateWarps][32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarp = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t ncell = (uint64_t)g.nx * g.ny * g.nz;
  for (uint64_t b = b0 + warp; b < b1; b += nwarp) {
    int ix, iy, iz;
    const bool own_valid = block_cell(g, b, lane, &ix, &iy, &iz);
    const uint64_t own = own_valid ? cell_index(g, ix, iy, iz) : 0;
    float accf[6];
#pragma unroll
    for (int s = 0; s < 6; s++) accf[s] = own_valid ? rates6[s * ncell + own] : 0.f;
    int bix, biy, biz;
    block_cell(g, b, 0, &bix, &biy, &biz);
    uint64_t r0, r1;
    if (!block_rays(blk_off, b, base, nray, &r0, &r1)) {
      if (lane == 0) atomicExch(err, 1);
      continue;
    }
    for (uint64_t rc = r0; rc < r1; rc += 32) {
      const uint64_t r = rc + lane;
      int t = -1;
      if (r < r1) {
        const uint32_t w = __ldg(rays + r);
        const uint32_t e = w >> 5;
        t = (int)(w & 31u);
        const int lx = bix + (t >> 4), ly = biy + ((t >> 2) & 3), lz = biz + (t & 3);
        const float4 ep = __ldg(emit_pos + e);
        const RayGeom geo = ray_geometry(g, g.ix0 + lx, g.iy0 + ly, g.iz0 + lz, ep.x, ep.y, ep.z);
        const float4 rw = __ldg(raw + cell_index(g, lx, ly, lz));
        const RayCols cols = ray_columns(g, __ldg(tau + r), __ldg(tau + nray + r), __ldg(tau + 2 * nray + r), rw, geo);
        double out[6];
        rate_bins_f64(cols, spec64 + (size_t)e * kNu, out);
#pragma unroll
        for (int s = 0; s < 6; s++) buf[wib][lane][s] = out[s];
      }
      tl[wib][lane] = t;
      __syncwarp();
      const int nk = (int)min((uint64_t)32, r1 - rc);
      for (int k = 0; k < nk; k++) {
        if (tl[wib][k] == lane) {
#pragma unroll
          for (int s = 0; s < 6; s++) accf[s] = __double2float_rn(__dadd_rn((double)accf[s], buf[wib][k][s]));
        }
      }
      __syncwarp();
    }
    if (own_valid) {
#pragma unroll
      for (int s = 0; s < 6; s++) rates6[s * ncell + own] = accf[s];
    }
  }
}

// ------------------------------------------------------------ FP32 rates
// One warp per target block, rays in chunks of 32.  Phase A: lane i forms
// the FP32 per-ray parameters of ray i of the chunk (ray_params_f32).
// Phase B: the warp splits into four groups of eight lanes; a group takes
// ARGOT_RATE_RAYS_PER_LANE rays at a time and its lanes share the 256
// frequency bins (lane j: bins j, j+8, ..., two at a time with the packed
// f32x2 arithmetic, ray_bins_packed2), reading the bin-pair table from
// shared memory; three butterfly steps sum the eight partial sums.  Phase C: every lane adds the
// rays that end in its cell, in ray order (add_chunk_in_order).  The
// kernel has no FP64 arithmetic.
// Launch shape: ARGOT_RATE_WARPS warps per CTA, at least ARGOT_RATE_MIN_CTAS
// CTAs resident per SM (which caps the registers per thread), and
// ARGOT_RATE_RAYS_PER_LANE rays per 8-lane group in phase B.  Measured on
// B200 (256^3, 4096 sources, 3.2e9 rays) with the per-cell sums in shared
// memory: one ray per group, 8 warps x 3 CTAs (80 registers, no spills)
// 0.93 s; two rays per group, 8 warps x 2 CTAs (112 registers) 0.85 s,
// x 3 CTAs (80 registers, spilling) 0.94 s.  With the later bin loop (the
// mid-cell form, the 48-byte table, the species stretches, 4-fold unroll)
// two rays per group at 8 warps x 2 CTAs (126 registers) take 0.75 s, at
// 4 warps x 4 CTAs 0.78 s; but the smaller CTAs share the SMs better with
// the march in the overlapped step, which runs 1.2% faster with them
// (1.437 s against 1.454 s); 4 warps x 5 CTAs (96 registers, the
// polynomial iterations unrolled twice, no spills) run the rates alone in
// the same time and the step 2.3% faster again (1.403 s; unrolled four
// times at 5 CTAs the loop spills: rates 0.83 s, step 1.435 s).
#ifndef ARGOT_RATE_WARPS
#define ARGOT_RATE_WARPS 4
#endif
#ifndef ARGOT_RATE_MIN_CTAS
#define ARGOT_RATE_MIN_CTAS 5
#endif
#ifndef ARGOT_RATE_RAYS_PER_LANE
#define ARGOT_RATE_RAYS_PER_LANE 2
#endif
constexpr int kF32Warps = ARGOT_RATE_WARPS;

template <bool kServed>
__global__ void __launch_bounds__(32 * kF32Warps, ARGOT_RATE_MIN_CTAS)
    k_rate_f32(GridDev g, const float4 *__restrict__ raw, const float4 *__restrict__ emit_pos,
               const float *__restrict__ specn, const double *__restrict__ total, uint64_t b0, uint64_t b1,
               const uint64_t *__restrict__ blk_off, uint64_t base, const uint32_t *__restrict__ rays,
               uint64_t nray, const float *__restrict__ tau, float *__restrict__ rates6,
               const float *__restrict__ pred, int *__restrict__ err) {
  __shared__ BinPair s_pairs[kBinPairs];
  __shared__ RateWarpSmem s_w[kF32Warps];
  load_bin_pairs(s_pairs);
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarp = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t b = b0 + warp; b < b1; b += nwarp) {
    uint64_t r0, r1;
    if (!block_rays(blk_off, b, base, nray, &r0, &r1)) {
      if (lane == 0) atomicExch(err, 1);
      continue;
    }
    rate_block_f32<kServed, ARGOT_RATE_RAYS_PER_LANE>(g, raw, emit_pos, specn, total, s_pairs, b, r0, r1, rays,
                                                      nray, tau, rates6, s_w[wib], lane, pred);
  }
}

// The FP32 rates of blocks [b0, b1) where the rays flagged in pred (7
// planes: six contributions and a flag, see rate_block_f32) keep their
// given contributions: the surrogate's second stage.
int launch_rate_f32_served(const GridDev &g, const float4 *raw, const float4 *emit_pos, const float *specn,
                           const double *total, uint64_t b0, uint64_t b1, const uint64_t *blk_off, uint64_t base,
                           const uint32_t *rays, uint64_t nray, const float *tau, float *rates6, const float *pred,
                           int *err, cudaStream_t st) {
  if (b0 >= b1) return 0;
  k_rate_f32<true><<<grid_blocks_for_rates((b1 - b0) * 32, 32 * kF32Warps), 32 * kF32Warps, 0, st>>>(
      g, raw, emit_pos, specn, total, b0, b1, blk_off, base, rays, nray, tau, rates6, pred, err);
  ARGOT_CUDA_TRY(cudaGetLastError());
  return 0;
}

int grid_blocks_for_rates(uint64_t n, int threads) {
  uint64_t b = (n + threads - 1) / threads;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t cap = (uint64_t)sms * 16;
  return (int)(b < cap ? (b ? b : 1) : cap);
}

}  // namespace argot

using namespace argot;

extern "C" int argot_b200_photoion_rays(const argot_b200_grid *gp, const void *packed,
                                        const argot_b200_dev_tree *t, uint64_t b0, uint64_t b1,
                                        const uint64_t *blk_off, uint64_t base, const uint32_t *rays,
                                        uint64_t nray, const float *tau, int mode, float *rates6,
                                        void *stream) {
  uint64_t nb = 0;
  if (!grid_valid(gp) || !packed || !t || !blk_off || !rates6 || (nray && (!rays || !tau)) ||
      argot_b200_num_blocks(gp, &nb) || b0 > b1 || b1 > nb) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  if (mode != ARGOT_B200_RATE_EXACT_F64 && mode != ARGOT_B200_RATE_EXACT_F32) {
    set_status(ARGOT_B200_ENOTSUP);
    return ARGOT_B200_ENOTSUP;
  }
  if (b0 == b1) { set_status(0); return 0; }
  int dev = 0;
  ARGOT_CUDA_TRY(cudaGetDevice(&dev));
  int rc = ensure_tables(dev);
  if (rc) return rc;
  int *err = err_flag(dev);
  if (!err) { set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  GridDev g = make_grid(*gp);
  const uint64_t ncell = (uint64_t)gp->nx * gp->ny * gp->nz;
  const float4 *raw = (const float4 *)packed + ncell;
  cudaStream_t st = (cudaStream_t)stream;
  const int threads = 32 * kRateWarps;
  const int blocks = grid_blocks_for_rates((b1 - b0) * 32, threads);
  if (mode == ARGOT_B200_RATE_EXACT_F64)
    k_rate_blocks<<<blocks, threads, 0, st>>>(g, raw, t->emit_pos, t->emit_spec64, b0, b1, blk_off, base, rays,
                                              nray, tau, rates6, err);
  else
    k_rate_f32<false><<<grid_blocks_for_rates((b1 - b0) * 32, 32 * kF32Warps), 32 * kF32Warps, 0, st>>>(
        g, raw, t->emit_pos, t->emit_specn, t->emit_total, b0, b1, blk_off, base, rays, nray, tau, rates6,
        nullptr, err);
  ARGOT_CUDA_TRY(cudaGetLastError());
  set_status(0);
  return 0;
}
