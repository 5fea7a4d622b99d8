// batch.cu -- many independent problems (meshes + source sets of uneven
// size) in one persistent launch, replayable as a CUDA graph.
//
// The unit of work is a run of consecutive target blocks of one problem (a
// "tile").  Each warp of the persistent grid takes tiles from a device
// queue (one atomic counter) and, for every block of its tile, marches the
// block's rays 32 at a time (one lane per ray, the count-down march with
// Kahan columns) and integrates their rates at once (exact FP32 quadrature,
// eight lanes per ray), so the columns never leave the registers; lane j
// sums the rays of cell j of the block in ray order.  The arithmetic is
// that of argot_b200_march_rays + argot_b200_photoion_rays (EXACT_F32), so
// every problem's rates equal those of the problem run alone, bit for bit.
//
// Tiles are queued largest first (estimated cost: rays x (mesh edge + a
// constant for the quadrature)), so the long tiles of the big meshes start
// early and the short ones fill the tail.
//
// Split mode runs the same tiles through two persistent kernels instead --
// the march (writing the columns of every ray to HBM) and the rates --
// each with its own launch shape, the tile list cut into parts so that
// the rates of one part overlap the march of the next on a second stream.
// The arithmetic is again that of the single-problem kernels.  The mode,
// the tile length, the fused kernel's warps per CTA and CTAs per SM and the
// number of parts are chosen by argot_b200_batch_tune, which times
// candidate configurations on the batch itself.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <new>
#include <numeric>
#include <vector>

#include "march.cuh"
#include "photoion.cuh"

namespace argot {

int *err_flag(int dev);

struct BatchProb {
  GridDev g;
  const float4 *cells;  // packed products (the march's gathers)
  const float4 *raw;    // packed raw fields (target cells of the rates)
  const float4 *emit_pos;
  const float *specn;
  const double *total;
  const uint64_t *blk_off;
  const uint32_t *rays;  // every ray of the problem, base 0
  float *rates6;
  uint64_t nray;
  float *tau;  // split mode: three column planes of nray (batch-owned)
};

struct BatchItem {
  uint32_t prob, b0, b1, pad;
};

// Launch shape: kWarps warps per CTA and at least ARGOT_BATCH_MIN_WARPS / kWarps
// CTAs resident per SM (which caps the registers per thread).  Measured on
// B200 (the 48-problem batch): 32 warps per SM (64 registers) run the step
// 22% faster than 16.
#ifndef ARGOT_BATCH_MIN_WARPS
#define ARGOT_BATCH_MIN_WARPS 32
#endif
template <int kWarps>
__global__ void __launch_bounds__(32 * kWarps, ARGOT_BATCH_MIN_WARPS / kWarps)
    k_batch(const BatchProb *__restrict__ probs, const BatchItem *__restrict__ items, uint32_t nitems,
            uint32_t *__restrict__ next, unsigned long long *__restrict__ crossings, int *__restrict__ err) {
  __shared__ BinPair s_pairs[kBinPairs];
  __shared__ float s_nd[kWarps][32][6];
  __shared__ float s_p[kWarps][32][3];
  __shared__ float s_out[kWarps][32][6];
  __shared__ int s_e[kWarps][32], s_t[kWarps][32], s_cnt[kWarps][32], s_src[kWarps][32];
  __shared__ int s_nsfu[kWarps][32];
  load_bin_pairs(s_pairs);
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int grp = lane >> 3, j = lane & 7;
  const unsigned gmask = 0xffu << (8 * grp);
  unsigned long long steps_total = 0;
  bool bad = false;
  for (;;) {
    uint32_t it = 0;
    if (lane == 0) it = atomicAdd(next, 1u);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= nitems) break;
    const BatchItem wi = items[it];
    const BatchProb &P = probs[wi.prob];
    const GridDev g = P.g;
    const float4 *__restrict__ cells = P.cells;
    const float4 *__restrict__ raw = P.raw;
    const float4 *__restrict__ emit_pos = P.emit_pos;
    const float *__restrict__ specn = P.specn;
    const double *__restrict__ total = P.total;
    const uint32_t *__restrict__ rays = P.rays;
    float *__restrict__ rates6 = P.rates6;
    const uint64_t ncell = (uint64_t)g.nx * g.ny * g.nz;
    for (uint64_t b = wi.b0; b < wi.b1; b++) {
      int ix, iy, iz;
      const bool own_valid = block_cell(g, b, lane, &ix, &iy, &iz);
      const uint64_t own = own_valid ? cell_index(g, ix, iy, iz) : 0;
      CellSum6 acc;
      acc.zero();
      int bix, biy, biz;
      block_cell(g, b, 0, &bix, &biy, &biz);
      const uint64_t r0 = P.blk_off[b], r1 = P.blk_off[b + 1];
      for (uint64_t rc = r0; rc < r1; rc += 32) {
        const uint64_t r = rc + lane;
        int t = -1;
        if (r < r1) {
          const uint32_t w = __ldg(rays + r);
          const uint32_t e = w >> 5;
          t = (int)(w & 31u);
          const int lx = bix + (t >> 4), ly = biy + ((t >> 2) & 3), lz = biz + (t & 3);
          // the march (as argot_b200_march_rays, Kahan columns)
          const float xe = cell_centre(g.xmin, g.ix0 + lx, g.dx);
          const float ye = cell_centre(g.ymin, g.iy0 + ly, g.dy);
          const float ze = cell_centre(g.zmin, g.iz0 + lz, g.dz);
          const float4 ep = __ldg(emit_pos + e);
          float xs, ys, zs;
          ray_start(g, ep.x, ep.y, ep.z, xe, ye, ze, &xs, &ys, &zs);
          int steps = 0;
          const Tau3 tt = march_kahan<0, true>(g, cells, xs, ys, zs, xe, ye, ze, &steps, &bad);
          steps_total += (unsigned long long)steps;
          // the rate parameters (as argot_b200_photoion_rays)
          const float4 rw = __ldg(raw + cell_index(g, lx, ly, lz));
          const RayParams p = ray_params_f32(g, g.ix0 + lx, g.iy0 + ly, g.iz0 + lz, ep.x, ep.y, ep.z, tt.hi, tt.hei,
                                             tt.heii, rw, __ldg(total + e));
#pragma unroll
          for (int s = 0; s < 3; s++) {
            s_nd[wib][lane][s] = p.N[s];
            s_nd[wib][lane][3 + s] = p.D[s];
            s_p[wib][lane][s] = p.P[s];
          }
          s_e[wib][lane] = (int)e;
          s_nsfu[wib][lane] = sfu_iters(p.D[0], p.D[1], p.D[2]);
        }
        s_t[wib][lane] = t;
        __syncwarp();
        const int nk = (int)min((uint64_t)32, r1 - rc);
        // rounds of four rays with one SFU count, as in rate_block_f32
        for (int q0 = 0; q0 < nk; q0 += 4) {
          const int q = q0 + grp < nk ? q0 + grp : q0;
          int nsfu = 0;
#pragma unroll
          for (int k = 0; k < 4; k++) nsfu = max(nsfu, q0 + k < nk ? s_nsfu[wib][q0 + k] : 0);
          const float N0 = s_nd[wib][q][0], N1 = s_nd[wib][q][1], N2 = s_nd[wib][q][2];
          const float D0 = s_nd[wib][q][3], D1 = s_nd[wib][q][4], D2 = s_nd[wib][q][5];
          const float *sp = specn + (size_t)s_e[wib][q] * kNu;
          float part[6];
          ray_bins_packed(s_pairs, sp, j, nsfu, s_nsfu[wib][q], N0, N1, N2, D0, D1, D2, part);
#pragma unroll
          for (int o = 1; o < 8; o <<= 1) {
#pragma unroll
            for (int s = 0; s < 6; s++) part[s] += __shfl_xor_sync(gmask, part[s], o);
          }
          if (j == 0 && q0 + grp < nk) {
            const float Pq[3] = {s_p[wib][q][0], s_p[wib][q][1], s_p[wib][q][2]};
            float out[6];
            ray_rates6(Pq, part[0], part[1], part[2], part[3], part[4], part[5], out);
#pragma unroll
            for (int s = 0; s < 6; s++) s_out[wib][q][s] = out[s];
          }
        }
        __syncwarp();
        add_chunk_in_order(acc, lane, t, s_out[wib], s_cnt[wib], s_src[wib]);
      }
      if (own_valid) {
#pragma unroll
        for (int s = 0; s < 6; s++) rates6[s * ncell + own] = acc.s[s];
      }
    }
  }
  if (crossings) {
    for (int o = 16; o; o >>= 1) steps_total += __shfl_xor_sync(0xffffffffu, steps_total, o);
    if (lane == 0 && steps_total) atomicAdd(crossings, steps_total);
  }
  if (bad) atomicExch(err, 1);
}

// ---- split mode: the march and the rates as two persistent kernels over
// the same tiles, their columns through HBM, so that each runs with its own
// launch shape; a part of the tile list is integrated while the next part
// is marched (two streams, one graph).

// Launch shapes of the split kernels (as the single-problem kernels).
#ifndef ARGOT_SPLIT_MARCH_MIN_CTAS
#define ARGOT_SPLIT_MARCH_MIN_CTAS 6
#endif
#ifndef ARGOT_SPLIT_RATE_MIN_CTAS
#define ARGOT_SPLIT_RATE_MIN_CTAS 2
#endif
#ifndef ARGOT_SPLIT_RATE_RAYS_PER_LANE
#define ARGOT_SPLIT_RATE_RAYS_PER_LANE 2
#endif
constexpr int kSplitRateWarps = 8;

__global__ void __launch_bounds__(256, ARGOT_SPLIT_MARCH_MIN_CTAS)
    k_batch_march(const BatchProb *__restrict__ probs, const BatchItem *__restrict__ items, uint32_t i0,
                  uint32_t i1, uint32_t *__restrict__ next, unsigned long long *__restrict__ crossings,
                  int *__restrict__ err) {
  const int lane = threadIdx.x & 31;
  unsigned long long steps_total = 0;
  bool bad = false;
  for (;;) {
    uint32_t it = 0;
    if (lane == 0) it = i0 + atomicAdd(next, 1u);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= i1) break;
    const BatchItem wi = items[it];
    const BatchProb &P = probs[wi.prob];
    const GridDev g = P.g;
    for (uint64_t b = wi.b0; b < wi.b1; b++) {
      const uint64_t r0 = P.blk_off[b], r1 = P.blk_off[b + 1];
      int bix, biy, biz;
      block_cell(g, b, 0, &bix, &biy, &biz);
      for (uint64_t r = r0 + lane; r < r1; r += 32) {
        const uint32_t w = __ldg(P.rays + r);
        const int l = (int)(w & 31u);
        const float xe = cell_centre(g.xmin, g.ix0 + bix + (l >> 4), g.dx);
        const float ye = cell_centre(g.ymin, g.iy0 + biy + ((l >> 2) & 3), g.dy);
        const float ze = cell_centre(g.zmin, g.iz0 + biz + (l & 3), g.dz);
        const float4 ep = __ldg(P.emit_pos + (w >> 5));
        float xs, ys, zs;
        ray_start(g, ep.x, ep.y, ep.z, xe, ye, ze, &xs, &ys, &zs);
        int steps = 0;
        const Tau3 t = march_kahan<0, true>(g, P.cells, xs, ys, zs, xe, ye, ze, &steps, &bad);
        P.tau[r] = t.hi;
        P.tau[P.nray + r] = t.hei;
        P.tau[2 * P.nray + r] = t.heii;
        steps_total += (unsigned long long)steps;
      }
    }
  }
  if (crossings) {
    for (int o = 16; o; o >>= 1) steps_total += __shfl_xor_sync(0xffffffffu, steps_total, o);
    if (lane == 0 && steps_total) atomicAdd(crossings, steps_total);
  }
  if (bad) atomicExch(err, 1);
}

__global__ void __launch_bounds__(32 * kSplitRateWarps, ARGOT_SPLIT_RATE_MIN_CTAS)
    k_batch_rates(const BatchProb *__restrict__ probs, const BatchItem *__restrict__ items, uint32_t i0,
                  uint32_t i1, uint32_t *__restrict__ next) {
  __shared__ BinPair s_pairs[kBinPairs];
  __shared__ RateWarpSmem s_w[kSplitRateWarps];
  load_bin_pairs(s_pairs);
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  for (;;) {
    uint32_t it = 0;
    if (lane == 0) it = i0 + atomicAdd(next, 1u);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= i1) break;
    const BatchItem wi = items[it];
    const BatchProb &P = probs[wi.prob];
    const GridDev g = P.g;
    for (uint64_t b = wi.b0; b < wi.b1; b++)
      rate_block_f32<false, ARGOT_SPLIT_RATE_RAYS_PER_LANE>(g, P.raw, P.emit_pos, P.specn, P.total, s_pairs, b,
                                                            P.blk_off[b], P.blk_off[b + 1], P.rays, P.nray, P.tau,
                                                            P.rates6, s_w[wib], lane);
  }
}

}  // namespace argot

using namespace argot;

struct argot_b200_batch {
  int device = 0;
  int sms = 148;
  std::vector<BatchProb> probs;
  std::vector<std::vector<uint64_t>> blk_off;  // host copies (tiles and costs)
  BatchProb *probs_dev = nullptr;
  BatchItem *items_dev = nullptr;
  size_t items_cap = 0;
  uint32_t nitems = 0;
  uint32_t *next_dev = nullptr;
  int *err = nullptr;
  argot_b200_batch_config cfg{8, 0, 4, 0, 0, 8};
  int grid = 0;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // split mode
  float *tau = nullptr;             // column planes of every problem
  uint64_t total_rays = 0;
  cudaStream_t side = nullptr;      // the rates' stream
  cudaStream_t side_cap = nullptr;  // the rates' stream while capturing
  std::vector<cudaEvent_t> ev;      // fork, one per part, join
  uint32_t *counters = nullptr;     // two per part
  int grid_march = 0, grid_rates = 0;
};

namespace {

void drop_graph(argot_b200_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

int max_ctas_per_sm(int warps) {
  int n = 0;
  cudaError_t e = warps == 4 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch<4>, 128, 0)
                             : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch<8>, 256, 0);
  return e == cudaSuccess ? n : 0;
}

constexpr int kMaxParts = 64;

bool config_valid(const argot_b200_batch_config &c) {
  return (c.warps_per_cta == 4 || c.warps_per_cta == 8) && c.ctas_per_sm >= 0 && c.ctas_per_sm <= 16 &&
         c.blocks_per_item >= 1 && c.blocks_per_item <= 4096 && (c.order == 0 || c.order == 1) &&
         (c.mode == 0 || c.mode == 1) && c.parts >= 1 && c.parts <= kMaxParts;
}

// The split mode's buffers (columns of every ray, counters, second stream
// and events), made on first use.
int ensure_split(argot_b200_batch *b) {
  if (b->tau) return 0;
  if (b->total_rays) {
    if (cudaMalloc(&b->tau, sizeof(float) * 3 * b->total_rays) != cudaSuccess) {
      cudaGetLastError();
      b->tau = nullptr;
      return ARGOT_B200_ENOMEM;
    }
  } else {
    ARGOT_CUDA_TRY(cudaMalloc(&b->tau, 16));
  }
  ARGOT_CUDA_TRY(cudaMalloc(&b->counters, sizeof(uint32_t) * 2 * kMaxParts));
  ARGOT_CUDA_TRY(cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking));
  ARGOT_CUDA_TRY(cudaStreamCreateWithFlags(&b->side_cap, cudaStreamNonBlocking));
  b->ev.resize(kMaxParts + 2);
  for (auto &e : b->ev) ARGOT_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  uint64_t off = 0;
  for (auto &q : b->probs) {
    q.tau = b->tau + 3 * off;
    off += q.nray;
  }
  ARGOT_CUDA_TRY(cudaMemcpy(b->probs_dev, b->probs.data(), sizeof(BatchProb) * b->probs.size(),
                            cudaMemcpyHostToDevice));
  int n = 0;
  ARGOT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_march, 256, 0));
  b->grid_march = b->sms * (n > 0 ? n : 1);
  ARGOT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_rates, 32 * kSplitRateWarps, 0));
  b->grid_rates = b->sms * (n > 0 ? n : 1);
  return 0;
}

// Work list of the configuration: tiles of blocks_per_item consecutive
// blocks, in problem order or by estimated cost (largest first; ties keep
// problem order, so the list is deterministic).
int build_items(argot_b200_batch *b) {
  std::vector<BatchItem> items;
  std::vector<double> cost;
  const uint32_t L = (uint32_t)b->cfg.blocks_per_item;
  for (size_t p = 0; p < b->probs.size(); p++) {
    const std::vector<uint64_t> &off = b->blk_off[p];
    const uint32_t nb = (uint32_t)(off.size() - 1);
    const double per_ray = (double)b->probs[p].g.nx + 64.0;  // march steps + quadrature, in march steps
    for (uint32_t b0 = 0; b0 < nb; b0 += L) {
      const uint32_t b1 = std::min(nb, b0 + L);
      items.push_back({(uint32_t)p, b0, b1, 0u});
      cost.push_back((double)(off[b1] - off[b0]) * per_ray + 1.0);
    }
  }
  if (b->cfg.order == 0) {
    std::vector<size_t> idx(items.size());
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t c) { return cost[a] > cost[c]; });
    std::vector<BatchItem> sorted(items.size());
    for (size_t i = 0; i < idx.size(); i++) sorted[i] = items[idx[i]];
    items.swap(sorted);
  }
  if (items.size() > 0xffffffffull) return ARGOT_B200_EINVAL;
  if (items.size() > b->items_cap) {
    cudaFree(b->items_dev);
    b->items_dev = nullptr;
    b->items_cap = 0;
    ARGOT_CUDA_TRY(cudaMalloc(&b->items_dev, sizeof(BatchItem) * std::max<size_t>(items.size(), 1)));
    b->items_cap = items.size();
  }
  if (!items.empty())
    ARGOT_CUDA_TRY(cudaMemcpy(b->items_dev, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice));
  b->nitems = (uint32_t)items.size();
  const int occ = max_ctas_per_sm(b->cfg.warps_per_cta);
  if (occ <= 0) return ARGOT_B200_ECUDA;
  const int per_sm = b->cfg.ctas_per_sm > 0 ? std::min(b->cfg.ctas_per_sm, occ) : occ;
  const uint64_t warps_needed = std::max<uint64_t>(1, b->nitems);
  const uint64_t ctas_needed = (warps_needed + b->cfg.warps_per_cta - 1) / b->cfg.warps_per_cta;
  b->grid = (int)std::min<uint64_t>((uint64_t)b->sms * per_sm, ctas_needed);
  drop_graph(b);
  return 0;
}

// Split mode: the tile list cut into parts; part p is marched on `st`,
// then integrated on the side stream once its march is done, while `st`
// marches part p + 1.  The side stream joins `st` at the end.
int launch_split(argot_b200_batch *b, unsigned long long *crossings, cudaStream_t st, cudaStream_t side) {
  const int parts = b->cfg.parts;
  ARGOT_CUDA_TRY(cudaMemsetAsync(b->counters, 0, sizeof(uint32_t) * 2 * parts, st));
  ARGOT_CUDA_TRY(cudaEventRecord(b->ev[0], st));
  ARGOT_CUDA_TRY(cudaStreamWaitEvent(side, b->ev[0], 0));
  for (int p = 0; p < parts; p++) {
    const uint32_t i0 = (uint32_t)((uint64_t)b->nitems * p / parts);
    const uint32_t i1 = (uint32_t)((uint64_t)b->nitems * (p + 1) / parts);
    k_batch_march<<<b->grid_march, 256, 0, st>>>(b->probs_dev, b->items_dev, i0, i1, b->counters + 2 * p,
                                                  crossings, b->err);
    ARGOT_CUDA_TRY(cudaGetLastError());
    ARGOT_CUDA_TRY(cudaEventRecord(b->ev[1 + p], st));
    ARGOT_CUDA_TRY(cudaStreamWaitEvent(side, b->ev[1 + p], 0));
    k_batch_rates<<<b->grid_rates, 32 * kSplitRateWarps, 0, side>>>(b->probs_dev, b->items_dev, i0, i1,
                                                                      b->counters + 2 * p + 1);
    ARGOT_CUDA_TRY(cudaGetLastError());
  }
  ARGOT_CUDA_TRY(cudaEventRecord(b->ev[1 + parts], side));
  ARGOT_CUDA_TRY(cudaStreamWaitEvent(st, b->ev[1 + parts], 0));
  return 0;
}

int launch(argot_b200_batch *b, unsigned long long *crossings, cudaStream_t st, bool capturing = false) {
  if (b->cfg.mode == 1) {
    int rc = ensure_split(b);
    if (rc) return rc;
    return launch_split(b, crossings, st, capturing ? b->side_cap : b->side);
  }
  ARGOT_CUDA_TRY(cudaMemsetAsync(b->next_dev, 0, sizeof(uint32_t), st));
  if (b->cfg.warps_per_cta == 4)
    k_batch<4><<<b->grid, 128, 0, st>>>(b->probs_dev, b->items_dev, b->nitems, b->next_dev, crossings, b->err);
  else
    k_batch<8><<<b->grid, 256, 0, st>>>(b->probs_dev, b->items_dev, b->nitems, b->next_dev, crossings, b->err);
  ARGOT_CUDA_TRY(cudaGetLastError());
  return 0;
}

}  // namespace

extern "C" {

int argot_b200_batch_create(const argot_b200_batch_problem *p, int n, argot_b200_batch **out) {
  if (!p || n <= 0 || !out) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  for (int i = 0; i < n; i++) {
    uint64_t nb = 0;
    const argot_b200_dev_tree *t = p[i].tree;
    if (!grid_valid(&p[i].grid) || !p[i].packed_dev || !t || !p[i].blk_offsets_dev || !p[i].blk_offsets_host ||
        !p[i].rates6_dev || argot_b200_num_blocks(&p[i].grid, &nb) || nb >= 0xffffffffull ||
        (p[i].blk_offsets_host[nb] && !p[i].rays_dev) || p[i].blk_offsets_host[0] != 0) {
      set_status(ARGOT_B200_EINVAL);
      return ARGOT_B200_EINVAL;
    }
  }
  auto *b = new (std::nothrow) argot_b200_batch();
  if (!b) { set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  auto fail = [&](int rc) {
    argot_b200_batch_free(b);
    set_status(rc);
    return rc;
  };
  if (cudaGetDevice(&b->device) != cudaSuccess) return fail(ARGOT_B200_ECUDA);
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
  int rc = ensure_rate_tables(b->device);
  if (rc) return fail(rc);
  b->err = err_flag(b->device);
  if (!b->err) return fail(ARGOT_B200_ENOMEM);
  for (int i = 0; i < n; i++) {
    uint64_t nb = 0;
    argot_b200_num_blocks(&p[i].grid, &nb);
    const uint64_t ncell = (uint64_t)p[i].grid.nx * p[i].grid.ny * p[i].grid.nz;
    BatchProb q;
    q.g = make_grid(p[i].grid);
    q.cells = (const float4 *)p[i].packed_dev;
    q.raw = (const float4 *)p[i].packed_dev + ncell;
    q.emit_pos = p[i].tree->emit_pos;
    q.specn = p[i].tree->emit_specn;
    q.total = p[i].tree->emit_total;
    q.blk_off = p[i].blk_offsets_dev;
    q.rays = p[i].rays_dev;
    q.rates6 = p[i].rates6_dev;
    q.nray = p[i].blk_offsets_host[nb];
    q.tau = nullptr;
    b->total_rays += q.nray;
    b->probs.push_back(q);
    b->blk_off.emplace_back(p[i].blk_offsets_host, p[i].blk_offsets_host + nb + 1);
  }
  if (cudaMalloc(&b->probs_dev, sizeof(BatchProb) * n) != cudaSuccess) return fail(ARGOT_B200_ENOMEM);
  if (cudaMemcpy(b->probs_dev, b->probs.data(), sizeof(BatchProb) * n, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(ARGOT_B200_ECUDA);
  if (cudaMalloc(&b->next_dev, sizeof(uint32_t)) != cudaSuccess) return fail(ARGOT_B200_ENOMEM);
  if (cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess) return fail(ARGOT_B200_ECUDA);
  rc = build_items(b);
  if (rc) return fail(rc);
  *out = b;
  set_status(0);
  return 0;
}

void argot_b200_batch_free(argot_b200_batch *b) {
  if (!b) return;
  drop_graph(b);
  if (b->cap) cudaStreamDestroy(b->cap);
  if (b->side) cudaStreamDestroy(b->side);
  if (b->side_cap) cudaStreamDestroy(b->side_cap);
  for (auto e : b->ev) cudaEventDestroy(e);
  cudaFree(b->tau);
  cudaFree(b->counters);
  cudaFree(b->probs_dev);
  cudaFree(b->items_dev);
  cudaFree(b->next_dev);
  delete b;
}

int argot_b200_batch_configure(argot_b200_batch *b, const argot_b200_batch_config *c) {
  if (!b || !c || !config_valid(*c)) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  b->cfg = *c;
  const int rc = build_items(b);
  set_status(rc);
  return rc;
}

int argot_b200_batch_get_config(const argot_b200_batch *b, argot_b200_batch_config *c) {
  if (!b || !c) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  *c = b->cfg;
  set_status(0);
  return 0;
}

int argot_b200_batch_num_items(const argot_b200_batch *b) { return b ? (int)b->nitems : -1; }

int argot_b200_batch_run(argot_b200_batch *b, unsigned long long *crossings_dev, void *stream) {
  if (!b) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  const int rc = launch(b, crossings_dev, (cudaStream_t)stream);
  set_status(rc);
  return rc;
}

int argot_b200_batch_graph_launch(argot_b200_batch *b, void *stream) {
  if (!b) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  if (!b->exec) {
    if (b->cfg.mode == 1) {
      const int r = ensure_split(b);  // allocates: must precede the capture
      if (r) { set_status(r); return r; }
    }
    ARGOT_CUDA_TRY(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    const int rc = launch(b, nullptr, b->cap, true);
    cudaGraph_t gr = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->cap, &gr);
    if (rc || e != cudaSuccess) {
      if (gr) cudaGraphDestroy(gr);
      const int r = rc ? rc : status_from_cuda(e);
      set_status(r);
      return r;
    }
    b->graph = gr;
    ARGOT_CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
  }
  ARGOT_CUDA_TRY(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
  set_status(0);
  return 0;
}

// Coordinate search over the configuration (the fused kernel's warps per
// CTA and CTAs per SM, tile length, queue order, fused or split mode, the
// split mode's number of parts): starting from the current one, each
// parameter in turn takes every candidate value with the others held;
// a candidate is timed by CUDA events around `reps` launches after one
// warm-up launch.  Leaves the best configuration set.
int argot_b200_batch_tune(argot_b200_batch *b, int reps, argot_b200_batch_config *best_out, float *best_ms,
                          void *stream) {
  if (!b || reps < 1) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  cudaStream_t st = (cudaStream_t)stream;
  cudaEvent_t e0, e1;
  ARGOT_CUDA_TRY(cudaEventCreate(&e0));
  ARGOT_CUDA_TRY(cudaEventCreate(&e1));
  auto time_cfg = [&](const argot_b200_batch_config &c, float *ms) -> int {
    b->cfg = c;
    int rc = build_items(b);
    if (rc) return rc;
    if ((rc = launch(b, nullptr, st))) return rc;
    ARGOT_CUDA_TRY(cudaEventRecord(e0, st));
    for (int i = 0; i < reps; i++)
      if ((rc = launch(b, nullptr, st))) return rc;
    ARGOT_CUDA_TRY(cudaEventRecord(e1, st));
    ARGOT_CUDA_TRY(cudaEventSynchronize(e1));
    ARGOT_CUDA_TRY(cudaEventElapsedTime(ms, e0, e1));
    *ms /= (float)reps;
    return 0;
  };
  argot_b200_batch_config best = b->cfg;
  float t_best = 0.f;
  int rc = time_cfg(best, &t_best);
  const int warps[] = {4, 8};
  const int per_sm[] = {1, 2, 3, 4, 6, 8};
  const int tiles[] = {1, 2, 4, 8, 16, 64};
  const int orders[] = {0, 1};
  const int modes[] = {0, 1};
  const int nparts[] = {2, 4, 8, 16};
  for (int pass = 0; pass < 2 && !rc; pass++) {
    for (int dim = 0; dim < 6 && !rc; dim++) {
      // the fused kernel's launch shape only matters in fused mode, the
      // number of parts only in split mode
      if ((dim <= 1 && best.mode == 1) || (dim == 5 && best.mode == 0)) continue;
      const int *vals = dim == 0 ? warps : dim == 1 ? per_sm : dim == 2 ? tiles : dim == 3 ? orders
                      : dim == 4 ? modes : nparts;
      const int nv = dim == 0 ? 2 : dim == 1 ? 6 : dim == 2 ? 6 : dim == 3 ? 2 : dim == 4 ? 2 : 4;
      for (int k = 0; k < nv && !rc; k++) {
        argot_b200_batch_config c = best;
        int *field = dim == 0 ? &c.warps_per_cta : dim == 1 ? &c.ctas_per_sm : dim == 2 ? &c.blocks_per_item
                   : dim == 3 ? &c.order : dim == 4 ? &c.mode : &c.parts;
        if (*field == vals[k]) continue;
        *field = vals[k];
        if (dim == 1 && vals[k] > max_ctas_per_sm(c.warps_per_cta)) continue;
        if (c.mode == 1 && ensure_split(b) != 0) continue;  // no room for the columns: fused only
        float t = 0.f;
        rc = time_cfg(c, &t);
        if (!rc && t < t_best) {
          t_best = t;
          best = c;
        }
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) { set_status(rc); return rc; }
  b->cfg = best;
  rc = build_items(b);
  if (rc) { set_status(rc); return rc; }
  if (best_out) *best_out = best;
  if (best_ms) *best_ms = t_best;
  set_status(0);
  return 0;
}

}  // extern "C"
