// march.cu -- field packing, light-ray generation (tree walk), the segment
// march (calc_optical_depth) and the stitching of segment columns
// (accum_optical_depth) on sm_100a.
#include <cub/device/device_scan.cuh>

#include "march.cuh"

namespace argot {

// ------------------------------------------------------------------ packing
// cells[c] = {n_HI, n_HeI, n_HeII, 0} with the reference's per-crossing
// products (calc_optical_depth.c:150-155): n_HI = dens*fHI in float,
// n_He = (float)(dens * HELIUM_FACT) in double, n_HeI = n_He*fHeI in float.
// raw[c] = {dens, fHI, fHeI, fHeII} for the rate stage, which forms its own
// products in double (calc_photoion_rate.c:211-218).
__global__ void k_pack_fields(uint64_t n, const float *__restrict__ dens, const float *__restrict__ fHI,
                              const float *__restrict__ fHeI, const float *__restrict__ fHeII,
                              float4 *__restrict__ cells, float4 *__restrict__ raw) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float d = dens[i], a = fHI[i], b = fHeI[i], c = fHeII[i];
    const float nhe = __double2float_rn(__dmul_rn((double)d, kHeliumFact));
    cells[i] = make_float4(__fmul_rn(d, a), __fmul_rn(nhe, b), __fmul_rn(nhe, c), 0.f);
    if (raw) raw[i] = make_float4(d, a, b, c);
  }
}

static int grid_blocks_for(uint64_t n, int threads) {
  uint64_t b = (n + threads - 1) / threads;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t cap = (uint64_t)sms * 16;
  return (int)(b < cap ? (b ? b : 1) : cap);
}

// --------------------------------------------------------------- tree walk
// One warp per block of 32 target cells.  The warp walks the preorder node
// array once for all its lanes; a lane that accepts node v (r^2 theta^2 >
// side^2, all in float as setup_light_ray_tree.c:341-354) records v's
// subtree end and stays idle until the walk leaves that subtree.  A node is
// opened when any lane needs it: internal nodes descend into their children
// (octant order), leaves (<= 1 source) emit one ray per source.  Each lane
// therefore sees the nodes in the reference's depth-first order and emits
// its rays in the reference's order.
template <bool kEmit>
__global__ void __launch_bounds__(256) k_walk(GridDev g, const DevNode *__restrict__ nodes, int n_nodes,
                                              const int *__restrict__ src_list, float theta_sq,
                                              uint64_t b0, uint64_t b1, uint64_t *__restrict__ blk_count,
                                              uint32_t *__restrict__ cell_count,
                                              const uint64_t *__restrict__ blk_off, uint64_t base,
                                              uint32_t *__restrict__ rays, int *__restrict__ err) {
  const int lane = threadIdx.x & 31;
  bool bad = false;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarp = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned lt = (1u << lane) - 1u;
  for (uint64_t b = b0 + warp; b < b1; b += nwarp) {
    int ix, iy, iz;
    const bool valid = block_cell(g, b, lane, &ix, &iy, &iz);
    const float px = cell_centre(g.xmin, g.ix0 + ix, g.dx);
    const float py = cell_centre(g.ymin, g.iy0 + iy, g.dy);
    const float pz = cell_centre(g.zmin, g.iz0 + iz, g.dz);
    int blocked_until = 0;
    uint32_t mine = 0;
    // emission: the block's rays go to [blk_off[b], blk_off[b + 1]) - base;
    // a ray past that range (offsets not counted for this tree and angle)
    // is dropped and the error flag set
    uint64_t off = 0, end = 0;
    if (kEmit) {
      const uint64_t a = blk_off[b], e = blk_off[b + 1];
      if (a < base || e < a) { bad = true; continue; }
      off = a - base;
      end = e - base;
    }
    int cur = 0;
    while (cur < n_nodes) {
      const DevNode nd = nodes[cur];
      const bool act = valid && cur >= blocked_until;
      const float ddx = __fsub_rn(px, nd.cx), ddy = __fsub_rn(py, nd.cy), ddz = __fsub_rn(pz, nd.cz);
      const float r2 = __fadd_rn(__fadd_rn(__fmul_rn(ddx, ddx), __fmul_rn(ddy, ddy)), __fmul_rn(ddz, ddz));
      const bool acc = act && (__fmul_rn(r2, theta_sq) > __fmul_rn(nd.len, nd.len));
      const bool opn = act && !acc;
      const unsigned macc = __ballot_sync(0xffffffffu, acc);
      const unsigned mopn = __ballot_sync(0xffffffffu, opn);
      if (macc) {
        if (kEmit) {
          const uint64_t at = off + __popc(macc & lt);
          if (acc) {
            if (at < end) rays[at] = ((uint32_t)cur << 5) | (uint32_t)lane;
            else bad = true;
          }
          off += __popc(macc);
        } else {
          mine += acc;
        }
      }
      int next = nd.skip;
      if (mopn) {
        if (nd.n > 1) {
          if (nd.has_child) {
            if (acc) blocked_until = nd.skip;
            next = cur + 1;
          }
        } else {
          for (int j = 0; j < nd.n; j++) {
            const uint32_t e = (uint32_t)(n_nodes + src_list[nd.src_first + j]);
            if (kEmit) {
              const uint64_t at = off + __popc(mopn & lt);
              if (opn) {
                if (at < end) rays[at] = (e << 5) | (uint32_t)lane;
                else bad = true;
              }
              off += __popc(mopn);
            } else {
              mine += opn;
            }
          }
        }
      }
      cur = next;
    }
    if (!kEmit) {
      if (cell_count && valid) cell_count[cell_index(g, ix, iy, iz)] = mine;
      uint32_t tot = mine;
      for (int o = 16; o; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
      if (lane == 0) blk_count[b] = tot;
    }
  }
  if (kEmit && bad) atomicExch(err, 1);
}

// -------------------------------------------------------------- ray march
// One warp per target block; the warp takes the block's rays 32 at a time.
// Consecutive rays of a block come from the same emitter and end in
// neighbouring cells, so the 32 lanes march nearly parallel paths of nearly
// equal length and their gathers hit the same cache lines.
// Launch shape: 256 threads, at least ARGOT_MARCH_MIN_CTAS CTAs resident per
// SM (which caps the registers per thread).  The march is bound by the
// latency of its cache-hit gathers, so resident warps matter more than
// registers: measured on B200 at 256^3 / 4096 sources with the fixed-point
// walk, 8 CTAs (32 registers) 1.15 s, 7 CTAs 1.15 s, 6 CTAs (40 registers)
// 1.21 s.  What lives across a ray's walk is kept out of registers: the
// Kahan columns in per-thread shared-memory slots, the block's state (block
// index, ray count, packed coordinates, first ray; the same for the warp's
// lanes) in per-warp shared memory, read back after each ray.  That took the
// 8-CTA launch from 1.76 s (spilling) to 1.15 s.  kInside: every emitter
// lies inside the box (the host checks the emitters' bounding box), so rays
// start at their emitter and the launch contains no call.
#ifndef ARGOT_MARCH_MIN_CTAS
#define ARGOT_MARCH_MIN_CTAS 8
#endif
#ifndef ARGOT_MARCH_CENTRE_END
#define ARGOT_MARCH_CENTRE_END true
#endif
// CTA size (measured at 256^3 / 4096 sources: 128 threads x 16 CTAs run the
// march alone 5% faster than 256 x 8, but the step that overlaps it with
// the rates 0.6% slower).
#ifndef ARGOT_MARCH_THREADS
#define ARGOT_MARCH_THREADS 256
#endif
constexpr int kMarchThreads = ARGOT_MARCH_THREADS;
template <int kPrec, bool kInside>
__global__ void __launch_bounds__(kMarchThreads, ARGOT_MARCH_MIN_CTAS) k_march_rays(GridDev g, const float4 *__restrict__ cells,
                                                    const float4 *__restrict__ emit_pos, uint32_t b0,
                                                    uint32_t b1, const uint64_t *__restrict__ blk_off,
                                                    uint64_t base, const uint32_t *__restrict__ rays,
                                                    uint64_t nray, float *__restrict__ tau,
                                                    unsigned long long *__restrict__ crossings,
                                                    int *__restrict__ err) {
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarp = (gridDim.x * blockDim.x) >> 5;
  __shared__ float kslot[6 * kMarchThreads];  // the Kahan columns, one slot per thread
  // the block's state, the same for the warp's lanes: it is read back from
  // shared memory after each ray instead of staying live in registers
  // across the walk (block index, ray count, packed coordinates, first ray)
  __shared__ uint32_t wstate[kMarchThreads / 32][5];
  volatile uint32_t *ws = wstate[threadIdx.x >> 5];
  bool bad = false;
  for (uint32_t b = b0 + warp; b < b1; b += nwarp) {
    uint64_t r0, r1;
    if (!block_rays(blk_off, b, base, nray, &r0, &r1)) { bad = true; continue; }
    // the block's coordinates in blocks (the host checks nbx < 4096 and
    // nby, nbz < 1024)
    const uint32_t nyz = (uint32_t)g.nby * (uint32_t)g.nbz;
    const uint32_t bx = b / nyz, by = (b - bx * nyz) / (uint32_t)g.nbz, bz = b - bx * nyz - by * (uint32_t)g.nbz;
    __syncwarp();
    if (lane == 0) {
      ws[0] = b;
      ws[1] = (uint32_t)(r1 - r0);
      ws[2] = bx | (by << 12) | (bz << 22);
      ws[3] = (uint32_t)r0;
      ws[4] = (uint32_t)(r0 >> 32);
    }
    __syncwarp();
    uint32_t bsteps = 0;
    for (uint32_t j = lane; j < ws[1]; j += 32) {
      const uint64_t r = (((uint64_t)ws[4] << 32) | ws[3]) + j;
      const uint32_t bpos = ws[2];
      const uint32_t w = __ldg(rays + r);
      const uint32_t e = w >> 5;
      const int l = (int)(w & 31u);
      const int gx = g.ix0 + kBlkX * (int)(bpos & 4095u) + (l >> 4);
      const int gy = g.iy0 + kBlkY * (int)((bpos >> 12) & 1023u) + ((l >> 2) & 3);
      const int gz = g.iz0 + kBlkZ * (int)(bpos >> 22) + (l & 3);
      const float xe = cell_centre(g.xmin, gx, g.dx);
      const float ye = cell_centre(g.ymin, gy, g.dy);
      const float ze = cell_centre(g.zmin, gz, g.dz);
      const float4 ep = __ldg(emit_pos + e);
      float xs = ep.x, ys = ep.y, zs = ep.z;
      if (!kInside) ray_start(g, ep.x, ep.y, ep.z, xe, ye, ze, &xs, &ys, &zs);
      int steps = 0;
      const Tau3 t = (kPrec == ARGOT_B200_PRECISION_REFERENCE)
                         ? march_reference(g, cells, xs, ys, zs, xe, ye, ze, &steps, &bad)
                         : march_kahan<kMarchThreads, ARGOT_MARCH_CENTRE_END>(g, cells, xs, ys, zs, xe, ye, ze,
                                                                              &steps, &bad, kslot + threadIdx.x);
      const uint64_t ro = (((uint64_t)ws[4] << 32) | ws[3]) + j;
      tau[ro] = t.hi;
      tau[nray + ro] = t.hei;
      tau[2 * nray + ro] = t.heii;
      bsteps += (uint32_t)steps;
    }
    if (crossings) {
      for (int o = 16; o; o >>= 1) bsteps += __shfl_xor_sync(0xffffffffu, bsteps, o);
      if (lane == 0 && bsteps) atomicAdd(crossings, (unsigned long long)bsteps);
    }
    b = ws[0];
  }
  if (bad) atomicExch(err, 1);
}

// -------------------------------------------------------- explicit segments
template <int kPrec>
__global__ void k_march_segments(GridDev g, const float4 *__restrict__ cells, uint64_t nseg,
                                 const float *__restrict__ pos6, float *__restrict__ tau3,
                                 int *__restrict__ err) {
  bool bad = false;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nseg;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float *p = pos6 + 6 * i;
    int steps;
    const Tau3 t = (kPrec == ARGOT_B200_PRECISION_REFERENCE)
                       ? march_reference(g, cells, p[0], p[1], p[2], p[3], p[4], p[5], &steps, &bad)
                       : march_kahan(g, cells, p[0], p[1], p[2], p[3], p[4], p[5], &steps, &bad);
    tau3[3 * i + 0] = t.hi;
    tau3[3 * i + 1] = t.hei;
    tau3[3 * i + 2] = t.heii;
  }
  if (bad) atomicExch(err, 1);
}

// ---------------------------------------------------------------- stitching
// Segments sorted by ray index: one thread per ray boundary run.  Each run
// of equal ray_indx is summed with Kahan compensation and written to its
// ray; rays without segments are zeroed first.
__global__ void k_zero3(uint64_t n, float *__restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < 3 * n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = 0.f;
}

__global__ void k_stitch(uint64_t nseg, const uint64_t *__restrict__ ray_indx,
                         const float *__restrict__ seg_tau3, uint64_t nray, float *__restrict__ ray_tau3,
                         int *__restrict__ err) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nseg;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = ray_indx[i];
    if (i > 0 && ray_indx[i - 1] == r) continue;  // not the head of a run
    if (r >= nray) {  // a segment of a ray the caller's array does not have: skipped, reported
      atomicExch(err, 1);
      continue;
    }
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, c0 = 0.f, c1 = 0.f, c2 = 0.f;
    for (uint64_t j = i; j < nseg && ray_indx[j] == r; j++) {
      kahan_add(s0, c0, seg_tau3[3 * j + 0]);
      kahan_add(s1, c1, seg_tau3[3 * j + 1]);
      kahan_add(s2, c2, seg_tau3[3 * j + 2]);
    }
    ray_tau3[3 * r + 0] = s0;
    ray_tau3[3 * r + 1] = s1;
    ray_tau3[3 * r + 2] = s2;
  }
}

// adds base to the n offsets (the scan's shift), on the device
__global__ void k_add_base(uint64_t n, uint64_t base, uint64_t *__restrict__ off) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    off[i] += base;
}

// per-device scratch: an error flag and a counter
struct DevScratch {
  int *err = nullptr;
};
static DevScratch g_scratch[64];

int *err_flag(int dev) {
  if (dev < 0 || dev >= 64) return nullptr;
  if (!g_scratch[dev].err) {
    if (cudaMalloc(&g_scratch[dev].err, sizeof(int)) != cudaSuccess) return nullptr;
    cudaMemset(g_scratch[dev].err, 0, sizeof(int));
  }
  return g_scratch[dev].err;
}

// Reads and clears the device error flag (synchronises the stream).
int check_err_flag(int *flag, cudaStream_t st) {
  int h = 0;
  ARGOT_CUDA_TRY(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  ARGOT_CUDA_TRY(cudaStreamSynchronize(st));
  if (h) {
    cudaMemsetAsync(flag, 0, sizeof(int), st);
    set_status(ARGOT_B200_EDEVICE);
    return ARGOT_B200_EDEVICE;
  }
  return 0;
}

}  // namespace argot

using namespace argot;

extern "C" {

int argot_b200_pack_fields(const argot_b200_grid *gp, const float *dens, const float *fHI,
                           const float *fHeI, const float *fHeII, void *packed_dev, void *stream) {
  if (!grid_valid(gp) || !dens || !fHI || !fHeI || !fHeII || !packed_dev) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  const uint64_t n = (uint64_t)gp->nx * gp->ny * gp->nz;
  float4 *cells = (float4 *)packed_dev;
  k_pack_fields<<<grid_blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, dens, fHI, fHeI, fHeII,
                                                                          cells, cells + n);
  ARGOT_CUDA_TRY(cudaGetLastError());
  set_status(0);
  return 0;
}

int argot_b200_num_blocks(const argot_b200_grid *gp, uint64_t *nblocks) {
  if (!grid_valid(gp) || !nblocks) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  GridDev g = make_grid(*gp);
  *nblocks = (uint64_t)g.nbx * g.nby * g.nbz;
  set_status(0);
  return 0;
}

int argot_b200_count_rays(const argot_b200_grid *gp, const argot_b200_dev_tree *t, uint64_t b0,
                          uint64_t b1, uint64_t *blk_count, uint32_t *cell_count, void *stream) {
  uint64_t nb = 0;
  if (!grid_valid(gp) || !t || !blk_count || argot_b200_num_blocks(gp, &nb) || b0 > b1 || b1 > nb) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  if (b0 == b1) { set_status(0); return 0; }
  GridDev g = make_grid(*gp);
  const int threads = 256;
  const int blocks = grid_blocks_for((b1 - b0) * 32, threads);
  k_walk<false><<<blocks, threads, 0, (cudaStream_t)stream>>>(g, t->nodes, t->n_nodes, t->src_list,
                                                              t->theta_sq, b0, b1, blk_count, cell_count,
                                                              nullptr, 0, nullptr, nullptr);
  ARGOT_CUDA_TRY(cudaGetLastError());
  set_status(0);
  return 0;
}

int argot_b200_scan_blocks(const uint64_t *blk_count, uint64_t nb, uint64_t base, uint64_t *blk_off,
                           uint64_t *total, void *stream) {
  if (!blk_count || !blk_off) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  cudaStream_t st = (cudaStream_t)stream;
  // blk_off[0] = base; blk_off[i+1] = base + sum(count[0..i])
  ARGOT_CUDA_TRY(cudaMemcpyAsync(blk_off, &base, sizeof(uint64_t), cudaMemcpyHostToDevice, st));
  if (nb) {
    size_t tmp_bytes = 0;
    ARGOT_CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, blk_count, blk_off + 1, (int64_t)nb, st));
    void *tmp = nullptr;
    ARGOT_CUDA_TRY(cudaMallocAsync(&tmp, tmp_bytes, st));
    cudaError_t e = cub::DeviceScan::InclusiveSum(tmp, tmp_bytes, blk_count, blk_off + 1, (int64_t)nb, st);
    cudaFreeAsync(tmp, st);
    ARGOT_CUDA_TRY(e);
    if (base) k_add_base<<<grid_blocks_for(nb, 256), 256, 0, st>>>(nb, base, blk_off + 1);
    ARGOT_CUDA_TRY(cudaGetLastError());
  }
  if (total) {
    ARGOT_CUDA_TRY(cudaMemcpyAsync(total, blk_off + nb, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    ARGOT_CUDA_TRY(cudaStreamSynchronize(st));
  }
  set_status(0);
  return 0;
}

int argot_b200_emit_rays(const argot_b200_grid *gp, const argot_b200_dev_tree *t, uint64_t b0,
                         uint64_t b1, const uint64_t *blk_off, uint64_t base, uint32_t *rays,
                         void *stream) {
  uint64_t nb = 0;
  if (!grid_valid(gp) || !t || !blk_off || !rays || argot_b200_num_blocks(gp, &nb) || b0 > b1 || b1 > nb) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  if (b0 == b1) { set_status(0); return 0; }
  int dev = 0;
  ARGOT_CUDA_TRY(cudaGetDevice(&dev));
  int *err = err_flag(dev);
  if (!err) { set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  GridDev g = make_grid(*gp);
  const int threads = 256;
  const int blocks = grid_blocks_for((b1 - b0) * 32, threads);
  k_walk<true><<<blocks, threads, 0, (cudaStream_t)stream>>>(g, t->nodes, t->n_nodes, t->src_list,
                                                             t->theta_sq, b0, b1, nullptr, nullptr, blk_off,
                                                             base, rays, err);
  ARGOT_CUDA_TRY(cudaGetLastError());
  set_status(0);
  return 0;
}

int argot_b200_march_rays(const argot_b200_grid *gp, const void *packed, const argot_b200_dev_tree *t,
                          uint64_t b0, uint64_t b1, const uint64_t *blk_off, uint64_t base,
                          const uint32_t *rays, uint64_t nray, float *tau, int prec,
                          unsigned long long *crossings, void *stream) {
  uint64_t nb = 0;
  if (!grid_valid(gp) || !packed || !t || !blk_off || (nray && (!rays || !tau)) ||
      argot_b200_num_blocks(gp, &nb) || b0 > b1 || b1 > nb ||
      (prec != ARGOT_B200_PRECISION_REFERENCE && prec != ARGOT_B200_PRECISION_KAHAN)) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  if (b0 == b1) { set_status(0); return 0; }
  GridDev g = make_grid(*gp);
  if (g.nbx >= 4096 || g.nby >= 1024 || g.nbz >= 1024) {  // the kernel packs block coordinates in 32 bits
    set_status(ARGOT_B200_ENOTSUP);
    return ARGOT_B200_ENOTSUP;
  }
  int dev = 0;
  ARGOT_CUDA_TRY(cudaGetDevice(&dev));
  int *err = err_flag(dev);
  if (!err) { set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  cudaStream_t st = (cudaStream_t)stream;
  const int threads = kMarchThreads;
  const int blocks = grid_blocks_for((b1 - b0) * 32, threads);
  const bool inside = t->emit_lo[0] >= gp->xmin && t->emit_lo[1] >= gp->ymin && t->emit_lo[2] >= gp->zmin &&
                      t->emit_hi[0] <= gp->xmax && t->emit_hi[1] <= gp->ymax && t->emit_hi[2] <= gp->zmax;
  const float4 *cells = (const float4 *)packed;
#define ARGOT_MARCH_LAUNCH(P, I)                                                                       \
  k_march_rays<P, I><<<blocks, threads, 0, st>>>(g, cells, t->emit_pos, (uint32_t)b0, (uint32_t)b1, blk_off, \
                                                 base, rays, nray, tau, crossings, err)
  if (prec == ARGOT_B200_PRECISION_REFERENCE) {
    if (inside) ARGOT_MARCH_LAUNCH(ARGOT_B200_PRECISION_REFERENCE, true);
    else ARGOT_MARCH_LAUNCH(ARGOT_B200_PRECISION_REFERENCE, false);
  } else {
    if (inside) ARGOT_MARCH_LAUNCH(ARGOT_B200_PRECISION_KAHAN, true);
    else ARGOT_MARCH_LAUNCH(ARGOT_B200_PRECISION_KAHAN, false);
  }
#undef ARGOT_MARCH_LAUNCH
  ARGOT_CUDA_TRY(cudaGetLastError());
  set_status(0);
  return 0;
}

int argot_b200_march_segments(const argot_b200_grid *gp, const void *packed, uint64_t nseg,
                              const float *pos6, float *tau3, int prec, void *stream) {
  if (!grid_valid(gp) || !packed || (nseg && (!pos6 || !tau3)) ||
      (prec != ARGOT_B200_PRECISION_REFERENCE && prec != ARGOT_B200_PRECISION_KAHAN)) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  if (!nseg) { set_status(0); return 0; }
  int dev = 0;
  ARGOT_CUDA_TRY(cudaGetDevice(&dev));
  int *err = err_flag(dev);
  if (!err) { set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  GridDev g = make_grid(*gp);
  cudaStream_t st = (cudaStream_t)stream;
  const int threads = 128;
  const int blocks = grid_blocks_for(nseg, threads);
  if (prec == ARGOT_B200_PRECISION_REFERENCE)
    k_march_segments<ARGOT_B200_PRECISION_REFERENCE><<<blocks, threads, 0, st>>>(g, (const float4 *)packed,
                                                                                 nseg, pos6, tau3, err);
  else
    k_march_segments<ARGOT_B200_PRECISION_KAHAN><<<blocks, threads, 0, st>>>(g, (const float4 *)packed,
                                                                             nseg, pos6, tau3, err);
  ARGOT_CUDA_TRY(cudaGetLastError());
  int rc = check_err_flag(err, st);
  set_status(rc);
  return rc;
}

int argot_b200_stitch(uint64_t nseg, const uint64_t *ray_indx, const float *seg_tau3, uint64_t nray,
                      float *ray_tau3, void *stream) {
  if ((nseg && (!ray_indx || !seg_tau3)) || (nray && !ray_tau3)) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  int dev = 0;
  ARGOT_CUDA_TRY(cudaGetDevice(&dev));
  int *err = err_flag(dev);
  if (!err) { set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  cudaStream_t st = (cudaStream_t)stream;
  if (nray) k_zero3<<<grid_blocks_for(3 * nray, 256), 256, 0, st>>>(nray, ray_tau3);
  if (nseg) k_stitch<<<grid_blocks_for(nseg, 256), 256, 0, st>>>(nseg, ray_indx, seg_tau3, nray, ray_tau3, err);
  ARGOT_CUDA_TRY(cudaGetLastError());
  set_status(0);
  return 0;
}

// Reads and clears the march error flag of the current device; returns
// ARGOT_B200_EDEVICE if any march since the last check hit its step cap.
int argot_b200_check_device_error(void *stream) {
  int dev = 0;
  ARGOT_CUDA_TRY(cudaGetDevice(&dev));
  int *err = err_flag(dev);
  if (!err) { set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  int rc = check_err_flag(err, (cudaStream_t)stream);
  set_status(rc);
  return rc;
}

}  // extern "C"
