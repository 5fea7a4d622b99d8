// scan_static.cu -- the ray-offset scan of argot_b200_scan_blocks in a form
// that allocates no memory, for callers that cannot allocate device memory
// while they run the path: hosts that hand all device memory to their own
// pool allocator up front, or a drop-in used from code that forbids
// cudaMalloc after start-up.
//
// The scan's scratch (one partial sum per tile of 2048 counts) lives in a
// file-scope device array of fixed size instead of a temporary allocation.
// Limits and behaviour:
//   * at most kMaxTiles tiles, i.e. nb <= kMaxTiles * kTile = 16 777 216
//     blocks of 32 cells (meshes up to ~812^3 cells); larger requests are
//     rejected with ARGOT_B200_EINVAL before anything is launched;
//   * the array belongs to the device (each GPU that loads the library holds
//     its 64 KiB until the process exits) and every call on that device
//     shares it: calls that overlap on the GPU (different streams, or
//     different host threads) race on it and must be serialised by the
//     caller;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture;
//   * the total on the host (total != NULL) needs a copy and a stream
//     synchronisation; with total == NULL the call only enqueues work and
//     the caller reads blk_offsets[nb] on the device.  A host total is
//     refused (ARGOT_B200_EINVAL, nothing launched) while `stream` is
//     capturing, where a synchronisation is not allowed.
#include <mutex>

#include "common.cuh"

namespace argot {

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 8;
constexpr int kTile = kThreads * kPerThread;  // counts per tile
constexpr int kMaxTiles = 8192;               // 64 KiB of scratch

// One partial sum per tile; entry t is written by k_tile_sums before
// anything reads it, so no call depends on what a previous call left.
static __device__ __align__(256) unsigned long long g_scan_scratch[kMaxTiles];

__device__ unsigned long long block_exclusive_scan(unsigned long long v, unsigned long long *total) {
  __shared__ unsigned long long warp_tot[kThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned long long x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    unsigned long long t = lane < kThreads / 32 ? warp_tot[lane] : 0ull;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < kThreads / 32) warp_tot[lane] = t;
  }
  __syncthreads();
  const unsigned long long before = (w ? warp_tot[w - 1] : 0ull) + x - v;
  if (total) *total = warp_tot[kThreads / 32 - 1];
  __syncthreads();
  return before;
}

__global__ void __launch_bounds__(kThreads) k_tile_sums(const unsigned long long *__restrict__ cnt, uint64_t nb,
                                                        unsigned long long *__restrict__ part) {
  const uint64_t t0 = (uint64_t)blockIdx.x * kTile;
  unsigned long long s = 0;
  for (int k = 0; k < kPerThread; k++) {
    const uint64_t i = t0 + (uint64_t)k * kThreads + threadIdx.x;
    if (i < nb) s += cnt[i];
  }
  unsigned long long tot;
  block_exclusive_scan(s, &tot);
  if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

// exclusive scan of the tile sums, in place, by one CTA
__global__ void __launch_bounds__(kThreads) k_scan_tiles(unsigned long long *__restrict__ part, int ntiles) {
  unsigned long long carry = 0;
  for (int b = 0; b < ntiles; b += kThreads) {
    const int i = b + threadIdx.x;
    const unsigned long long v = i < ntiles ? part[i] : 0ull;
    unsigned long long tot;
    const unsigned long long ex = block_exclusive_scan(v, &tot);
    if (i < ntiles) part[i] = carry + ex;
    carry += tot;
  }
}

// out[0] = base; out[i+1] = base + cnt[0] + ... + cnt[i]
__global__ void __launch_bounds__(kThreads) k_tile_scan(const unsigned long long *__restrict__ cnt, uint64_t nb,
                                                        const unsigned long long *__restrict__ part,
                                                        unsigned long long base, unsigned long long *__restrict__ out) {
  const uint64_t t0 = (uint64_t)blockIdx.x * kTile;
  // each thread owns kPerThread consecutive counts
  unsigned long long v[kPerThread];
  unsigned long long s = 0;
  for (int k = 0; k < kPerThread; k++) {
    const uint64_t i = t0 + (uint64_t)threadIdx.x * kPerThread + k;
    v[k] = i < nb ? cnt[i] : 0ull;
    s += v[k];
  }
  unsigned long long run = base + part[blockIdx.x] + block_exclusive_scan(s, nullptr);
  for (int k = 0; k < kPerThread; k++) {
    const uint64_t i = t0 + (uint64_t)threadIdx.x * kPerThread + k;
    run += v[k];
    if (i < nb) out[i + 1] = run;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[0] = base;
}

// device address of g_scan_scratch, looked up once per device
std::mutex g_mu;
void *g_addr[64] = {nullptr};

int scratch_address(int dev, void **ptr) {
  if (dev < 0 || dev >= 64) return ARGOT_B200_EINVAL;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scan_scratch);
    if (e != cudaSuccess) return status_from_cuda(e);
    g_addr[dev] = p;
  }
  *ptr = g_addr[dev];
  return 0;
}

}  // namespace
}  // namespace argot

using namespace argot;

extern "C" int argot_b200_scan_blocks_static(const uint64_t *blk_count, uint64_t nb, uint64_t base,
                                             uint64_t *blk_off, uint64_t *total, void *stream) {
  if (!blk_count || !blk_off) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  const uint64_t ntiles = (nb + kTile - 1) / kTile;
  if (ntiles > (uint64_t)kMaxTiles) {
    // beyond the fixed scratch: nothing is launched
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (total) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    ARGOT_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) {  // a synchronisation cannot be captured
      set_status(ARGOT_B200_EINVAL);
      return ARGOT_B200_EINVAL;
    }
  }
  int dev = 0;
  ARGOT_CUDA_TRY(cudaGetDevice(&dev));
  void *scratch = nullptr;
  int rc = scratch_address(dev, &scratch);
  if (rc) { set_status(rc); return rc; }
  unsigned long long *part = (unsigned long long *)scratch;
  const unsigned long long *cnt = (const unsigned long long *)blk_count;
  unsigned long long *out = (unsigned long long *)blk_off;
  if (ntiles) {
    k_tile_sums<<<(unsigned)ntiles, kThreads, 0, st>>>(cnt, nb, part);
    k_scan_tiles<<<1, kThreads, 0, st>>>(part, (int)ntiles);
    k_tile_scan<<<(unsigned)ntiles, kThreads, 0, st>>>(cnt, nb, part, (unsigned long long)base, out);
  } else {
    k_tile_scan<<<1, kThreads, 0, st>>>(cnt, 0, part, (unsigned long long)base, out);
  }
  ARGOT_CUDA_TRY(cudaGetLastError());
  if (total) {
    ARGOT_CUDA_TRY(cudaMemcpyAsync(total, blk_off + nb, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    ARGOT_CUDA_TRY(cudaStreamSynchronize(st));
  }
  set_status(0);
  return 0;
}
