// run.cu -- the device fast path of one ray group in one call: ray
// generation, march and rates, with the march of one part of the group's
// target blocks overlapping the rates of the previous part on a second
// stream.  The calls are the library's own (argot_b200_emit_rays,
// argot_b200_march_rays, argot_b200_photoion_rays), so the result equals
// the sequential calls bit for bit; a caller capturing its stream into a
// CUDA graph captures the two internal streams too (they fork from and
// join into the caller's stream through events).
#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace argot {
namespace {

struct RunStreams {
  cudaStream_t march = nullptr, rates = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  std::vector<cudaEvent_t> part;
  bool init = false;
};

std::mutex g_run_mu;
RunStreams g_run[64];

int ensure_run_streams(RunStreams &r, size_t parts) {
  if (!r.init) {
    ARGOT_CUDA_TRY(cudaStreamCreateWithFlags(&r.march, cudaStreamNonBlocking));
    ARGOT_CUDA_TRY(cudaStreamCreateWithFlags(&r.rates, cudaStreamNonBlocking));
    ARGOT_CUDA_TRY(cudaEventCreateWithFlags(&r.fork, cudaEventDisableTiming));
    ARGOT_CUDA_TRY(cudaEventCreateWithFlags(&r.join, cudaEventDisableTiming));
    r.init = true;
  }
  while (r.part.size() < parts) {
    cudaEvent_t e;
    ARGOT_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    r.part.push_back(e);
  }
  return 0;
}

}  // namespace
}  // namespace argot

using namespace argot;

extern "C" {

int argot_b200_run_group(const argot_b200_grid *g, const void *packed_dev, const argot_b200_dev_tree *t,
                         uint64_t b0, uint64_t b1, const uint64_t *blk_off_dev, const uint64_t *blk_off_host,
                         uint64_t base, uint32_t *rays_dev, float *tau_dev, int emit, int precision, int mode,
                         int parts, float *rates6_dev, unsigned long long *crossings_dev, void *stream) {
  uint64_t nb = 0;
  if (!grid_valid(g) || !packed_dev || !t || !blk_off_dev || !blk_off_host || !rays_dev || !tau_dev ||
      !rates6_dev || parts < 1 || parts > 4096 || (emit != 0 && emit != 1) || argot_b200_num_blocks(g, &nb) ||
      b0 > b1 || b1 > nb || blk_off_host[b0] < base || blk_off_host[b1] < blk_off_host[b0]) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  if (b0 == b1) { set_status(0); return 0; }
  // part boundaries: block ranges of about nray / parts rays each
  std::vector<uint64_t> cut{b0};
  for (int p = 1; p < parts; p++) {
    const uint64_t want = blk_off_host[b0] + (uint64_t)((double)(blk_off_host[b1] - blk_off_host[b0]) * p / parts);
    const uint64_t *it = std::lower_bound(blk_off_host + cut.back(), blk_off_host + b1, want);
    const uint64_t b = (uint64_t)(it - blk_off_host);
    if (b > cut.back() && b < b1) cut.push_back(b);
  }
  cut.push_back(b1);
  const size_t np = cut.size() - 1;
  int dev = 0;
  ARGOT_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  std::lock_guard<std::mutex> lock(g_run_mu);
  RunStreams &r = g_run[dev];
  int rc = ensure_run_streams(r, np);
  if (rc) return rc;
  cudaStream_t caller = (cudaStream_t)stream;
  ARGOT_CUDA_TRY(cudaEventRecord(r.fork, caller));
  ARGOT_CUDA_TRY(cudaStreamWaitEvent(r.march, r.fork, 0));
  ARGOT_CUDA_TRY(cudaStreamWaitEvent(r.rates, r.fork, 0));
  if (emit && (rc = argot_b200_emit_rays(g, t, b0, b1, blk_off_dev, base, rays_dev, r.march))) return rc;
  // the march of every part on one stream, the rates of part p on the other
  // once part p's columns are complete; part p's rays and columns start at
  // its first ray, its three column planes hold its own rays only
  for (size_t p = 0; p < np; p++) {
    const uint64_t lo = blk_off_host[cut[p]] - base, n = blk_off_host[cut[p + 1]] - blk_off_host[cut[p]];
    if ((rc = argot_b200_march_rays(g, packed_dev, t, cut[p], cut[p + 1], blk_off_dev, base + lo, rays_dev + lo, n,
                                    tau_dev + 3 * lo, precision, crossings_dev, r.march)))
      return rc;
    ARGOT_CUDA_TRY(cudaEventRecord(r.part[p], r.march));
  }
  for (size_t p = 0; p < np; p++) {
    const uint64_t lo = blk_off_host[cut[p]] - base, n = blk_off_host[cut[p + 1]] - blk_off_host[cut[p]];
    ARGOT_CUDA_TRY(cudaStreamWaitEvent(r.rates, r.part[p], 0));
    if ((rc = argot_b200_photoion_rays(g, packed_dev, t, cut[p], cut[p + 1], blk_off_dev, base + lo, rays_dev + lo,
                                       n, tau_dev + 3 * lo, mode, rates6_dev, r.rates)))
      return rc;
  }
  // the last rates follow the last march, so joining the rate stream
  // orders the caller after everything
  ARGOT_CUDA_TRY(cudaEventRecord(r.join, r.rates));
  ARGOT_CUDA_TRY(cudaStreamWaitEvent(caller, r.join, 0));
  set_status(0);
  return 0;
}

}  // extern "C"
