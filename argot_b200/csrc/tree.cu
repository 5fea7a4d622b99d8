// tree.cu -- the oct-tree over the sources built on the device, with the
// construction rules of the host builder in host.cu (itself the
// reference's construct_tree, setup_light_ray_tree.c:100-239, 465-571),
// bit for bit: the same nodes in the same depth-first preorder, the same
// FP64 sums in the same order, the same emitter table.
//
//  1. k_src_keys: per source its 63-bit Morton key (21 bits per axis of
//     (pos - box_min) / L * 2^21, a leading 1 bit for the root) and its
//     luminosity (the sum of its 256 bins in order).
//  2. A stable radix sort of (key, source index): sources with equal keys
//     keep their input order, as the host's stable sort.
//  3. k_node_counts: the node at depth d = 1..21 (key level 63 - 3 d) that
//     starts at sorted position i exists when i starts a new key prefix at
//     that depth and the parent splits: the root always does, a deeper
//     parent when it holds two or more sources.  Depth-first preorder is the
//     order of (first source, depth), so an exclusive scan of the counts per
//     position gives every node its preorder index; a node's subtree ends
//     where its source range ends.
//  4. k_node_fill: per node its source range, side, depth, skip link.
//  5. k_node_sums, one launch per depth from the leaves up: a leaf sums
//     its sources' spectra, luminosities and luminosity-weighted positions
//     in sorted order; an internal node sums its children's in octant
//     order; centres as the host divides them.  The root's spectrum and
//     centre are the host's flat sums over the sources in input order (the
//     centre weighted by the first bin).
//  6. The emitter table (nodes, then sources in input order): positions,
//     FP64 spectra, totals and the normalised FP32 spectra in bin-pair
//     order, and the emitters' bounding box.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "common.cuh"

namespace argot {

namespace {

constexpr int kMaxDepth = 21;

__global__ void k_src_keys(int n, const float *__restrict__ pos, float xmin, float ymin, float zmin, float base,
                           const double *__restrict__ spec, unsigned long long *__restrict__ keys,
                           int *__restrict__ idx, double *__restrict__ lum) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double scale = 2097152.0;  // 2^21
  const float p0 = pos[3 * i], p1 = pos[3 * i + 1], p2 = pos[3 * i + 2];
  // (uint64_t)(int)((p - min) / L * 2^21): float subtraction and division,
  // double product, truncation to int
  const unsigned long long ip0 = (unsigned long long)(long long)__double2int_rz(
      __dmul_rn((double)__fdiv_rn(__fsub_rn(p0, xmin), base), scale));
  const unsigned long long ip1 = (unsigned long long)(long long)__double2int_rz(
      __dmul_rn((double)__fdiv_rn(__fsub_rn(p1, ymin), base), scale));
  const unsigned long long ip2 = (unsigned long long)(long long)__double2int_rz(
      __dmul_rn((double)__fdiv_rn(__fsub_rn(p2, zmin), base), scale));
  unsigned long long k = 1ull << 63;
  for (int bit = 0; bit < 21; bit++) {
    const unsigned long long tri = (((ip0 >> bit) & 1ull) << 2) | (((ip1 >> bit) & 1ull) << 1) | ((ip2 >> bit) & 1ull);
    k |= tri << (3 * bit);
  }
  keys[i] = k;
  idx[i] = i;
  double L = 0.0;
  for (int b = 0; b < kNu; b++) L = __dadd_rn(L, spec[(size_t)i * kNu + b]);
  lum[i] = L;
}

// does the node at depth d start at sorted position i?
__device__ __forceinline__ bool node_starts(const unsigned long long *__restrict__ key, int n, int i, int d) {
  const int level = 63 - 3 * d;
  const unsigned long long me = key[i] >> level;
  if (i > 0 && (key[i - 1] >> level) == me) return false;
  if (d == 1) return true;  // the root always splits
  const unsigned long long par = key[i] >> (level + 3);
  return (i > 0 && (key[i - 1] >> (level + 3)) == par) || (i + 1 < n && (key[i + 1] >> (level + 3)) == par);
}

// nodes starting at each sorted position (the root counts at position 0)
__global__ void k_node_counts(int n, const unsigned long long *__restrict__ key, int *__restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > n) return;
  if (i == n) { cnt[n] = 0; return; }
  int c = i == 0 ? 1 : 0;
  for (int d = 1; d <= kMaxDepth; d++) c += node_starts(key, n, i, d);
  cnt[i] = c;
}

// end of the prefix group at depth d that starts at i (binary search in the
// sorted keys)
__device__ __forceinline__ int group_end(const unsigned long long *__restrict__ key, int n, int i, int d) {
  const int level = 63 - 3 * d;
  const unsigned long long me = key[i] >> level;
  int lo = i + 1, hi = n;  // first position in [lo, hi] whose prefix differs
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if ((key[mid] >> level) == me) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__global__ void k_node_fill(int n, const unsigned long long *__restrict__ key, const int *__restrict__ first,
                            const float *__restrict__ side, DevNode *__restrict__ nodes, int *__restrict__ depth) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int p = first[i];
  if (i == 0) {
    DevNode r{};
    r.len = side[0];
    r.n = n;
    r.src_first = 0;
    r.has_child = 1;
    r.skip = first[n];
    nodes[p] = r;
    depth[p] = 0;
    p++;
  }
  for (int d = 1; d <= kMaxDepth; d++) {
    if (!node_starts(key, n, i, d)) continue;
    const int e = group_end(key, n, i, d);
    DevNode nd{};
    nd.len = side[d];
    nd.n = e - i;
    nd.src_first = i;
    nd.has_child = (e - i > 1 && d < kMaxDepth) ? 1 : 0;
    nd.skip = first[e];
    nodes[p] = nd;
    depth[p] = d;
    p++;
  }
}

// Node sums of one depth: one warp per node (lists[l0 .. l1) of node
// indices), lanes over the bins for the spectrum; lane 0 forms the
// luminosity, the weighted position and the centre.
__global__ void k_node_sums(const int *__restrict__ list, int m, DevNode *__restrict__ nodes,
                            const int *__restrict__ idx, const float *__restrict__ pos,
                            const double *__restrict__ spec, const double *__restrict__ lum,
                            double *__restrict__ nspec, double *__restrict__ nlum, double *__restrict__ ncm) {
  const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (wid >= m) return;
  const int p = list[wid];
  const DevNode nd = nodes[p];
  if (!nd.has_child) {
    for (int b = lane; b < kNu; b += 32) {
      double s = 0.0;
      for (int j = nd.src_first; j < nd.src_first + nd.n; j++) s = __dadd_rn(s, spec[(size_t)idx[j] * kNu + b]);
      nspec[(size_t)p * kNu + b] = s;
    }
    if (lane == 0) {
      double mm = 0.0, c0 = 0.0, c1 = 0.0, c2 = 0.0;
      for (int j = nd.src_first; j < nd.src_first + nd.n; j++) {
        const int is = idx[j];
        const double mj = lum[is];
        mm = __dadd_rn(mm, mj);
        c0 = __dadd_rn(c0, __dmul_rn(mj, (double)pos[3 * is + 0]));
        c1 = __dadd_rn(c1, __dmul_rn(mj, (double)pos[3 * is + 1]));
        c2 = __dadd_rn(c2, __dmul_rn(mj, (double)pos[3 * is + 2]));
      }
      const double minv = __ddiv_rn(1.0, mm);
      nodes[p].cx = __double2float_rn(__dmul_rn(c0, minv));
      nodes[p].cy = __double2float_rn(__dmul_rn(c1, minv));
      nodes[p].cz = __double2float_rn(__dmul_rn(c2, minv));
      nlum[p] = mm;
      ncm[3 * (size_t)p + 0] = c0;
      ncm[3 * (size_t)p + 1] = c1;
      ncm[3 * (size_t)p + 2] = c2;
    }
    return;
  }
  // children: p + 1, then each child's skip link, while inside the subtree
  const int end = nd.skip;
  for (int b = lane; b < kNu; b += 32) {
    double s = 0.0;
    for (int c = p + 1; c < end; c = nodes[c].skip) s = __dadd_rn(s, nspec[(size_t)c * kNu + b]);
    nspec[(size_t)p * kNu + b] = s;
  }
  if (lane == 0) {
    double L = 0.0, c0 = 0.0, c1 = 0.0, c2 = 0.0;
    for (int c = p + 1; c < end; c = nodes[c].skip) {
      L = __dadd_rn(L, nlum[c]);
      c0 = __dadd_rn(c0, ncm[3 * (size_t)c + 0]);
      c1 = __dadd_rn(c1, ncm[3 * (size_t)c + 1]);
      c2 = __dadd_rn(c2, ncm[3 * (size_t)c + 2]);
    }
    nlum[p] = L;
    ncm[3 * (size_t)p + 0] = c0;
    ncm[3 * (size_t)p + 1] = c1;
    ncm[3 * (size_t)p + 2] = c2;
    nodes[p].cx = __double2float_rn(__ddiv_rn(c0, L));
    nodes[p].cy = __double2float_rn(__ddiv_rn(c1, L));
    nodes[p].cz = __double2float_rn(__ddiv_rn(c2, L));
  }
}

// The root: spectrum and first-bin-weighted centre summed over the sources
// in input order (one block; the centre by thread 0, bins by all threads).
__global__ void k_root_sums(int n, const float *__restrict__ pos, const double *__restrict__ spec,
                            DevNode *__restrict__ nodes, double *__restrict__ nspec) {
  for (int b = threadIdx.x; b < kNu; b += blockDim.x) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s = __dadd_rn(s, spec[(size_t)i * kNu + b]);
    nspec[b] = s;
  }
  if (threadIdx.x == 0) {
    double xc = 0.0, yc = 0.0, zc = 0.0, l0 = 0.0;
    for (int i = 0; i < n; i++) {
      const double w = spec[(size_t)i * kNu];
      xc = __dadd_rn(xc, __dmul_rn((double)pos[3 * i + 0], w));
      yc = __dadd_rn(yc, __dmul_rn((double)pos[3 * i + 1], w));
      zc = __dadd_rn(zc, __dmul_rn((double)pos[3 * i + 2], w));
      l0 = __dadd_rn(l0, w);
    }
    nodes[0].cx = __double2float_rn(__ddiv_rn(xc, l0));
    nodes[0].cy = __double2float_rn(__ddiv_rn(yc, l0));
    nodes[0].cz = __double2float_rn(__ddiv_rn(zc, l0));
  }
}

// The emitter table: emitter e < nn is node e, else source e - nn (input
// order).  total = sum of the bins in order; specn in bin-pair order.
__global__ void k_emitters(int nn, int n, const DevNode *__restrict__ nodes, const float *__restrict__ pos,
                           const double *__restrict__ spec, float4 *__restrict__ epos,
                           double *__restrict__ espec, float *__restrict__ especn, double *__restrict__ etot) {
  const int e = blockIdx.x;
  if (e >= nn + n) return;
  const double *s = e < nn ? espec + (size_t)e * kNu : spec + (size_t)(e - nn) * kNu;
  if (e >= nn) {
    for (int b = threadIdx.x; b < kNu; b += blockDim.x) espec[(size_t)e * kNu + b] = s[b];
  }
  __shared__ double tot;
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int b = 0; b < kNu; b++) t = __dadd_rn(t, s[b]);
    tot = t;
    etot[e] = t;
    epos[e] = e < nn ? make_float4(nodes[e].cx, nodes[e].cy, nodes[e].cz, 0.f)
                     : make_float4(pos[3 * (e - nn)], pos[3 * (e - nn) + 1], pos[3 * (e - nn) + 2], 0.f);
  }
  __syncthreads();
  const double inv = tot > 0.0 ? __ddiv_rn(1.0, tot) : 0.0;
  for (int b = threadIdx.x; b < kNu; b += blockDim.x)
    especn[(size_t)e * kNu + spec_pair_index(b)] = __double2float_rn(__dmul_rn(s[b], inv));
}

// bounding box of the emitter positions (one block)
__global__ void k_emit_bounds(int ne, const float4 *__restrict__ epos, float *__restrict__ out6) {
  __shared__ float lo[3][256], hi[3][256];
  float l[3], h[3];
  for (int a = 0; a < 3; a++) {
    l[a] = 3.4e38f;
    h[a] = -3.4e38f;
  }
  for (int e = threadIdx.x; e < ne; e += blockDim.x) {
    const float4 p = epos[e];
    l[0] = fminf(l[0], p.x); l[1] = fminf(l[1], p.y); l[2] = fminf(l[2], p.z);
    h[0] = fmaxf(h[0], p.x); h[1] = fmaxf(h[1], p.y); h[2] = fmaxf(h[2], p.z);
  }
  for (int a = 0; a < 3; a++) {
    lo[a][threadIdx.x] = l[a];
    hi[a][threadIdx.x] = h[a];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int a = 0; a < 3; a++) {
      float L = lo[a][0], H = hi[a][0];
      for (int t = 1; t < blockDim.x; t++) {
        L = fminf(L, lo[a][t]);
        H = fmaxf(H, hi[a][t]);
      }
      out6[a] = L;
      out6[3 + a] = H;
    }
  }
}

// per-depth node lists (counting sort of the node indices by depth)
__global__ void k_depth_lists(int nn, const int *__restrict__ depth, const int *__restrict__ dstart,
                              int *__restrict__ dfill, int *__restrict__ lists) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nn || p == 0) return;
  const int d = depth[p];
  lists[dstart[d] + atomicAdd(&dfill[d], 1)] = p;
}
__global__ void k_depth_hist(int nn, const int *__restrict__ depth, int *__restrict__ hist) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nn || p == 0) return;
  atomicAdd(&hist[depth[p]], 1);
}

}  // namespace
}  // namespace argot

using namespace argot;

extern "C" {

int argot_b200_dev_tree_build(const argot_b200_grid *g, int nsrc, const float *src_pos, const double *spectra,
                              float theta, argot_b200_dev_tree **out, void *stream) {
  if (!g || nsrc <= 0 || !src_pos || !spectra || !out) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0;
  ARGOT_CUDA_TRY(cudaGetDevice(&dev));
  int rc = ensure_tables(dev);
  if (rc) { set_status(rc); return rc; }
  const int n = nsrc;
  const float xl = g->xmax - g->xmin, yl = g->ymax - g->ymin, zl = g->zmax - g->zmin;
  const float base = std::max(xl, std::max(yl, zl));
  // side of a node at depth d, as the host builder forms it
  float side[kMaxDepth + 1];
  side[0] = base;
  for (int d = 1; d <= kMaxDepth; d++) {
    const int level = 63 - 3 * d;
    side[d] = (float)(base * std::pow(2.0, -(63.0 - level) / 3.0));
  }
  // scratch
  unsigned long long *keys = nullptr, *keys_s = nullptr;
  int *idx = nullptr, *idx_s = nullptr, *cnt = nullptr, *first = nullptr, *depth = nullptr, *dlist = nullptr;
  int *dhist = nullptr;
  double *lum = nullptr, *nlum = nullptr, *ncm = nullptr;
  float *side_d = nullptr, *bounds = nullptr;
  void *tmp = nullptr;
  size_t tmp_bytes = 0, t1 = 0, t2 = 0;
  argot_b200_dev_tree *d = nullptr;
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void **p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes ? bytes : 16);
  };
  auto cleanup = [&]() {
    cudaFree(keys); cudaFree(keys_s); cudaFree(idx); cudaFree(cnt); cudaFree(first);
    cudaFree(depth); cudaFree(dlist); cudaFree(dhist); cudaFree(lum); cudaFree(nlum); cudaFree(ncm);
    cudaFree(side_d); cudaFree(bounds); cudaFree(tmp);
  };
  alloc((void **)&keys, sizeof(unsigned long long) * n);
  alloc((void **)&keys_s, sizeof(unsigned long long) * n);
  alloc((void **)&idx, sizeof(int) * n);
  alloc((void **)&cnt, sizeof(int) * (n + 1));
  alloc((void **)&first, sizeof(int) * (n + 1));
  alloc((void **)&lum, sizeof(double) * n);
  alloc((void **)&side_d, sizeof(side));
  alloc((void **)&bounds, sizeof(float) * 6);
  d = new (std::nothrow) argot_b200_dev_tree();
  if (!d) { cleanup(); set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  alloc((void **)&d->src_list, sizeof(int) * n);
  idx_s = d->src_list;
  if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(nullptr, t1, keys, keys_s, idx, idx_s, n, 0, 64, st);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, t2, cnt, first, n + 1, st);
  tmp_bytes = std::max(t1, t2);
  alloc(&tmp, tmp_bytes);
  if (e == cudaSuccess) e = cudaMemcpyAsync(side_d, side, sizeof(side), cudaMemcpyHostToDevice, st);
  const int T = 256;
  if (e == cudaSuccess) {
    k_src_keys<<<(n + T - 1) / T, T, 0, st>>>(n, src_pos, g->xmin, g->ymin, g->zmin, base, spectra, keys, idx, lum);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(tmp, t1, keys, keys_s, idx, idx_s, n, 0, 64, st);
  if (e == cudaSuccess) {
    k_node_counts<<<(n + 1 + T - 1) / T, T, 0, st>>>(n, keys_s, cnt);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, t2, cnt, first, n + 1, st);
  int nn = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&nn, first + n, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  const size_t ne = (size_t)nn + n;
  alloc((void **)&d->nodes, sizeof(DevNode) * nn);
  alloc((void **)&depth, sizeof(int) * nn);
  alloc((void **)&dlist, sizeof(int) * nn);
  alloc((void **)&dhist, sizeof(int) * 2 * (kMaxDepth + 1));
  alloc((void **)&nlum, sizeof(double) * nn);
  alloc((void **)&ncm, sizeof(double) * 3 * nn);
  alloc((void **)&d->emit_pos, sizeof(float4) * ne);
  alloc((void **)&d->emit_spec64, sizeof(double) * ne * kNu);
  alloc((void **)&d->emit_specn, sizeof(float) * ne * kNu);
  alloc((void **)&d->emit_total, sizeof(double) * ne);
  if (e == cudaSuccess) {
    k_node_fill<<<(n + T - 1) / T, T, 0, st>>>(n, keys_s, first, side_d, d->nodes, depth);
    e = cudaGetLastError();
  }
  // per-depth lists
  int hist[kMaxDepth + 1] = {0}, dstart[kMaxDepth + 2] = {0};
  if (e == cudaSuccess) e = cudaMemsetAsync(dhist, 0, sizeof(int) * 2 * (kMaxDepth + 1), st);
  if (e == cudaSuccess && nn > 1) {
    k_depth_hist<<<(nn + T - 1) / T, T, 0, st>>>(nn, depth, dhist);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(hist, dhist, sizeof(hist), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  for (int k = 0; k <= kMaxDepth; k++) dstart[k + 1] = dstart[k] + hist[k];
  int *dstart_d = dhist + (kMaxDepth + 1);  // reuse: starts (device), then fill counters in dhist
  if (e == cudaSuccess) e = cudaMemcpyAsync(dstart_d, dstart, sizeof(int) * (kMaxDepth + 1), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(dhist, 0, sizeof(int) * (kMaxDepth + 1), st);
  if (e == cudaSuccess && nn > 1) {
    k_depth_lists<<<(nn + T - 1) / T, T, 0, st>>>(nn, depth, dstart_d, dhist, dlist);
    e = cudaGetLastError();
  }
  // node sums from the deepest level up; lists in any order within a
  // depth (nodes of one depth are independent)
  for (int k = kMaxDepth; k >= 1 && e == cudaSuccess; k--) {
    const int m = hist[k];
    if (!m) continue;
    k_node_sums<<<(m * 32 + T - 1) / T, T, 0, st>>>(dlist + dstart[k], m, d->nodes, idx_s, src_pos, spectra, lum,
                                                     d->emit_spec64, nlum, ncm);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_root_sums<<<1, 256, 0, st>>>(n, src_pos, spectra, d->nodes, d->emit_spec64);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_emitters<<<(unsigned)ne, 128, 0, st>>>(nn, n, d->nodes, src_pos, spectra, d->emit_pos, d->emit_spec64,
                                               d->emit_specn, d->emit_total);
    e = cudaGetLastError();
  }
  float b6[6] = {0, 0, 0, 0, 0, 0};
  if (e == cudaSuccess) {
    k_emit_bounds<<<1, 256, 0, st>>>((int)ne, d->emit_pos, bounds);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(b6, bounds, sizeof(b6), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cleanup();
  if (e != cudaSuccess) {
    argot_b200_dev_tree_free(d);
    return status_from_cuda(e);
  }
  d->device = dev;
  d->n_nodes = nn;
  d->n_src = n;
  d->n_emit = (int)ne;
  d->theta_sq = theta * theta;
  for (int a = 0; a < 3; a++) {
    d->emit_lo[a] = b6[a];
    d->emit_hi[a] = b6[3 + a];
  }
  *out = d;
  set_status(0);
  return 0;
}

int argot_b200_dev_tree_copy(const argot_b200_dev_tree *d, float *pos4, double *spec64, int *nodes8,
                             int *src_list, void *stream) {
  if (!d) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  cudaStream_t st = (cudaStream_t)stream;
  const size_t ne = (size_t)d->n_emit;
  if (pos4) ARGOT_CUDA_TRY(cudaMemcpyAsync(pos4, d->emit_pos, sizeof(float4) * ne, cudaMemcpyDeviceToHost, st));
  if (spec64)
    ARGOT_CUDA_TRY(cudaMemcpyAsync(spec64, d->emit_spec64, sizeof(double) * ne * kNu, cudaMemcpyDeviceToHost, st));
  if (nodes8)
    ARGOT_CUDA_TRY(cudaMemcpyAsync(nodes8, d->nodes, sizeof(DevNode) * (size_t)d->n_nodes, cudaMemcpyDeviceToHost, st));
  if (src_list)
    ARGOT_CUDA_TRY(cudaMemcpyAsync(src_list, d->src_list, sizeof(int) * (size_t)d->n_src, cudaMemcpyDeviceToHost, st));
  ARGOT_CUDA_TRY(cudaStreamSynchronize(st));
  set_status(0);
  return 0;
}

int argot_b200_dev_tree_info(const argot_b200_dev_tree *d, int *n_nodes, int *n_emit, float *bounds6) {
  if (!d) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  if (n_nodes) *n_nodes = d->n_nodes;
  if (n_emit) *n_emit = d->n_emit;
  if (bounds6) {
    for (int a = 0; a < 3; a++) {
      bounds6[a] = d->emit_lo[a];
      bounds6[3 + a] = d->emit_hi[a];
    }
  }
  set_status(0);
  return 0;
}

}  // extern "C"
