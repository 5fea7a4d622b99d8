// host.cu -- host-side parts of libargot_b200: status codes, ABI
// identification, the frequency/cross-section tables, source spectra and the
// oct-tree over the sources.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "common.cuh"
#include "ref_layout.h"

namespace argot {

static thread_local int t_status = 0;
void set_status(int code) { t_status = code; }
int status_from_cuda(cudaError_t e) {
  t_status = (e == cudaErrorMemoryAllocation) ? ARGOT_B200_ENOMEM : ARGOT_B200_ECUDA;
  return t_status;
}

bool grid_valid(const argot_b200_grid *g) {
  return g && g->nx > 0 && g->ny > 0 && g->nz > 0 && g->dx > 0.f && g->dy > 0.f &&
         g->dz > 0.f && (uint64_t)g->nx * g->ny * g->nz < (1ull << 40);
}

GridDev make_grid(const argot_b200_grid &g) {
  GridDev d;
  d.nx = g.nx; d.ny = g.ny; d.nz = g.nz;
  d.ix0 = g.ix0; d.iy0 = g.iy0; d.iz0 = g.iz0;
  d.xmin = g.xmin; d.ymin = g.ymin; d.zmin = g.zmin;
  d.xmax = g.xmax; d.ymax = g.ymax; d.zmax = g.zmax;
  d.xminl = g.xmin_local; d.yminl = g.ymin_local; d.zminl = g.zmin_local;
  d.dx = g.dx; d.dy = g.dy; d.dz = g.dz;
  d.lunit = g.lunit; d.denstonh = g.denstonh;
  d.nbx = (g.nx + kBlkX - 1) / kBlkX;
  d.nby = (g.ny + kBlkY - 1) / kBlkY;
  d.nbz = (g.nz + kBlkZ - 1) / kBlkZ;
  d.cdf = (float)(g.lunit * g.denstonh);
  int e = 0;
  const double m = std::frexp(1.0 / (4.0 * kPi * g.lunit * g.lunit), &e);  // m in [0.5, 1)
  d.pcm = (float)(2.0 * m);
  d.pce = e - 1;
  return d;
}

// ------------------------------------------------------------------ tables
// Frequency grid: 256 bins evenly spaced in log10(nu) over [0, 1.5] (nu in
// units of the HI Lyman limit), bin centres (source.c:38-53; the bin width
// is divided by a float-converted 256 as there).  Cross sections: the
// analytic fits of prim_chem/cross_section.c:20-53 for HI, HeI and HeII.
double sigma_hi(double nu) {
  if (nu < kThrHI) return 0.0;
  double e = std::sqrt(nu - kThrHI);
  return 6.3e-18 / (nu * nu * nu * nu) * std::exp(4.0 - 4.0 * std::atan(e) / e) /
         (1.0 - std::exp(-2.0 * kPi / e));
}
double sigma_hei(double nu) {
  if (nu < kThrHeI) return 0.0;
  return 7.83e-18 * (1.66 * std::pow(nu / kThrHeI, -2.05) - 0.66 * std::pow(nu / kThrHeI, -3.05));
}
double sigma_heii(double nu) {
  if (nu < kThrHeII) return 0.0;
  double e = std::sqrt(nu / kThrHeII - 1.0);
  return 6.3e-18 * 256.0 / (nu * nu * nu * nu) * std::exp(4.0 - 4.0 * std::atan(e) / e) /
         (1.0 - std::exp(-2.0 * kPi / e)) / 4.0;
}

static double dlog_nu() { return (1.5 - 0.0) / (float)kNu; }

void host_tables(double *nu, float *cs3) {
  const double dl = dlog_nu();
  for (int i = 0; i < kNu; i++) {
    double v = std::pow(10.0, 0.0 + (i + 0.5) * dl);
    if (nu) nu[i] = v;
    cs3[3 * i + 0] = (float)sigma_hi(v);
    cs3[3 * i + 1] = (float)sigma_hei(v);
    cs3[3 * i + 2] = (float)sigma_heii(v);
  }
}

void host_rate_weights(double *w6) {
  double nu[kNu];
  float cs3[3 * kNu];
  host_tables(nu, cs3);
  const double thr[3] = {kThrHI, kThrHeI, kThrHeII};
  for (int k = 0; k < kNu; k++) {
    const double nf = (double)(float)nu[k];
    for (int s = 0; s < 3; s++) {
      const double c = cs3[3 * k + s];
      w6[s * kNu + k] = c;
      w6[(3 + s) * kNu + k] = c * (nf > thr[s] ? nf - thr[s] : 0.0);
    }
  }
}

// ----------------------------------------------------------- photon rates
// Blackbody (photon-number shape nu^2/(e^{h nu/kT}-1), normalised at the
// Lyman limit) or power law nu^p; per-bin photon counts by the iterated
// (tripling) midpoint rule to 1e-8 or 5 stages, scaled so that the bins sum
// to the total rate over [1, 10^1.5] nu_L (source.c:10-138).
static double shape(int type, double nu, double p) {
  if (type == 0) {
    double a = (nu * kNuL) * (nu * kNuL) / (std::exp(kHPlanck * nu * kNuL / (1.38066e-16 * p)) - 1.0);
    double b = kNuL * kNuL / (std::exp(kHPlanck * kNuL / (1.38066e-16 * p)) - 1.0);
    return a / b;
  }
  return std::pow(nu, p);
}

static double midpoint_stages(int type, double p, double a, double b) {
  double s = 0.0, prev = 0.0;
  for (int stage = 1; stage <= 5; stage++) {
    if (stage == 1) {
      s = (b - a) * shape(type, 0.5 * (a + b), p);
    } else {
      int npts = 1;
      for (int j = 1; j < stage - 1; j++) npts *= 3;
      double h = (b - a) / (3.0 * npts);
      double x = a + 0.5 * h, acc = 0.0;
      for (int j = 1; j <= npts; j++) {
        acc += shape(type, x, p);
        x += h + h;
        acc += shape(type, x, p);
        x += h;
      }
      s = (s + (b - a) * acc / npts) / 3.0;
    }
    if (stage > 1 && std::fabs(s - prev) < 1.0e-8 * std::fabs(prev)) return s;
    prev = s;
  }
  return s;
}

}  // namespace argot

using namespace argot;

extern "C" {

int argot_b200_last_error(void) { return t_status; }

const char *argot_b200_error_string(int code) {
  switch (code) {
    case ARGOT_B200_OK: return "ok";
    case ARGOT_B200_EINVAL: return "invalid argument";
    case ARGOT_B200_ECUDA: return "CUDA runtime error";
    case ARGOT_B200_ENOMEM: return "out of memory";
    case ARGOT_B200_EDEVICE: return "kernel reported an internal error";
    case ARGOT_B200_ENOTSUP: return "not supported";
    default: return "unknown error";
  }
}

const char *argot_b200_version(void) { return "argot_b200 0.1 (sm_100a)"; }

void argot_b200_struct_sizes(uint64_t *s) {
  s[0] = sizeof(argot::ray_segment);
  s[1] = sizeof(argot::light_ray);
  s[2] = sizeof(argot::light_ray_IO);
  s[3] = sizeof(argot::radiation_src);
  s[4] = sizeof(argot::fluid_mesh);
  s[5] = sizeof(argot::prim_chem);
  s[6] = sizeof(argot::run_param);
  s[7] = sizeof(argot::cross_section);
  s[8] = sizeof(argot::freq_param);
  s[9] = sizeof(argot::photoion_rate);
}

int argot_b200_abi_check(const uint64_t *caller, int n) {
  uint64_t mine[10];
  argot_b200_struct_sizes(mine);
  if (!caller || n <= 0 || n > 10) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  for (int i = 0; i < n; i++)
    if (caller[i] != mine[i]) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  set_status(0);
  return 0;
}

void argot_b200_tables(double *nu, float *csect3) { host_tables(nu, csect3); }

void argot_b200_photon_counts(int type, float param, double *counts, double *norm) {
  const double dl = dlog_nu();
  *norm = midpoint_stages(type, (double)param, 1.0, std::pow(10.0, 1.5));
  for (int i = 0; i < kNu; i++) {
    double a = 0.0 + dl * (double)i;
    double b = a + dl;
    counts[i] = midpoint_stages(type, (double)param, std::pow(10.0, a), std::pow(10.0, b));
  }
}

void argot_b200_photon_rate(int type, float param, double total, double *out) {
  double norm;
  argot_b200_photon_counts(type, param, out, &norm);
  for (int i = 0; i < kNu; i++) out[i] *= total / norm;
}

}  // extern "C"

// ================================================================== tree
// Oct-tree over the sources with the reference's construction rules
// (setup_light_ray_tree.c:100-239, 465-571):
//  * 63-bit Morton keys, 21 bits per axis, of (pos - box_min)/L * 2^21 with
//    L = the longest box side; a leading 1 bit marks the root;
//  * a node at key level k (63 for the root, minus 3 per level) is split
//    into its non-empty octants (children in octant order 0..7) while it
//    holds more than one source and k > 0;
//  * node side = L * 2^-(63-k)/3;
//  * node spectrum = sum of its children's spectra (leaves: of their
//    sources, in sorted order); node centre = luminosity-weighted mean
//    position, luminosity = sum over bins of the photon rate; internal nodes
//    divide the weighted sum by the luminosity, leaves multiply by its
//    reciprocal; the root's centre is weighted by the first bin only
//    (setup_light_ray_tree.c:533-554).
// Nodes are stored in depth-first preorder with "skip" links so that the
// device walk needs no stack.
struct argot_b200_tree {
  float theta_sq;
  int nsrc;
  std::vector<DevNode> nodes;
  std::vector<int> src_list;        // sorted source indices
  std::vector<double> spec;         // n_nodes x 256
  std::vector<float> src_pos;       // nsrc x 3
  std::vector<double> src_spec;     // nsrc x 256
};

namespace {

struct Builder {
  const float *pos;
  const double *spectra;
  std::vector<uint64_t> key;   // sorted keys
  std::vector<int> idx;        // sorted source index
  float base_length;
  argot_b200_tree *t;

  static double lum(const double *s) {
    double L = 0.0;
    for (int k = 0; k < kNu; k++) L += s[k];
    return L;
  }

  // Children of the node at `self` (already appended), holding sorted
  // entries [first, first+n) at key level `level` (before the split).
  // Returns via the out-parameters the node's luminosity, spectrum and
  // luminosity-weighted position sums.
  void split(int self, int first, int n, int level, double *tot_L, double *tot_spec,
             double *tot_cm) {
    level -= 3;
    int cnt[8] = {0}, beg[8] = {0};
    int prev = -1;
    for (int i = first; i < first + n; i++) {
      int f = (int)((key[i] >> level) & 7);
      cnt[f]++;
      if (f != prev) beg[f] = i;
      prev = f;
    }
    *tot_L = 0.0;
    for (int k = 0; k < kNu; k++) tot_spec[k] = 0.0;
    tot_cm[0] = tot_cm[1] = tot_cm[2] = 0.0;
    t->nodes[self].has_child = 0;
    const float side = (float)(base_length * std::pow(2.0, -(63.0 - level) / 3.0));
    for (int c = 0; c < 8; c++) {
      if (!cnt[c]) continue;
      const int me = (int)t->nodes.size();
      t->nodes[self].has_child = 1;
      DevNode nd{};
      nd.len = side;
      nd.n = cnt[c];
      nd.src_first = beg[c];
      t->nodes.push_back(nd);
      t->spec.resize(t->nodes.size() * kNu);
      double L, cm[3];
      std::vector<double> s(kNu, 0.0);
      if (cnt[c] > 1 && level > 0) {
        split(me, beg[c], cnt[c], level, &L, s.data(), cm);
        for (int k = 0; k < 3; k++) cm[k] = cm[k];
        t->nodes[me].cx = (float)(cm[0] / L);
        t->nodes[me].cy = (float)(cm[1] / L);
        t->nodes[me].cz = (float)(cm[2] / L);
      } else {
        double m = 0.0;
        cm[0] = cm[1] = cm[2] = 0.0;
        for (int j = beg[c]; j < beg[c] + cnt[c]; j++) {
          const int is = idx[j];
          const double *ss = spectra + (size_t)is * kNu;
          double mj = lum(ss);
          for (int k = 0; k < kNu; k++) s[k] += ss[k];
          m += mj;
          cm[0] += mj * pos[3 * is + 0];
          cm[1] += mj * pos[3 * is + 1];
          cm[2] += mj * pos[3 * is + 2];
        }
        L = m;
        const double minv = 1.0 / m;
        t->nodes[me].cx = (float)(cm[0] * minv);
        t->nodes[me].cy = (float)(cm[1] * minv);
        t->nodes[me].cz = (float)(cm[2] * minv);
        t->nodes[me].has_child = 0;
      }
      std::memcpy(&t->spec[(size_t)me * kNu], s.data(), sizeof(double) * kNu);
      t->nodes[me].skip = (int)t->nodes.size();
      *tot_L += L;
      for (int k = 0; k < kNu; k++) tot_spec[k] += s[k];
      for (int k = 0; k < 3; k++) tot_cm[k] += cm[k];
    }
  }
};

}  // namespace

extern "C" {

int argot_b200_tree_build(const argot_b200_grid *g, int nsrc, const float *src_pos,
                          const double *spectra, float theta, argot_b200_tree **out) {
  if (!g || nsrc <= 0 || !src_pos || !spectra || !out) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  argot_b200_tree *t = new (std::nothrow) argot_b200_tree();
  if (!t) { set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  t->theta_sq = theta * theta;
  t->nsrc = nsrc;
  t->src_pos.assign(src_pos, src_pos + 3 * (size_t)nsrc);
  t->src_spec.assign(spectra, spectra + (size_t)kNu * nsrc);

  Builder b;
  b.pos = src_pos;
  b.spectra = spectra;
  b.t = t;
  const float xl = g->xmax - g->xmin, yl = g->ymax - g->ymin, zl = g->zmax - g->zmin;
  b.base_length = std::max(xl, std::max(yl, zl));
  const double scale = (double)(1 << 21);
  std::vector<std::pair<uint64_t, int>> kv(nsrc);
  for (int i = 0; i < nsrc; i++) {
    uint64_t ip[3];
    ip[0] = (uint64_t)(int)((src_pos[3 * i + 0] - g->xmin) / b.base_length * scale);
    ip[1] = (uint64_t)(int)((src_pos[3 * i + 1] - g->ymin) / b.base_length * scale);
    ip[2] = (uint64_t)(int)((src_pos[3 * i + 2] - g->zmin) / b.base_length * scale);
    uint64_t k = 1ull << 63;
    for (int bit = 0; bit < 21; bit++) {
      uint64_t tri = (((ip[0] >> bit) & 1) << 2) | (((ip[1] >> bit) & 1) << 1) | ((ip[2] >> bit) & 1);
      k |= tri << (3 * bit);
    }
    kv[i] = {k, i};
  }
  // Sorted by key; sources sharing a key (closer than 2^-21 of the box) keep
  // their input order.
  std::stable_sort(kv.begin(), kv.end(),
                   [](const std::pair<uint64_t, int> &a, const std::pair<uint64_t, int> &c) {
                     return a.first < c.first;
                   });
  b.key.resize(nsrc);
  b.idx.resize(nsrc);
  for (int i = 0; i < nsrc; i++) { b.key[i] = kv[i].first; b.idx[i] = kv[i].second; }
  t->src_list = b.idx;

  // root
  DevNode root{};
  root.len = b.base_length;
  root.n = nsrc;
  root.src_first = 0;
  t->nodes.push_back(root);
  t->spec.assign(kNu, 0.0);
  double xc = 0, yc = 0, zc = 0, l0 = 0;
  for (int i = 0; i < nsrc; i++) {
    const double w = spectra[(size_t)i * kNu + 0];
    xc += src_pos[3 * i + 0] * w;
    yc += src_pos[3 * i + 1] * w;
    zc += src_pos[3 * i + 2] * w;
    l0 += w;
    for (int k = 0; k < kNu; k++) t->spec[k] += spectra[(size_t)i * kNu + k];
  }
  xc /= l0; yc /= l0; zc /= l0;
  t->nodes[0].cx = (float)xc;
  t->nodes[0].cy = (float)yc;
  t->nodes[0].cz = (float)zc;
  double L, cm[3];
  std::vector<double> s(kNu);
  b.split(0, 0, nsrc, 63, &L, s.data(), cm);
  t->nodes[0].skip = (int)t->nodes.size();
  *out = t;
  set_status(0);
  return 0;
}

void argot_b200_tree_free(argot_b200_tree *t) { delete t; }

int argot_b200_tree_num_nodes(const argot_b200_tree *t) { return t ? (int)t->nodes.size() : 0; }
int argot_b200_tree_num_emitters(const argot_b200_tree *t) {
  return t ? (int)t->nodes.size() + t->nsrc : 0;
}

int argot_b200_tree_emitters(const argot_b200_tree *t, float *pos4, double *spec64) {
  if (!t) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  const size_t nn = t->nodes.size();
  for (size_t i = 0; i < nn; i++) {
    if (pos4) {
      pos4[4 * i + 0] = t->nodes[i].cx;
      pos4[4 * i + 1] = t->nodes[i].cy;
      pos4[4 * i + 2] = t->nodes[i].cz;
      pos4[4 * i + 3] = 0.f;
    }
    if (spec64) std::memcpy(spec64 + i * kNu, &t->spec[i * kNu], sizeof(double) * kNu);
  }
  for (int j = 0; j < t->nsrc; j++) {
    const size_t e = nn + j;
    if (pos4) {
      pos4[4 * e + 0] = t->src_pos[3 * j + 0];
      pos4[4 * e + 1] = t->src_pos[3 * j + 1];
      pos4[4 * e + 2] = t->src_pos[3 * j + 2];
      pos4[4 * e + 3] = 0.f;
    }
    if (spec64) std::memcpy(spec64 + e * kNu, &t->src_spec[(size_t)j * kNu], sizeof(double) * kNu);
  }
  set_status(0);
  return 0;
}

int argot_b200_dev_tree_upload(const argot_b200_tree *t, argot_b200_dev_tree **out,
                               void *stream) {
  if (!t || !out) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0;
  ARGOT_CUDA_TRY(cudaGetDevice(&dev));
  int rc = ensure_tables(dev);
  if (rc) return rc;
  auto *d = new (std::nothrow) argot_b200_dev_tree();
  if (!d) { set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  d->device = dev;
  d->n_nodes = (int)t->nodes.size();
  d->n_src = t->nsrc;
  d->n_emit = d->n_nodes + d->n_src;
  d->theta_sq = t->theta_sq;
  const size_t ne = (size_t)d->n_emit;
  std::vector<float> pos4(4 * ne);
  std::vector<double> spec(ne * kNu);
  argot_b200_tree_emitters(t, pos4.data(), spec.data());
  for (int a = 0; a < 3; a++) {
    d->emit_lo[a] = ne ? pos4[a] : 0.f;
    d->emit_hi[a] = ne ? pos4[a] : 0.f;
  }
  for (size_t e = 0; e < ne; e++) {
    for (int a = 0; a < 3; a++) {
      d->emit_lo[a] = std::min(d->emit_lo[a], pos4[4 * e + a]);
      d->emit_hi[a] = std::max(d->emit_hi[a], pos4[4 * e + a]);
    }
  }
  std::vector<float> specn(ne * kNu);
  std::vector<double> total(ne);
  for (size_t e = 0; e < ne; e++) {
    double s = 0.0;
    for (int k = 0; k < kNu; k++) s += spec[e * kNu + k];
    total[e] = s;
    const double inv = s > 0.0 ? 1.0 / s : 0.0;
    // bin-pair order of the packed rate loop: position 2 p + h holds bin
    // (p % 8) + 16 (p / 8) + 8 h (spec_pair_index)
    for (int k = 0; k < kNu; k++) specn[e * kNu + spec_pair_index(k)] = (float)(spec[e * kNu + k] * inv);
  }
  cudaError_t err = cudaSuccess;
  auto alloc = [&](void **p, size_t bytes) {
    if (err == cudaSuccess) err = cudaMalloc(p, bytes ? bytes : 16);
  };
  alloc((void **)&d->nodes, sizeof(DevNode) * d->n_nodes);
  alloc((void **)&d->src_list, sizeof(int) * d->n_src);
  alloc((void **)&d->emit_pos, sizeof(float4) * ne);
  alloc((void **)&d->emit_spec64, sizeof(double) * ne * kNu);
  alloc((void **)&d->emit_specn, sizeof(float) * ne * kNu);
  alloc((void **)&d->emit_total, sizeof(double) * ne);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(d->nodes, t->nodes.data(), sizeof(DevNode) * d->n_nodes,
                          cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(d->src_list, t->src_list.data(), sizeof(int) * d->n_src,
                          cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(d->emit_pos, pos4.data(), sizeof(float4) * ne, cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(d->emit_spec64, spec.data(), sizeof(double) * ne * kNu,
                          cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(d->emit_specn, specn.data(), sizeof(float) * ne * kNu,
                          cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(d->emit_total, total.data(), sizeof(double) * ne, cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  if (err != cudaSuccess) {
    argot_b200_dev_tree_free(d);
    return status_from_cuda(err);
  }
  *out = d;
  set_status(0);
  return 0;
}

void argot_b200_dev_tree_free(argot_b200_dev_tree *d) {
  if (!d) return;
  cudaFree(d->nodes);
  cudaFree(d->src_list);
  cudaFree(d->emit_pos);
  cudaFree(d->emit_spec64);
  cudaFree(d->emit_specn);
  cudaFree(d->emit_total);
  cudaFree(d->emit_logT);
  cudaFree(d->emit_i0);
  cudaFree(d->emit_m);
  delete d;
}

// Spectral temperature of every emitter for the surrogate: a node whose
// sources are all blackbodies of one temperature T (src_T[i] > 0) has the
// normalised spectrum of that blackbody; any other emitter gets NaN and
// is always integrated exactly.  Also uploads each emitter's six thin-limit
// integrals I_j0 = sum_nu w_j(nu) s_nu of its own normalised spectrum and
// the first moments m_js = sum_nu w_j s_nu sigma_s(nu) / sigma_s0 / I_j0.
int argot_b200_dev_tree_set_blackbody(const argot_b200_tree *t, argot_b200_dev_tree *d, const float *src_T,
                                      void *stream) {
  if (!t || !d || !src_T || d->n_src != t->nsrc) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  const size_t nn = t->nodes.size(), ne = nn + t->nsrc;
  std::vector<float> logT(ne);
  const float qnan = std::nanf("");
  auto temp_of = [&](float T) { return (T > 0.f) ? (float)std::log10((double)T) : qnan; };
  for (size_t i = 0; i < nn; i++) {
    const DevNode &nd = t->nodes[i];
    float T0 = src_T[t->src_list[nd.src_first]];
    bool same = T0 > 0.f;
    for (int j = 1; j < nd.n && same; j++) same = src_T[t->src_list[nd.src_first + j]] == T0;
    logT[i] = same ? temp_of(T0) : qnan;
  }
  for (int j = 0; j < t->nsrc; j++) logT[nn + j] = temp_of(src_T[j]);
  std::vector<double> w(6 * kNu), i0(6 * ne);
  std::vector<float> mom(18 * ne);
  host_rate_weights(w.data());
  double sig0[3];
  for (int s = 0; s < 3; s++) {
    sig0[s] = 0.0;
    for (int k = 0; k < kNu && sig0[s] == 0.0; k++) sig0[s] = w[s * kNu + k];
  }
  std::vector<double> spec(ne * kNu);
  argot_b200_tree_emitters(t, nullptr, spec.data());
  for (size_t e = 0; e < ne; e++) {
    double tot = 0.0;
    for (int k = 0; k < kNu; k++) tot += spec[e * kNu + k];
    for (int j = 0; j < 6; j++) {
      double s0 = 0.0, m[3] = {0.0, 0.0, 0.0};
      for (int k = 0; k < kNu; k++) {
        const double a = w[j * kNu + k] * (spec[e * kNu + k] / tot);
        s0 += a;
        for (int s = 0; s < 3; s++) m[s] += a * (w[s * kNu + k] / sig0[s]);
      }
      i0[e * 6 + j] = s0;
      for (int s = 0; s < 3; s++) mom[e * 18 + 3 * j + s] = s0 > 0.0 ? (float)(m[s] / s0) : 0.f;
    }
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (!d->emit_logT) ARGOT_CUDA_TRY(cudaMalloc(&d->emit_logT, sizeof(float) * ne));
  if (!d->emit_i0) ARGOT_CUDA_TRY(cudaMalloc(&d->emit_i0, sizeof(double) * 6 * ne));
  if (!d->emit_m) ARGOT_CUDA_TRY(cudaMalloc(&d->emit_m, sizeof(float) * 18 * ne));
  ARGOT_CUDA_TRY(cudaMemcpyAsync(d->emit_logT, logT.data(), sizeof(float) * ne, cudaMemcpyHostToDevice, st));
  ARGOT_CUDA_TRY(cudaMemcpyAsync(d->emit_i0, i0.data(), sizeof(double) * 6 * ne, cudaMemcpyHostToDevice, st));
  ARGOT_CUDA_TRY(cudaMemcpyAsync(d->emit_m, mom.data(), sizeof(float) * 18 * ne, cudaMemcpyHostToDevice, st));
  ARGOT_CUDA_TRY(cudaStreamSynchronize(st));
  set_status(0);
  return 0;
}

}  // extern "C"
