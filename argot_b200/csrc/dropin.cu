// dropin.cu -- the reference's own entry points (src/prototype.h:47,89,93,
// 124-125) on one GPU, for argot_mpi / argot_hydro_mpi to link in place of
// calc_optical_depth_cuda.o, calc_photoion_rate_cuda.o,
// accum_optical_depth.o and smooth_photoion_rate.o on a single rank.
//
// Every kernel here follows the caller's flag set (flagset.h): the columns
// of a segment, the cross-section channels and the rate fields are those
// of the struct layouts the library is compiled for, and the rate formula
// is the photon-conserving or the plain one, with or without the scale
// factor, as the reference's calc_photoion_rate.c selects them.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "march.cuh"
#include "ref_layout.h"

namespace argot {

int launch_smooth_planes(int nx, int ny, int nz, const float *in, float *out, int nplanes, int isolated,
                         cudaStream_t st);
int grid_blocks_for_rates(uint64_t n, int threads);
int *err_flag(int dev);
int check_err_flag(int *flag, cudaStream_t st);

using flags::kNCol;
using flags::kNChan;
using flags::kNOut;

// ------------------------------------------------------------------ packing
// kNG float4 per cell: the species densities of the march in column order,
// each the product the reference forms per crossing
// (calc_optical_depth.c:150-161): n_HI = dens*fHI and n_HM, n_H2I, n_H2II
// likewise in float; n_He = (float)(dens * HELIUM_FACT) in double, then
// n_HeI = n_He*fHeI in float.
constexpr int kNG = (kNCol + 3) / 4;

__global__ void k_pack_cols(uint64_t n, const fluid_mesh *__restrict__ mesh, float4 *__restrict__ cells) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const fluid_mesh &m = mesh[i];
    const float d = m.dens;
    float v[4 * kNG];
#pragma unroll
    for (int q = 0; q < 4 * kNG; q++) v[q] = 0.f;
    v[0] = __fmul_rn(d, m.chem.fHI);
#ifdef __HELIUM__
    const float nhe = __double2float_rn(__dmul_rn((double)d, kHeliumFact));
    v[flags::kColHeI] = __fmul_rn(nhe, m.chem.fHeI);
    v[flags::kColHeII] = __fmul_rn(nhe, m.chem.fHeII);
#endif
#ifdef __HYDROGEN_MOL__
    v[flags::kColHM] = __fmul_rn(d, m.chem.fHM);
    v[flags::kColH2I] = __fmul_rn(d, m.chem.fH2I);
    v[flags::kColH2II] = __fmul_rn(d, m.chem.fH2II);
#endif
#pragma unroll
    for (int q = 0; q < kNG; q++) cells[i * kNG + q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  }
}

// ------------------------------------------------------------------ march
// The reference's struct ray_segment array, in place: every column of the
// flag set, by the reference-order march (bit-identical) or the
// compensated one.
template <int kPrec>
__global__ void k_march_aos(GridDev g, const float4 *__restrict__ cells, uint64_t nseg,
                            ray_segment *__restrict__ seg, int *__restrict__ err) {
  bool bad = false;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nseg;
       i += (uint64_t)gridDim.x * blockDim.x) {
    ray_segment &s = seg[i];
    int steps;
    const Cols<kNCol> t = (kPrec == ARGOT_B200_PRECISION_REFERENCE)
                              ? march_reference_n<kNCol>(g, cells, s.xpos_start, s.ypos_start, s.zpos_start,
                                                         s.xpos_end, s.ypos_end, s.zpos_end, &steps, &bad)
                              : march_kahan_n<kNCol>(g, cells, s.xpos_start, s.ypos_start, s.zpos_start,
                                                     s.xpos_end, s.ypos_end, s.zpos_end, &steps, &bad);
    float *o = s.col();
#pragma unroll
    for (int q = 0; q < kNCol; q++) o[q] = t.v[q];
  }
  if (bad) atomicExch(err, 1);
}

// ------------------------------------------------------------------ rates
// The frequency grid and cross sections of the caller's run_param
// (freq.nu, csect[]; filled by its setup_freq_param / setup_cross_section),
// copied to the device on every call, and the Lyman-Werner bin of the H2
// photo-dissociation term (calc_photoion_rate.c:107-120).
struct DropinTab {
  double nu[kNu];
  double cs[kNChan][kNu];  // the float cross sections, as double
  double dnu_lw;           // width of the LW bin [Hz]
  int lw;                  // LW bin
};

// shielding_func_H2 (prim_chem/cross_section.c:142-161), Wolcott-Green,
// Haiman & Bryan (2011)
__device__ __forceinline__ double shielding_h2(double nh2, double tmpr) {
  const double x = __ddiv_rn(nh2, 5.0e14);
  const double bth = __ddiv_rn(__dmul_rn(0.90854e4, sqrt(tmpr)), 1.0e5);
  const double a = __ddiv_rn(0.965, pow(__dadd_rn(1.0, __ddiv_rn(x, bth)), 1.1));
  const double sx = sqrt(__dadd_rn(1.0, x));
  return __dadd_rn(a, __dmul_rn(__ddiv_rn(0.035, sx), exp(__dmul_rn(-8.5e4, sx))));
}

// The rates of one light ray in the reference's order and precision
// (calc_photoion_rate.c:159-425, FP64 with round-to-nearest single
// operations; only the device exp/pow differ by an ulp from the host's):
// out[k] is the ray's contribution to rate field k of prim_chem (GammaHI
// on), heating already times h nu_L except HeatH2I_II, which the
// reference adds as it is.
__device__ void ray_rates_f64(const GridDev &g, const DropinTab *__restrict__ T, const light_ray_IO &r,
                              const fluid_mesh &m, float anow, double (&out)[kNOut]) {
  using namespace flags;
  const double cd = __dmul_rn(g.lunit, g.denstonh);
  const float *col = r.col();
  double od[kNCol];
#pragma unroll
  for (int q = 0; q < kNCol; q++) od[q] = __dmul_rn((double)col[q], cd);
  const RayGeom geo = ray_geometry(g, r.ix_target, r.iy_target, r.iz_target, r.src.xpos, r.src.ypos, r.src.zpos);
  [[maybe_unused]] float dist2 = geo.dist2;
#ifdef __PHOTON_CONSERVING__
  // per-species densities, the cell's own columns and 1/(n V_shell + TINY)
  double n[kNCol], dd[kNCol], rN[kNCol];
  const double nH = __dmul_rn((double)m.dens, g.denstonh);
  n[0] = __dmul_rn(nH, (double)m.chem.fHI);
#ifdef __HELIUM__
  const double nHe = __dmul_rn(nH, kHeliumFact);
  n[kColHeI] = __dmul_rn(nHe, (double)m.chem.fHeI);
  n[kColHeII] = __dmul_rn(nHe, (double)m.chem.fHeII);
#endif
#ifdef __HYDROGEN_MOL__
  n[kColHM] = __dmul_rn(nH, (double)m.chem.fHM);
  n[kColH2I] = __dmul_rn(nH, (double)m.chem.fH2I);
  n[kColH2II] = __dmul_rn(nH, (double)m.chem.fH2II);
#endif
  const double a = __dadd_rn((double)geo.dist, __dmul_rn(0.5, (double)geo.delta));
  const double b = __dsub_rn((double)geo.dist, __dmul_rn(0.5, (double)geo.delta));
  const double l3 = __dmul_rn(__dmul_rn(g.lunit, g.lunit), g.lunit);
  const double vsh =
      __dmul_rn(__dmul_rn(4.0 * kPi / 3.0, __dsub_rn(__dmul_rn(__dmul_rn(a, a), a), __dmul_rn(__dmul_rn(b, b), b))), l3);
#pragma unroll
  for (int q = 0; q < kNCol; q++) {
    dd[q] = __dmul_rn(__dmul_rn(n[q], (double)geo.delta), g.lunit);
    od[q] = __dsub_rn(od[q], __dmul_rn(0.5, dd[q]));
    rN[q] = __ddiv_rn(1.0, __dadd_rn(__dmul_rn(n[q], vsh), kTiny));
  }
#endif
#ifdef __COSMOLOGICAL__
  {
    const float a2 = __fmul_rn(anow, anow);
#pragma unroll
    for (int q = 0; q < kNCol; q++) od[q] = __ddiv_rn(od[q], (double)a2);
    dist2 = __fmul_rn(dist2, a2);
#ifdef __PHOTON_CONSERVING__
#pragma unroll
    for (int q = 0; q < kNCol; q++) dd[q] = __ddiv_rn(dd[q], (double)a2);
#endif
  }
#else
  (void)anow;
#endif
  double acc[kNOut];
#pragma unroll
  for (int k = 0; k < kNOut; k++) acc[k] = 0.0;
  const double *rate = r.src.photon_rate;
#ifndef __PHOTON_CONSERVING__
  const double geom = __dmul_rn(__dmul_rn(4.0 * kPi, (double)dist2), __dmul_rn(g.lunit, g.lunit));
#endif
  for (int k = 0; k < kNu; k++) {
    const float nu = __double2float_rn(__ldg(T->nu + k));
    const double vn = (double)nu;
    double cs[kNChan];
#pragma unroll
    for (int c = 0; c < kNChan; c++) cs[c] = __ldg(&T->cs[c][k]);
    // channel order: HI, [HeI, HeII], [HM, H2I_I, H2II_I, H2II_II]
    [[maybe_unused]] constexpr int cHM = kHe ? 3 : 1;
    double tau = __dmul_rn(od[0], cs[0]);
#ifdef __HELIUM__
    tau = __dadd_rn(tau, __dmul_rn(od[kColHeI], cs[1]));
    tau = __dadd_rn(tau, __dmul_rn(od[kColHeII], cs[2]));
#endif
#ifdef __HYDROGEN_MOL__
    tau = __dadd_rn(tau, __dmul_rn(od[kColHM], cs[cHM]));
    tau = __dadd_rn(tau, __dmul_rn(od[kColH2I], cs[cHM + 1]));
    tau = __dadd_rn(tau, __dmul_rn(od[kColH2II], cs[cHM + 2]));
    tau = __dadd_rn(tau, __dmul_rn(od[kColH2II], cs[cHM + 3]));
#endif
#ifdef __PHOTON_CONSERVING__
    // photon-conserving branch (calc_photoion_rate.c:327-386)
    double dt[kNChan];
    dt[0] = __dmul_rn(dd[0], cs[0]);
    double dtot = dt[0];
#ifdef __HELIUM__
    dt[1] = __dmul_rn(dd[kColHeI], cs[1]);
    dt[2] = __dmul_rn(dd[kColHeII], cs[2]);
    dtot = __dadd_rn(dtot, __dadd_rn(dt[1], dt[2]));
#endif
#ifdef __HYDROGEN_MOL__
    dt[cHM] = __dmul_rn(dd[kColHM], cs[cHM]);
    dt[cHM + 1] = __dmul_rn(dd[kColH2I], cs[cHM + 1]);
    dt[cHM + 2] = __dmul_rn(dd[kColH2II], cs[cHM + 2]);
    dt[cHM + 3] = __dmul_rn(dd[kColH2II], cs[cHM + 3]);
    dtot = __dadd_rn(dtot, __dadd_rn(__dadd_rn(__dadd_rn(dt[cHM], dt[cHM + 1]), dt[cHM + 2]), dt[cHM + 3]));
#endif
    const double pabs = __dmul_rn(__dmul_rn(__ldg(rate + k), exp(-tau)), __dsub_rn(1.0, exp(-dtot)));
    const double den = __dadd_rn(dtot, kTiny);
    // the share of channel c, its Gamma field, its heating field, the
    // species' 1/(n V), the heating threshold and the subtracted energy
    // (the reference tests H2I_I above 1.144 but subtracts 1.134)
    auto add = [&](int c, int fg, int fh, double rn, double thr, double sub) {
      const double w = __dmul_rn(__ddiv_rn(dt[c], den), pabs);
      acc[fg] = __dadd_rn(acc[fg], __dmul_rn(w, rn));
      if (vn > thr) acc[fh] = __dadd_rn(acc[fh], __dmul_rn(__dmul_rn(w, __dsub_rn(vn, sub)), rn));
    };
    add(0, kOutGHI, kOutHHI, rN[0], 1.0, 1.0);
#ifdef __HELIUM__
    add(1, kOutGHeI, kOutHHeI, rN[kColHeI], 1.8125, 1.8125);
    add(2, kOutGHeII, kOutHHeII, rN[kColHeII], 4.0, 4.0);
#endif
#ifdef __HYDROGEN_MOL__
    add(cHM, kOutGHM, kOutHHM, rN[kColHM], 5.551e-2, 5.551e-2);
    add(cHM + 1, kOutGH2I_I, kOutHH2I_I, rN[kColH2I], 1.144, 1.134);
    add(cHM + 2, kOutGH2II_I, kOutHH2II_I, rN[kColH2II], 0.195, 0.195);
    add(cHM + 3, kOutGH2II_II, kOutHH2II_II, rN[kColH2II], 2.2058, 2.2058);
#endif
#else
    // plain branch (calc_photoion_rate.c:291-326)
    const double flux = __ddiv_rn(__dmul_rn(__ldg(rate + k), exp(-tau)), geom);
    auto add = [&](int c, int fg, int fh, double thr, double sub) {
      acc[fg] = __dadd_rn(acc[fg], __dmul_rn(flux, cs[c]));
      if (vn > thr) acc[fh] = __dadd_rn(acc[fh], __dmul_rn(__dmul_rn(flux, __dsub_rn(vn, sub)), cs[c]));
    };
    add(0, kOutGHI, kOutHHI, 1.0, 1.0);
#ifdef __HELIUM__
    add(1, kOutGHeI, kOutHHeI, 1.8125, 1.8125);
    add(2, kOutGHeII, kOutHHeII, 4.0, 4.0);
#endif
#ifdef __HYDROGEN_MOL__
    add(cHM, kOutGHM, kOutHHM, 5.551e-2, 5.551e-2);
    add(cHM + 1, kOutGH2I_I, kOutHH2I_I, 1.144, 1.134);
    add(cHM + 2, kOutGH2II_I, kOutHH2II_I, 0.195, 0.195);
    add(cHM + 3, kOutGH2II_II, kOutHH2II_II, 2.2058, 2.2058);
#endif
#endif
  }
#ifdef __HYDROGEN_MOL__
  {
    // H2 photo-dissociation in the LW band (calc_photoion_rate.c:391-401)
    constexpr int cHM = kHe ? 3 : 1;
    const int L = T->lw;
    const double tl = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(od[kColHM], __ldg(&T->cs[cHM][L])),
                                                    __dmul_rn(od[kColH2I], __ldg(&T->cs[cHM + 1][L]))),
                                          __dmul_rn(od[kColH2II], __ldg(&T->cs[cHM + 2][L]))),
                                __dmul_rn(od[kColH2II], __ldg(&T->cs[cHM + 3][L])));
    const double geom_lw = __dmul_rn(__dmul_rn(4.0 * kPi, (double)dist2), __dmul_rn(g.lunit, g.lunit));
    const double flux = __ddiv_rn(__dmul_rn(__ldg(rate + L), exp(-tl)), geom_lw);
    const double jnu = __ddiv_rn(__dmul_rn(flux, kHPlanck * (12.87 / 13.6) * kNuL), T->dnu_lw);
    acc[kOutGH2I_II] = __dmul_rn(__dmul_rn(1.13e8, jnu), shielding_h2(od[kColH2I], 1.0e2));
    acc[kOutHH2I_II] = __dmul_rn(6.4e-13, acc[kOutGH2I_II]);
  }
#endif
  // Gamma as it is, heating times h nu_L (HeatH2I_II as it is)
#pragma unroll
  for (int k = 0; k < kNOut; k++) {
    const bool heat = (k == kOutHHI) || (kHe && (k == kOutHHeI || k == kOutHHeII)) ||
                      (kH2 && k >= kOutHHM && k != kOutHH2I_II);
    out[k] = heat ? __dmul_rn(acc[k], kHPlanck * kNuL) : acc[k];
  }
}

// Per-ray rates of the reference's light_ray_IO array (one thread per ray);
// per[kNOut i + k] = field k of ray i (zero for a target outside the mesh).
__global__ void k_rate_rayio(GridDev g, const fluid_mesh *__restrict__ mesh, const light_ray_IO *__restrict__ rays,
                             uint64_t nray, int rank_x, int rank_y, int rank_z, const DropinTab *__restrict__ T,
                             float anow, double *__restrict__ per) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nray;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const light_ray_IO &r = rays[i];
    const int lx = r.ix_target - rank_x * g.nx, ly = r.iy_target - rank_y * g.ny, lz = r.iz_target - rank_z * g.nz;
    double out[kNOut];
#pragma unroll
    for (int k = 0; k < kNOut; k++) out[k] = 0.0;
    if ((unsigned)lx < (unsigned)g.nx && (unsigned)ly < (unsigned)g.ny && (unsigned)lz < (unsigned)g.nz)
      ray_rates_f64(g, T, r, mesh[cell_index(g, lx, ly, lz)], anow, out);
#pragma unroll
    for (int k = 0; k < kNOut; k++) per[kNOut * i + k] = out[k];
  }
}

// Adds per-ray rates into mesh[].prev_chem in ray order.  One thread per run
// of consecutive rays with the same target (the reference emits the rays of
// a cell consecutively); each field is updated with a compare-and-swap so
// that a cell appearing in several runs still receives every contribution,
// with the reference's float += double rounding per ray
// (calc_photoion_rate.c:403-425).  A CAS fails only when another run of the
// same cell has just landed, so the loop ends after at most that many
// retries; past 2^20 of them (more than a million runs of one cell in
// flight) the run's sum is added with one float atomicAdd instead, its
// per-ray float rounding is lost, and the device error flag reports it.
__device__ __forceinline__ void add_run(float *field, const double *per, int k, uint64_t i0, uint64_t i1,
                                        int *err) {
  unsigned int *addr = (unsigned int *)field;
  unsigned int old = *((volatile unsigned int *)addr);
  for (int attempt = 0; attempt < 1 << 20; attempt++) {
    float v = __uint_as_float(old);
    for (uint64_t i = i0; i < i1; i++) v = __double2float_rn(__dadd_rn((double)v, per[kNOut * i + k]));
    const unsigned int prev = atomicCAS(addr, old, __float_as_uint(v));
    if (prev == old) return;
    old = prev;
  }
  double sum = 0.0;
  for (uint64_t i = i0; i < i1; i++) sum += per[kNOut * i + k];
  atomicAdd(field, (float)sum);
  atomicExch(err, 1);
}

__global__ void k_accum_runs(GridDev g, const light_ray_IO *__restrict__ rays, uint64_t nray, int rank_x,
                             int rank_y, int rank_z, const double *__restrict__ per, fluid_mesh *__restrict__ mesh,
                             int *__restrict__ err) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nray;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const int tx = rays[i].ix_target, ty = rays[i].iy_target, tz = rays[i].iz_target;
    if (i > 0 && rays[i - 1].ix_target == tx && rays[i - 1].iy_target == ty && rays[i - 1].iz_target == tz)
      continue;
    uint64_t j = i + 1;
    while (j < nray && rays[j].ix_target == tx && rays[j].iy_target == ty && rays[j].iz_target == tz) j++;
    const int lx = tx - rank_x * g.nx, ly = ty - rank_y * g.ny, lz = tz - rank_z * g.nz;
    if ((unsigned)lx >= (unsigned)g.nx || (unsigned)ly >= (unsigned)g.ny || (unsigned)lz >= (unsigned)g.nz) continue;
    float *f = &mesh[cell_index(g, lx, ly, lz)].prev_chem.GammaHI;
    for (int k = 0; k < kNOut; k++) add_run(f + k, per, k, i, j, err);
  }
}

// zero_out_photoion_rate: every rate field of prev_chem
__global__ void k_zero_rates(uint64_t n, fluid_mesh *__restrict__ mesh) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    float *f = &mesh[i].prev_chem.GammaHI;
#pragma unroll
    for (int k = 0; k < kNOut; k++) f[k] = 0.f;
  }
}

// ------------------------------------------------------------------ smoothing
// The rate fields of prev_chem to and from kNOut planes of ncell floats
// (prim_chem order).
__global__ void __launch_bounds__(256) k_rates_from_mesh(uint64_t n, const fluid_mesh *__restrict__ mesh,
                                                        float *__restrict__ planes) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float *f = &mesh[i].prev_chem.GammaHI;
#pragma unroll
    for (int k = 0; k < kNOut; k++) planes[k * n + i] = f[k];
  }
}
__global__ void __launch_bounds__(256) k_rates_to_mesh(uint64_t n, const float *__restrict__ planes,
                                                      fluid_mesh *__restrict__ mesh) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    float *f = &mesh[i].prev_chem.GammaHI;
#pragma unroll
    for (int k = 0; k < kNOut; k++) f[k] = planes[k * n + i];
  }
}

static int blocks_for(uint64_t n, int threads) { return grid_blocks_for_rates(n, threads); }

namespace dropin_detail {

// Device buffers kept across calls (the reference allocates and frees its
// segment / ray buffers on every call).
struct Pool {
  void *ptr = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t want) {
    if (want <= bytes) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e == cudaSuccess) bytes = want;
    return e;
  }
};

struct DropinState {
  Pool cells;   // packed species densities, kNG float4 per cell
  Pool work[2]; // double-buffered segment / ray chunks
  Pool per;     // per-ray rates, kNOut doubles per ray
  Pool tab;     // frequency grid and cross sections (DropinTab)
  Pool smooth;  // rate planes of the smoothing: 2 kNOut floats per cell
  cudaStream_t lane[2] = {nullptr, nullptr};
  cudaEvent_t ev = nullptr;
  cudaEvent_t rate_done[2] = {nullptr, nullptr};
  cudaEvent_t accum_done[2] = {nullptr, nullptr};
  bool init = false;
};

std::mutex g_mu;
DropinState g_state;
int g_march_mode = -1;
int g_smooth_isolated = 1;

int march_mode() {
  if (g_march_mode < 0) {
    const char *e = std::getenv("ARGOT_B200_MARCH");
    g_march_mode = (e && (!std::strcmp(e, "kahan") || !std::strcmp(e, "1"))) ? ARGOT_B200_PRECISION_KAHAN
                                                                            : ARGOT_B200_PRECISION_REFERENCE;
  }
  return g_march_mode;
}

// The local mesh of run_param as the library's grid; false when its sizes
// or cell widths are not positive.
bool grid_from_run(const run_param *r, GridDev *out) {
  argot_b200_grid g{};
  g.nx = r->nmesh_x_local; g.ny = r->nmesh_y_local; g.nz = r->nmesh_z_local;
  g.ix0 = r->rank_x * r->nmesh_x_local;
  g.iy0 = r->rank_y * r->nmesh_y_local;
  g.iz0 = r->rank_z * r->nmesh_z_local;
  g.xmin = r->xmin; g.ymin = r->ymin; g.zmin = r->zmin;
  g.xmax = r->xmax; g.ymax = r->ymax; g.zmax = r->zmax;
  g.xmin_local = r->xmin_local; g.ymin_local = r->ymin_local; g.zmin_local = r->zmin_local;
  g.dx = r->delta_x; g.dy = r->delta_y; g.dz = r->delta_z;
  g.lunit = r->lunit; g.denstonh = r->denstonh;
  if (!grid_valid(&g)) return false;
  *out = make_grid(g);
  return true;
}

// Makes device 0 current for the call and restores the caller's device.
struct DeviceScope {
  int prev = 0;
  bool ok = false;
  DeviceScope() {
    if (cudaGetDevice(&prev) == cudaSuccess && cudaSetDevice(0) == cudaSuccess) ok = true;
  }
  ~DeviceScope() { cudaSetDevice(prev); }
};

int ensure_state(DropinState &s) {
  if (s.init) return 0;
  for (int i = 0; i < 2; i++) ARGOT_CUDA_TRY(cudaStreamCreateWithFlags(&s.lane[i], cudaStreamNonBlocking));
  ARGOT_CUDA_TRY(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming));
  for (int i = 0; i < 2; i++) {
    ARGOT_CUDA_TRY(cudaEventCreateWithFlags(&s.rate_done[i], cudaEventDisableTiming));
    ARGOT_CUDA_TRY(cudaEventCreateWithFlags(&s.accum_done[i], cudaEventDisableTiming));
  }
  s.init = true;
  return 0;
}

cudaStream_t caller_stream(const cuda_param *c) {
  return (c && c->num_cuda_dev > 0) ? (cudaStream_t)c->strm[0] : (cudaStream_t)0;
}

// lane streams start after the caller's stream's pending work, and the
// caller's stream waits for both lanes at the end
int fork_lanes(DropinState &s, cudaStream_t caller) {
  ARGOT_CUDA_TRY(cudaEventRecord(s.ev, caller));
  for (int i = 0; i < 2; i++) ARGOT_CUDA_TRY(cudaStreamWaitEvent(s.lane[i], s.ev, 0));
  return 0;
}
int join_lanes(DropinState &s, cudaStream_t caller) {
  for (int i = 0; i < 2; i++) {
    ARGOT_CUDA_TRY(cudaEventRecord(s.ev, s.lane[i]));
    ARGOT_CUDA_TRY(cudaStreamWaitEvent(caller, s.ev, 0));
  }
  return 0;
}

int do_march(ray_segment *seg, cuda_mem_space *cm, cuda_param *cp, run_param *run) {
  if (!seg || !cm || !run) return ARGOT_B200_EINVAL;
  const uint64_t nseg = run->nseg;
  GridDev g;
  if (!grid_from_run(run, &g) || !cm[0].mesh_dev) return ARGOT_B200_EINVAL;
  const uint64_t ncell = (uint64_t)g.nx * g.ny * g.nz;
  DeviceScope dscope;
  if (!dscope.ok) return ARGOT_B200_ECUDA;
  std::lock_guard<std::mutex> lock(g_mu);
  DropinState &s = g_state;
  int rc = ensure_state(s);
  if (rc) return rc;
  ARGOT_CUDA_TRY(s.cells.ensure(sizeof(float4) * kNG * ncell));
  int *err = err_flag(0);
  if (!err) return ARGOT_B200_ENOMEM;
  cudaStream_t caller = caller_stream(cp);
  float4 *cells = (float4 *)s.cells.ptr;
  // the mesh may have changed since the last call (send_mesh_data): repack
  k_pack_cols<<<blocks_for(ncell, 256), 256, 0, caller>>>(ncell, cm[0].mesh_dev, cells);
  ARGOT_CUDA_TRY(cudaGetLastError());
  if ((rc = fork_lanes(s, caller))) return rc;
  const uint64_t chunk = 1ull << 20;  // segments per pipelined chunk (56 MB)
  for (int i = 0; i < 2; i++) ARGOT_CUDA_TRY(s.work[i].ensure(sizeof(ray_segment) * std::min(chunk, std::max<uint64_t>(nseg, 1))));
  const int mode = march_mode();
  for (uint64_t c0 = 0, k = 0; c0 < nseg; c0 += chunk, k++) {
    const uint64_t n = std::min(chunk, nseg - c0);
    cudaStream_t st = s.lane[k & 1];
    void *dbuf = s.work[k & 1].ptr;
    ARGOT_CUDA_TRY(cudaMemcpyAsync(dbuf, seg + c0, sizeof(ray_segment) * n, cudaMemcpyHostToDevice, st));
    if (mode == ARGOT_B200_PRECISION_REFERENCE)
      k_march_aos<ARGOT_B200_PRECISION_REFERENCE>
          <<<blocks_for(n, 128), 128, 0, st>>>(g, cells, n, (ray_segment *)dbuf, err);
    else
      k_march_aos<ARGOT_B200_PRECISION_KAHAN><<<blocks_for(n, 128), 128, 0, st>>>(g, cells, n, (ray_segment *)dbuf, err);
    ARGOT_CUDA_TRY(cudaGetLastError());
    ARGOT_CUDA_TRY(cudaMemcpyAsync(seg + c0, dbuf, sizeof(ray_segment) * n, cudaMemcpyDeviceToHost, st));
  }
  if ((rc = join_lanes(s, caller))) return rc;
  ARGOT_CUDA_TRY(cudaStreamSynchronize(caller));
  return check_err_flag(err, caller);
}

// The caller's frequency grid and cross sections, and (with H2) the LW bin:
// the bin whose edges nu / 10^(dlog_nu / 2), nu 10^(dlog_nu / 2) enclose
// 12.87 eV, the last one if several do (calc_photoion_rate.c:107-120, whose
// asserts become ARGOT_B200_EINVAL).
int fill_tables(const run_param *run, DropinTab *t) {
  for (int k = 0; k < kNu; k++) {
    t->nu[k] = run->freq.nu[k];
    const float *c = &run->csect[k].csect_HI;
    for (int q = 0; q < kNChan; q++) t->cs[q][k] = (double)c[q];
  }
  t->lw = 0;
  t->dnu_lw = 1.0;
  if (flags::kH2) {
    const double nu_lw = 12.87 / 13.6;
    int lw = -1;
    double dnu = 0.0;
    for (int k = 0; k < kNu - 1; k++) {
      const double f = std::pow(10.0, 0.5 * run->freq.dlog_nu);
      const double lo = run->freq.nu[k] / f, hi = run->freq.nu[k] * f;
      if (lo < nu_lw && hi > nu_lw) {
        lw = k;
        dnu = (hi - lo) * kNuL;
      }
    }
    if (lw < 0 || lw >= kNu - 2) return ARGOT_B200_EINVAL;
    t->lw = lw;
    t->dnu_lw = dnu;
  }
  return 0;
}

void fill_ray_io(const light_ray *ray, light_ray_IO *io, uint64_t nray) {
  auto work = [&](uint64_t a, uint64_t b) {
    for (uint64_t i = a; i < b; i++) {
      std::memcpy(&io[i].src, &ray[i].src, sizeof(radiation_src));
      io[i].ix_target = ray[i].ix_target;
      io[i].iy_target = ray[i].iy_target;
      io[i].iz_target = ray[i].iz_target;
      for (int q = 0; q < kNCol; q++) io[i].col()[q] = ray[i].col()[q];
    }
  };
  const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  if (nray < 65536 || hw == 1) { work(0, nray); return; }
  std::vector<std::thread> th;
  const uint64_t per = (nray + hw - 1) / hw;
  for (unsigned t = 0; t < hw; t++) {
    const uint64_t a = t * per, b = std::min(nray, a + per);
    if (a < b) th.emplace_back(work, a, b);
  }
  for (auto &x : th) x.join();
}

int do_rates(cuda_mem_space *cm, light_ray *ray, light_ray_IO *ray_io, cuda_param *cp, run_param *run) {
  if (!cm || !run || (run->nray && (!ray || !ray_io))) return ARGOT_B200_EINVAL;
  const uint64_t nray = run->nray;
  GridDev g;
  if (!grid_from_run(run, &g) || !cm[0].mesh_dev) return ARGOT_B200_EINVAL;
  DeviceScope dscope;
  if (!dscope.ok) return ARGOT_B200_ECUDA;
  std::lock_guard<std::mutex> lock(g_mu);
  DropinState &s = g_state;
  int rc = ensure_state(s);
  if (rc) return rc;
  DropinTab tab;
  if ((rc = fill_tables(run, &tab))) return rc;
  fill_ray_io(ray, ray_io, nray);
  int *err = err_flag(0);
  if (!err) return ARGOT_B200_ENOMEM;
  cudaStream_t caller = caller_stream(cp);
  ARGOT_CUDA_TRY(s.tab.ensure(sizeof(DropinTab)));
  const DropinTab *tab_dev = (const DropinTab *)s.tab.ptr;
  ARGOT_CUDA_TRY(cudaMemcpyAsync(s.tab.ptr, &tab, sizeof(DropinTab), cudaMemcpyHostToDevice, caller));
  const uint64_t chunk = 1ull << 15;  // rays per chunk (69 MB of light_ray_IO)
  const uint64_t cn = std::min(chunk, std::max<uint64_t>(nray, 1));
  for (int i = 0; i < 2; i++) ARGOT_CUDA_TRY(s.work[i].ensure(sizeof(light_ray_IO) * cn));
  ARGOT_CUDA_TRY(s.per.ensure(2 * kNOut * sizeof(double) * cn));
  // Copies and per-ray rates of consecutive chunks alternate between two
  // lanes; the accumulation into the mesh runs on the caller's stream, chunk
  // after chunk, so the rays of a cell are added in ray order.
  if ((rc = fork_lanes(s, caller))) return rc;
  for (uint64_t c0 = 0, k = 0; c0 < nray; c0 += chunk, k++) {
    const uint64_t n = std::min(chunk, nray - c0);
    const int bi = (int)(k & 1);
    cudaStream_t st = s.lane[bi];
    void *dbuf = s.work[bi].ptr;
    double *per = (double *)s.per.ptr + bi * kNOut * cn;
    if (k >= 2) ARGOT_CUDA_TRY(cudaStreamWaitEvent(st, s.accum_done[bi], 0));
    ARGOT_CUDA_TRY(cudaMemcpyAsync(dbuf, ray_io + c0, sizeof(light_ray_IO) * n, cudaMemcpyHostToDevice, st));
    k_rate_rayio<<<blocks_for(n, 128), 128, 0, st>>>(g, cm[0].mesh_dev, (const light_ray_IO *)dbuf, n,
                                                      run->rank_x, run->rank_y, run->rank_z, tab_dev, run->anow,
                                                      per);
    ARGOT_CUDA_TRY(cudaGetLastError());
    ARGOT_CUDA_TRY(cudaEventRecord(s.rate_done[bi], st));
    ARGOT_CUDA_TRY(cudaStreamWaitEvent(caller, s.rate_done[bi], 0));
    k_accum_runs<<<blocks_for(n, 128), 128, 0, caller>>>(g, (const light_ray_IO *)dbuf, n, run->rank_x,
                                                          run->rank_y, run->rank_z, per, cm[0].mesh_dev, err);
    ARGOT_CUDA_TRY(cudaGetLastError());
    ARGOT_CUDA_TRY(cudaEventRecord(s.accum_done[bi], caller));
  }
  if ((rc = join_lanes(s, caller))) return rc;
  ARGOT_CUDA_TRY(cudaStreamSynchronize(caller));
  return check_err_flag(err, caller);
}

// smooth_photoion_rate with __USE_GPU__ on one rank
// (src/smooth_photoion_rate.c:27-1588): the reference copies the rates of
// mesh_dev to the host (recv_photoion_data), smooths them there, copies the
// result back into mesh_dev (send_photoion_data) and into the host mesh.
// Here the smoothing runs on mesh_dev in place; only the host copy of the
// result crosses PCIe.
int do_smooth(fluid_mesh *mesh, run_param *run, cuda_mem_space *cm, cuda_param *cp) {
  if (!cm || !run || !cm[0].mesh_dev) return ARGOT_B200_EINVAL;
  const int nx = run->nmesh_x_local, ny = run->nmesh_y_local, nz = run->nmesh_z_local;
  if (nx <= 0 || ny <= 0 || nz <= 0) return ARGOT_B200_EINVAL;
  const uint64_t ncell = (uint64_t)nx * ny * nz;
  if (ncell >= (1ull << 32)) return ARGOT_B200_EINVAL;
  DeviceScope dscope;
  if (!dscope.ok) return ARGOT_B200_ECUDA;
  std::lock_guard<std::mutex> lock(g_mu);
  DropinState &s = g_state;
  int rc = ensure_state(s);
  if (rc) return rc;
  ARGOT_CUDA_TRY(s.smooth.ensure(2 * kNOut * sizeof(float) * ncell));
  cudaStream_t caller = caller_stream(cp);
  float *work = (float *)s.smooth.ptr;
  // mesh -> planes (work), smoothed planes (work + kNOut ncell), -> mesh
  const int nb = blocks_for(ncell, 256);
  k_rates_from_mesh<<<nb, 256, 0, caller>>>(ncell, cm[0].mesh_dev, work);
  ARGOT_CUDA_TRY(cudaGetLastError());
  if ((rc = launch_smooth_planes(nx, ny, nz, work, work + kNOut * ncell, kNOut, g_smooth_isolated, caller)))
    return rc;
  k_rates_to_mesh<<<nb, 256, 0, caller>>>(ncell, work + kNOut * ncell, cm[0].mesh_dev);
  ARGOT_CUDA_TRY(cudaGetLastError());
  if (mesh) {
    std::vector<float> host(kNOut * ncell);
    ARGOT_CUDA_TRY(cudaMemcpyAsync(host.data(), work + kNOut * ncell, kNOut * sizeof(float) * ncell,
                                   cudaMemcpyDeviceToHost, caller));
    ARGOT_CUDA_TRY(cudaStreamSynchronize(caller));
    auto scatter = [&](uint64_t a, uint64_t b) {
      for (uint64_t i = a; i < b; i++) {
        float *f = &mesh[i].prev_chem.GammaHI;
        for (int k = 0; k < kNOut; k++) f[k] = host[k * ncell + i];
      }
    };
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (ncell < 65536 || hw == 1) {
      scatter(0, ncell);
      return 0;
    }
    std::vector<std::thread> th;
    const uint64_t per = (ncell + hw - 1) / hw;
    for (unsigned t = 0; t < hw; t++) {
      const uint64_t a = t * per, b = std::min(ncell, a + per);
      if (a < b) th.emplace_back(scatter, a, b);
    }
    for (auto &x : th) x.join();
    return 0;
  }
  ARGOT_CUDA_TRY(cudaStreamSynchronize(caller));
  return 0;
}

}  // namespace dropin_detail
using namespace dropin_detail;

void dropin_status(const run_param *run, const char *entry, int rc) {
  set_status(rc);
  if (rc && run && run->proc_file) {
    std::fprintf(run->proc_file, "# argot_b200 %s: %s (%d)\n", entry, argot_b200_error_string(rc), rc);
    std::fflush(run->proc_file);
  }
}
}  // namespace argot

using argot::set_status;

extern "C" {

int argot_b200_set_dropin_march_mode(int mode) {
  if (mode != ARGOT_B200_MARCH_REFERENCE && mode != ARGOT_B200_MARCH_KAHAN) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  argot::g_march_mode =
      mode == ARGOT_B200_MARCH_KAHAN ? ARGOT_B200_PRECISION_KAHAN : ARGOT_B200_PRECISION_REFERENCE;
  set_status(0);
  return 0;
}

int argot_b200_set_dropin_smooth_faces(int faces) {
  if (faces != ARGOT_B200_FACES_PERIODIC && faces != ARGOT_B200_FACES_ISOLATED) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  argot::g_smooth_isolated = faces == ARGOT_B200_FACES_ISOLATED;
  set_status(0);
  return 0;
}

void smooth_photoion_rate(::fluid_mesh *mesh, ::run_param *this_run, ::cuda_mem_space *cuda_mem,
                          ::cuda_param *this_cuda, struct mpi_param *this_mpi) {
  (void)this_mpi;
  argot::dropin_status((argot::run_param *)this_run, "smooth_photoion_rate",
                       argot::do_smooth((argot::fluid_mesh *)mesh, (argot::run_param *)this_run,
                                        (argot::cuda_mem_space *)cuda_mem, (argot::cuda_param *)this_cuda));
}

void calc_optical_depth_cuda(::ray_segment *seg, ::cuda_mem_space *cuda_mem,
                             struct cuda_param *this_cuda, ::run_param *this_run) {
  argot::dropin_status((argot::run_param *)this_run, "calc_optical_depth_cuda",
                       argot::do_march((argot::ray_segment *)seg, (argot::cuda_mem_space *)cuda_mem,
                                       (argot::cuda_param *)this_cuda, (argot::run_param *)this_run));
}

void calc_photoion_rate_cuda(::cuda_mem_space *cuda_mem, ::light_ray *ray, ::light_ray_IO *ray_IO,
                             struct cuda_param *this_cuda, ::run_param *this_run) {
  argot::dropin_status((argot::run_param *)this_run, "calc_photoion_rate_cuda",
                       argot::do_rates((argot::cuda_mem_space *)cuda_mem, (argot::light_ray *)ray,
                                       (argot::light_ray_IO *)ray_IO, (argot::cuda_param *)this_cuda,
                                       (argot::run_param *)this_run));
}

void zero_out_photoion_rate_cuda(::cuda_mem_space *cuda_mem, ::cuda_param *this_cuda,
                                 struct run_param *this_run) {
  argot::cuda_mem_space *cm = (argot::cuda_mem_space *)cuda_mem;
  argot::run_param *run = (argot::run_param *)this_run;
  if (!cm || !run || !cm[0].mesh_dev || run->nmesh_x_local <= 0 || run->nmesh_y_local <= 0 ||
      run->nmesh_z_local <= 0) {
    argot::dropin_status(run, "zero_out_photoion_rate_cuda", ARGOT_B200_EINVAL);
    return;
  }
  const uint64_t n = (uint64_t)run->nmesh_x_local * run->nmesh_y_local * run->nmesh_z_local;
  argot::DeviceScope dscope;
  if (!dscope.ok) { argot::dropin_status(run, "zero_out_photoion_rate_cuda", ARGOT_B200_ECUDA); return; }
  cudaStream_t st = argot::caller_stream((argot::cuda_param *)this_cuda);
  argot::k_zero_rates<<<argot::blocks_for(n, 256), 256, 0, st>>>(n, cm[0].mesh_dev);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  const int rc = e == cudaSuccess ? 0 : argot::status_from_cuda(e);
  argot::dropin_status(run, "zero_out_photoion_rate_cuda", rc);
}

// One rank: the send buffer of accum_optical_depth.c:59-104 is the only
// contribution, so each ray's columns are those of the (single) segment
// that carries its index; rays without a segment get zero.
void accum_optical_depth(::light_ray *ray_, ::ray_segment *seg_, ::run_param *run_,
                         struct omp_param *omp) {
  (void)omp;
  argot::light_ray *ray = (argot::light_ray *)ray_;
  argot::ray_segment *seg = (argot::ray_segment *)seg_;
  argot::run_param *run = (argot::run_param *)run_;
  if (!run || (run->nray && !ray) || (run->nseg && !seg)) { set_status(ARGOT_B200_EINVAL); return; }
  constexpr int nc = argot::flags::kNCol;
  std::vector<float> send(nc * run->nray, 0.f);
  for (uint64_t i = 0; i < run->nseg; i++) {
    if (seg[i].target_rank != run->mpi_rank) continue;
    const uint64_t r = seg[i].ray_indx;
    if (r >= run->nray) continue;
    for (int q = 0; q < nc; q++) send[nc * r + q] = seg[i].col()[q];
  }
  for (uint64_t r = 0; r < run->nray; r++)
    for (int q = 0; q < nc; q++) ray[r].col()[q] = 0.f + send[nc * r + q];
  set_status(0);
}

}  // extern "C"

// ---- device API pieces tied to the struct layouts ----------------------
namespace argot {
#ifdef ARGOT_HELIUM_LAYOUT
// The device path's packed fields from a struct fluid_mesh array:
// cells[c] = {n_HI, n_HeI, n_HeII, 0} as k_pack_cols forms them and
// raw[c] = {dens, fHI, fHeI, fHeII} for the rate stage.
__global__ void k_pack_mesh_he(uint64_t n, const fluid_mesh *__restrict__ mesh, float4 *__restrict__ cells,
                               float4 *__restrict__ raw) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float d = mesh[i].dens, a = mesh[i].chem.fHI, b = mesh[i].chem.fHeI, c = mesh[i].chem.fHeII;
    const float nhe = __double2float_rn(__dmul_rn((double)d, kHeliumFact));
    cells[i] = make_float4(__fmul_rn(d, a), __fmul_rn(nhe, b), __fmul_rn(nhe, c), 0.f);
    raw[i] = make_float4(d, a, b, c);
  }
}
#endif
}  // namespace argot

extern "C" {

const char *argot_b200_flagset(void) { return argot::flags::kName; }

int argot_b200_pack_fluid_mesh(const argot_b200_grid *gp, const void *mesh_dev, void *packed_dev, void *stream) {
  if (!argot::grid_valid(gp) || !mesh_dev || !packed_dev) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
#ifdef ARGOT_HELIUM_LAYOUT
  const uint64_t n = (uint64_t)gp->nx * gp->ny * gp->nz;
  float4 *cells = (float4 *)packed_dev;
  argot::k_pack_mesh_he<<<argot::blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
      n, (const argot::fluid_mesh *)mesh_dev, cells, cells + n);
  const cudaError_t e = cudaGetLastError();
  const int rc = e == cudaSuccess ? 0 : argot::status_from_cuda(e);
  set_status(rc);
  return rc;
#else
  (void)stream;
  set_status(ARGOT_B200_ENOTSUP);
  return ARGOT_B200_ENOTSUP;
#endif
}

}  // extern "C"
