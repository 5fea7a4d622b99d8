// dropin.cu -- the reference's own entry points (src/prototype.h:47,89,93,
// 124-125) on one GPU, for argot_mpi / argot_hydro_mpi to link in place of
// calc_optical_depth_cuda.o, calc_photoion_rate_cuda.o,
// accum_optical_depth.o and smooth_photoion_rate.o on a single rank.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "common.cuh"
#include "ref_layout.h"

namespace argot {

int launch_march_aos(const GridDev &g, const float4 *cells, uint64_t nseg, void *seg_dev, int prec, int *err_dev,
                     cudaStream_t st);
int launch_pack_mesh(uint64_t n, const void *mesh, float4 *cells, float4 *raw, cudaStream_t st);
int launch_rate_rayio(const GridDev &g, const float4 *raw, const void *rays_io, uint64_t nray, int rx, int ry,
                      int rz, double *per6, cudaStream_t st);
int launch_accum_runs(const GridDev &g, const void *rays_io, uint64_t nray, int rx, int ry, int rz,
                      const double *per6, void *mesh, int *err, cudaStream_t st);
int launch_zero_rates(uint64_t n, void *mesh, cudaStream_t st);
int launch_smooth_mesh(int nx, int ny, int nz, void *mesh, float *work, int isolated, cudaStream_t st);
int *err_flag(int dev);
int check_err_flag(int *flag, cudaStream_t st);

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
  Pool cells;   // packed fields: cells + raw, 32 B per cell
  Pool work[2]; // double-buffered segment / ray chunks
  Pool per6;    // per-ray rates
  Pool smooth;  // rate planes of the smoothing: 12 floats per cell
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
  ARGOT_CUDA_TRY(s.cells.ensure(32 * ncell));
  int *err = err_flag(0);
  if (!err) return ARGOT_B200_ENOMEM;
  cudaStream_t caller = caller_stream(cp);
  float4 *cells = (float4 *)s.cells.ptr;
  // the mesh may have changed since the last call (send_mesh_data): repack
  rc = launch_pack_mesh(ncell, cm[0].mesh_dev, cells, cells + ncell, caller);
  if (rc) return rc;
  if ((rc = fork_lanes(s, caller))) return rc;
  const uint64_t chunk = 1ull << 20;  // segments per pipelined chunk (56 MB)
  for (int i = 0; i < 2; i++) ARGOT_CUDA_TRY(s.work[i].ensure(sizeof(ray_segment) * std::min(chunk, std::max<uint64_t>(nseg, 1))));
  const int mode = march_mode();
  for (uint64_t c0 = 0, k = 0; c0 < nseg; c0 += chunk, k++) {
    const uint64_t n = std::min(chunk, nseg - c0);
    cudaStream_t st = s.lane[k & 1];
    void *dbuf = s.work[k & 1].ptr;
    ARGOT_CUDA_TRY(cudaMemcpyAsync(dbuf, seg + c0, sizeof(ray_segment) * n, cudaMemcpyHostToDevice, st));
    if ((rc = launch_march_aos(g, cells, n, dbuf, mode, err, st))) return rc;
    ARGOT_CUDA_TRY(cudaMemcpyAsync(seg + c0, dbuf, sizeof(ray_segment) * n, cudaMemcpyDeviceToHost, st));
  }
  if ((rc = join_lanes(s, caller))) return rc;
  ARGOT_CUDA_TRY(cudaStreamSynchronize(caller));
  return check_err_flag(err, caller);
}

void fill_ray_io(const light_ray *ray, light_ray_IO *io, uint64_t nray) {
  auto work = [&](uint64_t a, uint64_t b) {
    for (uint64_t i = a; i < b; i++) {
      std::memcpy(&io[i].src, &ray[i].src, sizeof(radiation_src));
      io[i].ix_target = ray[i].ix_target;
      io[i].iy_target = ray[i].iy_target;
      io[i].iz_target = ray[i].iz_target;
      io[i].optical_depth_HI = ray[i].optical_depth_HI;
      io[i].optical_depth_HeI = ray[i].optical_depth_HeI;
      io[i].optical_depth_HeII = ray[i].optical_depth_HeII;
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
  const uint64_t ncell = (uint64_t)g.nx * g.ny * g.nz;
  DeviceScope dscope;
  if (!dscope.ok) return ARGOT_B200_ECUDA;
  std::lock_guard<std::mutex> lock(g_mu);
  DropinState &s = g_state;
  int rc = ensure_state(s);
  if (rc) return rc;
  if ((rc = ensure_tables(0))) return rc;
  fill_ray_io(ray, ray_io, nray);
  ARGOT_CUDA_TRY(s.cells.ensure(32 * ncell));
  int *err = err_flag(0);
  if (!err) return ARGOT_B200_ENOMEM;
  cudaStream_t caller = caller_stream(cp);
  float4 *cells = (float4 *)s.cells.ptr;
  if ((rc = launch_pack_mesh(ncell, cm[0].mesh_dev, cells, cells + ncell, caller))) return rc;
  const uint64_t chunk = 1ull << 15;  // rays per chunk (69 MB of light_ray_IO)
  const uint64_t cn = std::min(chunk, std::max<uint64_t>(nray, 1));
  for (int i = 0; i < 2; i++) ARGOT_CUDA_TRY(s.work[i].ensure(sizeof(light_ray_IO) * cn));
  ARGOT_CUDA_TRY(s.per6.ensure(2 * 6 * sizeof(double) * cn));
  // Copies and per-ray rates of consecutive chunks alternate between two
  // lanes; the accumulation into the mesh runs on the caller's stream, chunk
  // after chunk, so the rays of a cell are added in ray order.
  if ((rc = fork_lanes(s, caller))) return rc;
  for (uint64_t c0 = 0, k = 0; c0 < nray; c0 += chunk, k++) {
    const uint64_t n = std::min(chunk, nray - c0);
    const int bi = (int)(k & 1);
    cudaStream_t st = s.lane[bi];
    void *dbuf = s.work[bi].ptr;
    double *per = (double *)s.per6.ptr + bi * 6 * cn;
    if (k >= 2) ARGOT_CUDA_TRY(cudaStreamWaitEvent(st, s.accum_done[bi], 0));
    ARGOT_CUDA_TRY(cudaMemcpyAsync(dbuf, ray_io + c0, sizeof(light_ray_IO) * n, cudaMemcpyHostToDevice, st));
    if ((rc = launch_rate_rayio(g, cells + ncell, dbuf, n, run->rank_x, run->rank_y, run->rank_z, per, st)))
      return rc;
    ARGOT_CUDA_TRY(cudaEventRecord(s.rate_done[bi], st));
    ARGOT_CUDA_TRY(cudaStreamWaitEvent(caller, s.rate_done[bi], 0));
    if ((rc = launch_accum_runs(g, dbuf, n, run->rank_x, run->rank_y, run->rank_z, per, cm[0].mesh_dev, err,
                                caller)))
      return rc;
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
  ARGOT_CUDA_TRY(s.smooth.ensure(12 * sizeof(float) * ncell));
  cudaStream_t caller = caller_stream(cp);
  float *work = (float *)s.smooth.ptr;
  if ((rc = launch_smooth_mesh(nx, ny, nz, cm[0].mesh_dev, work, g_smooth_isolated, caller))) return rc;
  if (mesh) {
    std::vector<float> host(6 * ncell);
    ARGOT_CUDA_TRY(cudaMemcpyAsync(host.data(), work + 6 * ncell, 6 * sizeof(float) * ncell,
                                   cudaMemcpyDeviceToHost, caller));
    ARGOT_CUDA_TRY(cudaStreamSynchronize(caller));
    auto scatter = [&](uint64_t a, uint64_t b) {
      for (uint64_t i = a; i < b; i++) {
        prim_chem &pc = mesh[i].prev_chem;
        pc.GammaHI = host[0 * ncell + i];
        pc.GammaHeI = host[1 * ncell + i];
        pc.GammaHeII = host[2 * ncell + i];
        pc.HeatHI = host[3 * ncell + i];
        pc.HeatHeI = host[4 * ncell + i];
        pc.HeatHeII = host[5 * ncell + i];
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
  int rc = argot::launch_zero_rates(n, cm[0].mesh_dev, st);
  if (!rc) {
    cudaError_t e = cudaStreamSynchronize(st);
    rc = e == cudaSuccess ? 0 : argot::status_from_cuda(e);
  }
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
  std::vector<float> send(3 * run->nray, 0.f);
  for (uint64_t i = 0; i < run->nseg; i++) {
    if (seg[i].target_rank != run->mpi_rank) continue;
    const uint64_t r = seg[i].ray_indx;
    if (r >= run->nray) continue;
    send[3 * r + 0] = seg[i].optical_depth_HI;
    send[3 * r + 1] = seg[i].optical_depth_HeI;
    send[3 * r + 2] = seg[i].optical_depth_HeII;
  }
  for (uint64_t r = 0; r < run->nray; r++) {
    ray[r].optical_depth_HI = 0.f + send[3 * r + 0];
    ray[r].optical_depth_HeI = 0.f + send[3 * r + 1];
    ray[r].optical_depth_HeII = 0.f + send[3 * r + 2];
  }
  set_status(0);
}

}  // extern "C"
