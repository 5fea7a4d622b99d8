/*
 * ref_gpu_driver.cu -- test-infrastructure glue that runs ARGOT's OWN GPU
 * entry points on a B200: calc_optical_depth_cuda, calc_photoion_rate_cuda
 * and zero_out_photoion_rate_cuda (src/calc_optical_depth_cuda.cu,
 * src/calc_photoion_rate_cuda.cu) and the pinned allocators of
 * src/allocate_pinned_segment.cu, compiled unmodified for sm_100a with the
 * reference Makefile's nvcc flags (src/Makefile:208: -use_fast_math -O3) by
 * oracle/build.py into oracle/_ref/libargot_refgpu_n<EDGE>.so, together with
 * the CPU reference and ref_driver.c.  Only bench.py's reference-GPU
 * baseline and tests/ load it.
 *
 * refgpu_run_range follows calc_ARGOT_part (src/step_radiation_tree.c:
 * 214-309) for the groups of a range of target cells: the reference's tree
 * builds the rays on the host, then calc_optical_depth_cuda,
 * accum_optical_depth and calc_photoion_rate_cuda run as ARGOT runs them,
 * each timed by the wall clock (what one call costs: its allocations,
 * copies and kernels).  A second, kernel-only pass launches the two
 * reference kernels themselves with the reference's launch geometry on
 * device-resident copies of the same segments and rays, timed with CUDA
 * events on the launching stream.  The same loop can call another
 * library's functions of the same signatures instead (a drop-in
 * replacement) for a like-for-like timing.  No arithmetic of the path lives
 * here.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <sys/time.h>

#include <cuda_runtime.h>

#include "run_param.h"
#include "constants.h"
#include "fluid.h"
#include "radiation.h"
#include "cuda_mem_space.h"

extern "C" {
void calc_optical_depth_cuda(struct ray_segment *, struct cuda_mem_space *, struct cuda_param *,
                             struct run_param *);
void calc_photoion_rate_cuda(struct cuda_mem_space *, struct light_ray *, struct light_ray_IO *,
                             struct cuda_param *, struct run_param *);
void zero_out_photoion_rate_cuda(struct cuda_mem_space *, struct cuda_param *, struct run_param *);
void allocate_pinned_segment(struct ray_segment **, uint64_t);
void deallocate_pinned_segment(struct ray_segment *);
void allocate_pinned_light_ray_IO(struct light_ray_IO **, uint64_t);
void deallocate_pinned_light_ray_IO(struct light_ray_IO *);

int ref_next_group(int im, int im_end, uint64_t *nray);
int64_t ref_setup_group(int im, int ge, struct light_ray *ray, uint64_t nray);
void ref_assign_group(struct light_ray *ray, struct ray_segment *seg);
void ref_accum_group(struct light_ray *ray, struct ray_segment *seg);
struct run_param *ref_run_param(void);
struct fluid_mesh *ref_mesh(void);
}

/* the reference's kernels (defined in its .cu files, launched here with its
 * own launch geometry for the kernel-only timing) */
__global__ void calc_optical_depth_kernel(const struct fluid_mesh *__restrict__, struct ray_segment *,
                                          const struct run_param *__restrict__, uint64_t);
__global__ void calc_photoion_rate_kernel(struct fluid_mesh *, const struct light_ray_IO *__restrict__,
                                          const struct run_param *__restrict__, uint64_t);

/* the march and rate entry points the group loop calls: the reference's
 * own by default, or another library's functions with the same signatures
 * (refgpu_use_entry_points), so that ARGOT's loop can be timed with a
 * drop-in replacement linked in */
typedef void (*march_fn)(struct ray_segment *, struct cuda_mem_space *, struct cuda_param *, struct run_param *);
typedef void (*rates_fn)(struct cuda_mem_space *, struct light_ray *, struct light_ray_IO *, struct cuda_param *,
                         struct run_param *);
static march_fn g_march = calc_optical_depth_cuda;
static rates_fn g_rates = calc_photoion_rate_cuda;

extern "C" void refgpu_use_entry_points(void *march, void *rates) {
  g_march = march ? (march_fn)march : calc_optical_depth_cuda;
  g_rates = rates ? (rates_fn)rates : calc_photoion_rate_cuda;
}

static struct cuda_param g_cp;
static struct cuda_mem_space g_cm[NMAX_CUDA_DEV];
static struct fluid_mesh *g_scratch_mesh = NULL;  /* target of the kernel-only rate pass */
static cudaStream_t g_stream = NULL;
static int g_ready = 0;

static double now_s(void) {
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return (double)tv.tv_sec + 1.0e-6 * (double)tv.tv_usec;
}

#define REFGPU_TRY(x)                      \
  do {                                     \
    cudaError_t e_ = (x);                  \
    if (e_ != cudaSuccess) return -(int)e_ - 1000; \
  } while (0)

extern "C" int refgpu_edge(void) { return NMESH_X_LOCAL; }

/* One device, as init_gpu (src/init_gpu.cu:40-140) sets it up for one rank,
 * and the mesh and run parameters copied to it as send_mesh_data /
 * send_run_param_data do.  Call after ref_init / ref_set_mesh /
 * ref_set_sources; call again after the mesh changes. */
extern "C" int refgpu_init(void) {
  if (!g_ready) {
    REFGPU_TRY(cudaSetDevice(0));
    memset(&g_cp, 0, sizeof(g_cp));
    memset(g_cm, 0, sizeof(g_cm));
    cudaDeviceProp prop;
    REFGPU_TRY(cudaGetDeviceProperties(&prop, 0));
    g_cp.num_cuda_dev = 1;
    g_cp.cuda_nblock = NMESH_LOCAL / NMESH_PER_BLOCK;
    g_cp.nmesh_per_dev = NMESH_LOCAL;
    g_cp.max_thread_dimx = prop.maxThreadsDim[0];
    g_cp.max_block_dimx = prop.maxGridSize[0];
    REFGPU_TRY(cudaStreamCreate(&g_stream));
    g_cp.strm[0] = g_stream;
    REFGPU_TRY(cudaMalloc((void **)&g_cm[0].mesh_dev, sizeof(struct fluid_mesh) * NMESH_LOCAL));
    REFGPU_TRY(cudaMalloc((void **)&g_cm[0].this_run_dev, sizeof(struct run_param)));
    REFGPU_TRY(cudaMalloc((void **)&g_scratch_mesh, sizeof(struct fluid_mesh) * NMESH_LOCAL));
    g_ready = 1;
  }
  REFGPU_TRY(cudaMemcpy(g_cm[0].mesh_dev, ref_mesh(), sizeof(struct fluid_mesh) * NMESH_LOCAL,
                        cudaMemcpyHostToDevice));
  REFGPU_TRY(cudaMemcpy(g_scratch_mesh, ref_mesh(), sizeof(struct fluid_mesh) * NMESH_LOCAL,
                        cudaMemcpyHostToDevice));
  REFGPU_TRY(cudaMemcpy(g_cm[0].this_run_dev, ref_run_param(), sizeof(struct run_param),
                        cudaMemcpyHostToDevice));
  return 0;
}

extern "C" void refgpu_free(void) {
  if (!g_ready) return;
  cudaFree(g_cm[0].mesh_dev);
  cudaFree(g_cm[0].this_run_dev);
  cudaFree(g_scratch_mesh);
  cudaStreamDestroy(g_stream);
  g_ready = 0;
}

extern "C" int refgpu_zero_rates(void) {
  if (!g_ready) return -1;
  zero_out_photoion_rate_cuda(g_cm, &g_cp, ref_run_param());
  REFGPU_TRY(cudaGetLastError());
  return 0;
}

/* the six rate planes (Gamma HI, HeI, HeII, heat HI, HeI, HeII) of mesh_dev */
extern "C" int refgpu_get_rates(float *out6) {
  if (!g_ready) return -1;
  struct fluid_mesh *h = (struct fluid_mesh *)malloc(sizeof(struct fluid_mesh) * NMESH_LOCAL);
  if (!h) return -2;
  cudaError_t e = cudaMemcpy(h, g_cm[0].mesh_dev, sizeof(struct fluid_mesh) * NMESH_LOCAL,
                             cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) { free(h); return -(int)e - 1000; }
  const uint64_t n = (uint64_t)NMESH_LOCAL;
  for (uint64_t i = 0; i < n; i++) {
    out6[0 * n + i] = h[i].prev_chem.GammaHI;
    out6[1 * n + i] = h[i].prev_chem.GammaHeI;
    out6[2 * n + i] = h[i].prev_chem.GammaHeII;
    out6[3 * n + i] = h[i].prev_chem.HeatHI;
    out6[4 * n + i] = h[i].prev_chem.HeatHeI;
    out6[5 * n + i] = h[i].prev_chem.HeatHeII;
  }
  free(h);
  return 0;
}

/* Kernel-only passes: the reference's launch loops
 * (calc_optical_depth_cuda.cu:84-113, calc_photoion_rate_cuda.cu:151-187)
 * over device copies, bracketed by CUDA events on the launching stream. */
static int time_march_kernel(const struct ray_segment *seg, uint64_t nseg, int reps, double *ms) {
  struct ray_segment *d = NULL;
  REFGPU_TRY(cudaMalloc((void **)&d, sizeof(struct ray_segment) * nseg));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaMemcpyAsync(d, seg, sizeof(struct ray_segment) * nseg, cudaMemcpyHostToDevice, g_stream);
  float total = 0.f;
  for (int r = 0; r < reps; r++) {
    cudaEventRecord(a, g_stream);
    uint64_t waiting = nseg, offset = 0;
    while (waiting > 0) {
      uint64_t nthread, nblock;
      if (waiting >= NSEG_MAX_PER_DEV) {
        nthread = NSEG_MAX_PER_BLOCK;
        nblock = NSEG_MAX_PER_DEV / NSEG_MAX_PER_BLOCK;
      } else if (waiting >= NSEG_MAX_PER_BLOCK) {
        nthread = NSEG_MAX_PER_BLOCK;
        nblock = waiting / NSEG_MAX_PER_BLOCK;
      } else {
        nthread = waiting;
        nblock = 1;
      }
      calc_optical_depth_kernel<<<(unsigned)nblock, (unsigned)nthread, 0, g_stream>>>(
          g_cm[0].mesh_dev, d, g_cm[0].this_run_dev, offset);
      waiting -= nthread * nblock;
      offset += nthread * nblock;
    }
    cudaEventRecord(b, g_stream);
    cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    total += t;
  }
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(d);
  if (e != cudaSuccess) return -(int)e - 1000;
  *ms += total / reps;
  return 0;
}

static int time_rate_kernel(const struct light_ray_IO *io, uint64_t nray, int reps, double *ms) {
  struct light_ray_IO *d = NULL;
  REFGPU_TRY(cudaMalloc((void **)&d, sizeof(struct light_ray_IO) * nray));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaMemcpyAsync(d, io, sizeof(struct light_ray_IO) * nray, cudaMemcpyHostToDevice, g_stream);
  float total = 0.f;
  for (int r = 0; r < reps; r++) {
    cudaEventRecord(a, g_stream);
    uint64_t waiting = nray, offset = 0;
    while (waiting > 0) {
      uint64_t nthread, nblock;
      if (waiting >= NMESH_PER_BLOCK) {
        nthread = NMESH_PER_BLOCK;
        nblock = waiting / NMESH_PER_BLOCK;
      } else {
        nthread = waiting;
        nblock = 1;
      }
      calc_photoion_rate_kernel<<<(unsigned)nblock, (unsigned)nthread, 0, g_stream>>>(
          g_scratch_mesh, d, g_cm[0].this_run_dev, offset);
      waiting -= nthread * nblock;
      offset += nthread * nblock;
    }
    cudaEventRecord(b, g_stream);
    cudaEventSynchronize(b);
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    total += t;
  }
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(d);
  if (e != cudaSuccess) return -(int)e - 1000;
  *ms += total / reps;
  return 0;
}

/*
 * The reference's GPU path over target cells [im_start, im_end) of the
 * current mesh and sources, group by group as calc_ARGOT_part runs it.
 * Rates accumulate into mesh_dev (refgpu_zero_rates first, refgpu_get_rates
 * after).  seg6 (optional, 6 floats per segment in the reference's order:
 * start xyz, end xyz) and tau3 (optional, the stitched columns per ray)
 * receive the group outputs; cap bounds them (segments, rays).  out[10]:
 *   0 rays, 1 segments, 2 setup wall s (tree walk, segment assignment,
 *   pinned allocations), 3 calc_optical_depth_cuda wall s,
 *   4 accum_optical_depth wall s, 5 calc_photoion_rate_cuda wall s,
 *   6 march kernel ms, 7 rate kernel ms (kernel-only passes, mean over
 *   reps), 8 groups.
 * Returns 0, or a negative code.
 */
extern "C" int refgpu_run_range(int im_start, int im_end, int kernel_reps, float *seg6, float *tau3, uint64_t cap,
                                double *out) {
  if (!g_ready) return -1;
  for (int i = 0; i < 10; i++) out[i] = 0.0;
  struct run_param *run = ref_run_param();
  struct light_ray *ray = NULL;
  uint64_t ray_cap = 0, nray_total = 0, nseg_total = 0;
  int im = im_start;
  while (im < im_end) {
    uint64_t nray = 0;
    const int ge = ref_next_group(im, im_end, &nray);
    if (nray > ray_cap) {
      free(ray);
      ray = (struct light_ray *)malloc(sizeof(struct light_ray) * (size_t)nray);
      if (!ray) return -2;
      ray_cap = nray;
    }
    const double t0 = now_s();
    const int64_t nseg = ref_setup_group(im, ge, ray, nray);
    if (nseg < 0) { free(ray); return -3; }
    struct ray_segment *seg = NULL;
    struct light_ray_IO *io = NULL;
    allocate_pinned_segment(&seg, (uint64_t)(nseg ? nseg : 1));
    allocate_pinned_light_ray_IO(&io, nray ? nray : 1);
    if (!seg || !io) { free(ray); return -4; }
    ref_assign_group(ray, seg);
    const double t1 = now_s();
    if (seg6) {
      for (int64_t k = 0; k < nseg && nseg_total + (uint64_t)k < cap; k++) {
        float *o = seg6 + 6 * (nseg_total + (uint64_t)k);
        o[0] = seg[k].xpos_start; o[1] = seg[k].ypos_start; o[2] = seg[k].zpos_start;
        o[3] = seg[k].xpos_end; o[4] = seg[k].ypos_end; o[5] = seg[k].zpos_end;
      }
    }
    g_march(seg, g_cm, &g_cp, run);
    const double t2 = now_s();
    ref_accum_group(ray, seg);
    const double t3 = now_s();
    g_rates(g_cm, ray, io, &g_cp, run);
    const double t4 = now_s();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { free(ray); return -(int)e - 1000; }
    out[2] += t1 - t0; out[3] += t2 - t1; out[4] += t3 - t2; out[5] += t4 - t3;
    if (tau3) {
      for (uint64_t r = 0; r < nray && nray_total + r < cap; r++) {
        float *o = tau3 + 3 * (nray_total + r);
        o[0] = ray[r].optical_depth_HI; o[1] = ray[r].optical_depth_HeI; o[2] = ray[r].optical_depth_HeII;
      }
    }
    if (kernel_reps > 0) {
      int rc = time_march_kernel(seg, (uint64_t)nseg, kernel_reps, &out[6]);
      if (!rc) rc = time_rate_kernel(io, nray, kernel_reps, &out[7]);
      if (rc) { free(ray); return rc; }
    }
    deallocate_pinned_segment(seg);
    deallocate_pinned_light_ray_IO(io);
    nray_total += nray;
    nseg_total += (uint64_t)nseg;
    out[8] += 1.0;
    im = ge;
  }
  free(ray);
  out[0] = (double)nray_total;
  out[1] = (double)nseg_total;
  return 0;
}
