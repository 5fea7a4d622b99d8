// ref_layout.h -- byte-identical mirrors of the ARGOT structs that cross the
// drop-in boundary, with the reference's own flag macros (flagset.h):
// __HELIUM__ and __HYDROGEN_MOL__ add fields exactly where the reference
// headers do; NGRID_NU = 256 (run_param.h:78), NSEG_PER_RAY = 5
// (run_param.h:60), NMAX_CUDA_DEV = 4 (run_param.h:141, GPU builds).
// Field order and types follow the reference headers; the sizes and offsets
// asserted below were measured from the reference headers compiled with gcc
// on x86-64 for each flag set (and are re-checked by the test suite against
// the reference built with those flags).
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstddef>

#include "flagset.h"

namespace argot {

constexpr int kNGridNu = 256;
constexpr int kNSegPerRay = 5;
constexpr int kNMaxCudaDev = 4;

// src/prim_chem/chemistry.h:41-63
struct prim_chem {
  float wmol, felec;
  float fHI, fHII;
#ifdef __HYDROGEN_MOL__
  float fH2I, fH2II, fHM;
#endif
#ifdef __HELIUM__
  float fHeI, fHeII, fHeIII;
#endif
  float GammaHI, HeatHI;
#ifdef __HELIUM__
  float GammaHeI, GammaHeII;
  float HeatHeI, HeatHeII;
#endif
#ifdef __HYDROGEN_MOL__
  float GammaHM, GammaH2I_I, GammaH2I_II, GammaH2II_I, GammaH2II_II;
  float HeatHM, HeatH2I_I, HeatH2I_II, HeatH2II_I, HeatH2II_II;
#endif
};

// src/fluid.h:101-116
struct fluid_mesh {
  float dens, eneg, momx, momy, momz;
  float uene, duene, durad, etrp, pot, dens_prev;
  prim_chem chem;
  prim_chem prev_chem;
  float prev_uene;
  short under_shock, high_mach;
};

// src/source.h:6-16
struct freq_param {
  double log_nu_min, log_nu_max, dlog_nu;
  double nu[kNGridNu];
};
struct radiation_src {
  int type;
  float param;
  float xpos, ypos, zpos;
  double photon_rate[kNGridNu];
};

// src/radiation.h:10-83
struct photoion_rate {
  float GammaHI, HeatHI;
#ifdef __HELIUM__
  float GammaHeI, GammaHeII, HeatHeI, HeatHeII;
#endif
#ifdef __HYDROGEN_MOL__
  float GammaHM, GammaH2I_I, GammaH2I_II, GammaH2II_I, GammaH2II_II;
  float HeatHM, HeatH2I_I, HeatH2I_II, HeatH2II_I, HeatH2II_II;
#endif
};
// The columns of a segment or ray, in the reference's order; as an array
// through col(): HI, [HeI, HeII], [HM, H2I, H2II] (flags::kNCol floats).
#ifdef __HELIUM__
#define ARGOT_HE_COLUMNS float optical_depth_HeI, optical_depth_HeII;
#else
#define ARGOT_HE_COLUMNS
#endif
#ifdef __HYDROGEN_MOL__
#define ARGOT_H2_COLUMNS float optical_depth_HM, optical_depth_H2I, optical_depth_H2II;
#else
#define ARGOT_H2_COLUMNS
#endif
struct ray_segment {
  uint64_t ray_indx;
  int local_rank, target_rank;
  float xpos_start, ypos_start, zpos_start;
  float xpos_end, ypos_end, zpos_end;
  float optical_depth_HI;
  ARGOT_HE_COLUMNS
  ARGOT_H2_COLUMNS
  __host__ __device__ float *col() { return &optical_depth_HI; }
  __host__ __device__ const float *col() const { return &optical_depth_HI; }
};
struct light_ray {
  radiation_src src;
  int num_segment;
  ray_segment segment[kNSegPerRay];
  int ix_target, iy_target, iz_target;
  float optical_depth_HI;
  ARGOT_HE_COLUMNS
  ARGOT_H2_COLUMNS
  const float *col() const { return &optical_depth_HI; }
  float *col() { return &optical_depth_HI; }
};
struct light_ray_IO {
  radiation_src src;
  int ix_target, iy_target, iz_target;
  float optical_depth_HI;
  ARGOT_HE_COLUMNS
  ARGOT_H2_COLUMNS
  __host__ __device__ const float *col() const { return &optical_depth_HI; }
  __host__ __device__ float *col() { return &optical_depth_HI; }
};
#undef ARGOT_HE_COLUMNS
#undef ARGOT_H2_COLUMNS

// src/cross_section.h:7-20, src/cosmology.h:9-12
struct cross_section {
  float csect_HI;
#ifdef __HELIUM__
  float csect_HeI, csect_HeII;
#endif
#ifdef __HYDROGEN_MOL__
  float csect_HM, csect_H2I_I, csect_H2II_I, csect_H2II_II;
#endif
};
struct cosmology {
  float omega_m, omega_v, omega_b, omega_nu, hubble, tend;
};

// src/run_param.h:171-235
struct run_param {
  char *model_name;
  FILE *proc_file, *diag_file, *err_file;
  int helium_flag, hydrogen_mol_flag, cosmology_flag, ngrid_nu;
  int mpi_rank, mpi_nproc;
  int rank_x, rank_y, rank_z;
  int nnode_x, nnode_y, nnode_z;
  double lunit, munit, tunit, eunit;
  double denstonh, uenetok, masstonh;
  float anow, tnow, znow, hnow;
  cosmology cosm;
  float tend, dtime;
  freq_param freq;
  cross_section csect[kNGridNu];
  int nspecies, nchannel, step, output_indx, noutput;
  float *output_timing;
  uint64_t nsrc, nray, nseg;
  float xmin, ymin, zmin, xmax, ymax, zmax;
  float xmin_local, ymin_local, zmin_local, xmax_local, ymax_local, zmax_local;
  int nmesh_x_total, nmesh_y_total, nmesh_z_total;
  int nmesh_x_local, nmesh_y_local, nmesh_z_local;
  float delta_x, delta_y, delta_z;
  float theta_crit;
  int nmesh_per_loop;
};

// src/cuda_mem_space.h:14-39 (cudaStream_t is a 64-bit handle)
struct cuda_param {
  int num_cuda_dev, nmesh_per_dev, cuda_nblock, max_thread_dimx, max_block_dimx;
  int64_t strm[kNMaxCudaDev];
  int64_t diffuse_strm[kNMaxCudaDev];
};
struct cuda_mem_space {
  fluid_mesh *mesh_dev;
  run_param *this_run_dev;
  freq_param *freq_dev;
  ray_segment *segment_dev;
  photoion_rate *rate_dev;
  prim_chem *chem_updated;
  light_ray_IO *ray_IO_dev;
  float *optical_depth_dev, *dtime_dev, *diff_chem_dev, *diff_uene_dev;
};

// src/diffuse_photon/diffuse_photon.h:76-79,130-154 (GPU build: the host
// parameters carry no radiation mesh)
struct angle_info {
  float xovr, yovr, zovr;
  short base_id, corner_id;
};
struct step_func_factor {
  float HI[2], HeI[2], HeII[2];
};
struct host_diffuse_param {
  int corner_id_num[8];
  step_func_factor *step_fact;
  angle_info *angle;
};

// Records a drop-in entry point's status for argot_b200_last_error and, on
// failure, writes one line to the caller's run->proc_file (the reference's
// log) when it has one.
void dropin_status(const run_param *run, const char *entry, int rc);

static_assert(sizeof(angle_info) == 16, "angle_info layout");
static_assert(sizeof(step_func_factor) == 24, "step_func_factor layout");
static_assert(sizeof(host_diffuse_param) == 48, "host_diffuse_param layout");
static_assert(sizeof(radiation_src) == 2072, "radiation_src layout");
static_assert(offsetof(radiation_src, photon_rate) == 24, "radiation_src.photon_rate");
static_assert(sizeof(freq_param) == 2072, "freq_param layout");
static_assert(offsetof(fluid_mesh, chem) == 44, "fluid_mesh.chem");
static_assert(offsetof(prim_chem, fHI) == 8, "prim_chem.fHI");
static_assert(offsetof(ray_segment, xpos_start) == 16, "ray_segment.xpos_start");
static_assert(offsetof(ray_segment, optical_depth_HI) == 40, "ray_segment.optical_depth_HI");
static_assert(offsetof(light_ray, num_segment) == 2072, "light_ray.num_segment");
static_assert(offsetof(light_ray, segment) == 2080, "light_ray.segment");
static_assert(offsetof(light_ray_IO, ix_target) == 2072, "light_ray_IO.ix_target");
static_assert(offsetof(light_ray_IO, optical_depth_HI) == 2084, "light_ray_IO.optical_depth_HI");
static_assert(offsetof(run_param, lunit) == 80, "run_param.lunit");
static_assert(offsetof(run_param, denstonh) == 112, "run_param.denstonh");
static_assert(offsetof(run_param, anow) == 136, "run_param.anow");
static_assert(offsetof(run_param, freq) == 184, "run_param.freq");
static_assert(offsetof(run_param, csect) == 2256, "run_param.csect");
static_assert(offsetof(run_param, rank_x) == 56, "run_param.rank_x");
static_assert(sizeof(cuda_param) == 88, "cuda_param layout");
static_assert(sizeof(cuda_mem_space) == 88, "cuda_mem_space layout");
// the rate fields of prim_chem are consecutive floats from GammaHI on
static_assert(sizeof(prim_chem) == offsetof(prim_chem, GammaHI) + 4 * flags::kNOut, "prim_chem rate fields");
static_assert(sizeof(cross_section) == 4 * flags::kNChan, "cross_section channels");
static_assert(offsetof(ray_segment, optical_depth_HI) + 4 * flags::kNCol <= sizeof(ray_segment), "columns");

// Per flag set (sizes measured from the reference headers with gcc, x86-64):
//   set            ray_segment light_ray light_ray_IO prim_chem fluid_mesh run_param
//   He             56          2384      2096         52        156        5480
//   H2             56          2392      2104         76        204        7528
//   He + H2        64          2440      2112         104       260        9576
//   neither        48          2336      2088         24        100        3432
#if defined(__HELIUM__) && !defined(__HYDROGEN_MOL__)
static_assert(sizeof(prim_chem) == 52 && sizeof(fluid_mesh) == 156 && offsetof(fluid_mesh, prev_chem) == 96,
              "prim_chem / fluid_mesh layout (helium)");
static_assert(offsetof(prim_chem, fHeI) == 16 && offsetof(prim_chem, GammaHI) == 28 &&
                  offsetof(prim_chem, HeatHeII) == 48,
              "prim_chem offsets (helium)");
static_assert(sizeof(ray_segment) == 56 && sizeof(light_ray) == 2384 && sizeof(light_ray_IO) == 2096,
              "ray layouts (helium)");
static_assert(offsetof(light_ray, ix_target) == 2360 && offsetof(light_ray, optical_depth_HI) == 2372,
              "light_ray offsets (helium)");
static_assert(sizeof(cross_section) == 12 && sizeof(photoion_rate) == 24, "tables (helium)");
static_assert(sizeof(run_param) == 5480 && offsetof(run_param, nsrc) == 5360 && offsetof(run_param, nseg) == 5376 &&
                  offsetof(run_param, xmin) == 5384 && offsetof(run_param, xmin_local) == 5408 &&
                  offsetof(run_param, nmesh_x_total) == 5432 && offsetof(run_param, nmesh_x_local) == 5444 &&
                  offsetof(run_param, delta_x) == 5456 && offsetof(run_param, theta_crit) == 5468 &&
                  offsetof(run_param, nmesh_per_loop) == 5472,
              "run_param layout (helium)");
#elif !defined(__HELIUM__) && defined(__HYDROGEN_MOL__)
static_assert(sizeof(prim_chem) == 76 && sizeof(fluid_mesh) == 204 && offsetof(fluid_mesh, prev_chem) == 120 &&
                  offsetof(prim_chem, GammaHI) == 28,
              "prim_chem / fluid_mesh layout (H2)");
static_assert(sizeof(ray_segment) == 56 && sizeof(light_ray) == 2392 && sizeof(light_ray_IO) == 2104 &&
                  offsetof(light_ray, ix_target) == 2360 && offsetof(light_ray, optical_depth_HI) == 2372,
              "ray layouts (H2)");
static_assert(sizeof(cross_section) == 20 && sizeof(photoion_rate) == 48 && sizeof(run_param) == 7528 &&
                  offsetof(run_param, nseg) == 7424 && offsetof(run_param, nmesh_x_local) == 7492 &&
                  offsetof(run_param, delta_x) == 7504,
              "tables / run_param (H2)");
#elif defined(__HELIUM__) && defined(__HYDROGEN_MOL__)
static_assert(sizeof(prim_chem) == 104 && sizeof(fluid_mesh) == 260 && offsetof(fluid_mesh, prev_chem) == 148 &&
                  offsetof(prim_chem, GammaHI) == 40,
              "prim_chem / fluid_mesh layout (helium + H2)");
static_assert(sizeof(ray_segment) == 64 && sizeof(light_ray) == 2440 && sizeof(light_ray_IO) == 2112 &&
                  offsetof(light_ray, ix_target) == 2400 && offsetof(light_ray, optical_depth_HI) == 2412,
              "ray layouts (helium + H2)");
static_assert(sizeof(cross_section) == 28 && sizeof(photoion_rate) == 64 && sizeof(run_param) == 9576 &&
                  offsetof(run_param, nseg) == 9472 && offsetof(run_param, nmesh_x_local) == 9540 &&
                  offsetof(run_param, delta_x) == 9552,
              "tables / run_param (helium + H2)");
#else
static_assert(sizeof(prim_chem) == 24 && sizeof(fluid_mesh) == 100 && offsetof(fluid_mesh, prev_chem) == 68 &&
                  offsetof(prim_chem, GammaHI) == 16,
              "prim_chem / fluid_mesh layout (hydrogen only)");
static_assert(sizeof(ray_segment) == 48 && sizeof(light_ray) == 2336 && sizeof(light_ray_IO) == 2088 &&
                  offsetof(light_ray, ix_target) == 2320 && offsetof(light_ray, optical_depth_HI) == 2332,
              "ray layouts (hydrogen only)");
static_assert(sizeof(cross_section) == 4 && sizeof(photoion_rate) == 8 && sizeof(run_param) == 3432 &&
                  offsetof(run_param, nseg) == 3328 && offsetof(run_param, nmesh_x_local) == 3396 &&
                  offsetof(run_param, delta_x) == 3408,
              "tables / run_param (hydrogen only)");
#endif

}  // namespace argot
