// ref_layout.h -- byte-identical mirrors of the ARGOT structs that cross the
// drop-in boundary, for the reference's default flag set:
//   -D__HELIUM__ -D__PHOTON_CONSERVING__, no __HYDROGEN_MOL__,
//   NGRID_NU = 256 (run_param.h:78), NSEG_PER_RAY = 5 (run_param.h:60),
//   NMAX_CUDA_DEV = 4 (run_param.h:141, GPU builds).
// Field order and types follow the reference headers; the sizes and offsets
// asserted below were measured from the reference compiled with gcc on
// x86-64 (and are re-checked by the test suite against that build).
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstddef>

namespace argot {

constexpr int kNGridNu = 256;
constexpr int kNSegPerRay = 5;
constexpr int kNMaxCudaDev = 4;

// src/prim_chem/chemistry.h:41-63
struct prim_chem {
  float wmol, felec;
  float fHI, fHII;
  float fHeI, fHeII, fHeIII;
  float GammaHI, HeatHI;
  float GammaHeI, GammaHeII;
  float HeatHeI, HeatHeII;
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
  float GammaHI, HeatHI, GammaHeI, GammaHeII, HeatHeI, HeatHeII;
};
struct ray_segment {
  uint64_t ray_indx;
  int local_rank, target_rank;
  float xpos_start, ypos_start, zpos_start;
  float xpos_end, ypos_end, zpos_end;
  float optical_depth_HI, optical_depth_HeI, optical_depth_HeII;
};
struct light_ray {
  radiation_src src;
  int num_segment;
  ray_segment segment[kNSegPerRay];
  int ix_target, iy_target, iz_target;
  float optical_depth_HI, optical_depth_HeI, optical_depth_HeII;
};
struct light_ray_IO {
  radiation_src src;
  int ix_target, iy_target, iz_target;
  float optical_depth_HI, optical_depth_HeI, optical_depth_HeII;
};

// src/cross_section.h:7-20, src/cosmology.h:9-12
struct cross_section {
  float csect_HI, csect_HeI, csect_HeII;
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
static_assert(sizeof(prim_chem) == 52, "prim_chem layout");
static_assert(sizeof(fluid_mesh) == 156, "fluid_mesh layout");
static_assert(offsetof(fluid_mesh, chem) == 44, "fluid_mesh.chem");
static_assert(offsetof(fluid_mesh, prev_chem) == 96, "fluid_mesh.prev_chem");
static_assert(offsetof(prim_chem, fHI) == 8, "prim_chem.fHI");
static_assert(offsetof(prim_chem, fHeI) == 16, "prim_chem.fHeI");
static_assert(offsetof(prim_chem, GammaHI) == 28, "prim_chem.GammaHI");
static_assert(offsetof(prim_chem, HeatHeII) == 48, "prim_chem.HeatHeII");
static_assert(sizeof(radiation_src) == 2072, "radiation_src layout");
static_assert(offsetof(radiation_src, photon_rate) == 24, "radiation_src.photon_rate");
static_assert(sizeof(ray_segment) == 56, "ray_segment layout");
static_assert(offsetof(ray_segment, xpos_start) == 16, "ray_segment.xpos_start");
static_assert(offsetof(ray_segment, optical_depth_HI) == 40, "ray_segment.optical_depth_HI");
static_assert(sizeof(light_ray) == 2384, "light_ray layout");
static_assert(offsetof(light_ray, num_segment) == 2072, "light_ray.num_segment");
static_assert(offsetof(light_ray, segment) == 2080, "light_ray.segment");
static_assert(offsetof(light_ray, ix_target) == 2360, "light_ray.ix_target");
static_assert(offsetof(light_ray, optical_depth_HI) == 2372, "light_ray.optical_depth_HI");
static_assert(sizeof(light_ray_IO) == 2096, "light_ray_IO layout");
static_assert(offsetof(light_ray_IO, ix_target) == 2072, "light_ray_IO.ix_target");
static_assert(offsetof(light_ray_IO, optical_depth_HI) == 2084, "light_ray_IO.optical_depth_HI");
static_assert(sizeof(cross_section) == 12, "cross_section layout");
static_assert(sizeof(freq_param) == 2072, "freq_param layout");
static_assert(sizeof(photoion_rate) == 24, "photoion_rate layout");
static_assert(sizeof(run_param) == 5480, "run_param layout");
static_assert(offsetof(run_param, lunit) == 80, "run_param.lunit");
static_assert(offsetof(run_param, denstonh) == 112, "run_param.denstonh");
static_assert(offsetof(run_param, anow) == 136, "run_param.anow");
static_assert(offsetof(run_param, freq) == 184, "run_param.freq");
static_assert(offsetof(run_param, csect) == 2256, "run_param.csect");
static_assert(offsetof(run_param, nsrc) == 5360, "run_param.nsrc");
static_assert(offsetof(run_param, nseg) == 5376, "run_param.nseg");
static_assert(offsetof(run_param, xmin) == 5384, "run_param.xmin");
static_assert(offsetof(run_param, xmin_local) == 5408, "run_param.xmin_local");
static_assert(offsetof(run_param, nmesh_x_total) == 5432, "run_param.nmesh_x_total");
static_assert(offsetof(run_param, nmesh_x_local) == 5444, "run_param.nmesh_x_local");
static_assert(offsetof(run_param, delta_x) == 5456, "run_param.delta_x");
static_assert(offsetof(run_param, theta_crit) == 5468, "run_param.theta_crit");
static_assert(offsetof(run_param, nmesh_per_loop) == 5472, "run_param.nmesh_per_loop");
static_assert(offsetof(run_param, rank_x) == 56, "run_param.rank_x");
static_assert(sizeof(cuda_param) == 88, "cuda_param layout");
static_assert(sizeof(cuda_mem_space) == 88, "cuda_mem_space layout");

}  // namespace argot
