/*
 * ref_driver.c -- test-infrastructure driver around ARGOT's OWN hot-path C
 * code (the "O1" parity oracle).  It is compiled together with the
 * reference sources, unmodified, by oracle/build_ref.py, into
 * oracle/_ref/libargot_ref_n<EDGE>.so (one library per mesh edge, because
 * the reference fixes the mesh size at compile time).  Only tests/, the
 * smoke check and bench.py's CPU-baseline / reference arm load it.
 *
 * Everything here is glue: it fills the reference's own structs from flat
 * arrays and calls the reference's functions in the order the reference's
 * driver calc_ARGOT_part uses (step_radiation_tree.c:214-309):
 *   setup_light_ray_range (setup_light_ray_tree.c:397)
 *   count_ray_segment / assign_ray_segment (assign_ray_segment.c:22,106)
 *   calc_optical_depth (calc_optical_depth.c:20)
 *   accum_optical_depth (accum_optical_depth.c:14)
 *   calc_photoion_rate (calc_photoion_rate.c:93)
 * No arithmetic of the hot path lives in this file.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <sys/time.h>
#include <omp.h>

#include "run_param.h"
#include "constants.h"
#include "fluid.h"
#include "radiation.h"
#include "source.h"
#include "cross_section.h"
#include "prototype.h"
#include "tree_clist.h"
#include "mpi_param.h"
#include "omp_param.h"
#include "diffuse_photon.h"
#include "diffuse_prototype.h"

static struct run_param g_run;
static struct fluid_mesh *g_mesh = NULL;
static struct radiation_src *g_src = NULL;
static struct clist_t *g_clist = NULL;
static uint64_t *g_key = NULL;
static int *g_index = NULL;
static struct mpi_param g_mpi;
static struct omp_param g_omp;
static int g_have_tree = 0;

static double now_s(void)
{
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return (double)tv.tv_sec + 1.0e-6 * (double)tv.tv_usec;
}

int ref_mesh_edge(void) { return NMESH_X_LOCAL; }

/* sizes of the reference structs under the flags this library was built
 * with; the test suite compares them with include/argot_b200.h */
void ref_struct_sizes(uint64_t *out)
{
  out[0] = sizeof(struct ray_segment);
  out[1] = sizeof(struct light_ray);
  out[2] = sizeof(struct light_ray_IO);
  out[3] = sizeof(struct radiation_src);
  out[4] = sizeof(struct fluid_mesh);
  out[5] = sizeof(struct prim_chem);
  out[6] = sizeof(struct run_param);
  out[7] = sizeof(struct cross_section);
  out[8] = sizeof(struct freq_param);
  out[9] = sizeof(struct photoion_rate);
}

/* byte offsets of the fields the hot path touches */
void ref_struct_offsets(uint64_t *out)
{
  int i = 0;
  out[i++] = offsetof(struct ray_segment, ray_indx);
  out[i++] = offsetof(struct ray_segment, xpos_start);
  out[i++] = offsetof(struct ray_segment, optical_depth_HI);
  out[i++] = offsetof(struct light_ray, num_segment);
  out[i++] = offsetof(struct light_ray, segment);
  out[i++] = offsetof(struct light_ray, ix_target);
  out[i++] = offsetof(struct light_ray, optical_depth_HI);
  out[i++] = offsetof(struct light_ray_IO, ix_target);
  out[i++] = offsetof(struct light_ray_IO, optical_depth_HI);
  out[i++] = offsetof(struct radiation_src, photon_rate);
  out[i++] = offsetof(struct fluid_mesh, chem);
  out[i++] = offsetof(struct fluid_mesh, prev_chem);
  out[i++] = offsetof(struct prim_chem, fHI);
  out[i++] = offsetof(struct prim_chem, fHeI);
  out[i++] = offsetof(struct prim_chem, GammaHI);
  out[i++] = offsetof(struct prim_chem, HeatHeII);
  out[i++] = offsetof(struct run_param, lunit);
  out[i++] = offsetof(struct run_param, denstonh);
  out[i++] = offsetof(struct run_param, freq);
  out[i++] = offsetof(struct run_param, csect);
  out[i++] = offsetof(struct run_param, nsrc);
  out[i++] = offsetof(struct run_param, nray);
  out[i++] = offsetof(struct run_param, nseg);
  out[i++] = offsetof(struct run_param, xmin);
  out[i++] = offsetof(struct run_param, xmin_local);
  out[i++] = offsetof(struct run_param, nmesh_x_total);
  out[i++] = offsetof(struct run_param, nmesh_x_local);
  out[i++] = offsetof(struct run_param, delta_x);
  out[i++] = offsetof(struct run_param, theta_crit);
  out[i++] = offsetof(struct run_param, nmesh_per_loop);
  out[i++] = offsetof(struct run_param, rank_x);
  out[i++] = offsetof(struct run_param, anow);
}

/* Fill run_param for a single rank covering the unit box [0,1)^3, the way
 * the reference's IC generators do (test_IC/cmpproj_test2_IC.c:51-75) and
 * init_run does for the tables (init_run.c:93). */
int ref_init(double lunit, double denstonh, float theta_crit, int nthreads)
{
  memset(&g_run, 0, sizeof(g_run));
  g_run.proc_file = fopen("/dev/null", "w");
  g_run.diag_file = g_run.proc_file;
  g_run.err_file = g_run.proc_file;
  g_run.helium_flag = 1;
  g_run.ngrid_nu = NGRID_NU;
  g_run.mpi_rank = 0;
  g_run.mpi_nproc = 1;
  g_run.nnode_x = g_run.nnode_y = g_run.nnode_z = 1;
  g_run.lunit = lunit;
  g_run.denstonh = denstonh;
  g_run.anow = 1.0f;
  g_run.nspecies = NSPECIES;
  g_run.nchannel = NCHANNEL;
  g_run.xmin = g_run.ymin = g_run.zmin = 0.0f;
  g_run.xmax = g_run.ymax = g_run.zmax = 1.0f;
  g_run.xmin_local = g_run.ymin_local = g_run.zmin_local = 0.0f;
  g_run.xmax_local = g_run.ymax_local = g_run.zmax_local = 1.0f;
  g_run.nmesh_x_total = NMESH_X_TOTAL;
  g_run.nmesh_y_total = NMESH_Y_TOTAL;
  g_run.nmesh_z_total = NMESH_Z_TOTAL;
  g_run.nmesh_x_local = NMESH_X_LOCAL;
  g_run.nmesh_y_local = NMESH_Y_LOCAL;
  g_run.nmesh_z_local = NMESH_Z_LOCAL;
  g_run.delta_x = (g_run.xmax - g_run.xmin) / (float)g_run.nmesh_x_total;
  g_run.delta_y = (g_run.ymax - g_run.ymin) / (float)g_run.nmesh_y_total;
  g_run.delta_z = (g_run.zmax - g_run.zmin) / (float)g_run.nmesh_z_total;
  g_run.theta_crit = theta_crit;
  g_run.nmesh_per_loop = NMESH_LOCAL;
  setup_freq_param(&g_run.freq);
  setup_cross_section(g_run.csect, &g_run.freq);
  g_run.rank_x = g_run.rank_y = g_run.rank_z = 0;
  g_mpi.photoion_rate_type = ARGOT_SHIM_SIZED_TYPE(sizeof(struct photoion_rate));
  omp_init_nest_lock(&g_omp.omp_lock);
  if (nthreads > 0) omp_set_num_threads(nthreads);
  if (!g_mesh) g_mesh = (struct fluid_mesh *)calloc(NMESH_LOCAL, sizeof(struct fluid_mesh));
  return g_mesh ? 0 : -1;
}

void ref_set_threads(int nthreads) { if (nthreads > 0) omp_set_num_threads(nthreads); }

void ref_tables(double *nu, float *csect3, double *freq_meta3)
{
  for (int i = 0; i < NGRID_NU; i++) {
    nu[i] = g_run.freq.nu[i];
    csect3[3 * i + 0] = g_run.csect[i].csect_HI;
    csect3[3 * i + 1] = g_run.csect[i].csect_HeI;
    csect3[3 * i + 2] = g_run.csect[i].csect_HeII;
  }
  freq_meta3[0] = g_run.freq.log_nu_min;
  freq_meta3[1] = g_run.freq.log_nu_max;
  freq_meta3[2] = g_run.freq.dlog_nu;
}

void ref_photon_rate(int type, float param, double total_rate, double *out)
{
  struct radiation_src s;
  memset(&s, 0, sizeof(s));
  s.type = type;
  s.param = param;
  setup_photon_rate(&g_run.freq, &s, total_rate);
  memcpy(out, s.photon_rate, sizeof(double) * NGRID_NU);
}

void ref_set_mesh(const float *dens, const float *fHI, const float *fHeI,
                  const float *fHeII)
{
  for (uint64_t i = 0; i < (uint64_t)NMESH_LOCAL; i++) {
    memset(&g_mesh[i], 0, sizeof(struct fluid_mesh));
    g_mesh[i].dens = dens[i];
    g_mesh[i].chem.fHI = fHI[i];
    g_mesh[i].chem.fHII = 1.0f - fHI[i];
    g_mesh[i].chem.fHeI = fHeI[i];
    g_mesh[i].chem.fHeII = fHeII[i];
    g_mesh[i].chem.fHeIII = 1.0f - fHeI[i] - fHeII[i];
  }
}

void ref_zero_rates(void) { zero_out_photoion_rate(g_mesh, &g_run); }

void ref_get_rates(float *out6)
{
  const uint64_t n = (uint64_t)NMESH_LOCAL;
  for (uint64_t i = 0; i < n; i++) {
    out6[0 * n + i] = g_mesh[i].prev_chem.GammaHI;
    out6[1 * n + i] = g_mesh[i].prev_chem.GammaHeI;
    out6[2 * n + i] = g_mesh[i].prev_chem.GammaHeII;
    out6[3 * n + i] = g_mesh[i].prev_chem.HeatHI;
    out6[4 * n + i] = g_mesh[i].prev_chem.HeatHeI;
    out6[5 * n + i] = g_mesh[i].prev_chem.HeatHeII;
  }
}

/* Sources: photon rates from the reference's setup_photon_rate
 * (source.c:104-138), then the reference's oct-tree (construct_tree,
 * setup_light_ray_tree.c:465). */
int ref_set_sources(int nsrc, const int *type, const float *param,
                    const float *xyz, const double *total_rate, int build_tree)
{
  free(g_src);
  g_src = (struct radiation_src *)calloc((size_t)nsrc, sizeof(struct radiation_src));
  if (!g_src) return -1;
  for (int i = 0; i < nsrc; i++) {
    g_src[i].type = type[i];
    g_src[i].param = param[i];
    g_src[i].xpos = xyz[3 * i + 0];
    g_src[i].ypos = xyz[3 * i + 1];
    g_src[i].zpos = xyz[3 * i + 2];
    setup_photon_rate(&g_run.freq, &g_src[i], total_rate[i]);
  }
  g_run.nsrc = (uint64_t)nsrc;
  free(g_clist); free(g_key); free(g_index);
  g_clist = NULL; g_key = NULL; g_index = NULL;
  g_have_tree = 0;
  if (!build_tree) return 0;
  int nclist = 0;
  init_tree_param(60, &g_run, &nclist);
  g_clist = (struct clist_t *)malloc(sizeof(struct clist_t) * (size_t)nclist);
  g_key = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)nsrc);
  g_index = (int *)malloc(sizeof(int) * (size_t)nsrc);
  if (!g_clist || !g_key || !g_index) return -2;
  construct_tree(g_clist, g_key, g_index, g_src, &g_run);
  g_have_tree = 1;
  return 0;
}

void ref_get_source_spectra(double *out)
{
  for (uint64_t i = 0; i < g_run.nsrc; i++)
    memcpy(out + i * NGRID_NU, g_src[i].photon_rate, sizeof(double) * NGRID_NU);
}

/* number of light rays that end in each local cell of [im_start, im_end)
 * (count_ray_to, setup_light_ray_tree.c:587) */
uint64_t ref_count_rays(int im_start, int im_end, uint64_t *per_cell)
{
  uint64_t total = 0;
  for (int im = im_start; im < im_end; im++) {
    int ix = im / (NMESH_Y_LOCAL * NMESH_Z_LOCAL);
    int iy = (im - ix * NMESH_Y_LOCAL * NMESH_Z_LOCAL) / NMESH_Z_LOCAL;
    int iz = im - ix * NMESH_Y_LOCAL * NMESH_Z_LOCAL - iy * NMESH_Z_LOCAL;
    uint64_t n = count_ray_to(ix, iy, iz, g_clist, g_index, &g_run);
    if (per_cell) per_cell[im - im_start] = n;
    total += n;
  }
  return total;
}

/* End of the group of target cells that starts at im: grown while its ray
 * count stays within MAX_NRAY_PER_TARGET, as calc_ARGOT_part does; *nray
 * receives the group's ray count. */
int ref_next_group(int im, int im_end, uint64_t *nray)
{
  const uint64_t max_rays = (uint64_t)MAX_NRAY_PER_TARGET;
  uint64_t n = 0;
  int ge = im;
  while (ge < im_end) {
    uint64_t c = ref_count_rays(ge, ge + 1, NULL);
    if (ge > im && n + c > max_rays) break;
    n += c;
    ge++;
  }
  *nray = n;
  return ge;
}

/* The first half of calc_ARGOT_part for one group [im, ge) whose ray count
 * is nray (from ref_next_group), for a caller that marches and integrates
 * with other functions (the reference's GPU entry points): the group's light
 * rays into ray[nray], their segments counted (returns nseg); then
 * ref_assign_group fills seg[nseg]. */
int64_t ref_setup_group(int im, int ge, struct light_ray *ray, uint64_t nray)
{
  if (!g_have_tree) return -1;
  g_run.nray = nray;
  setup_light_ray_range(im, ge, ray, 1, g_clist, g_src, g_index, &g_run);
  count_ray_segment(ray, &g_run, &g_omp);
  return (int64_t)g_run.nseg;
}

void ref_assign_group(struct light_ray *ray, struct ray_segment *seg)
{
  assign_ray_segment(ray, seg, &g_run, &g_mpi, &g_omp);
}

void ref_accum_group(struct light_ray *ray, struct ray_segment *seg)
{
  accum_optical_depth(ray, seg, &g_run, &g_omp);
}

struct run_param *ref_run_param(void) { return &g_run; }
struct fluid_mesh *ref_mesh(void) { return g_mesh; }

/*
 * Runs the reference's hot path over target cells [im_start, im_end), in
 * groups whose ray count stays within the reference's MAX_NRAY_PER_TARGET
 * (run_param.h:125, asserted at setup_light_ray_tree.c:432), exactly like
 * calc_ARGOT_part.  Per-ray outputs (in the reference's ray order) are
 * written to the optional arrays; times[0..3] receive the wall time spent in
 * ray setup, calc_optical_depth, accum_optical_depth, calc_photoion_rate.
 * The photo-ionisation rates accumulate into the internal mesh (read them
 * with ref_get_rates after ref_zero_rates).  Returns the number of rays.
 */
int64_t ref_run_range(int im_start, int im_end, int do_photo,
                      int32_t *tgt3, float *src3, float *seg6, float *tau3,
                      double *spec_sum, double *spectra, double *times)
{
  if (!g_have_tree) return -1;
  uint64_t nray_total = 0;
  double t_setup = 0, t_march = 0, t_accum = 0, t_photo = 0;
  struct light_ray *ray = NULL;
  uint64_t ray_cap = 0;

  int im = im_start;
  while (im < im_end) {
    uint64_t nray = 0;
    const int ge = ref_next_group(im, im_end, &nray);
    double t0 = now_s();
    if (nray > ray_cap) {
      free(ray);
      ray = (struct light_ray *)malloc(sizeof(struct light_ray) * (size_t)nray);
      if (!ray) return -2;
      ray_cap = nray;
    }
    g_run.nray = nray;
    setup_light_ray_range(im, ge, ray, 1, g_clist, g_src, g_index, &g_run);
    count_ray_segment(ray, &g_run, &g_omp);
    struct ray_segment *seg =
        (struct ray_segment *)malloc(sizeof(struct ray_segment) * (size_t)(g_run.nseg ? g_run.nseg : 1));
    if (!seg) return -3;
    assign_ray_segment(ray, seg, &g_run, &g_mpi, &g_omp);
    double t1 = now_s();
    calc_optical_depth(seg, g_mesh, &g_run);
    double t2 = now_s();
    accum_optical_depth(ray, seg, &g_run, &g_omp);
    double t3 = now_s();
    if (do_photo) calc_photoion_rate(g_mesh, ray, &g_run);
    double t4 = now_s();
    t_setup += t1 - t0; t_march += t2 - t1; t_accum += t3 - t2; t_photo += t4 - t3;

    for (uint64_t r = 0; r < nray; r++) {
      uint64_t o = nray_total + r;
      if (tgt3) {
        tgt3[3 * o + 0] = ray[r].ix_target;
        tgt3[3 * o + 1] = ray[r].iy_target;
        tgt3[3 * o + 2] = ray[r].iz_target;
      }
      if (src3) {
        src3[3 * o + 0] = ray[r].src.xpos;
        src3[3 * o + 1] = ray[r].src.ypos;
        src3[3 * o + 2] = ray[r].src.zpos;
      }
      if (seg6) {
        seg6[6 * o + 0] = ray[r].segment[0].xpos_start;
        seg6[6 * o + 1] = ray[r].segment[0].ypos_start;
        seg6[6 * o + 2] = ray[r].segment[0].zpos_start;
        seg6[6 * o + 3] = ray[r].segment[0].xpos_end;
        seg6[6 * o + 4] = ray[r].segment[0].ypos_end;
        seg6[6 * o + 5] = ray[r].segment[0].zpos_end;
      }
      if (tau3) {
        tau3[3 * o + 0] = ray[r].optical_depth_HI;
        tau3[3 * o + 1] = ray[r].optical_depth_HeI;
        tau3[3 * o + 2] = ray[r].optical_depth_HeII;
      }
      if (spec_sum) {
        double s = 0.0;
        for (int k = 0; k < NGRID_NU; k++) s += ray[r].src.photon_rate[k];
        spec_sum[o] = s;
      }
      if (spectra)
        memcpy(spectra + o * NGRID_NU, ray[r].src.photon_rate, sizeof(double) * NGRID_NU);
    }
    nray_total += nray;
    free(seg);
    im = ge;
  }
  free(ray);
  if (times) { times[0] = t_setup; times[1] = t_march; times[2] = t_accum; times[3] = t_photo; }
  return (int64_t)nray_total;
}

/* calc_optical_depth on caller-given segments (single rank: every segment
 * lies in this domain).  pos6 = (xs,ys,zs,xe,ye,ze) per segment. */
int ref_march_segments(uint64_t nseg, const float *pos6, float *tau3, double *wall)
{
  struct ray_segment *seg =
      (struct ray_segment *)calloc((size_t)(nseg ? nseg : 1), sizeof(struct ray_segment));
  if (!seg) return -1;
  for (uint64_t i = 0; i < nseg; i++) {
    seg[i].ray_indx = i;
    seg[i].xpos_start = pos6[6 * i + 0];
    seg[i].ypos_start = pos6[6 * i + 1];
    seg[i].zpos_start = pos6[6 * i + 2];
    seg[i].xpos_end = pos6[6 * i + 3];
    seg[i].ypos_end = pos6[6 * i + 4];
    seg[i].zpos_end = pos6[6 * i + 5];
  }
  g_run.nseg = nseg;
  double t0 = now_s();
  calc_optical_depth(seg, g_mesh, &g_run);
  double t1 = now_s();
  if (wall) *wall = t1 - t0;
  for (uint64_t i = 0; i < nseg; i++) {
    tau3[3 * i + 0] = seg[i].optical_depth_HI;
    tau3[3 * i + 1] = seg[i].optical_depth_HeI;
    tau3[3 * i + 2] = seg[i].optical_depth_HeII;
  }
  free(seg);
  return 0;
}

/* accum_optical_depth on caller-given segments -> per-ray columns
 * (rays[ray_indx] receives the segment's columns; one rank). */
int ref_accum_segments(uint64_t nray, uint64_t nseg, const uint64_t *ray_indx,
                       const float *seg_tau3, float *ray_tau3)
{
  struct ray_segment *seg =
      (struct ray_segment *)calloc((size_t)(nseg ? nseg : 1), sizeof(struct ray_segment));
  struct light_ray *ray =
      (struct light_ray *)calloc((size_t)(nray ? nray : 1), sizeof(struct light_ray));
  if (!seg || !ray) { free(seg); free(ray); return -1; }
  for (uint64_t i = 0; i < nseg; i++) {
    seg[i].ray_indx = ray_indx[i];
    seg[i].target_rank = 0;
    seg[i].local_rank = 0;
    seg[i].optical_depth_HI = seg_tau3[3 * i + 0];
    seg[i].optical_depth_HeI = seg_tau3[3 * i + 1];
    seg[i].optical_depth_HeII = seg_tau3[3 * i + 2];
  }
  g_run.nseg = nseg;
  g_run.nray = nray;
  accum_optical_depth(ray, seg, &g_run, &g_omp);
  for (uint64_t r = 0; r < nray; r++) {
    ray_tau3[3 * r + 0] = ray[r].optical_depth_HI;
    ray_tau3[3 * r + 1] = ray[r].optical_depth_HeI;
    ray_tau3[3 * r + 2] = ray[r].optical_depth_HeII;
  }
  free(seg); free(ray);
  return 0;
}

/* calc_photoion_rate on caller-given rays, in chunks (each light_ray is
 * 2.3 kB).  Adds into the internal mesh's prev_chem rates, like the
 * reference.  spectra: nray x NGRID_NU photon rates (s^-1 per bin). */
int ref_photoion_rays(uint64_t nray, const int32_t *tgt3, const float *src3,
                      const double *spectra, const float *tau3, double *wall)
{
  const uint64_t chunk = 1u << 14;
  struct light_ray *ray =
      (struct light_ray *)calloc((size_t)chunk, sizeof(struct light_ray));
  if (!ray) return -1;
  double t = 0.0;
  for (uint64_t r0 = 0; r0 < nray; r0 += chunk) {
    uint64_t n = (nray - r0 < chunk) ? (nray - r0) : chunk;
    for (uint64_t i = 0; i < n; i++) {
      uint64_t r = r0 + i;
      ray[i].src.xpos = src3[3 * r + 0];
      ray[i].src.ypos = src3[3 * r + 1];
      ray[i].src.zpos = src3[3 * r + 2];
      memcpy(ray[i].src.photon_rate, spectra + r * NGRID_NU, sizeof(double) * NGRID_NU);
      ray[i].ix_target = tgt3[3 * r + 0];
      ray[i].iy_target = tgt3[3 * r + 1];
      ray[i].iz_target = tgt3[3 * r + 2];
      ray[i].optical_depth_HI = tau3[3 * r + 0];
      ray[i].optical_depth_HeI = tau3[3 * r + 1];
      ray[i].optical_depth_HeII = tau3[3 * r + 2];
    }
    g_run.nray = n;
    double t0 = now_s();
    calc_photoion_rate(g_mesh, ray, &g_run);
    t += now_s() - t0;
  }
  free(ray);
  if (wall) *wall = t;
  return 0;
}

/* The reference's smooth_photoion_rate (27-point stencil, central weight 30,
 * halo by MPI one-sided puts; on one rank: a copy of the nearest cell when
 * built with __ISOLATED__, the periodic image otherwise) applied to six rate
 * planes rates6 (Gamma HI, HeI, HeII, Heat HI, HeI, HeII; ncell floats
 * each), in place. */
void ref_smooth_rates(float *rates6)
{
  const size_t n = NMESH_LOCAL;
  for (size_t i = 0; i < n; i++) {
    g_mesh[i].prev_chem.GammaHI = rates6[0 * n + i];
    g_mesh[i].prev_chem.GammaHeI = rates6[1 * n + i];
    g_mesh[i].prev_chem.GammaHeII = rates6[2 * n + i];
    g_mesh[i].prev_chem.HeatHI = rates6[3 * n + i];
    g_mesh[i].prev_chem.HeatHeI = rates6[4 * n + i];
    g_mesh[i].prev_chem.HeatHeII = rates6[5 * n + i];
  }
  smooth_photoion_rate(g_mesh, &g_run, &g_mpi);
  for (size_t i = 0; i < n; i++) {
    rates6[0 * n + i] = g_mesh[i].prev_chem.GammaHI;
    rates6[1 * n + i] = g_mesh[i].prev_chem.GammaHeI;
    rates6[2 * n + i] = g_mesh[i].prev_chem.GammaHeII;
    rates6[3 * n + i] = g_mesh[i].prev_chem.HeatHI;
    rates6[4 * n + i] = g_mesh[i].prev_chem.HeatHeI;
    rates6[5 * n + i] = g_mesh[i].prev_chem.HeatHeII;
  }
}

/* The reference's own writers on the loaded mesh and sources:
 * output_mesh_single (output_data.c:14-44) to mesh_file and output_src
 * (output_data.c:59-73) to <src_prefix>_src.dat. */
void ref_write_files(const char *mesh_file, const char *src_prefix)
{
  output_mesh_single(g_mesh, &g_run, (char *)mesh_file);
  output_src(g_src, &g_run, (char *)src_prefix);
}

/* The reference's own readers (input_data.c:112-150, 196-223) into scratch
 * state: the mesh's dens, fHI, fHeI, fHeII and the sources' type, param,
 * position and photon rates (up to max_src).  Returns nsrc, or -1 when the
 * file holds more than max_src.  The mesh header must match this build
 * (the reader exits otherwise). */
int64_t ref_read_files(const char *mesh_file, const char *src_file, float *dens, float *fHI, float *fHeI,
                       float *fHeII, int *type, float *param, float *xyz, double *spectra, int64_t max_src)
{
  static struct run_param tmp_run;
  struct fluid_mesh *m = (struct fluid_mesh *)calloc(NMESH_LOCAL, sizeof(struct fluid_mesh));
  if (!m) return -1;
  input_mesh_single(m, &tmp_run, (char *)mesh_file);
  for (size_t i = 0; i < NMESH_LOCAL; i++) {
    dens[i] = m[i].dens;
    fHI[i] = m[i].chem.fHI;
    fHeI[i] = m[i].chem.fHeI;
    fHeII[i] = m[i].chem.fHeII;
  }
  free(m);
  struct radiation_src *s = (struct radiation_src *)calloc(NSOURCE_MAX, sizeof(struct radiation_src));
  if (!s) return -1;
  input_src_file(s, &tmp_run, (char *)src_file);
  int64_t n = (int64_t)tmp_run.nsrc;
  if (n > max_src) { free(s); return -1; }
  for (int64_t i = 0; i < n; i++) {
    type[i] = s[i].type;
    param[i] = s[i].param;
    xyz[3 * i + 0] = s[i].xpos;
    xyz[3 * i + 1] = s[i].ypos;
    xyz[3 * i + 2] = s[i].zpos;
    memcpy(spectra + i * NGRID_NU, s[i].photon_rate, sizeof(double) * NGRID_NU);
  }
  free(s);
  return n;
}


/* ------------------------------------------------------------------------
 * ART diffuse radiation (src/diffuse_photon, CPU build, single rank): the
 * angle table and step-function factors of setup_diffuse_photon
 * (setup_diffuse.c:8-15), and calc_diffuse_photon_radiation
 * (calc_diffuse_photon_radiation.c:37-128), which adds the diffuse rates to
 * mesh[].prev_chem.  Its inputs are the mesh's prev_chem fractions, dens
 * and prev_uene.
 */
static struct host_diffuse_param g_hd;
static int g_have_hd = 0;

int ref_art_init(double uenetok)
{
  if (!g_have_hd) { init_hd_param(&g_hd); g_have_hd = 1; }
  g_run.uenetok = uenetok;
  setup_diffuse_photon(&g_hd, &g_run);
  return N_ANG;
}

/* dir3[3 N_ANG] (xovr, yovr, zovr), bc2[2 N_ANG] (base_id, corner_id) in the
 * processing order, corner8 the angles per corner, step6 (HI, HeI, HeII x
 * ionisation, heating) */
void ref_art_table(float *dir3, int *bc2, int *corner8, float *step6)
{
  for (int i = 0; i < N_ANG; i++) {
    dir3[3 * i + 0] = g_hd.angle[i].xovr;
    dir3[3 * i + 1] = g_hd.angle[i].yovr;
    dir3[3 * i + 2] = g_hd.angle[i].zovr;
    bc2[2 * i + 0] = g_hd.angle[i].base_id;
    bc2[2 * i + 1] = g_hd.angle[i].corner_id;
  }
  for (int c = 0; c < 8; c++) corner8[c] = g_hd.corner_id_num[c];
  step6[0] = g_hd.step_fact->HI[0]; step6[1] = g_hd.step_fact->HI[1];
  step6[2] = g_hd.step_fact->HeI[0]; step6[3] = g_hd.step_fact->HeI[1];
  step6[4] = g_hd.step_fact->HeII[0]; step6[5] = g_hd.step_fact->HeII[1];
}

/* planes8: dens, fHI, fHII, fHeI, fHeII, fHeIII, felec, prev_uene */
void ref_art_set_mesh(const float *planes8)
{
  const uint64_t n = (uint64_t)NMESH_LOCAL;
  for (uint64_t i = 0; i < n; i++) {
    memset(&g_mesh[i], 0, sizeof(struct fluid_mesh));
    g_mesh[i].dens = planes8[0 * n + i];
    g_mesh[i].prev_chem.fHI = planes8[1 * n + i];
    g_mesh[i].prev_chem.fHII = planes8[2 * n + i];
    g_mesh[i].prev_chem.fHeI = planes8[3 * n + i];
    g_mesh[i].prev_chem.fHeII = planes8[4 * n + i];
    g_mesh[i].prev_chem.fHeIII = planes8[5 * n + i];
    g_mesh[i].prev_chem.felec = planes8[6 * n + i];
    g_mesh[i].prev_uene = planes8[7 * n + i];
    g_mesh[i].chem = g_mesh[i].prev_chem;
  }
}

/* the diffuse rates alone (prev_chem rates zeroed first) into out6; returns
 * the wall time of calc_diffuse_photon_radiation */
double ref_art_run(float *out6)
{
  zero_out_photoion_rate(g_mesh, &g_run);
  const double t0 = now_s();
  calc_diffuse_photon_radiation(g_mesh, &g_run, &g_hd, &g_omp);
  const double t1 = now_s();
  ref_get_rates(out6);
  return t1 - t0;
}
