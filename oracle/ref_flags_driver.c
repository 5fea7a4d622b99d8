/*
 * ref_flags_driver.c -- test-infrastructure driver around ARGOT's OWN C for
 * the hot path compiled with a flag set other than the default one (the
 * stock -D__HYDROGEN_MOL__ build of src/Makefile, helium with H2, no photon
 * conservation, the scale factor, hydrogen only).  oracle/build.py compiles
 * it with the reference sources, unmodified, into
 * oracle/_ref/libargot_ref_flags_<tag>_n<EDGE>.so.  Only tests/ load it.
 *
 * The callers use the reference's own entry points directly
 * (calc_optical_depth, zero_out_photoion_rate, calc_photoion_rate,
 * setup_photon_rate); this file only owns the run_param, the mesh and the
 * MPI / OpenMP parameter structs a single rank needs, filled the way the
 * reference's init_run does (init_run.c:93).  No arithmetic of the hot path
 * lives here.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <stddef.h>
#include <omp.h>

#include "run_param.h"
#include "constants.h"
#include "fluid.h"
#include "radiation.h"
#include "source.h"
#include "cross_section.h"
#include "prototype.h"
#include "mpi_param.h"
#include "omp_param.h"

static struct run_param g_run;
static struct fluid_mesh *g_mesh = NULL;
static struct mpi_param g_mpi;

int refv_mesh_edge(void) { return NMESH_X_LOCAL; }

/* same order as argot_b200_struct_sizes */
void refv_struct_sizes(uint64_t *s)
{
  s[0] = sizeof(struct ray_segment);
  s[1] = sizeof(struct light_ray);
  s[2] = sizeof(struct light_ray_IO);
  s[3] = sizeof(struct radiation_src);
  s[4] = sizeof(struct fluid_mesh);
  s[5] = sizeof(struct prim_chem);
  s[6] = sizeof(struct run_param);
  s[7] = sizeof(struct cross_section);
  s[8] = sizeof(struct freq_param);
  s[9] = sizeof(struct photoion_rate);
}

/* offsets of the fields the test mirrors position by name */
void refv_offsets(uint64_t *o)
{
  int i = 0;
  o[i++] = offsetof(struct prim_chem, fHI);
  o[i++] = offsetof(struct prim_chem, GammaHI);
  o[i++] = offsetof(struct fluid_mesh, chem);
  o[i++] = offsetof(struct fluid_mesh, prev_chem);
  o[i++] = offsetof(struct ray_segment, optical_depth_HI);
  o[i++] = offsetof(struct light_ray, ix_target);
  o[i++] = offsetof(struct light_ray, optical_depth_HI);
  o[i++] = offsetof(struct light_ray_IO, optical_depth_HI);
  o[i++] = offsetof(struct run_param, csect);
  o[i++] = offsetof(struct run_param, nseg);
  o[i++] = offsetof(struct run_param, nmesh_x_local);
  o[i++] = offsetof(struct run_param, delta_x);
}

/* single rank over the unit box; tables by the reference's own setup */
int refv_init(double lunit, double denstonh, float anow, int nthreads)
{
  memset(&g_run, 0, sizeof(g_run));
  g_run.proc_file = fopen("/dev/null", "w");
  g_run.diag_file = g_run.proc_file;
  g_run.err_file = g_run.proc_file;
#ifdef __HELIUM__
  g_run.helium_flag = 1;
#endif
#ifdef __HYDROGEN_MOL__
  g_run.hydrogen_mol_flag = 1;
#endif
#ifdef __COSMOLOGICAL__
  g_run.cosmology_flag = 1;
#endif
  g_run.ngrid_nu = NGRID_NU;
  g_run.mpi_nproc = 1;
  g_run.nnode_x = g_run.nnode_y = g_run.nnode_z = 1;
  g_run.lunit = lunit;
  g_run.denstonh = denstonh;
  g_run.anow = anow;
  g_run.nspecies = NSPECIES;
  g_run.nchannel = NCHANNEL;
  g_run.xmax = g_run.ymax = g_run.zmax = 1.0f;
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
  g_run.theta_crit = 0.5f;
  g_run.nmesh_per_loop = NMESH_LOCAL;
  setup_freq_param(&g_run.freq);
  setup_cross_section(g_run.csect, &g_run.freq);
  g_mpi.photoion_rate_type = ARGOT_SHIM_SIZED_TYPE(sizeof(struct photoion_rate));
  if (nthreads > 0) omp_set_num_threads(nthreads);
  if (!g_mesh) g_mesh = (struct fluid_mesh *)calloc(NMESH_LOCAL, sizeof(struct fluid_mesh));
  return g_mesh ? 0 : -1;
}

struct run_param *refv_run(void) { return &g_run; }
struct fluid_mesh *refv_mesh(void) { return g_mesh; }

/* the spectrum of one source (setup_photon_rate, source.c:104-138) */
void refv_photon_rate(int type, float param, double total, double *out)
{
  struct radiation_src s;
  memset(&s, 0, sizeof(s));
  s.type = type;
  s.param = param;
  setup_photon_rate(&g_run.freq, &s, total);
  memcpy(out, s.photon_rate, sizeof(s.photon_rate));
}

/* the reference's smoothing of the rate fields of g_mesh, in place */
void refv_smooth(void) { smooth_photoion_rate(g_mesh, &g_run, &g_mpi); }
