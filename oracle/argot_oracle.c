/*
 * argot_oracle.c -- CPU restatement of ARGOT's point-source radiative-transfer
 * hot path.  TEST INFRASTRUCTURE ONLY: the CUDA library never links, loads or
 * calls this file; tests/, the smoke check and bench.py's CPU baseline use it
 * as the checker.
 *
 * Two families of functions:
 *
 *  1. "ref-order" restatements that follow the reference's arithmetic step by
 *     step, including its float/double promotions, so that their results can
 *     be pinned bit for bit against the reference's own C compiled in this
 *     tree (oracle/_ref, see build_ref.py):
 *       orc_march_f32ref     calc_optical_depth.c:38-228
 *       orc_accum            accum_optical_depth.c:56-139 (one rank)
 *       orc_photoion_f64ref  calc_photoion_rate.c:124-426 (photon-conserving
 *                            branch, helium, no H2, not cosmological)
 *       orc_tables           source.c:38-53 + prim_chem/cross_section.c:20-53
 *       orc_photon_rate      source.c:10-138 (blackbody / power law)
 *
 *  2. FP64 "precision oracle" variants that compute the same quantities with
 *     every intermediate in double precision and per-cell sums in double:
 *       orc_march_f64, orc_photoion_f64
 *     These are the reference values the FP32 / surrogate GPU paths are
 *     scored against.
 *
 * Conventions (all as in the reference): mesh index
 * MESH(ix,iy,iz) = f[iz + nz*(iy + ny*ix)] (calc_optical_depth.c:18); He
 * number density = HELIUM_FACT * n_H (prim_chem/chemistry.h:25); columns in
 * code units (length x code density); TINY = 1e-31.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_TINY (1.0e-31)
#define ORC_HELIUM_FACT (0.0811258278)
#define ORC_PI (3.1415926535897932384626433)
#define ORC_HPLANCK (6.626e-27)
#define ORC_NUL (3.28e15)
#define ORC_KBOLTZ (1.38066e-16)
#define ORC_NGRID_NU 256

typedef struct {
  int nx, ny, nz;                 /* local mesh (run_param.nmesh_*_local)  */
  int rank_x, rank_y, rank_z;     /* rank coordinates (0 on one rank)       */
  float xmin, ymin, zmin;         /* global box lower corner               */
  float xmin_local, ymin_local, zmin_local;
  float delta_x, delta_y, delta_z;
  double lunit, denstonh;
} orc_grid;

static inline int imin_(int a, int b) { return a < b ? a : b; }
static inline int imax_(int a, int b) { return a > b ? a : b; }

/* ------------------------------------------------------------------ tables */

void orc_tables(double *nu, float *csect3, double *meta3)
{
  const double log_nu_min = 0.0, log_nu_max = 1.5;
  /* dlog_nu is divided by a float-converted NGRID_NU (source.c:46) */
  const double dlog = (log_nu_max - log_nu_min) / (float)ORC_NGRID_NU;
  for (int i = 0; i < ORC_NGRID_NU; i++) {
    double v = pow(10.0, log_nu_min + (i + 0.5) * dlog);
    nu[i] = v;
    double s_hi = 0.0, s_hei = 0.0, s_heii = 0.0;
    if (v >= 1.0) {
      double e = sqrt(v - 1.0);
      s_hi = 6.3e-18 / (v * v * v * v) * exp(4.0 - 4.0 * atan(e) / e) /
             (1.0 - exp(-2.0 * ORC_PI / e));
    }
    if (v >= 1.8125) {
      s_hei = 7.83e-18 * (1.66 * pow(v / 1.8125, -2.05) - 0.66 * pow(v / 1.8125, -3.05));
    }
    if (v >= 4.0) {
      double e = sqrt(v / 4.0 - 1.0);
      s_heii = 6.3e-18 * 256.0 / (v * v * v * v) * exp(4.0 - 4.0 * atan(e) / e) /
               (1.0 - exp(-2.0 * ORC_PI / e)) / 4.0;
    }
    csect3[3 * i + 0] = (float)s_hi;
    csect3[3 * i + 1] = (float)s_hei;
    csect3[3 * i + 2] = (float)s_heii;
  }
  meta3[0] = log_nu_min;
  meta3[1] = log_nu_max;
  meta3[2] = dlog;
}

/* spectral shapes, both normalised at the Lyman limit (source.c:10-36) */
static double shape_bb(double nu, double T)
{
  double i_nu = (nu * ORC_NUL) * (nu * ORC_NUL) / (exp(ORC_HPLANCK * nu * ORC_NUL / (ORC_KBOLTZ * T)) - 1.0);
  double i_l = ORC_NUL * ORC_NUL / (exp(ORC_HPLANCK * ORC_NUL / (ORC_KBOLTZ * T)) - 1.0);
  return i_nu / i_l;
}

static double shape_pl(double nu, double idx) { return pow(nu, idx); }

/* Iterated midpoint rule on [a,b]: stage 1 is one midpoint; every further
 * stage triples the number of points and reuses the previous sum
 * (the open "midpnt" extended rule); the iteration stops when two successive
 * stages agree to 1e-8 relative or after 5 stages (source.c:56-101). */
static double midpoint_integral(double (*f)(double, double), double p, double a, double b)
{
  double s = 0.0, prev = 0.0;
  for (int stage = 1; stage <= 5; stage++) {
    if (stage == 1) {
      s = (b - a) * f(0.5 * (a + b), p);
    } else {
      int npts = 1;
      for (int j = 1; j < stage - 1; j++) npts *= 3;
      double h = (b - a) / (3.0 * npts);
      double x = a + 0.5 * h, acc = 0.0;
      for (int j = 1; j <= npts; j++) {
        acc += f(x, p);
        x += 2.0 * h;
        acc += f(x, p);
        x += h;
      }
      s = (s + (b - a) * acc / npts) / 3.0;
    }
    if (stage > 1 && fabs(s - prev) < 1.0e-8 * fabs(prev)) return s;
    prev = s;
  }
  return s;
}

void orc_photon_rate(int type, float param, double total_rate, double *out)
{
  const double log_nu_min = 0.0;
  const double dlog = (1.5 - 0.0) / (float)ORC_NGRID_NU;
  double (*f)(double, double) = (type == 0) ? shape_bb : shape_pl;
  double norm = midpoint_integral(f, (double)param, 1.0, pow(10.0, 1.5));
  for (int i = 0; i < ORC_NGRID_NU; i++) {
    double a = log_nu_min + dlog * (double)i;
    double b = a + dlog;
    out[i] = midpoint_integral(f, (double)param, pow(10.0, a), pow(10.0, b));
    out[i] *= total_rate / norm;
  }
}

/* ----------------------------------------------------------- march (FP32) */

/* One segment, the reference's float arithmetic in the reference's order
 * (calc_optical_depth.c:65-227).  The comments mark where the reference
 * promotes to double because TINY and HELIUM_FACT are double literals. */
static void march_f32ref_one(const orc_grid *g, const float *dens, const float *fHI,
                             const float *fHeI, const float *fHeII, const float *p,
                             float *tau)
{
  const int NX = g->nx, NY = g->ny, NZ = g->nz;
  float t_hi = 0.0f, t_hei = 0.0f, t_heii = 0.0f;
  float xs = p[0], ys = p[1], zs = p[2], xe = p[3], ye = p[4], ze = p[5];

  int ix_end = (int)((xe - g->xmin_local) / g->delta_x);
  int iy_end = (int)((ye - g->ymin_local) / g->delta_y);
  int iz_end = (int)((ze - g->zmin_local) / g->delta_z);
  ix_end = imax_(imin_(ix_end, NX - 1), 0);
  iy_end = imax_(imin_(iy_end, NY - 1), 0);
  iz_end = imax_(imin_(iz_end, NZ - 1), 0);
  int ix = (int)((xs - g->xmin_local) / g->delta_x);
  int iy = (int)((ys - g->ymin_local) / g->delta_y);
  int iz = (int)((zs - g->zmin_local) / g->delta_z);
  ix = imax_(imin_(ix, NX - 1), 0);
  iy = imax_(imin_(iy, NY - 1), 0);
  iz = imax_(imin_(iz, NZ - 1), 0);

  float dx = xe - xs, dy = ye - ys, dz = ze - zs;
  float dl = (float)sqrt((double)(dx * dx + dy * dy + dz * dz) + ORC_TINY); /* double */
  float dxy = (float)sqrt((double)(dx * dx + dy * dy));
  float cos_t = dz / dl, sin_t = dxy / dl;
  float cos_p = (float)((double)dx / ((double)dxy + ORC_TINY)); /* double */
  float sin_p = (float)((double)dy / ((double)dxy + ORC_TINY));
  float xo = cos_p * sin_t, yo = sin_p * sin_t, zo = cos_t;
  if (fabs((double)xo) < ORC_TINY) xo = (xo >= 0.0f) ? (float)ORC_TINY : -(float)ORC_TINY;
  if (fabs((double)yo) < ORC_TINY) yo = (yo >= 0.0f) ? (float)ORC_TINY : -(float)ORC_TINY;
  if (fabs((double)zo) < ORC_TINY) zo = (zo >= 0.0f) ? (float)ORC_TINY : -(float)ORC_TINY;
  int xs_step = xo > 0.0f ? 1 : 0, xn = xo > 0.0f ? 1 : -1;
  int ys_step = yo > 0.0f ? 1 : 0, yn = yo > 0.0f ? 1 : -1;
  int zs_step = zo > 0.0f ? 1 : 0, zn = zo > 0.0f ? 1 : -1;

  float xc = xs - g->xmin_local, yc = ys - g->ymin_local, zc = zs - g->zmin_local;

  while ((ix != ix_end || iy != iy_end || iz != iz_end) &&
         (0 <= ix && ix < NX) && (0 <= iy && iy < NY) && (0 <= iz && iz < NZ)) {
    size_t c = (size_t)iz + (size_t)NZ * ((size_t)iy + (size_t)NY * (size_t)ix);
    float nH = dens[c];
    float nHI = nH * fHI[c];
    float nHe = (float)((double)nH * ORC_HELIUM_FACT); /* double */
    float nHeI = nHe * fHeI[c];
    float nHeII = nHe * fHeII[c];
    float ddx = g->delta_x * (float)(xs_step + ix) - xc;
    float ddy = g->delta_y * (float)(ys_step + iy) - yc;
    float ddz = g->delta_z * (float)(zs_step + iz) - zc;
    float rx = ddx / xo, ry = ddy / yo, rz = ddz / zo;
    float rmin = fminf(rx, fminf(ry, rz));
    if (rmin == rx) ix += xn;
    if (rmin == ry) iy += yn;
    if (rmin == rz) iz += zn;
    xc += rmin * xo;
    yc += rmin * yo;
    zc += rmin * zo;
    t_hi += rmin * nHI;
    t_hei += rmin * nHeI;
    t_heii += rmin * nHeII;
  }
  xc += g->xmin_local;
  yc += g->ymin_local;
  zc += g->zmin_local;
  float ex = xe - xc, ey = ye - yc, ez = ze - zc;
  float depth = (float)sqrt((double)(ex * ex + ey * ey + ez * ez));
  size_t c = (size_t)iz_end + (size_t)NZ * ((size_t)iy_end + (size_t)NY * (size_t)ix_end);
  float nH = dens[c];
  float nHI = nH * fHI[c];
  float nHe = (float)((double)nH * ORC_HELIUM_FACT);
  float nHeI = nHe * fHeI[c];
  float nHeII = nHe * fHeII[c];
  t_hi += depth * nHI;
  t_hei += depth * nHeI;
  t_heii += depth * nHeII;
  tau[0] = t_hi;
  tau[1] = t_hei;
  tau[2] = t_heii;
}

void orc_march_f32ref(const orc_grid *g, const float *dens, const float *fHI,
                      const float *fHeI, const float *fHeII, uint64_t nseg,
                      const float *pos6, float *tau3)
{
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < (int64_t)nseg; i++)
    march_f32ref_one(g, dens, fHI, fHeI, fHeII, pos6 + 6 * i, tau3 + 3 * i);
}

/* ----------------------------------------------------------- march (FP64) */

/* Same traversal semantics in double precision throughout: start/end cell
 * from the (float) endpoints, cell-by-cell chords until the end cell is
 * reached or the walk leaves the local mesh, then the partial chord from the
 * last crossing to the end point.  Positions are recomputed from the start
 * point and the path parameter (no drift), and columns are summed in
 * double. */
static void march_f64_one(const orc_grid *g, const float *dens, const float *fHI,
                          const float *fHeI, const float *fHeII, const float *p,
                          double *tau)
{
  const int NX = g->nx, NY = g->ny, NZ = g->nz;
  const double dX = g->delta_x, dY = g->delta_y, dZ = g->delta_z;
  const double x0 = (double)p[0] - g->xmin_local, y0 = (double)p[1] - g->ymin_local,
               z0 = (double)p[2] - g->zmin_local;
  const double x1 = (double)p[3] - g->xmin_local, y1 = (double)p[4] - g->ymin_local,
               z1 = (double)p[5] - g->zmin_local;
  double s_hi = 0, s_hei = 0, s_heii = 0;

  int ix_end = (int)((p[3] - g->xmin_local) / g->delta_x);
  int iy_end = (int)((p[4] - g->ymin_local) / g->delta_y);
  int iz_end = (int)((p[5] - g->zmin_local) / g->delta_z);
  ix_end = imax_(imin_(ix_end, NX - 1), 0);
  iy_end = imax_(imin_(iy_end, NY - 1), 0);
  iz_end = imax_(imin_(iz_end, NZ - 1), 0);
  int ix = (int)((p[0] - g->xmin_local) / g->delta_x);
  int iy = (int)((p[1] - g->ymin_local) / g->delta_y);
  int iz = (int)((p[2] - g->zmin_local) / g->delta_z);
  ix = imax_(imin_(ix, NX - 1), 0);
  iy = imax_(imin_(iy, NY - 1), 0);
  iz = imax_(imin_(iz, NZ - 1), 0);

  double dx = x1 - x0, dy = y1 - y0, dz = z1 - z0;
  double len = sqrt(dx * dx + dy * dy + dz * dz + ORC_TINY);
  double ux = dx / len, uy = dy / len, uz = dz / len;
  if (fabs(ux) < ORC_TINY) ux = (ux >= 0.0) ? ORC_TINY : -ORC_TINY;
  if (fabs(uy) < ORC_TINY) uy = (uy >= 0.0) ? ORC_TINY : -ORC_TINY;
  if (fabs(uz) < ORC_TINY) uz = (uz >= 0.0) ? ORC_TINY : -ORC_TINY;
  const int sx = ux > 0 ? 1 : 0, nx_ = ux > 0 ? 1 : -1;
  const int sy = uy > 0 ? 1 : 0, ny_ = uy > 0 ? 1 : -1;
  const int sz = uz > 0 ? 1 : 0, nz_ = uz > 0 ? 1 : -1;

  double t = 0.0; /* path length travelled from the start point */
  while ((ix != ix_end || iy != iy_end || iz != iz_end) &&
         (0 <= ix && ix < NX) && (0 <= iy && iy < NY) && (0 <= iz && iz < NZ)) {
    size_t c = (size_t)iz + (size_t)NZ * ((size_t)iy + (size_t)NY * (size_t)ix);
    double nH = dens[c];
    double nHe = nH * ORC_HELIUM_FACT;
    double tx = (dX * (sx + ix) - x0) / ux;
    double ty = (dY * (sy + iy) - y0) / uy;
    double tz = (dZ * (sz + iz) - z0) / uz;
    double tn = fmin(tx, fmin(ty, tz));
    double r = tn - t;
    if (tn == tx) ix += nx_;
    if (tn == ty) iy += ny_;
    if (tn == tz) iz += nz_;
    t = tn;
    s_hi += r * nH * fHI[c];
    s_hei += r * nHe * fHeI[c];
    s_heii += r * nHe * fHeII[c];
  }
  double xc = x0 + t * ux, yc = y0 + t * uy, zc = z0 + t * uz;
  double depth = sqrt((x1 - xc) * (x1 - xc) + (y1 - yc) * (y1 - yc) + (z1 - zc) * (z1 - zc));
  size_t c = (size_t)iz_end + (size_t)NZ * ((size_t)iy_end + (size_t)NY * (size_t)ix_end);
  double nH = dens[c], nHe = nH * ORC_HELIUM_FACT;
  s_hi += depth * nH * fHI[c];
  s_hei += depth * nHe * fHeI[c];
  s_heii += depth * nHe * fHeII[c];
  tau[0] = s_hi;
  tau[1] = s_hei;
  tau[2] = s_heii;
}

void orc_march_f64(const orc_grid *g, const float *dens, const float *fHI,
                   const float *fHeI, const float *fHeII, uint64_t nseg,
                   const float *pos6, double *tau3)
{
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < (int64_t)nseg; i++)
    march_f64_one(g, dens, fHI, fHeI, fHeII, pos6 + 6 * i, tau3 + 3 * i);
}

/* number of cells each segment's walk visits before the end cell, plus one
 * for the end cell itself: the unit of the "ray-cell crossings" metric */
void orc_count_crossings(const orc_grid *g, uint64_t nseg, const float *pos6, uint64_t *out)
{
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < (int64_t)nseg; i++) {
    const float *p = pos6 + 6 * i;
    const int NX = g->nx, NY = g->ny, NZ = g->nz;
    int ix_end = imax_(imin_((int)((p[3] - g->xmin_local) / g->delta_x), NX - 1), 0);
    int iy_end = imax_(imin_((int)((p[4] - g->ymin_local) / g->delta_y), NY - 1), 0);
    int iz_end = imax_(imin_((int)((p[5] - g->zmin_local) / g->delta_z), NZ - 1), 0);
    int ix = imax_(imin_((int)((p[0] - g->xmin_local) / g->delta_x), NX - 1), 0);
    int iy = imax_(imin_((int)((p[1] - g->ymin_local) / g->delta_y), NY - 1), 0);
    int iz = imax_(imin_((int)((p[2] - g->zmin_local) / g->delta_z), NZ - 1), 0);
    /* |di|+|dj|+|dk| + 1 cells for a walk that steps one axis at a time */
    out[i] = (uint64_t)(abs(ix_end - ix) + abs(iy_end - iy) + abs(iz_end - iz) + 1);
  }
}

/* --------------------------------------------------------------- stitching */

/* One rank: every ray's columns are the sum of its segments' columns
 * (accum_optical_depth.c:89-139 writes send[ray_indx] = seg and adds the
 * remote accumulation, which is zero on one rank). */
void orc_accum(uint64_t nray, uint64_t nseg, const uint64_t *ray_indx,
               const float *seg_tau3, float *ray_tau3)
{
  memset(ray_tau3, 0, sizeof(float) * 3 * nray);
  for (uint64_t i = 0; i < nseg; i++) {
    uint64_t r = ray_indx[i];
    ray_tau3[3 * r + 0] += seg_tau3[3 * i + 0];
    ray_tau3[3 * r + 1] += seg_tau3[3 * i + 1];
    ray_tau3[3 * r + 2] += seg_tau3[3 * i + 2];
  }
}

/* ---------------------------------------------------- photo-ionisation rate */

/* delta_length (calc_photoion_rate.c:52-90): float arithmetic with double
 * promotions where TINY is involved. */
static float delta_length_ref(float dx, float dy, float dz, const orc_grid *g)
{
  float dl = (float)sqrt((double)(dx * dx + dy * dy + dz * dz) + ORC_TINY);
  float dxy = (float)sqrt((double)(dx * dx + dy * dy) + ORC_TINY);
  float cos_t = dz / dl, sin_t = dxy / dl;
  float cos_p = dx / dxy, sin_p = dy / dxy;
  float xo = cos_p * sin_t, yo = sin_p * sin_t, zo = cos_t;
  if (fabsf(xo) < ORC_TINY) xo = (xo >= 0.0f) ? (float)ORC_TINY : -(float)ORC_TINY;
  if (fabsf(yo) < ORC_TINY) yo = (yo >= 0.0f) ? (float)ORC_TINY : -(float)ORC_TINY;
  if (fabsf(zo) < ORC_TINY) zo = (zo >= 0.0f) ? (float)ORC_TINY : -(float)ORC_TINY;
  float rx = fabsf(g->delta_x / xo), ry = fabsf(g->delta_y / yo), rz = fabsf(g->delta_z / zo);
  return fminf(rx, fminf(ry, rz));
}

/* Per-ray rates (6 doubles: Gamma HI/HeI/HeII, Heat HI/HeI/HeII) in the
 * reference's order and precision.  tau3: code-unit columns of the ray;
 * tgt: global target indices; src: source position; spec: photon rate per
 * bin.  Heat is returned already multiplied by h*nu_L. */
static void photoion_ray_ref(const orc_grid *g, const float *dens, const float *fHI,
                             const float *fHeI, const float *fHeII, const double *nu,
                             const float *cs3, const float *tau3, const int32_t *tgt,
                             const float *src, const double *spec, double *out6)
{
  double tHI = tau3[0] * (g->lunit * g->denstonh);
  double tHeI = tau3[1] * (g->lunit * g->denstonh);
  double tHeII = tau3[2] * (g->lunit * g->denstonh);
  int ix = tgt[0] - g->rank_x * g->nx;
  int iy = tgt[1] - g->rank_y * g->ny;
  int iz = tgt[2] - g->rank_z * g->nz;
  size_t c = (size_t)iz + (size_t)g->nz * ((size_t)iy + (size_t)g->ny * (size_t)ix);
  float x = (float)(g->delta_x * ((float)tgt[0] + 0.5) + g->xmin);
  float y = (float)(g->delta_y * ((float)tgt[1] + 0.5) + g->ymin);
  float z = (float)(g->delta_z * ((float)tgt[2] + 0.5) + g->zmin);
  float dx = x - src[0], dy = y - src[1], dz = z - src[2];

  float delta = delta_length_ref(dx, dy, dz, g);
  float dist = (float)sqrt((double)(dx * dx + dy * dy + dz * dz));
  double nH = dens[c] * g->denstonh;
  double nHI = nH * fHI[c];
  double dHI = nHI * delta * (g->lunit);
  tHI -= 0.5 * dHI;
  double nHe = nH * ORC_HELIUM_FACT;
  double nHeI = nHe * fHeI[c];
  double nHeII = nHe * fHeII[c];
  double dHeI = nHeI * delta * (g->lunit);
  double dHeII = nHeII * delta * (g->lunit);
  tHeI -= 0.5 * dHeI;
  tHeII -= 0.5 * dHeII;
  double L3 = g->lunit * g->lunit * g->lunit;
  double Vsh = 4.0 * ORC_PI / 3.0 *
               ((dist + 0.5 * delta) * (dist + 0.5 * delta) * (dist + 0.5 * delta) -
                (dist - 0.5 * delta) * (dist - 0.5 * delta) * (dist - 0.5 * delta)) * L3;
  double rNHI = 1.0 / (nHI * Vsh + ORC_TINY);
  double rNHeI = 1.0 / (nHeI * Vsh + ORC_TINY);
  double rNHeII = 1.0 / (nHeII * Vsh + ORC_TINY);

  double GHI = 0, HHI = 0, GHeI = 0, GHeII = 0, HHeI = 0, HHeII = 0;
  for (int k = 0; k < ORC_NGRID_NU; k++) {
    float v = (float)nu[k];
    double tau = tHI * cs3[3 * k + 0];
    double dtHI = dHI * cs3[3 * k + 0];
    double dtot = dtHI;
    tau += tHeI * cs3[3 * k + 1];
    tau += tHeII * cs3[3 * k + 2];
    double dtHeI = dHeI * cs3[3 * k + 1];
    double dtHeII = dHeII * cs3[3 * k + 2];
    dtot += dtHeI + dtHeII;
    double pabs = spec[k] * exp(-tau) * (1.0e0 - exp(-dtot));
    dtHI /= (dtot + ORC_TINY);
    GHI += dtHI * pabs * rNHI;
    if (v > 1.0) HHI += dtHI * pabs * (v - 1.0) * rNHI;
    dtHeI /= (dtot + ORC_TINY);
    dtHeII /= (dtot + ORC_TINY);
    GHeI += dtHeI * pabs * rNHeI;
    GHeII += dtHeII * pabs * rNHeII;
    if (v > 1.8125) HHeI += dtHeI * pabs * (v - 1.8125) * rNHeI;
    if (v > 4.0) HHeII += dtHeII * pabs * (v - 4.0) * rNHeII;
  }
  out6[0] = GHI;
  out6[1] = GHeI;
  out6[2] = GHeII;
  out6[3] = HHI * (ORC_HPLANCK * ORC_NUL);
  out6[4] = HHeI * (ORC_HPLANCK * ORC_NUL);
  out6[5] = HHeII * (ORC_HPLANCK * ORC_NUL);
}

/* Rates accumulated into float per-cell fields in ray order, the way the
 * reference's single-threaded loop does (calc_photoion_rate.c:403-425: a
 * float field += a double value).  rates6: 6 x ncell SoA (Gamma HI, HeI,
 * HeII, Heat HI, HeI, HeII), added to. */
void orc_photoion_f64ref(const orc_grid *g, const float *dens, const float *fHI,
                         const float *fHeI, const float *fHeII, const double *nu,
                         const float *cs3, uint64_t nray, const float *tau3,
                         const int32_t *tgt3, const float *src3, const double *spectra,
                         const uint64_t *spec_index, float *rates6)
{
  const size_t ncell = (size_t)g->nx * g->ny * g->nz;
  double *per = (double *)malloc(sizeof(double) * 6 * (nray ? nray : 1));
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t r = 0; r < (int64_t)nray; r++) {
    const double *spec = spectra + (spec_index ? spec_index[r] : (uint64_t)r) * ORC_NGRID_NU;
    photoion_ray_ref(g, dens, fHI, fHeI, fHeII, nu, cs3, tau3 + 3 * r, tgt3 + 3 * r,
                     src3 + 3 * r, spec, per + 6 * r);
  }
  for (uint64_t r = 0; r < nray; r++) {
    int ix = tgt3[3 * r + 0] - g->rank_x * g->nx;
    int iy = tgt3[3 * r + 1] - g->rank_y * g->ny;
    int iz = tgt3[3 * r + 2] - g->rank_z * g->nz;
    size_t c = (size_t)iz + (size_t)g->nz * ((size_t)iy + (size_t)g->ny * (size_t)ix);
    for (int s = 0; s < 6; s++)
      rates6[s * ncell + c] = (float)((double)rates6[s * ncell + c] + per[6 * r + s]);
  }
  free(per);
}

/* FP64 precision oracle: per-ray rates from double columns with double
 * geometry, summed per cell in double. */
void orc_photoion_f64(const orc_grid *g, const float *dens, const float *fHI,
                      const float *fHeI, const float *fHeII, const double *nu,
                      const float *cs3, uint64_t nray, const double *tau3,
                      const int32_t *tgt3, const float *src3, const double *spectra,
                      const uint64_t *spec_index, double *rates6)
{
  const size_t ncell = (size_t)g->nx * g->ny * g->nz;
  double *per = (double *)malloc(sizeof(double) * 6 * (nray ? nray : 1));
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t r = 0; r < (int64_t)nray; r++) {
    const double *spec = spectra + (spec_index ? spec_index[r] : (uint64_t)r) * ORC_NGRID_NU;
    const int32_t *tgt = tgt3 + 3 * r;
    const float *src = src3 + 3 * r;
    int ix = tgt[0] - g->rank_x * g->nx;
    int iy = tgt[1] - g->rank_y * g->ny;
    int iz = tgt[2] - g->rank_z * g->nz;
    size_t c = (size_t)iz + (size_t)g->nz * ((size_t)iy + (size_t)g->ny * (size_t)ix);
    double x = (double)g->delta_x * ((double)tgt[0] + 0.5) + g->xmin;
    double y = (double)g->delta_y * ((double)tgt[1] + 0.5) + g->ymin;
    double z = (double)g->delta_z * ((double)tgt[2] + 0.5) + g->zmin;
    double dx = x - src[0], dy = y - src[1], dz = z - src[2];
    double d2 = dx * dx + dy * dy + dz * dz;
    double dl = sqrt(d2 + ORC_TINY), dxy = sqrt(dx * dx + dy * dy + ORC_TINY);
    double xo = (dx / dxy) * (dxy / dl), yo = (dy / dxy) * (dxy / dl), zo = dz / dl;
    if (fabs(xo) < ORC_TINY) xo = xo >= 0 ? ORC_TINY : -ORC_TINY;
    if (fabs(yo) < ORC_TINY) yo = yo >= 0 ? ORC_TINY : -ORC_TINY;
    if (fabs(zo) < ORC_TINY) zo = zo >= 0 ? ORC_TINY : -ORC_TINY;
    double delta = fmin(fabs(g->delta_x / xo), fmin(fabs(g->delta_y / yo), fabs(g->delta_z / zo)));
    double dist = sqrt(d2);
    double lu = g->lunit, cd = g->lunit * g->denstonh;
    double nH = dens[c] * g->denstonh, nHe = nH * ORC_HELIUM_FACT;
    double n3[3] = {nH * fHI[c], nHe * fHeI[c], nHe * fHeII[c]};
    double d3[3], t3[3], rN[3];
    double Vsh = 4.0 * ORC_PI / 3.0 *
                 (pow(dist + 0.5 * delta, 3) - pow(dist - 0.5 * delta, 3)) * lu * lu * lu;
    for (int s = 0; s < 3; s++) {
      d3[s] = n3[s] * delta * lu;
      t3[s] = tau3[3 * r + s] * cd - 0.5 * d3[s];
      rN[s] = 1.0 / (n3[s] * Vsh + ORC_TINY);
    }
    double G[3] = {0, 0, 0}, H[3] = {0, 0, 0};
    const double thr[3] = {1.0, 1.8125, 4.0};
    for (int k = 0; k < ORC_NGRID_NU; k++) {
      double v = (float)nu[k];
      double tau = 0, dtot = 0, dts[3];
      for (int s = 0; s < 3; s++) {
        tau += t3[s] * cs3[3 * k + s];
        dts[s] = d3[s] * cs3[3 * k + s];
        dtot += dts[s];
      }
      /* (1 - e^-dtot)/dtot without cancellation */
      double phi = dtot > 1e-300 ? -expm1(-dtot) / dtot : 1.0;
      double a = spec[k] * exp(-tau) * phi;
      for (int s = 0; s < 3; s++) {
        double gs = dts[s] * a * rN[s];
        G[s] += gs;
        if (v > thr[s]) H[s] += gs * (v - thr[s]);
      }
    }
    for (int s = 0; s < 3; s++) {
      per[6 * r + s] = G[s];
      per[6 * r + 3 + s] = H[s] * (ORC_HPLANCK * ORC_NUL);
    }
    (void)c;
  }
  for (uint64_t r = 0; r < nray; r++) {
    int ix = tgt3[3 * r + 0] - g->rank_x * g->nx;
    int iy = tgt3[3 * r + 1] - g->rank_y * g->ny;
    int iz = tgt3[3 * r + 2] - g->rank_z * g->nz;
    size_t c = (size_t)iz + (size_t)g->nz * ((size_t)iy + (size_t)g->ny * (size_t)ix);
    for (int s = 0; s < 6; s++) rates6[s * ncell + c] += per[6 * r + s];
  }
  free(per);
}

/* Per-ray (not per-cell) FP64 rates, for parity checks at ray granularity. */
void orc_photoion_f64ref_per_ray(const orc_grid *g, const float *dens, const float *fHI,
                                 const float *fHeI, const float *fHeII, const double *nu,
                                 const float *cs3, uint64_t nray, const float *tau3,
                                 const int32_t *tgt3, const float *src3,
                                 const double *spectra, const uint64_t *spec_index,
                                 double *per6)
{
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t r = 0; r < (int64_t)nray; r++) {
    const double *spec = spectra + (spec_index ? spec_index[r] : (uint64_t)r) * ORC_NGRID_NU;
    photoion_ray_ref(g, dens, fHI, fHeI, fHeII, nu, cs3, tau3 + 3 * r, tgt3 + 3 * r,
                     src3 + 3 * r, spec, per6 + 6 * r);
  }
}
