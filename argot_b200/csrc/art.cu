// art.cu -- ARGOT's ART diffuse-radiation transfer (src/diffuse_photon:
// calc_diffuse_photon_radiation.c, ray_tracing.c, calc_rmesh_data.c,
// calc_GH_tot.c, set_angle.c, set_step_func_factor.c) for one rank on the
// device: the second radiative-transfer path of ARGOT, recombination
// photons carried along long characteristics in N_ANG = 12 nside^2 HEALPix
// directions.
//
// Per angle every cell of the start face (the face a direction enters
// through: base 0..5 = -z, +z, -x, +x, -y, +y side of the box) launches one
// ray at a fixed sub-cell offset.  The ray marches with the reference's
// float DDA (same operations, IEEE rounding, so the cell sequence and the
// chord lengths are the reference's), wraps through the two side faces to
// the opposite side with its intensity reset to zero (a single rank is its
// own, isolated, neighbour: ray_tracing.c:276-372 with reset_I), and ends at
// the far face.  In every cell it crosses it adds, for three frequencies
// (HI, HeI, HeII edges), I (1 - e^-tau) and the chord length to the angle's
// accumulators, and updates I = I e^-tau + S (1 - e^-tau).
//
// B200 design.  A pass takes a batch of angles: one thread per ray, all
// rays of all angles of the batch in one launch (a single angle has only
// N^2 rays), each angle with its own accumulator planes, so the per-angle
// sums stay separate as the reference needs them.  Rays of one angle are
// parallel lines, several may cross a cell, so the accumulators take vector
// float atomics (one 16-byte reduction per crossing).  The per-cell
// quantities (absorption, source function) are one 32-byte record per cell,
// one 256-bit load per step.  A second kernel folds the batch's angles into the six
// per-cell totals in angle order, as calc_GH_tot does angle after angle.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "ref_layout.h"

namespace argot {

// src/diffuse_photon/diffuse_photon.h:39-73 (He without the
// two-photon/bound-bound lines), prim_chem/chemistry.h:10-34
constexpr double kRcrossHI2 = 1.9529766579e-01, kRcrossHI3 = 1.9513732355e-02;
constexpr double kRcrossHeI3 = 2.6858709594e-01;
constexpr double kRintJHI2 = 1.128855608262e-01, kRintJHI3 = 5.288790581895e-03;
constexpr double kRintJHeI3 = 1.2404369898e-01;
constexpr double kRintHHI2 = 3.1154224364e+00, kRintHHI3 = 5.2452188546e-01;
constexpr double kRintHHeI3 = 8.7872474963e+00;
constexpr double kKtoEV = 8.61623e-5, kEVtoErg = 1.6022e-12, kNuLeV = 13.6;
constexpr double kXHydrogen = 0.755, kYHelium = 0.245;
constexpr double kStepRange = 0.0632353;
constexpr int kStepBins = 64;

struct ArtAngle {
  float ox, oy, oz;
  int base;
};

// Per-cell data of the march: absorption coefficients [cm^-1] and source
// functions of the three frequencies in one 32-byte record, read with one
// 256-bit load per step.
struct __align__(32) ArtCell {
  float a1, a2, a3, s1, s2, s3, pad0, pad1;
};
__device__ __forceinline__ ArtCell load_cell(const ArtCell *p) {
  ArtCell c;
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(c.a1), "=f"(c.a2), "=f"(c.a3), "=f"(c.s1), "=f"(c.s2), "=f"(c.s3), "=f"(c.pad0), "=f"(c.pad1)
      : "l"(p));
  return c;
}

struct ArtGeom {
  int nx, ny, nz;
  float dx, dy, dz;
  float xminl, yminl, zminl, xmaxl, ymaxl, zmaxl;
  float xmin, ymin, zmin, xmax, ymax, zmax;
  double lunit;
};

// ------------------------------------------------------- recombination fits
// Case-A and case-B recombination coefficients [cm^3 s^-1] of HII, HeII and
// HeIII at temperature t [K] (diffuse_photon/diffuse_chemistry.c:13-103:
// Abel et al. 1997, Hui & Gnedin 1997 and the reference's own low-T fit);
// their difference is the rate of recombinations to the ground state,
// whose photons ionise.
__device__ double rec_hii_a(double t) {
  const double l = log(t * kKtoEV);
  double p = -3.071135243196595e-9;
  p = p * l - 1.856767039775261e-8;
  p = p * l + 5.755614137575758e-7;
  p = p * l + 4.989108920299513e-6;
  p = p * l - 0.00001421502914054107;
  p = p * l - 0.0003212605213188796;
  p = p * l - 0.002380861877349834;
  p = p * l - 0.02026044731984691;
  p = p * l - 0.7241125657826851;
  p = p * l - 28.61303380689232;
  return exp(p);
}
__device__ double rec_hii_b(double t) {
  const double lam = 2.0 * 157807.0 / t;
  return 2.753e-14 * pow(lam, 1.5) / pow(1.0 + pow(lam / 2.740, 0.407), 2.242);
}
__device__ double rec_heii_a(double t) {
  const double tev = t * kKtoEV;
  const double low = 3.92e-13 / pow(tev, 0.6353);
  if (!(tev > 0.8)) return low;
  return 1.54e-9 * (1.0 + 0.3 / exp(8.099328789667 / tev)) / (exp(40.49664394833662 / tev) * pow(tev, 1.5)) + low;
}
__device__ double rec_heii_b(double t) {
  if (t > 500.3) return 1.26e-14 * pow(2.0 * 285335.0 / t, 0.75);
  return (1.12e-10 - 2.1e-11 * log10(t)) / sqrt(t);
}
__device__ double rec_heiii_a(double t) {
  return 3.36e-10 / sqrt(t) / pow(t / 1.e3, 0.2) / (1.0 + pow(t / 1.e6, 0.7));
}
__device__ double rec_heiii_b(double t) {
  const double lam = 2.0 * 631515.0 / t;
  return 1.3765e-14 * pow(lam, 1.5) / pow(1.0 + pow(lam / 2.740, 0.407), 2.242);
}

// ------------------------------------------------------------- per cell
// Absorption coefficients [cm^-1] and source functions of the three
// frequencies (calc_rmesh_data.c:33-111, with the reference's float
// storage), and zeroed totals.  fields: 8 planes of ncell floats: dens,
// fHI, fHII, fHeI, fHeII, fHeIII, felec, uene (the prev_chem fractions and
// prev_uene of fluid_mesh).
__global__ void __launch_bounds__(256) k_art_cells(uint64_t n, const float *__restrict__ f, double denstonh,
                                                  double uenetok, float cs_hi, float cs_hei, float cs_heii,
                                                  ArtCell *__restrict__ cells, float *__restrict__ gh6) {
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < n; c += (uint64_t)gridDim.x * blockDim.x) {
    const float dens = f[c], fhi = f[n + c], fhii = f[2 * n + c], fhei = f[3 * n + c];
    const float fheii = f[4 * n + c], fheiii = f[5 * n + c], felec = f[6 * n + c], uene = f[7 * n + c];
    const float wmol = (float)(1.0 / ((1.0 + (double)felec) * kXHydrogen + 0.25 * kYHelium));
    float temper = (float)((double)uene * uenetok * (double)wmol);
    if (temper < 1.0f) temper = 1.0f;
    const double nh = (double)dens * denstonh;
    const double nhi = (double)fhi * nh, nhii = (double)fhii * nh;
    const double nhei = (double)fhei * kHeliumFact * nh;
    const double nheii = (double)fheii * kHeliumFact * nh;
    const double nheiii = (double)fheiii * kHeliumFact * nh;
    const double ne = nhii + (nheii + 2.0 * nheiii);
    const double ahi = (double)cs_hi * nhi;
    const double ahei = (double)cs_hei * nhei, aheii = (double)cs_heii * nheii;
    const float a1 = (float)(ahi + kTiny);
    const float a2 = (float)(ahi * kRcrossHI2 + ahei + kTiny);
    const float a3 = (float)(ahi * kRcrossHI3 + ahei * kRcrossHeI3 + aheii + kTiny);
    const double t = temper;
    const double e1 = (rec_hii_a(t) - rec_hii_b(t)) * ne * nhii * kNuLeV * kThrHI * kEVtoErg / (4.0 * kPi);
    const double e2 = (rec_heii_a(t) - rec_heii_b(t)) * ne * nheii * kNuLeV * kThrHeI * kEVtoErg / (4.0 * kPi);
    const double e3 = (rec_heiii_a(t) - rec_heiii_b(t)) * ne * nheiii * kNuLeV * kThrHeII * kEVtoErg / (4.0 * kPi);
    cells[c] = ArtCell{a1, a2, a3, (float)(e1 / (double)a1), (float)(e2 / (double)a2), (float)(e3 / (double)a3),
                       0.f, 0.f};
#pragma unroll
    for (int s = 0; s < 6; s++) gh6[s * n + c] = 0.f;
  }
}

// e^-tau and 1 - e^-tau in FP32: the exponential on the SFU, the
// difference by its Taylor series below tau = 1/2 (no cancellation; the
// truncation after the tau^9 term is below 3e-9 relative there).
__device__ __forceinline__ void att(float tau, float *et, float *em1) {
  *et = __expf(-tau);
  if (tau < 0.5f) {
    float p = 1.f / 362880.f;
    p = fmaf(p, -tau, 1.f / 40320.f);
    p = fmaf(p, -tau, 1.f / 5040.f);
    p = fmaf(p, -tau, 1.f / 720.f);
    p = fmaf(p, -tau, 1.f / 120.f);
    p = fmaf(p, -tau, 1.f / 24.f);
    p = fmaf(p, -tau, 1.f / 6.f);
    p = fmaf(p, -tau, 0.5f);
    p = fmaf(p, -tau, 1.f);
    *em1 = tau * p;
  } else {
    *em1 = 1.f - *et;
  }
}

// ------------------------------------------------------------- rays
// Launch shape: 256 threads, at least ARGOT_ART_MIN_CTAS CTAs per SM (the
// register cap that sets the number of rays in flight): 6 (40 registers)
// measured 8% faster than 8 (32 registers, with spills).
#ifndef ARGOT_ART_MIN_CTAS
#define ARGOT_ART_MIN_CTAS 6
#endif
// One thread per ray of angles [a0, a0 + na); acc: na planes of ncell
// float4 (sum of I (1 - e^-tau) per frequency, chord length).  A ray that
// exceeds its step bound sets *err and stops.
__global__ void __launch_bounds__(256, ARGOT_ART_MIN_CTAS) k_art_trace(ArtGeom g, const ArtAngle *__restrict__ ang, int a0, int na,
                                                  uint32_t face_max, const ArtCell *__restrict__ cells,
                                                  float4 *__restrict__ acc,
                                                  unsigned long long *__restrict__ crossings, int *__restrict__ err) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t ncell = (uint64_t)g.nx * g.ny * g.nz;
  unsigned long long steps = 0;
  if (tid < (uint64_t)na * face_max) {
    const int al = (int)(tid / face_max);
    const uint32_t r = (uint32_t)(tid % face_max);
    const ArtAngle A = ang[a0 + al];
    // start cell on the face (set_start_pos.c:150-190); consecutive threads
    // take consecutive cells along z where the face contains z, so that a
    // warp's loads and reductions fall on contiguous cells
    int i0, j0, k0;
    bool ok = true;
    if (A.base <= 1) {
      ok = r < (uint32_t)(g.nx * g.ny);
      i0 = (int)(r / g.ny); j0 = (int)(r % g.ny); k0 = A.base == 0 ? 0 : g.nz - 1;
    } else if (A.base <= 3) {
      ok = r < (uint32_t)(g.ny * g.nz);
      j0 = (int)(r / g.nz); k0 = (int)(r % g.nz); i0 = A.base == 2 ? 0 : g.nx - 1;
    } else {
      ok = r < (uint32_t)(g.nz * g.nx);
      i0 = (int)(r / g.nz); k0 = (int)(r % g.nz); j0 = A.base == 4 ? 0 : g.ny - 1;
    }
    if (ok) {
      float x = __double2float_rn(__dadd_rn((double)g.xminl, __dmul_rn(__dadd_rn((double)i0, 0.521212345), (double)g.dx)));
      float y = __double2float_rn(__dadd_rn((double)g.yminl, __dmul_rn(__dadd_rn((double)j0, 0.508512345), (double)g.dy)));
      float z = __double2float_rn(__dadd_rn((double)g.zminl, __dmul_rn(__dadd_rn((double)k0, 0.468287655), (double)g.dz)));
      switch (A.base) {
        case 0: z = g.zmin; break;
        case 1: z = g.zmax; break;
        case 2: x = g.xmin; break;
        case 3: x = g.xmax; break;
        case 4: y = g.ymin; break;
        default: y = g.ymax; break;
      }
      const float ox = A.ox, oy = A.oy, oz = A.oz;
      const int xs = ox > 0.f ? 1 : 0, ys = oy > 0.f ? 1 : 0, zs = oz > 0.f ? 1 : 0;
      const int xn = ox > 0.f ? 1 : -1, yn = oy > 0.f ? 1 : -1, zn = oz > 0.f ? 1 : -1;
      int ix = __float2int_rz(__fdiv_rn(__fsub_rn(x, g.xminl), g.dx));
      int iy = __float2int_rz(__fdiv_rn(__fsub_rn(y, g.yminl), g.dy));
      int iz = __float2int_rz(__fdiv_rn(__fsub_rn(z, g.zminl), g.dz));
      if (ox < 0.f && ix == g.nx) --ix;
      if (oy < 0.f && iy == g.ny) --iy;
      if (oz < 0.f && iz == g.nz) --iz;
      float4 *accA = acc + (uint64_t)al * ncell;
      float i1 = 0.f, i2 = 0.f, i3 = 0.f;
      const unsigned long long cap = 8ull * (g.nx + g.ny + g.nz) + 16;
      bool inside = ix >= 0 && iy >= 0 && iz >= 0 && ix < g.nx && iy < g.ny && iz < g.nz;
      while (inside) {
        if (steps >= cap) {
          atomicExch(err, 1);
          break;
        }
        steps++;
        const uint32_t pos = (uint32_t)((iz + (uint64_t)g.nz * (iy + (uint64_t)g.ny * ix)));
        // geometry in the reference's float operations (ray_tracing.c:219-246)
        const float ddx = __fsub_rn(__fmul_rn(g.dx, (float)(xs + ix)), __fsub_rn(x, g.xminl));
        const float ddy = __fsub_rn(__fmul_rn(g.dy, (float)(ys + iy)), __fsub_rn(y, g.yminl));
        const float ddz = __fsub_rn(__fmul_rn(g.dz, (float)(zs + iz)), __fsub_rn(z, g.zminl));
        float rdx = __fdiv_rn(ddx, ox), rdy = __fdiv_rn(ddy, oy), rdz = __fdiv_rn(ddz, oz);
        if (rdx < 0.f) rdx = 0.f;
        if (rdy < 0.f) rdy = 0.f;
        if (rdz < 0.f) rdz = 0.f;
        float rmin = fminf(fminf(rdx, rdy), rdz);
        x = __fadd_rn(x, __fmul_rn(rmin, ox));
        y = __fadd_rn(y, __fmul_rn(rmin, oy));
        z = __fadd_rn(z, __fmul_rn(rmin, oz));
        if (rdx == rmin) ix += xn;
        if (rdy == rmin) iy += yn;
        if (rdz == rmin) iz += zn;
        rmin = __double2float_rn(__dmul_rn((double)rmin, g.lunit));
        // intensities (calc_intensity, ray_tracing.c:71-157)
        const ArtCell cl = load_cell(cells + pos);
        float et, em;
        float4 add;
        att(__fmul_rn(cl.a1, rmin), &et, &em);
        add.x = i1 * em;
        i1 = fmaf(i1, et, cl.s1 * em);
        att(__fmul_rn(cl.a2, rmin), &et, &em);
        add.y = i2 * em;
        i2 = fmaf(i2, et, cl.s2 * em);
        att(__fmul_rn(cl.a3, rmin), &et, &em);
        add.z = i3 * em;
        i3 = fmaf(i3, et, cl.s3 * em);
        add.w = rmin;
        atomicAdd(accA + pos, add);
        // leaving the box: stop at the far face, wrap through the side faces
        // with the intensity reset (ray_tracing.c:276-372, one rank)
        if (ix >= g.nx || iy >= g.ny || iz >= g.nz || ix < 0 || iy < 0 || iz < 0) {
          if (A.base <= 1) {
            if (iz >= g.nz || iz < 0) break;
            if (ix >= g.nx) { ix = 0; x = g.xminl; i1 = i2 = i3 = 0.f; }
            else if (ix < 0) { ix = g.nx - 1; x = g.xmaxl; i1 = i2 = i3 = 0.f; }
            if (iy >= g.ny) { iy = 0; y = g.yminl; i1 = i2 = i3 = 0.f; }
            else if (iy < 0) { iy = g.ny - 1; y = g.ymaxl; i1 = i2 = i3 = 0.f; }
          } else if (A.base <= 3) {
            if (ix >= g.nx || ix < 0) break;
            if (iy >= g.ny) { iy = 0; y = g.yminl; i1 = i2 = i3 = 0.f; }
            else if (iy < 0) { iy = g.ny - 1; y = g.ymaxl; i1 = i2 = i3 = 0.f; }
            if (iz >= g.nz) { iz = 0; z = g.zminl; i1 = i2 = i3 = 0.f; }
            else if (iz < 0) { iz = g.nz - 1; z = g.zmaxl; i1 = i2 = i3 = 0.f; }
          } else {
            if (iy >= g.ny || iy < 0) break;
            if (iz >= g.nz) { iz = 0; z = g.zminl; i1 = i2 = i3 = 0.f; }
            else if (iz < 0) { iz = g.nz - 1; z = g.zmaxl; i1 = i2 = i3 = 0.f; }
            if (ix >= g.nx) { ix = 0; x = g.xminl; i1 = i2 = i3 = 0.f; }
            else if (ix < 0) { ix = g.nx - 1; x = g.xmaxl; i1 = i2 = i3 = 0.f; }
          }
        }
      }
    }
  }
  if (crossings) {
    for (int o = 16; o; o >>= 1) steps += __shfl_xor_sync(0xffffffffu, steps, o);
    if ((threadIdx.x & 31) == 0 && steps) atomicAdd(crossings, steps);
  }
}

// The batch's angles, in order, into the six per-cell totals
// (calc_GH_tot.c:178-228).  The reference evaluates each angle's terms in
// double with six divisions; here the divisions by the cell's absorption
// coefficients are hoisted out of the angle loop as FP32 reciprocals and
// each angle costs one reciprocal of its chord length and FP32 FMAs, the
// totals kept in float as the reference keeps them.  step: ionisation and
// heating factors of HI, HeI, HeII.
struct ArtStep {
  float f[6];
};
__global__ void __launch_bounds__(256) k_art_fold(uint64_t n, int na, const float4 *__restrict__ acc,
                                                 const ArtCell *__restrict__ cells, ArtStep st,
                                                 float *__restrict__ gh6) {
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < n; c += (uint64_t)gridDim.x * blockDim.x) {
    const ArtCell cl = load_cell(cells + c);
    const float4 ab = make_float4(cl.a1, cl.a2, cl.a3, 0.f), sf = make_float4(cl.s1, cl.s2, cl.s3, 0.f);
    const float ia1 = 1.f / ab.x, ia2 = 1.f / ab.y, ia3 = 1.f / ab.z;
    const float c2j = (float)kRintJHI2 * ia2, c3j = (float)kRintJHI3 * ia3;
    const float c2h = (float)kRintHHI2 * ia2, c3h = (float)kRintHHI3 * ia3;
    const float c3ej = (float)kRintJHeI3 * ia3, c3eh = (float)kRintHHeI3 * ia3;
    const float src_ghi = fmaf(sf.z, (float)kRintJHI3, fmaf(sf.y, (float)kRintJHI2, sf.x));
    const float src_hhi = fmaf(sf.z, (float)kRintHHI3, fmaf(sf.y, (float)kRintHHI2, sf.x));
    const float src_ghei = fmaf(sf.z, (float)kRintJHeI3, sf.y);
    const float src_hhei = fmaf(sf.z, (float)kRintHHeI3, sf.y);
    float g[6];
#pragma unroll
    for (int s = 0; s < 6; s++) g[s] = gh6[s * n + c];
    for (int a = 0; a < na; a++) {
      const float4 v = acc[(uint64_t)a * n + c];
      const float il = 1.f / v.w;
      const float t1 = v.x * ia1, t2 = v.y * ia2;
      g[0] = fmaf(fmaf(fmaf(v.z, c3j, fmaf(v.y, c2j, t1)), il, src_ghi), st.f[0], g[0]);
      g[3] = fmaf(fmaf(fmaf(v.z, c3h, fmaf(v.y, c2h, t1)), il, src_hhi), st.f[1], g[3]);
      g[1] = fmaf(fmaf(fmaf(v.z, c3ej, t2), il, src_ghei), st.f[2], g[1]);
      g[4] = fmaf(fmaf(fmaf(v.z, c3eh, t2), il, src_hhei), st.f[3], g[4]);
      const float t3 = fmaf(v.z * ia3, il, sf.z);
      g[2] = fmaf(t3, st.f[4], g[2]);
      g[5] = fmaf(t3, st.f[5], g[5]);
    }
#pragma unroll
    for (int s = 0; s < 6; s++) gh6[s * n + c] = g[s];
  }
}

// rates6 += totals / N_ANG (calc_GH_sum, calc_GH_tot.c:232-247)
__global__ void __launch_bounds__(256) k_art_add(uint64_t n, const float *__restrict__ gh6, float r_nang,
                                                float *__restrict__ rates6) {
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < n; c += (uint64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int s = 0; s < 6; s++) rates6[s * n + c] = __fadd_rn(rates6[s * n + c], __fmul_rn(gh6[s * n + c], r_nang));
  }
}

#ifdef ARGOT_HELIUM_LAYOUT
// fluid_mesh AoS <-> the planes of the ART kernels (the drop-in)
__global__ void __launch_bounds__(256) k_art_from_mesh(uint64_t n, const fluid_mesh *__restrict__ mesh,
                                                      float *__restrict__ f8, float *__restrict__ rates6) {
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < n; c += (uint64_t)gridDim.x * blockDim.x) {
    const fluid_mesh &m = mesh[c];
    f8[c] = m.dens;
    f8[n + c] = m.prev_chem.fHI;
    f8[2 * n + c] = m.prev_chem.fHII;
    f8[3 * n + c] = m.prev_chem.fHeI;
    f8[4 * n + c] = m.prev_chem.fHeII;
    f8[5 * n + c] = m.prev_chem.fHeIII;
    f8[6 * n + c] = m.prev_chem.felec;
    f8[7 * n + c] = m.prev_uene;
    rates6[c] = m.prev_chem.GammaHI;
    rates6[n + c] = m.prev_chem.GammaHeI;
    rates6[2 * n + c] = m.prev_chem.GammaHeII;
    rates6[3 * n + c] = m.prev_chem.HeatHI;
    rates6[4 * n + c] = m.prev_chem.HeatHeI;
    rates6[5 * n + c] = m.prev_chem.HeatHeII;
  }
}
__global__ void __launch_bounds__(256) k_art_to_mesh(uint64_t n, const float *__restrict__ rates6,
                                                    fluid_mesh *__restrict__ mesh) {
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < n; c += (uint64_t)gridDim.x * blockDim.x) {
    prim_chem &p = mesh[c].prev_chem;
    p.GammaHI = rates6[c];
    p.GammaHeI = rates6[n + c];
    p.GammaHeII = rates6[2 * n + c];
    p.HeatHI = rates6[3 * n + c];
    p.HeatHeI = rates6[4 * n + c];
    p.HeatHeII = rates6[5 * n + c];
  }
}

#endif  // ARGOT_HELIUM_LAYOUT

int art_blocks(uint64_t n) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t want = (n + 255) / 256;
  return (int)(want < (uint64_t)sms * 8 ? (want ? want : 1) : (uint64_t)sms * 8);
}

// ------------------------------------------------------------- host tables
// HEALPix RING pixel centres (Gorski et al. 2005, ApJ 622, 759, section 4):
// polar-cap rings i = 1..nside-1 with 4 i pixels at z = 1 - i^2/(3 nside^2),
// equatorial rings of 4 nside pixels at z = 4/3 - 2 i/(3 nside) with every
// other ring shifted by half a pixel, the south cap mirrored.
long isqrt_l(long v) {
  long r = (long)std::sqrt((double)v + 0.5);
  while (r * r > v) r--;
  while ((r + 1) * (r + 1) <= v) r++;
  return r;
}
void ring_pix2ang(long nside, long ipix, double *theta, double *phi) {
  const long npix = 12 * nside * nside;
  const long ncap = 2 * nside * (nside - 1);
  const double pi = 3.141592653589793238462643383279502884197;
  double z;
  if (ipix < ncap) {
    const long iring = (1 + isqrt_l(1 + 2 * ipix)) >> 1;
    const long iphi = ipix + 1 - 2 * iring * (iring - 1);
    z = 1.0 - (double)(iring * iring) / (3.0 * (double)(nside * nside));
    *phi = ((double)iphi - 0.5) * pi / (2.0 * (double)iring);
  } else if (ipix < npix - ncap) {
    const long ip = ipix - ncap;
    const long iring = ip / (4 * nside) + nside;
    const long iphi = ip % (4 * nside) + 1;
    const double fodd = ((iring + nside) & 1) ? 1.0 : 0.5;
    z = (double)(2 * nside - iring) * 2.0 / (3.0 * (double)nside);
    *phi = ((double)iphi - fodd) * pi / (2.0 * (double)nside);
  } else {
    const long ip = npix - ipix;
    const long iring = (1 + isqrt_l(2 * ip - 1)) >> 1;
    const long iphi = 4 * iring + 1 - (ip - 2 * iring * (iring - 1));
    z = -1.0 + (double)(iring * iring) / (3.0 * (double)(nside * nside));
    *phi = ((double)iphi - 0.5) * pi / (2.0 * (double)iring);
  }
  *theta = std::acos(z);
}

// the start face of a direction (set_angle.c:70-96): the axis whose
// component dominates, entered from its low side (even id) or high side
int start_face(double cphi, double sphi, double ttheta) {
  const double c4 = std::cos(0.7853981633974483096156608458198757);
  const double rc = 1.0 / std::fabs(cphi), rs = 1.0 / std::fabs(sphi);
  if (std::fabs(cphi) >= c4) {
    if (0.0 <= ttheta && ttheta <= rc) return 0;
    if (-rc <= ttheta && ttheta < 0.0) return 1;
    return cphi >= 0.0 ? 2 : 3;
  }
  if (0.0 <= ttheta && ttheta <= rs) return 0;
  if (-rs <= ttheta && ttheta < 0.0) return 1;
  return sphi >= 0.0 ? 4 : 5;
}

// the octant (set_angle.c:100-147)
int octant(double cphi, double sphi, double ctheta) {
  return (cphi > 0.0 ? 0 : 4) + (sphi > 0.0 ? 0 : 2) + (ctheta > 0.0 ? 0 : 1);
}

// Integrals over the first 0.063 nu_L above each edge of 4 pi sigma / (h nu)
// (ionisation) and of the same times (nu - nu_s) (heating), trapezoidal on
// 64 bins with the reference's float accumulation (set_step_func_factor.c)
void step_factors(float out[6]) {
  const double thr[3] = {kThrHI, kThrHeI, kThrHeII};
  const double nul[3] = {3.2885e15, 5.9483e15, 1.3154e16};
  double (*sig[3])(double) = {sigma_hi, sigma_hei, sigma_heii};
  float f[3][2] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
  const double block = kStepRange / kStepBins;
  for (int k = 0; k < kStepBins; k++) {
    for (int s = 0; s < 3; s++) {
      double nu = thr[s] + k * block, nu1 = thr[s] + (k + 1) * block;
      if (nu == thr[s]) nu = thr[s] + 1e-7;
      if (nu1 == thr[s]) nu1 = thr[s] + 1e-7;
      const double c0 = 4.0e0 * kPi * sig[s](nu) / (kHPlanck * (nu * nul[s]));
      const double c0n = 4.0e0 * kPi * sig[s](nu1) / (kHPlanck * (nu1 * nul[s]));
      const double h0 = k == 0 ? 0.0 : c0 * (nu - thr[s]);
      const double h0n = c0 * (nu1 - thr[s]);
      f[s][0] = (float)((double)f[s][0] + (c0 + c0n) * 0.5e0);
      f[s][1] = (float)((double)f[s][1] + (h0 + h0n) * 0.5e0);
    }
  }
  for (int s = 0; s < 3; s++) {
    out[2 * s] = f[s][0] / (float)kStepBins;
    out[2 * s + 1] = (float)((double)f[s][1] / ((double)kStepBins / (kHPlanck * nul[s])));
  }
}

}  // namespace argot

struct argot_b200_art {
  int device;
  int nang;
  argot::ArtAngle *dev_ang;
  argot::ArtStep step;
};

using namespace argot;

namespace {

int art_run(const argot_b200_art *a, const ArtGeom &g, double denstonh, double uenetok, const float *fields8,
            float *rates6, void *work, int apass, unsigned long long *crossings, int *err, cudaStream_t st) {
  const uint64_t n = (uint64_t)g.nx * g.ny * g.nz;
  ArtCell *cells = (ArtCell *)work;
  float4 *acc = (float4 *)(cells + n);
  float *gh6 = (float *)(acc + (uint64_t)apass * n);
  const int blocks = art_blocks(n);
  const float cs1 = (float)sigma_hi(kThrHI + 1.0e-7), cs2 = (float)sigma_hei(kThrHeI + 1.0e-7);
  const float cs3 = (float)sigma_heii(kThrHeII + 1.0e-7);
  k_art_cells<<<blocks, 256, 0, st>>>(n, fields8, denstonh, uenetok, cs1, cs2, cs3, cells, gh6);
  ARGOT_CUDA_TRY(cudaGetLastError());
  const uint32_t face_max = (uint32_t)std::max<uint64_t>(
      (uint64_t)g.nx * g.ny, std::max<uint64_t>((uint64_t)g.ny * g.nz, (uint64_t)g.nz * g.nx));
  for (int a0 = 0; a0 < a->nang; a0 += apass) {
    const int na = std::min(apass, a->nang - a0);
    ARGOT_CUDA_TRY(cudaMemsetAsync(acc, 0, sizeof(float4) * n * (uint64_t)na, st));
    const uint64_t threads = (uint64_t)na * face_max;
    k_art_trace<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(g, a->dev_ang, a0, na, face_max, cells, acc,
                                                                    crossings, err);
    ARGOT_CUDA_TRY(cudaGetLastError());
    k_art_fold<<<blocks, 256, 0, st>>>(n, na, acc, cells, a->step, gh6);
    ARGOT_CUDA_TRY(cudaGetLastError());
  }
  const float r_nang = (float)(1.0e0 / a->nang);
  k_art_add<<<blocks, 256, 0, st>>>(n, gh6, r_nang, rates6);
  ARGOT_CUDA_TRY(cudaGetLastError());
  return 0;
}

bool art_geom_from_grid(const argot_b200_grid *gp, ArtGeom *g) {
  if (!grid_valid(gp)) return false;
  const uint64_t n = (uint64_t)gp->nx * gp->ny * gp->nz;
  if (n >= (1ull << 32)) return false;
  g->nx = gp->nx; g->ny = gp->ny; g->nz = gp->nz;
  g->dx = gp->dx; g->dy = gp->dy; g->dz = gp->dz;
  g->xminl = gp->xmin_local; g->yminl = gp->ymin_local; g->zminl = gp->zmin_local;
  // one rank: the local domain is the box
  g->xmaxl = gp->xmax; g->ymaxl = gp->ymax; g->zmaxl = gp->zmax;
  g->xmin = gp->xmin; g->ymin = gp->ymin; g->zmin = gp->zmin;
  g->xmax = gp->xmax; g->ymax = gp->ymax; g->zmax = gp->zmax;
  g->lunit = gp->lunit;
  return true;
}

}  // namespace

namespace argot {
int *err_flag(int dev);
int check_err_flag(int *flag, cudaStream_t st);
}  // namespace argot

#ifdef ARGOT_HELIUM_LAYOUT
namespace argot {

// Buffers of the drop-in, kept across calls.
struct ArtDropin {
  std::mutex mu;
  argot_b200_art *art = nullptr;
  std::vector<angle_info> table;
  std::vector<float> step;
  void *buf = nullptr;
  size_t bytes = 0;
};
ArtDropin g_art_dropin;

int art_dropin(run_param *run, cuda_mem_space *cm, cuda_param *cp, host_diffuse_param *hd) {
  if (!run || !cm || !cm[0].mesh_dev || !hd || !hd->angle || !hd->step_fact) return ARGOT_B200_EINVAL;
  int nang = 0;
  for (int c = 0; c < 8; c++) {
    if (hd->corner_id_num[c] < 0) return ARGOT_B200_EINVAL;
    nang += hd->corner_id_num[c];
  }
  if (nang < 1) return ARGOT_B200_EINVAL;
  ArtGeom g;
  g.nx = run->nmesh_x_local; g.ny = run->nmesh_y_local; g.nz = run->nmesh_z_local;
  if (g.nx <= 0 || g.ny <= 0 || g.nz <= 0) return ARGOT_B200_EINVAL;
  const uint64_t n = (uint64_t)g.nx * g.ny * g.nz;
  if (n >= (1ull << 32)) return ARGOT_B200_EINVAL;
  g.dx = run->delta_x; g.dy = run->delta_y; g.dz = run->delta_z;
  if (!(g.dx > 0.f && g.dy > 0.f && g.dz > 0.f)) return ARGOT_B200_EINVAL;
  g.xminl = run->xmin_local; g.yminl = run->ymin_local; g.zminl = run->zmin_local;
  g.xmaxl = run->xmax_local; g.ymaxl = run->ymax_local; g.zmaxl = run->zmax_local;
  g.xmin = run->xmin; g.ymin = run->ymin; g.zmin = run->zmin;
  g.xmax = run->xmax; g.ymax = run->ymax; g.zmax = run->zmax;
  g.lunit = run->lunit;
  int prev = 0;
  ARGOT_CUDA_TRY(cudaGetDevice(&prev));
  ARGOT_CUDA_TRY(cudaSetDevice(0));
  struct Restore {
    int d;
    ~Restore() { cudaSetDevice(d); }
  } restore{prev};
  std::lock_guard<std::mutex> lock(g_art_dropin.mu);
  ArtDropin &D = g_art_dropin;
  const float step6[6] = {hd->step_fact->HI[0], hd->step_fact->HI[1], hd->step_fact->HeI[0],
                          hd->step_fact->HeI[1], hd->step_fact->HeII[0], hd->step_fact->HeII[1]};
  const bool same = D.art && D.table.size() == (size_t)nang &&
                    !std::memcmp(D.table.data(), hd->angle, sizeof(angle_info) * (size_t)nang) &&
                    !std::memcmp(D.step.data(), step6, sizeof(step6));
  if (!same) {
    std::vector<float> dir(3 * (size_t)nang);
    std::vector<int> bc(2 * (size_t)nang);
    for (int i = 0; i < nang; i++) {
      dir[3 * i] = hd->angle[i].xovr; dir[3 * i + 1] = hd->angle[i].yovr; dir[3 * i + 2] = hd->angle[i].zovr;
      bc[2 * i] = hd->angle[i].base_id; bc[2 * i + 1] = hd->angle[i].corner_id;
    }
    argot_b200_art *a = nullptr;
    const int rc = argot_b200_art_create(dir.data(), bc.data(), nang, step6, &a);
    if (rc) return rc;
    argot_b200_art_destroy(D.art);
    D.art = a;
    D.table.assign(hd->angle, hd->angle + nang);
    D.step.assign(step6, step6 + 6);
  }
  // angles per pass: about a million rays in flight, within 2 GB of
  // accumulators
  const uint64_t face = std::max<uint64_t>((uint64_t)g.nx * g.ny,
                                           std::max<uint64_t>((uint64_t)g.ny * g.nz, (uint64_t)g.nz * g.nx));
  int apass = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)nang, (1ull << 20) / face));
  apass = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)apass, (2ull << 30) / (16 * n)));
  const size_t need = sizeof(float) * 14 * n + 32 + (size_t)(n * (32 + 24) + n * 16 * (uint64_t)apass);
  if (need > D.bytes) {
    if (D.buf) cudaFree(D.buf);
    D.buf = nullptr;
    D.bytes = 0;
    ARGOT_CUDA_TRY(cudaMalloc(&D.buf, need));
    D.bytes = need;
  }
  float *f8 = (float *)D.buf;
  float *r6 = f8 + 8 * n;
  void *work = (void *)(((uintptr_t)(r6 + 6 * n) + 31) & ~(uintptr_t)31);
  cudaStream_t st = (cp && cp->num_cuda_dev > 0) ? (cudaStream_t)cp->strm[0] : (cudaStream_t)0;
  int *err = err_flag(0);
  if (!err) return ARGOT_B200_ENOMEM;
  const int blocks = art_blocks(n);
  k_art_from_mesh<<<blocks, 256, 0, st>>>(n, cm[0].mesh_dev, f8, r6);
  ARGOT_CUDA_TRY(cudaGetLastError());
  int rc = art_run(D.art, g, run->denstonh, run->uenetok, f8, r6, work, apass, nullptr, err, st);
  if (rc) return rc;
  k_art_to_mesh<<<blocks, 256, 0, st>>>(n, r6, cm[0].mesh_dev);
  ARGOT_CUDA_TRY(cudaGetLastError());
  return check_err_flag(err, st);
}

}  // namespace argot
#endif  // ARGOT_HELIUM_LAYOUT

extern "C" {

int argot_b200_art_angle_table(int nside, float *dir3, int *base_corner2, int *corner_count8) {
  if (nside < 1 || nside > 1024 || !dir3 || !base_corner2) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  const long npix = 12L * nside * nside;
  struct Row {
    float d[3];
    int base, corner;
  };
  std::vector<Row> rows((size_t)npix);
  for (long p = 0; p < npix; p++) {
    double th, ph;
    ring_pix2ang(nside, p, &th, &ph);
    const double ct = std::cos(th), st = std::sin(th), cp = std::cos(ph), sp = std::sin(ph), tt = std::tan(th);
    double o[3] = {st * cp, st * sp, ct};
    Row &r = rows[(size_t)p];
    for (int k = 0; k < 3; k++) {
      if (std::fabs(o[k]) < kTiny) o[k] = o[k] >= 0.0 ? kTiny : -kTiny;
      r.d[k] = (float)o[k];
    }
    r.base = start_face(cp, sp, tt);
    r.corner = octant(cp, sp, ct);
  }
  // the reference's processing order: by octant, then by start face, the
  // pixel order kept within each (sort_angle_id, set_angle.c:174-246)
  std::stable_sort(rows.begin(), rows.end(), [](const Row &a, const Row &b) {
    return a.corner != b.corner ? a.corner < b.corner : a.base < b.base;
  });
  if (corner_count8)
    for (int c = 0; c < 8; c++) corner_count8[c] = 0;
  for (long p = 0; p < npix; p++) {
    const Row &r = rows[(size_t)p];
    for (int k = 0; k < 3; k++) dir3[3 * p + k] = r.d[k];
    base_corner2[2 * p] = r.base;
    base_corner2[2 * p + 1] = r.corner;
    if (corner_count8) corner_count8[r.corner]++;
  }
  set_status(0);
  return (int)npix;
}

void argot_b200_art_step_factors(float *step6) {
  if (step6) step_factors(step6);
}

int argot_b200_art_create(const float *dir3, const int *base_corner2, int nang, const float *step6,
                          argot_b200_art **out) {
  if (!dir3 || !base_corner2 || !step6 || !out || nang < 1) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  std::vector<ArtAngle> h((size_t)nang);
  for (int i = 0; i < nang; i++) {
    const int b = base_corner2[2 * i];
    if (b < 0 || b > 5 || !(dir3[3 * i] != 0.f) || !(dir3[3 * i + 1] != 0.f) || !(dir3[3 * i + 2] != 0.f)) {
      set_status(ARGOT_B200_EINVAL);
      return ARGOT_B200_EINVAL;
    }
    h[(size_t)i] = ArtAngle{dir3[3 * i], dir3[3 * i + 1], dir3[3 * i + 2], b};
  }
  argot_b200_art *a = new (std::nothrow) argot_b200_art();
  if (!a) { set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  a->nang = nang;
  for (int s = 0; s < 6; s++) a->step.f[s] = step6[s];
  cudaError_t e = cudaGetDevice(&a->device);
  if (e == cudaSuccess) e = cudaMalloc(&a->dev_ang, sizeof(ArtAngle) * (size_t)nang);
  if (e == cudaSuccess)
    e = cudaMemcpy(a->dev_ang, h.data(), sizeof(ArtAngle) * (size_t)nang, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    if (a->dev_ang) cudaFree(a->dev_ang);
    delete a;
    return status_from_cuda(e);
  }
  *out = a;
  set_status(0);
  return 0;
}

void argot_b200_art_destroy(argot_b200_art *a) {
  if (!a) return;
  cudaFree(a->dev_ang);
  delete a;
}

int argot_b200_art_num_angles(const argot_b200_art *a) { return a ? a->nang : 0; }

#ifdef ARGOT_HELIUM_LAYOUT
// calc_diffuse_photon_radiation as built with __USE_GPU__
// (calc_diffuse_photon_radiation.c:37-128) on one rank: the angle table and
// step factors the caller's setup_diffuse_photon filled in hd_param, the
// mesh from cuda_mem[0].mesh_dev, the diffuse rates added to its prev_chem
// there.  cd_param and this_omp are not used (the device buffers are this
// library's own).
void calc_diffuse_photon_radiation(::fluid_mesh *mesh, ::run_param *this_run, ::cuda_mem_space *cuda_mem,
                                   ::cuda_param *this_cuda, ::host_diffuse_param *hd_param,
                                   ::cuda_diffuse_param *cd_param, ::omp_param *this_omp) {
  (void)mesh; (void)cd_param; (void)this_omp;
  argot::dropin_status((argot::run_param *)this_run, "calc_diffuse_photon_radiation",
                       argot::art_dropin((argot::run_param *)this_run, (argot::cuda_mem_space *)cuda_mem,
                                         (argot::cuda_param *)this_cuda, (argot::host_diffuse_param *)hd_param));
}
#endif  // ARGOT_HELIUM_LAYOUT

uint64_t argot_b200_art_workspace(const argot_b200_grid *g, int angles_per_pass) {
  if (!grid_valid(g) || angles_per_pass < 1) return 0;
  const uint64_t n = (uint64_t)g->nx * g->ny * g->nz;
  return n * (sizeof(ArtCell) + 6 * sizeof(float)) + n * sizeof(float4) * (uint64_t)angles_per_pass;
}

int argot_b200_art_rates(const argot_b200_art *a, const argot_b200_grid *gp, double uenetok, const float *fields8,
                         float *rates6, void *work, int angles_per_pass, unsigned long long *crossings,
                         void *stream) {
  ArtGeom g;
  if (!a || !fields8 || !rates6 || !work || ((uintptr_t)work & 31) || angles_per_pass < 1 ||
      !art_geom_from_grid(gp, &g) || !(uenetok > 0.0)) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  int dev = 0;
  ARGOT_CUDA_TRY(cudaGetDevice(&dev));
  int *err = err_flag(dev);
  if (!err) { set_status(ARGOT_B200_ENOMEM); return ARGOT_B200_ENOMEM; }
  const int rc = art_run(a, g, gp->denstonh, uenetok, fields8, rates6, work, angles_per_pass, crossings, err,
                         (cudaStream_t)stream);
  set_status(rc);
  return rc;
}

}  // extern "C"
