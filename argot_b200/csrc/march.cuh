// march.cuh -- device functions of the segment march (calc_optical_depth).
#pragma once
#include "common.cuh"

namespace argot {

struct Tau3 {
  float hi, hei, heii;
};

// NC columns of a segment (the drop-in's flag sets carry 1 to 6 species).
template <int NC>
struct Cols {
  float v[NC];
};

// Packed cells with NC species: (NC + 3) / 4 float4 per cell, species in
// column order (one float4 {n_HI, n_HeI, n_HeII, 0} for the default set).
template <int NC>
__device__ __forceinline__ void ld_cols(const float4 *__restrict__ cells, size_t c, float (&n)[NC]) {
  constexpr int NG = (NC + 3) / 4;
#pragma unroll
  for (int q = 0; q < NG; q++) {
    const float4 f = __ldg(cells + c * NG + q);
    if (4 * q + 0 < NC) n[(4 * q + 0) % NC] = f.x;
    if (4 * q + 1 < NC) n[(4 * q + 1) % NC] = f.y;
    if (4 * q + 2 < NC) n[(4 * q + 2) % NC] = f.z;
    if (4 * q + 3 < NC) n[(4 * q + 3) % NC] = f.w;
  }
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ size_t cell_index(const GridDev &g, int ix, int iy, int iz) {
  return (size_t)iz + (size_t)g.nz * ((size_t)iy + (size_t)g.ny * (size_t)ix);
}

// Cell index of a coordinate along one axis, truncated toward zero and
// clamped into the local mesh (calc_optical_depth.c:76-90).
__device__ __forceinline__ int axis_cell(float p, float lo, float d, int n) {
  return clampi(__float2int_rz(__fdiv_rn(__fsub_rn(p, lo), d)), 0, n - 1);
}

// The reference's guard against vanishing direction cosines: |c| < TINY
// becomes +-TINY with the sign test c >= 0 (calc_optical_depth.c:107-120).
__device__ __forceinline__ float cosine_guard(float c) {
  return (fabs((double)c) < kTiny) ? ((c >= 0.f) ? (float)kTiny : -(float)kTiny) : c;
}

// ---------------------------------------------------------------------------
// Reference-order march.  Every operation is the reference's, in its order
// and precision (calc_optical_depth.c:65-227): round-to-nearest single
// operations with no contraction into FMA, double where the reference's
// double literals promote, IEEE division.  Results equal the reference CPU
// build bit for bit.  `*steps` receives the number of cells visited (the
// loop iterations plus the end cell); `*bad` is set when the walk exceeds
// nx+ny+nz+2 steps (only possible for non-finite input).
template <int NC>
static __device__ __noinline__ Cols<NC> march_reference_n(const GridDev &g, const float4 *__restrict__ cells,
                                                          float xs, float ys, float zs, float xe, float ye,
                                                          float ze, int *steps, bool *bad) {
  const int ixe = axis_cell(xe, g.xminl, g.dx, g.nx);
  const int iye = axis_cell(ye, g.yminl, g.dy, g.ny);
  const int ize = axis_cell(ze, g.zminl, g.dz, g.nz);
  int ix = axis_cell(xs, g.xminl, g.dx, g.nx);
  int iy = axis_cell(ys, g.yminl, g.dy, g.ny);
  int iz = axis_cell(zs, g.zminl, g.dz, g.nz);

  const float dx = __fsub_rn(xe, xs), dy = __fsub_rn(ye, ys), dz = __fsub_rn(ze, zs);
  const float sxy = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
  const float s3 = __fadd_rn(sxy, __fmul_rn(dz, dz));
  const float dl = __double2float_rn(__dsqrt_rn(__dadd_rn((double)s3, kTiny)));
  const float dxy = __double2float_rn(__dsqrt_rn((double)sxy));
  const float cos_t = __fdiv_rn(dz, dl), sin_t = __fdiv_rn(dxy, dl);
  const double den = __dadd_rn((double)dxy, kTiny);
  const float cos_p = __double2float_rn(__ddiv_rn((double)dx, den));
  const float sin_p = __double2float_rn(__ddiv_rn((double)dy, den));
  const float xo = cosine_guard(__fmul_rn(cos_p, sin_t));
  const float yo = cosine_guard(__fmul_rn(sin_p, sin_t));
  const float zo = cosine_guard(cos_t);
  const int sx = xo > 0.f ? 1 : 0, nxs = xo > 0.f ? 1 : -1;
  const int sy = yo > 0.f ? 1 : 0, nys = yo > 0.f ? 1 : -1;
  const int sz = zo > 0.f ? 1 : 0, nzs = zo > 0.f ? 1 : -1;

  float xc = __fsub_rn(xs, g.xminl), yc = __fsub_rn(ys, g.yminl), zc = __fsub_rn(zs, g.zminl);
  Cols<NC> t;
#pragma unroll
  for (int q = 0; q < NC; q++) t.v[q] = 0.f;
  int it = 0;
  const int cap = g.nx + g.ny + g.nz + 2;
  while ((ix != ixe || iy != iye || iz != ize) && (unsigned)ix < (unsigned)g.nx &&
         (unsigned)iy < (unsigned)g.ny && (unsigned)iz < (unsigned)g.nz) {
    if (++it > cap) { *bad = true; break; }
    float n[NC];
    ld_cols<NC>(cells, cell_index(g, ix, iy, iz), n);
    const float ddx = __fsub_rn(__fmul_rn(g.dx, __int2float_rn(sx + ix)), xc);
    const float ddy = __fsub_rn(__fmul_rn(g.dy, __int2float_rn(sy + iy)), yc);
    const float ddz = __fsub_rn(__fmul_rn(g.dz, __int2float_rn(sz + iz)), zc);
    const float rx = __fdiv_rn(ddx, xo), ry = __fdiv_rn(ddy, yo), rz = __fdiv_rn(ddz, zo);
    const float rmin = fminf(rx, fminf(ry, rz));
    if (rmin == rx) ix += nxs;
    if (rmin == ry) iy += nys;
    if (rmin == rz) iz += nzs;
    xc = __fadd_rn(xc, __fmul_rn(rmin, xo));
    yc = __fadd_rn(yc, __fmul_rn(rmin, yo));
    zc = __fadd_rn(zc, __fmul_rn(rmin, zo));
#pragma unroll
    for (int q = 0; q < NC; q++) t.v[q] = __fadd_rn(t.v[q], __fmul_rn(rmin, n[q]));
  }
  xc = __fadd_rn(xc, g.xminl);
  yc = __fadd_rn(yc, g.yminl);
  zc = __fadd_rn(zc, g.zminl);
  const float ex = __fsub_rn(xe, xc), ey = __fsub_rn(ye, yc), ez = __fsub_rn(ze, zc);
  const float e3 = __fadd_rn(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)), __fmul_rn(ez, ez));
  const float depth = __double2float_rn(__dsqrt_rn((double)e3));
  float ne[NC];
  ld_cols<NC>(cells, cell_index(g, ixe, iye, ize), ne);
#pragma unroll
  for (int q = 0; q < NC; q++) t.v[q] = __fadd_rn(t.v[q], __fmul_rn(depth, ne[q]));
  *steps = it + 1;
  return t;
}

// The three-column march of the device path.
__device__ __forceinline__ Tau3 march_reference(const GridDev &g, const float4 *__restrict__ cells, float xs,
                                                float ys, float zs, float xe, float ye, float ze, int *steps,
                                                bool *bad) {
  const Cols<3> c = march_reference_n<3>(g, cells, xs, ys, zs, xe, ye, ze, steps, bad);
  return Tau3{c.v[0], c.v[1], c.v[2]};
}

// Compensated (Kahan) summation step: s + c carries the running sum.
__device__ __forceinline__ void kahan_add(float &s, float &c, float v) {
  const float y = v - c;
  const float tt = s + y;
  c = (tt - s) - y;
  s = tt;
}

// ---------------------------------------------------------------------------
// Count-down march with compensated sums.  Same start / end cell rules as
// the reference.  Along each axis the walk must cross exactly
// |i_end - i_start| faces.  Per axis it keeps the number of faces still to
// cross and the path length from the start point to the next one; every
// step takes the nearest face among the axes that still have faces to
// cross, the chord from the previous crossing to it belongs to the current
// cell, and the crossed axes advance to their following face by the face
// spacing dX/|u_x|.  The walk always ends in the end cell after at most
// sum|di| steps.  Columns are FP32 with compensated (Kahan) summation.
// (Testing the next face against the position of each axis's last face
// instead of keeping counts executes 9% fewer instructions but takes more
// selects and spills at 32 registers: 4% slower, measured.)
//
// Path lengths are unsigned fixed-point integers.  Every chord is a
// difference of two path lengths to faces, and the face spacing of a
// slanted axis is a multi-cell distance: FP32 countdowns round both (1e-7
// of them per step and per reset), which drifts along the ray and, measured
// on a 32^3 lognormal mesh, put 2e-5 relative error into minor-species
// columns that one short chord dominates.  Integer differences are exact.
// The unit is 2^-k of the largest cell side, with k per ray the largest
// that keeps the ray length below 2^31 units (2^-22 of a cell for rays of
// up to 256 cells); a face position is held as 32.32 bits, so the spacing
// is added with a 64-bit carry and its rounding (2^-32 unit per face) never
// accumulates to a unit.  The chord, an integer number of units below 2^31,
// converts to FP32 with one rounding and the column sums are scaled back by
// the unit at the end.  The per-ray set-up (cosines, spacings, first
// faces) is formed once per ray in FP64: its inputs are differences of
// box-scale coordinates.  Columns agree with an FP64 march to ~3e-7.
//
// The walk's geometry does not depend on the densities, so the compiler
// issues a step's gather ahead of the previous steps' sums (an explicit
// one-step-ahead gather held four more registers and measured no faster).
// Chords are summed with FMA into per-species partial sums that are folded
// into the Kahan sums every 16 steps (compensated summation over blocks of
// 16 terms).  The last chord runs from the latest face crossing to the end
// point.  kSlotStride > 0: the Kahan sums live in per-thread shared-memory
// slots (`slot`, words kSlotStride apart), touched once per 16 steps, which
// frees six registers for the walk.
// kCentreEnd: the end point is the centre of its cell (every ray of the
// device path).  Then every face still to cross lies at least half a cell
// before the end point along the ray and the next face of an axis that has
// none left at least half a cell past it, both far more than the 2^-32
// unit per face that the fixed-point positions can drift, so the walk
// needs no face counts: it ends when the nearest face lies at or past the
// end point, and a crossed axis always advances to its next face.  The
// faces taken, their order and the columns are those of the counting walk
// (three registers and about six instructions per step fewer).
// Kahan step on a column kept in per-thread shared-memory slots: sum in
// word q, compensation in word q + NC (words kStride apart).
template <int NC, int kStride>
__device__ __forceinline__ void kahan_slot(float *slot, int q, float v) {
  float s = slot[q * kStride], c = slot[(q + NC) * kStride];
  kahan_add(s, c, v);
  slot[q * kStride] = s;
  slot[(q + NC) * kStride] = c;
}

// The step of one axis in the end-tested walk: when the axis's next face
// is the nearest (h == m), its face position t moves on by the spacing T
// and the cell index by ds.  Written as two predicated adds, where the
// compiler's form (both sums formed, then selected) took twice the
// instructions (ncu, 256^3 / 4096 sources: march 0.98 s -> 0.93 s).
__device__ __forceinline__ void advance_if_hit(uint64_t &t, int &idx, uint32_t h, uint32_t m, uint64_t T, int ds) {
  asm("{\n\t.reg .pred p;\n\tsetp.eq.u32 p, %2, %3;\n\t@p add.u64 %0, %0, %4;\n\t@p add.s32 %1, %1, %5;\n\t}"
      : "+l"(t), "+r"(idx)
      : "r"(h), "r"(m), "l"(T), "r"(ds));
}

__device__ __forceinline__ uint64_t fixed_32_32(double units) {
  return (uint64_t)__double2ull_rz(units * 4294967296.0);
}

template <int NC, int kSlotStride = 0, bool kCentreEnd = false>
static __device__ __forceinline__ Cols<NC> march_kahan_n(const GridDev &g, const float4 *__restrict__ cells,
                                                         float xs, float ys, float zs, float xe, float ye,
                                                         float ze, int *steps, bool *bad, float *slot = nullptr) {
  const int ixe = axis_cell(xe, g.xminl, g.dx, g.nx);
  const int iye = axis_cell(ye, g.yminl, g.dy, g.ny);
  const int ize = axis_cell(ze, g.zminl, g.dz, g.nz);
  const int ix = axis_cell(xs, g.xminl, g.dx, g.nx);
  const int iy = axis_cell(ys, g.yminl, g.dy, g.ny);
  const int iz = axis_cell(zs, g.zminl, g.dz, g.nz);
  // differences of floats are exact in double
  const double x0 = (double)xs - (double)g.xminl, y0 = (double)ys - (double)g.yminl,
               z0 = (double)zs - (double)g.zminl;
  const double dx = (double)xe - (double)xs, dy = (double)ye - (double)ys, dz = (double)ze - (double)zs;
  const double len = sqrt(fma(dx, dx, fma(dy, dy, dz * dz)));
  if (!(len <= 1.0e30)) *bad = true;  // non-finite end points
  // 1/|cosine| per axis, with the reference's floor of 1e-31 on |cosine|
  const double iax = len / fmax(fabs(dx), kTiny * len), iay = len / fmax(fabs(dy), kTiny * len),
               iaz = len / fmax(fabs(dz), kTiny * len);
  int cx = abs(ixe - ix), cy = abs(iye - iy), cz = abs(ize - iz);
  const int stx = ixe > ix ? 1 : -1, sty = iye > iy ? 1 : -1, stz = ize > iz ? 1 : -1;
  // the unit: 2^-k of the largest cell side, the ray length below 2^31 units
  const double dmax = fmax((double)g.dx, fmax((double)g.dy, (double)g.dz));
  const int k = min(40, 30 - ilogb(len / dmax + 2.0));
  const double sc = ldexp(1.0, k) / dmax;  // box lengths -> units
  // path lengths of the first face of each axis and the face spacings,
  // 32.32 fixed point; an axis without faces to cross never comes next
  const uint64_t kNone = ~0ull;
  uint64_t tx = cx ? fixed_32_32(fabs(fma((double)g.dx, (double)(ix + (stx > 0)), -x0)) * iax * sc) : kNone;
  uint64_t ty = cy ? fixed_32_32(fabs(fma((double)g.dy, (double)(iy + (sty > 0)), -y0)) * iay * sc) : kNone;
  uint64_t tz = cz ? fixed_32_32(fabs(fma((double)g.dz, (double)(iz + (stz > 0)), -z0)) * iaz * sc) : kNone;
  // a spacing is used only while its axis has faces left, then it is
  // shorter than the ray (below 2^31 units)
  const uint64_t Tx = fixed_32_32(fmin((double)g.dx * iax * sc, 2147483648.0));
  const uint64_t Ty = fixed_32_32(fmin((double)g.dy * iay * sc, 2147483648.0));
  const uint64_t Tz = fixed_32_32(fmin((double)g.dz * iaz * sc, 2147483648.0));
  const uint32_t lu = (uint32_t)__double2uint_rn(fmin(len * sc, 2147483648.0));
  const int dsz = stz, dsy = sty * g.nz, dsx = stx * g.nz * g.ny;
  int idx = iz + g.nz * (iy + g.ny * ix);

  float p[NC], s[NC], c[NC];
#pragma unroll
  for (int q = 0; q < NC; q++) p[q] = s[q] = c[q] = 0.f;
  if (kSlotStride) {
#pragma unroll
    for (int q = 0; q < 2 * NC; q++) slot[q * kSlotStride] = 0.f;
  }
  uint32_t t = 0;  // path length of the latest crossing (units)
  int it = 0;
  // blocks of 16 steps (unrolled; the Kahan fold once per block, so only
  // "faces left" is tested per step).  Every step crosses the face of at
  // least one axis with faces left, so the walk ends.
  for (;;) {
    int kk = 0;
#pragma unroll
    for (; kk < 16; kk++) {
      const uint32_t xh = (uint32_t)(tx >> 32), yh = (uint32_t)(ty >> 32), zh = (uint32_t)(tz >> 32);
      const uint32_t m = min(xh, min(yh, zh));
      if (kCentreEnd ? m >= lu : !(cx | cy | cz)) break;
      if (kCentreEnd) {
        float n[NC];
        ld_cols<NC>(cells, (size_t)idx, n);
        advance_if_hit(tx, idx, xh, m, Tx, dsx);
        advance_if_hit(ty, idx, yh, m, Ty, dsy);
        advance_if_hit(tz, idx, zh, m, Tz, dsz);
        const float rf = __uint2float_rn(m - t);
        t = m;
#pragma unroll
        for (int q = 0; q < NC; q++) p[q] = fmaf(rf, n[q], p[q]);
        continue;
      }
      const bool hx = xh == m, hy = yh == m, hz = zh == m;
      float n[NC];
      ld_cols<NC>(cells, (size_t)idx, n);
      idx += (hx ? dsx : 0) + (hy ? dsy : 0) + (hz ? dsz : 0);
      const float rf = __uint2float_rn(m - t);
      t = m;
#pragma unroll
      for (int q = 0; q < NC; q++) p[q] = fmaf(rf, n[q], p[q]);
      cx -= hx; cy -= hy; cz -= hz;
      if (hx) tx = cx ? tx + Tx : kNone;
      if (hy) ty = cy ? ty + Ty : kNone;
      if (hz) tz = cz ? tz + Tz : kNone;
    }
    it += kk;
    if (kk < 16) break;
#pragma unroll
    for (int q = 0; q < NC; q++) {
      if (kSlotStride)
        kahan_slot<NC, kSlotStride>(slot, q, p[q]);
      else
        kahan_add(s[q], c[q], p[q]);
      p[q] = 0.f;
    }
  }
  // the last chord: from the latest crossing to the end point
  const float df = __int2float_rn(max((int)(lu - t), 0));
  float n[NC];
  ld_cols<NC>(cells, (size_t)idx, n);
  const float unit = (float)(dmax * ldexp(1.0, -k));  // exact: dmax is a float
  Cols<NC> out;
#pragma unroll
  for (int q = 0; q < NC; q++) {
    p[q] = fmaf(df, n[q], p[q]);
    if (kSlotStride) {
      s[q] = slot[q * kSlotStride];
      c[q] = slot[(q + NC) * kSlotStride];
    }
    kahan_add(s[q], c[q], p[q]);
    out.v[q] = s[q] * unit;
  }
  *steps = it + 1;
  return out;
}

// The three-column march of the device path.
template <int kSlotStride = 0, bool kCentreEnd = false>
__device__ __forceinline__ Tau3 march_kahan(const GridDev &g, const float4 *__restrict__ cells, float xs, float ys,
                                            float zs, float xe, float ye, float ze, int *steps, bool *bad,
                                            float *slot = nullptr) {
  const Cols<3> c = march_kahan_n<3, kSlotStride, kCentreEnd>(g, cells, xs, ys, zs, xe, ye, ze, steps, bad, slot);
  return Tau3{c.v[0], c.v[1], c.v[2]};
}

// Rate geometry shared by both precisions (calc_photoion_rate.c:176-246, FP32
// where the reference uses float): target centre, squared distance and
// distance, and the cell chord `delta` along the ray (delta_length, :52-90).
struct RayGeom {
  float dist2, dist, delta;
};

__device__ __forceinline__ RayGeom ray_geometry(const GridDev &g, int gix, int giy, int giz, float sx,
                                                float sy, float sz) {
  // x = delta_x*((float)ix + 0.5) + xmin, in double, stored as float
  const float x = __double2float_rn(__dadd_rn(__dmul_rn((double)g.dx, __dadd_rn((double)__int2float_rn(gix), 0.5)), (double)g.xmin));
  const float y = __double2float_rn(__dadd_rn(__dmul_rn((double)g.dy, __dadd_rn((double)__int2float_rn(giy), 0.5)), (double)g.ymin));
  const float z = __double2float_rn(__dadd_rn(__dmul_rn((double)g.dz, __dadd_rn((double)__int2float_rn(giz), 0.5)), (double)g.zmin));
  const float dx = __fsub_rn(x, sx), dy = __fsub_rn(y, sy), dz = __fsub_rn(z, sz);
  const float sxy = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
  const float s3 = __fadd_rn(sxy, __fmul_rn(dz, dz));
  const float dl = __double2float_rn(__dsqrt_rn(__dadd_rn((double)s3, kTiny)));
  const float dxy = __double2float_rn(__dsqrt_rn(__dadd_rn((double)sxy, kTiny)));
  const float ct = __fdiv_rn(dz, dl), st = __fdiv_rn(dxy, dl);
  const float cp = __fdiv_rn(dx, dxy), sp = __fdiv_rn(dy, dxy);
  const float xo = cosine_guard(__fmul_rn(cp, st));
  const float yo = cosine_guard(__fmul_rn(sp, st));
  const float zo = cosine_guard(ct);
  const float rx = fabsf(__fdiv_rn(g.dx, xo)), ry = fabsf(__fdiv_rn(g.dy, yo)), rz = fabsf(__fdiv_rn(g.dz, zo));
  RayGeom r;
  r.delta = fminf(rx, fminf(ry, rz));
  r.dist2 = s3;
  r.dist = __double2float_rn(__dsqrt_rn((double)s3));
  return r;
}

// ---------------------------------------------------------------------------
// Segment end points of a light ray on one rank (calc_ray_segment.c:47-126):
// the end is the centre of the target cell (global indices), the start is
// the emitter, moved onto the box surface along the ray when the emitter
// lies outside the box (with that file's TINY of 1e-30).
__device__ __forceinline__ float cell_centre(float lo, int i, float d) {
  // lo + ((float)i + 0.5) * d, evaluated in double as the reference does
  return __double2float_rn(__dadd_rn((double)lo, __dmul_rn(__dadd_rn((double)__int2float_rn(i), 0.5), (double)d)));
}

// Emitters outside the box (rare: only sources placed outside it).  The box
// bounds come by value and the point returns in registers, so that the
// call does not make its callers keep the grid or the end points in memory.
static __device__ __noinline__ float3 ray_start_outside(float xmin, float ymin, float zmin, float xmax,
                                                        float ymax, float zmax, float sx, float sy,
                                                        float sz, float xt, float yt, float zt) {
  const double tiny = 1.0e-30;
  const float dx = __fsub_rn(xt, sx), dy = __fsub_rn(yt, sy), dz = __fsub_rn(zt, sz);
  const float s3 = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
  const float dl = __double2float_rn(__dsqrt_rn(__dadd_rn((double)s3, tiny)));
  const float ct = __fdiv_rn(dz, dl);
  const float st = __double2float_rn(__dsqrt_rn(__dsub_rn(1.0, (double)__fmul_rn(ct, ct))));
  const float dxy = __fmul_rn(dl, st);
  const double den = __dadd_rn((double)dxy, tiny);
  const float cp = __double2float_rn(__ddiv_rn((double)dx, den));
  const float sp = __double2float_rn(__ddiv_rn((double)dy, den));
  float xo = __fmul_rn(cp, st), yo = __fmul_rn(sp, st), zo = ct;
  if (fabs((double)xo) < tiny) xo = (xo >= 0.f) ? (float)tiny : -(float)tiny;
  if (fabs((double)yo) < tiny) yo = (yo >= 0.f) ? (float)tiny : -(float)tiny;
  if (fabs((double)zo) < tiny) zo = (zo >= 0.f) ? (float)tiny : -(float)tiny;
  float out = 0.f;
  if (sx < xmin) out = __fdiv_rn(__fsub_rn(xmin, sx), xo);
  if (sx > xmax) out = __fdiv_rn(__fsub_rn(xmax, sx), xo);
  if (sy < ymin) out = __fdiv_rn(__fsub_rn(ymin, sy), yo);
  if (sy > ymax) out = __fdiv_rn(__fsub_rn(ymax, sy), yo);
  if (sz < zmin) out = __fdiv_rn(__fsub_rn(zmin, sz), zo);
  if (sz > zmax) out = __fdiv_rn(__fsub_rn(zmax, sz), zo);
  if (out == 0.f) return make_float3(sx, sy, sz);
  return make_float3(__fadd_rn(sx, __fmul_rn(out, xo)), __fadd_rn(sy, __fmul_rn(out, yo)),
                     __fadd_rn(sz, __fmul_rn(out, zo)));
}

__device__ __forceinline__ void ray_start(const GridDev &g, float sx, float sy, float sz, float xt,
                                          float yt, float zt, float *ox, float *oy, float *oz) {
  *ox = sx; *oy = sy; *oz = sz;
  if (sx >= g.xmin && sx <= g.xmax && sy >= g.ymin && sy <= g.ymax && sz >= g.zmin && sz <= g.zmax)
    return;
  const float3 o = ray_start_outside(g.xmin, g.ymin, g.zmin, g.xmax, g.ymax, g.zmax, sx, sy, sz, xt, yt, zt);
  *ox = o.x; *oy = o.y; *oz = o.z;
}

// Target cell of lane `lane` in block b (local indices); false if the lane's
// cell lies outside a partial block.
__device__ __forceinline__ bool block_cell(const GridDev &g, uint64_t b, int lane, int *ix, int *iy,
                                           int *iz) {
  const uint64_t nyz = (uint64_t)g.nby * g.nbz;
  const int bx = (int)(b / nyz);
  const uint64_t rem = b - (uint64_t)bx * nyz;
  const int by = (int)(rem / g.nbz);
  const int bz = (int)(rem - (uint64_t)by * g.nbz);
  *ix = bx * kBlkX + (lane >> 4);
  *iy = by * kBlkY + ((lane >> 2) & 3);
  *iz = bz * kBlkZ + (lane & 3);
  return *ix < g.nx && *iy < g.ny && *iz < g.nz;
}

// The rays [r0, r1) of block b in a buffer of nray rays that starts at ray
// `base` of the caller's offsets; false when blk_off[b], blk_off[b + 1] do
// not lie in order within [base, base + nray] (the caller's offsets do not
// match its buffers): the block is then skipped and the error flag set.
__device__ __forceinline__ bool block_rays(const uint64_t *__restrict__ blk_off, uint64_t b, uint64_t base,
                                           uint64_t nray, uint64_t *r0, uint64_t *r1) {
  const uint64_t a = blk_off[b], e = blk_off[b + 1];
  if (a < base || e < a || e - base > nray) return false;
  *r0 = a - base;
  *r1 = e - base;
  return true;
}

}  // namespace argot
