// march.cuh -- device functions of the segment march (calc_optical_depth).
#pragma once
#include "common.cuh"

namespace argot {

struct Tau3 {
  float hi, hei, heii;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ size_t cell_index(const GridDev &g, int ix, int iy, int iz) {
  return (size_t)iz + (size_t)g.nz * ((size_t)iy + (size_t)g.ny * (size_t)ix);
}

__device__ __forceinline__ float4 ld_cell(const float4 *__restrict__ cells, size_t c) {
  return __ldg(cells + c);
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
static __device__ __noinline__ Tau3 march_reference(const GridDev &g, const float4 *__restrict__ cells,
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
  Tau3 t = {0.f, 0.f, 0.f};
  int it = 0;
  const int cap = g.nx + g.ny + g.nz + 2;
  while ((ix != ixe || iy != iye || iz != ize) && (unsigned)ix < (unsigned)g.nx &&
         (unsigned)iy < (unsigned)g.ny && (unsigned)iz < (unsigned)g.nz) {
    if (++it > cap) { *bad = true; break; }
    const float4 n = ld_cell(cells, cell_index(g, ix, iy, iz));
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
    t.hi = __fadd_rn(t.hi, __fmul_rn(rmin, n.x));
    t.hei = __fadd_rn(t.hei, __fmul_rn(rmin, n.y));
    t.heii = __fadd_rn(t.heii, __fmul_rn(rmin, n.z));
  }
  xc = __fadd_rn(xc, g.xminl);
  yc = __fadd_rn(yc, g.yminl);
  zc = __fadd_rn(zc, g.zminl);
  const float ex = __fsub_rn(xe, xc), ey = __fsub_rn(ye, yc), ez = __fsub_rn(ze, zc);
  const float e3 = __fadd_rn(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)), __fmul_rn(ez, ez));
  const float depth = __double2float_rn(__dsqrt_rn((double)e3));
  const float4 ne = ld_cell(cells, cell_index(g, ixe, iye, ize));
  t.hi = __fadd_rn(t.hi, __fmul_rn(depth, ne.x));
  t.hei = __fadd_rn(t.hei, __fmul_rn(depth, ne.y));
  t.heii = __fadd_rn(t.heii, __fmul_rn(depth, ne.z));
  *steps = it + 1;
  return t;
}

// ---------------------------------------------------------------------------
// Count-down march with compensated sums.  Same start / end cell rules as
// the reference.  Along each axis the walk must cross exactly
// |i_end - i_start| faces, so it keeps per axis the number of faces still
// to cross and the distance along the ray to the next one.  Every step
// takes the nearest face among the axes that still have faces to cross,
// resets that axis's distance to the face spacing dX/|u_x| and shortens the
// others by the step.  Distances therefore stay of cell size, and their
// rounding scales with the cell rather than with the ray length as a running
// position or an absolute path parameter would; the walk always ends in the
// end cell after at most sum|di| steps.  The last chord is measured from
// the face through which the end cell was entered.  Columns are FP32 with
// compensated (Kahan) summation.
__device__ __forceinline__ void kahan_add(float &s, float &c, float v) {
  const float y = v - c;
  const float tt = s + y;
  c = (tt - s) - y;
  s = tt;
}

// The walk.  Per step: the nearest face among the axes with faces left;
// the chord belongs to the current cell; the crossed axes advance the
// 32-bit cell index by their precomputed strides and reset their distance
// to the face spacing, the others shorten theirs.  The gather of the next
// cell is issued before the current one is accumulated.  Chords are summed
// with FMA into per-species partial sums that are folded into Kahan sums
// every 16 steps (compensated summation over blocks of 16 terms).  The last
// chord runs from the end cell's entry face to the end point.
static __device__ __forceinline__ Tau3 march_kahan(const GridDev &g, const float4 *__restrict__ cells,
                                                   float xs, float ys, float zs, float xe, float ye,
                                                   float ze, int *steps, bool *bad) {
  const int ixe = axis_cell(xe, g.xminl, g.dx, g.nx);
  const int iye = axis_cell(ye, g.yminl, g.dy, g.ny);
  const int ize = axis_cell(ze, g.zminl, g.dz, g.nz);
  const int ix = axis_cell(xs, g.xminl, g.dx, g.nx);
  const int iy = axis_cell(ys, g.yminl, g.dy, g.ny);
  const int iz = axis_cell(zs, g.zminl, g.dz, g.nz);
  const float x0 = xs - g.xminl, y0 = ys - g.yminl, z0 = zs - g.zminl;
  const float dx = xe - xs, dy = ye - ys, dz = ze - zs;
  const float len = sqrtf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
  const float il = len > 0.f ? 1.0f / len : 0.f;
  const float ax = fabsf(cosine_guard(dx * il)), ay = fabsf(cosine_guard(dy * il)),
              az = fabsf(cosine_guard(dz * il));
  const float iax = 1.0f / ax, iay = 1.0f / ay, iaz = 1.0f / az;
  int cx = abs(ixe - ix), cy = abs(iye - iy), cz = abs(ize - iz);
  const int stx = ixe > ix ? 1 : -1, sty = iye > iy ? 1 : -1, stz = ize > iz ? 1 : -1;
  const float kInf = __int_as_float(0x7f800000);
  float rx = cx ? fmaxf(fabsf(fmaf(g.dx, (float)(ix + (stx > 0)), -x0)) * iax, 0.f) : kInf;
  float ry = cy ? fmaxf(fabsf(fmaf(g.dy, (float)(iy + (sty > 0)), -y0)) * iay, 0.f) : kInf;
  float rz = cz ? fmaxf(fabsf(fmaf(g.dz, (float)(iz + (stz > 0)), -z0)) * iaz, 0.f) : kInf;
  const float tdx = g.dx * iax, tdy = g.dy * iay, tdz = g.dz * iaz;
  const int dsz = stz, dsy = sty * g.nz, dsx = stx * g.nz * g.ny;
  int idx = iz + g.nz * (iy + g.ny * ix);

  float4 n = __ldg(cells + idx);
  float p0 = 0.f, p1 = 0.f, p2 = 0.f;
  float s0 = 0.f, s1 = 0.f, s2 = 0.f, c0 = 0.f, c1 = 0.f, c2 = 0.f;
  const int cap = cx + cy + cz;  // every finite step crosses at least one face
  const bool crx = cx != 0, cry = cy != 0, crz = cz != 0;  // axes with faces to cross
  int it = 0;
  // blocks of 16 steps (unrolled; the Kahan fold and the step bound are
  // checked once per block, so only "faces left" is tested per step)
  while ((cx | cy | cz) && it < cap) {
    int k = 0;
#pragma unroll
    for (; k < 16; k++) {
      if (!(cx | cy | cz)) break;
      const float r = fminf(rx, fminf(ry, rz));
      const bool hx = rx == r, hy = ry == r, hz = rz == r;
      idx += (hx ? dsx : 0) + (hy ? dsy : 0) + (hz ? dsz : 0);
      const float4 nn = __ldg(cells + idx);
      p0 = fmaf(r, n.x, p0);
      p1 = fmaf(r, n.y, p1);
      p2 = fmaf(r, n.z, p2);
      cx -= hx; cy -= hy; cz -= hz;
      rx = hx ? (cx ? tdx : kInf) : rx - r;
      ry = hy ? (cy ? tdy : kInf) : ry - r;
      rz = hz ? (cz ? tdz : kInf) : rz - r;
      n = nn;
    }
    it += k;
    if (k == 16) {
      kahan_add(s0, c0, p0);
      kahan_add(s1, c1, p1);
      kahan_add(s2, c2, p2);
      p0 = p1 = p2 = 0.f;
    }
  }
  if (cx | cy | cz) *bad = true;  // only non-finite input leaves faces uncrossed
  // the ray enters the end cell at its latest face crossing, so the last
  // chord is the shortest distance from an axis's entry face of the end
  // cell to the end point, over the axes that had faces to cross
  float depth = len;
  if (crx | cry | crz) {
    depth = kInf;
    if (crx) depth = fminf(depth, fabsf((xe - g.xminl) - g.dx * (float)(ixe + (stx < 0))) * iax);
    if (cry) depth = fminf(depth, fabsf((ye - g.yminl) - g.dy * (float)(iye + (sty < 0))) * iay);
    if (crz) depth = fminf(depth, fabsf((ze - g.zminl) - g.dz * (float)(ize + (stz < 0))) * iaz);
  }
  p0 = fmaf(depth, n.x, p0);
  p1 = fmaf(depth, n.y, p1);
  p2 = fmaf(depth, n.z, p2);
  kahan_add(s0, c0, p0);
  kahan_add(s1, c1, p1);
  kahan_add(s2, c2, p2);
  *steps = it + 1;
  return Tau3{s0, s1, s2};
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

static __device__ __noinline__ void ray_start_outside(const GridDev &g, float sx, float sy, float sz,
                                                      float xt, float yt, float zt, float *ox, float *oy,
                                                      float *oz);

__device__ __forceinline__ void ray_start(const GridDev &g, float sx, float sy, float sz, float xt,
                                          float yt, float zt, float *ox, float *oy, float *oz) {
  *ox = sx; *oy = sy; *oz = sz;
  if (sx >= g.xmin && sx <= g.xmax && sy >= g.ymin && sy <= g.ymax && sz >= g.zmin && sz <= g.zmax)
    return;
  ray_start_outside(g, sx, sy, sz, xt, yt, zt, ox, oy, oz);
}

// emitters outside the box (rare: only sources placed outside it)
static __device__ __noinline__ void ray_start_outside(const GridDev &g, float sx, float sy, float sz,
                                                      float xt, float yt, float zt, float *ox, float *oy,
                                                      float *oz) {
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
  if (sx < g.xmin) out = __fdiv_rn(__fsub_rn(g.xmin, sx), xo);
  if (sx > g.xmax) out = __fdiv_rn(__fsub_rn(g.xmax, sx), xo);
  if (sy < g.ymin) out = __fdiv_rn(__fsub_rn(g.ymin, sy), yo);
  if (sy > g.ymax) out = __fdiv_rn(__fsub_rn(g.ymax, sy), yo);
  if (sz < g.zmin) out = __fdiv_rn(__fsub_rn(g.zmin, sz), zo);
  if (sz > g.zmax) out = __fdiv_rn(__fsub_rn(g.zmax, sz), zo);
  if (out != 0.f) {
    *ox = __fadd_rn(sx, __fmul_rn(out, xo));
    *oy = __fadd_rn(sy, __fmul_rn(out, yo));
    *oz = __fadd_rn(sz, __fmul_rn(out, zo));
  }
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
