// smooth.cu -- the photo-ionisation-rate smoothing of smooth_photoion_rate.c
// on the device, so that the rates stay in HBM through the iteration loop
// (the reference copies them to the host, smooths there and copies back).
//
// Per cell and field: the 27 cells ix-1..ix+1 (outer), iy-1..iy+1,
// iz-1..iz+1 (inner) with the centre weighted by 30, summed in the
// reference's order and precision (smooth_photoion_rate.c:1060-1517): the
// first 13 terms in single precision, the weighted centre and the rest in
// double (its double literal promotes the running sum), times 1/56 in
// double, stored as float.  At the mesh faces: a copy of the nearest cell
// (the reference's default build, `isolated = yes`, with no neighbour rank)
// or the periodic image.  Bit-identical to the reference.
#include "march.cuh"

namespace argot {

__global__ void __launch_bounds__(256) k_smooth(int nx, int ny, int nz, const float *__restrict__ in,
                                               float *__restrict__ out, int nplanes, int isolated) {
  const uint64_t ncell = (uint64_t)nx * ny * nz;
  const double kNormal = 1.0 / (30.0 + 26.0);
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < ncell;
       c += (uint64_t)gridDim.x * blockDim.x) {
    const int iz = (int)(c % nz);
    const int iy = (int)((c / nz) % ny);
    const int ix = (int)(c / ((uint64_t)nz * ny));
    int jx[3], jy[3], jz[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const int x = ix + a - 1, y = iy + a - 1, z = iz + a - 1;
      jx[a] = isolated ? clampi(x, 0, nx - 1) : (x + nx) % nx;
      jy[a] = isolated ? clampi(y, 0, ny - 1) : (y + ny) % ny;
      jz[a] = isolated ? clampi(z, 0, nz - 1) : (z + nz) % nz;
    }
    uint32_t off[27];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++)
#pragma unroll
        for (int d = 0; d < 3; d++) off[9 * a + 3 * b + d] = (uint32_t)((jx[a] * ny + jy[b]) * nz + jz[d]);
#pragma unroll 1
    for (int s = 0; s < nplanes; s++) {
      const float *__restrict__ f = in + s * ncell;
      float acc = __ldg(f + off[0]);
#pragma unroll
      for (int k = 1; k < 13; k++) acc = __fadd_rn(acc, __ldg(f + off[k]));
      double d = __dadd_rn((double)acc, __dmul_rn(30.0, (double)__ldg(f + off[13])));
#pragma unroll
      for (int k = 14; k < 27; k++) d = __dadd_rn(d, (double)__ldg(f + off[k]));
      out[s * ncell + c] = __double2float_rn(__dmul_rn(kNormal, d));
    }
  }
}

int smooth_blocks(uint64_t ncell) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint64_t want = (ncell + 255) / 256;
  return (int)(want < (uint64_t)sms * 8 ? (want ? want : 1) : (uint64_t)sms * 8);
}

// Smooths nplanes planes of ncell floats (in -> out).
int launch_smooth_planes(int nx, int ny, int nz, const float *in, float *out, int nplanes, int isolated,
                         cudaStream_t st) {
  const uint64_t ncell = (uint64_t)nx * ny * nz;
  if (!ncell || nplanes <= 0) return 0;
  k_smooth<<<smooth_blocks(ncell), 256, 0, st>>>(nx, ny, nz, in, out, nplanes, isolated);
  ARGOT_CUDA_TRY(cudaGetLastError());
  return 0;
}

}  // namespace argot

using namespace argot;

extern "C" {

int argot_b200_smooth_rates(const argot_b200_grid *gp, const float *in6, float *out6, int isolated, void *stream) {
  if (!grid_valid(gp) || !in6 || !out6 || in6 == out6 || (isolated != 0 && isolated != 1)) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  const uint64_t ncell = (uint64_t)gp->nx * gp->ny * gp->nz;
  if (ncell >= (1ull << 32)) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  const int blocks = smooth_blocks(ncell);
  k_smooth<<<blocks, 256, 0, (cudaStream_t)stream>>>(gp->nx, gp->ny, gp->nz, in6, out6, 6, isolated);
  ARGOT_CUDA_TRY(cudaGetLastError());
  set_status(0);
  return 0;
}

}  // extern "C"
