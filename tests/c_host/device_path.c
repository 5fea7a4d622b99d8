/*
 * device_path.c -- a C host of the device fast path (no Python): the calls
 * an ARGOT-like C program makes to libargot_b200 to generate the rays of a
 * problem on the device, march them and integrate the rates, with one call
 * of argot_b200_run_group.  tests/test_c_host.py builds it, feeds it a
 * problem and compares its rates with the Python driver's, bit for bit.
 *
 * usage: device_path <input> <output>
 * input:  int32 edge, int32 nsrc, float theta, double lunit, double denstonh,
 *         float fields[4][edge^3] (dens, fHI, fHeI, fHeII),
 *         float src_pos[nsrc][3], double spectra[nsrc][256]
 * output: float rates6[6][edge^3], uint64 crossings
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "argot_b200.h"

#define CHECK(call)                                                             \
  do {                                                                          \
    int rc_ = (call);                                                           \
    if (rc_ != 0) {                                                             \
      fprintf(stderr, "%s failed: %d (%s)\n", #call, rc_, argot_b200_error_string(rc_)); \
      return 1;                                                                 \
    }                                                                           \
  } while (0)
#define CUDA(call)                                                              \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      fprintf(stderr, "%s failed: %s\n", #call, cudaGetErrorString(e_));        \
      return 1;                                                                 \
    }                                                                           \
  } while (0)

static int read_all(FILE *f, void *p, size_t n) { return fread(p, 1, n, f) == n ? 0 : 1; }

int main(int argc, char **argv) {
  if (argc != 3) { fprintf(stderr, "usage: %s <input> <output>\n", argv[0]); return 2; }
  FILE *in = fopen(argv[1], "rb");
  if (!in) { perror("input"); return 2; }
  int edge = 0, nsrc = 0;
  float theta = 0.f;
  double lunit = 0.0, denstonh = 0.0;
  if (read_all(in, &edge, 4) || read_all(in, &nsrc, 4) || read_all(in, &theta, 4) || read_all(in, &lunit, 8) ||
      read_all(in, &denstonh, 8) || edge <= 0 || nsrc <= 0) { fprintf(stderr, "bad header\n"); return 2; }
  const size_t ncell = (size_t)edge * edge * edge;
  float *fields = (float *)malloc(4 * ncell * sizeof(float));
  float *pos = (float *)malloc(3 * (size_t)nsrc * sizeof(float));
  double *spec = (double *)malloc(256 * (size_t)nsrc * sizeof(double));
  float *rates = (float *)malloc(6 * ncell * sizeof(float));
  if (!fields || !pos || !spec || !rates) return 2;
  if (read_all(in, fields, 4 * ncell * sizeof(float)) || read_all(in, pos, 3 * (size_t)nsrc * sizeof(float)) ||
      read_all(in, spec, 256 * (size_t)nsrc * sizeof(double))) { fprintf(stderr, "short input\n"); return 2; }
  fclose(in);

  /* one rank covering the unit box */
  argot_b200_grid g;
  memset(&g, 0, sizeof(g));
  g.nx = g.ny = g.nz = edge;
  g.xmax = g.ymax = g.zmax = 1.0f;
  g.dx = g.dy = g.dz = 1.0f / (float)edge;
  g.lunit = lunit;
  g.denstonh = denstonh;

  CUDA(cudaSetDevice(0));
  cudaStream_t st;
  CUDA(cudaStreamCreate(&st));
  float *d_fields = NULL, *d_packed = NULL, *d_rates = NULL, *d_tau = NULL;
  uint64_t *d_count = NULL, *d_off = NULL;
  unsigned long long *d_cross = NULL;
  uint32_t *d_rays = NULL;
  CUDA(cudaMalloc((void **)&d_fields, 4 * ncell * sizeof(float)));
  CUDA(cudaMalloc((void **)&d_packed, 8 * ncell * sizeof(float)));
  CUDA(cudaMalloc((void **)&d_rates, 6 * ncell * sizeof(float)));
  CUDA(cudaMalloc((void **)&d_cross, sizeof(unsigned long long)));
  CUDA(cudaMemcpy(d_fields, fields, 4 * ncell * sizeof(float), cudaMemcpyHostToDevice));
  CUDA(cudaMemset(d_rates, 0, 6 * ncell * sizeof(float)));
  CUDA(cudaMemset(d_cross, 0, sizeof(unsigned long long)));

  CHECK(argot_b200_pack_fields(&g, d_fields, d_fields + ncell, d_fields + 2 * ncell, d_fields + 3 * ncell,
                               d_packed, st));
  argot_b200_tree *tree = NULL;
  argot_b200_dev_tree *dtree = NULL;
  CHECK(argot_b200_tree_build(&g, nsrc, pos, spec, theta, &tree));
  CHECK(argot_b200_dev_tree_upload(tree, &dtree, st));
  uint64_t nb = 0, nray = 0;
  CHECK(argot_b200_num_blocks(&g, &nb));
  CUDA(cudaMalloc((void **)&d_count, nb * sizeof(uint64_t)));
  CUDA(cudaMalloc((void **)&d_off, (nb + 1) * sizeof(uint64_t)));
  CHECK(argot_b200_count_rays(&g, dtree, 0, nb, d_count, NULL, st));
  CHECK(argot_b200_scan_blocks(d_count, nb, 0, d_off, &nray, st));
  uint64_t *off = (uint64_t *)malloc((nb + 1) * sizeof(uint64_t));
  if (!off) return 2;
  CUDA(cudaMemcpyAsync(off, d_off, (nb + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
  CUDA(cudaStreamSynchronize(st));
  CUDA(cudaMalloc((void **)&d_rays, (nray ? nray : 1) * sizeof(uint32_t)));
  CUDA(cudaMalloc((void **)&d_tau, 3 * (nray ? nray : 1) * sizeof(float)));

  /* the whole fast path in one call: rays, march, rates (4 overlapped parts) */
  CHECK(argot_b200_run_group(&g, d_packed, dtree, 0, nb, d_off, off, 0, d_rays, d_tau, 1,
                             ARGOT_B200_PRECISION_KAHAN, ARGOT_B200_RATE_EXACT_F32, 4, d_rates, d_cross, st));
  CUDA(cudaStreamSynchronize(st));
  CHECK(argot_b200_check_device_error(st));
  unsigned long long cross = 0;
  CUDA(cudaMemcpy(rates, d_rates, 6 * ncell * sizeof(float), cudaMemcpyDeviceToHost));
  CUDA(cudaMemcpy(&cross, d_cross, sizeof(cross), cudaMemcpyDeviceToHost));

  FILE *out = fopen(argv[2], "wb");
  if (!out) { perror("output"); return 2; }
  fwrite(rates, sizeof(float), 6 * ncell, out);
  fwrite(&cross, sizeof(cross), 1, out);
  fclose(out);
  printf("device_path: %llu rays, %llu crossings\n", (unsigned long long)nray, cross);

  argot_b200_dev_tree_free(dtree);
  argot_b200_tree_free(tree);
  cudaFree(d_fields); cudaFree(d_packed); cudaFree(d_rates); cudaFree(d_tau); cudaFree(d_rays);
  cudaFree(d_count); cudaFree(d_off); cudaFree(d_cross);
  cudaStreamDestroy(st);
  free(fields); free(pos); free(spec); free(rates); free(off);
  return 0;
}
