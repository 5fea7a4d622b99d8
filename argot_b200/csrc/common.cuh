// common.cuh -- shared definitions of libargot_b200 (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../include/argot_b200.h"

namespace argot {

// Physical constants and flags exactly as the reference spells them
// (constants.h, prim_chem/chemistry.h:14,25, calc_optical_depth.c:15).
constexpr double kTiny = 1.0e-31;
constexpr double kHeliumFact = 0.0811258278;
constexpr double kPi = 3.1415926535897932384626433;
constexpr double kHPlanck = 6.626e-27;
constexpr double kNuL = 3.28e15;
constexpr double kThrHI = 1.0, kThrHeI = 1.8125, kThrHeII = 4.0;
constexpr int kNu = 256;

// Rays are generated and consumed per block of 32 target cells.
constexpr int kBlkX = 2, kBlkY = 4, kBlkZ = 4;

// Thread-local status of the last API call (argot_b200_last_error).
void set_status(int code);
int status_from_cuda(cudaError_t e);

#define ARGOT_CUDA_TRY(expr)                                   \
  do {                                                         \
    cudaError_t _e = (expr);                                   \
    if (_e != cudaSuccess) return argot::status_from_cuda(_e); \
  } while (0)

// Geometry as the kernels see it (by value in kernel parameters).
struct GridDev {
  int nx, ny, nz;
  int ix0, iy0, iz0;
  float xmin, ymin, zmin, xmax, ymax, zmax;
  float xminl, yminl, zminl;
  float dx, dy, dz;
  double lunit, denstonh;
  int nbx, nby, nbz;  // blocks per axis
  // FP32 forms of the unit conversions of the FP32 rate path: lunit *
  // denstonh (code column -> cm^-2), and 1 / (4 pi lunit^2) = pcm * 2^pce
  // (below the FP32 range, so its power of two is kept apart)
  float cdf, pcm;
  int pce;
};

GridDev make_grid(const argot_b200_grid &g);
bool grid_valid(const argot_b200_grid *g);

// Tables in constant memory (filled once per device by ensure_tables()).
struct RateTables {
  float nu_f[kNu];        // (float) nu, as the reference compares it
  float cs[3][kNu];       // sigma_s(nu) [cm^2]
  float cs_l2e[3][kNu];   // sigma_s(nu) * log2(e)
  float hw[3][kNu];       // sigma_s(nu) * max((float)nu - nu_s, 0)
  float smax16[3][16];    // max of sigma_s(nu) over the bins k >= 16 i
  // the bin loop's iterations (16 bins each) before iter_he have sigma_HeI =
  // sigma_HeII = 0 in every bin, those before iter_heii sigma_HeII = 0
  int iter_he, iter_heii;
};
// Uploads the tables to the constant bank of the translation unit that owns
// the rate kernels (photoion.cu), once per device.
int ensure_tables(int device);

// Photo-ionisation cross sections [cm^2] at nu in units of the HI Lyman
// limit (prim_chem/cross_section.c:20-53).
double sigma_hi(double nu);
double sigma_hei(double nu);
double sigma_heii(double nu);

// Host copies of the tables (computed with the reference's formulas).
void host_tables(double *nu, float *cs3);
// Weights of the six rate integrals per bin (6 x 256): sigma_s(nu) and
// sigma_s(nu) * ((float)nu - nu_s)^+ for s = HI, HeI, HeII.
void host_rate_weights(double *w6);

// Position of bin k in an emitter's normalised spectrum (emit_specn): the
// bins are stored in the pair order of the packed rate loop, pair
// p = (k % 8) + 8 (k / 16) holding bins k0 = (p % 8) + 16 (p / 8) and k0 + 8
// at 2 p and 2 p + 1, so one 8-byte load fetches a pair.
__host__ __device__ __forceinline__ int spec_pair_index(int k) {
  return 2 * ((k & 7) + 8 * (k >> 4)) + ((k >> 3) & 1);
}

// Emitters and tree on the device.
struct DevNode {
  float cx, cy, cz, len;   // centre (float, as stored by the reference), side
  int n;                   // number of sources below
  int skip;                // preorder index after this subtree
  int has_child;           // children follow at index+1 in preorder
  int src_first;           // first entry of the leaf's source list
};

}  // namespace argot

// Opaque handle bodies (C ABI types).
struct argot_b200_dev_tree {
  int device;
  int n_nodes, n_src, n_emit;
  float theta_sq;          // SQR(theta) in float, as the reference's walk
  argot::DevNode *nodes;   // n_nodes (preorder)
  int *src_list;           // n_src: source index per leaf slot
  float4 *emit_pos;        // n_emit (x, y, z, 0)
  float emit_lo[3], emit_hi[3];  // bounding box of the emitter positions
  double *emit_spec64;     // n_emit x 256
  float *emit_specn;       // n_emit x 256: spectrum / total, in bin-pair order (spec_pair_index)
  double *emit_total;      // n_emit
  // surrogate inputs (set by argot_b200_dev_tree_set_blackbody): log10 T of
  // an emitter whose spectrum is a single-temperature blackbody (NaN
  // otherwise), its six thin-limit integrals I_j0 = sum_nu w_j(nu) s_nu and
  // the first moments m_js = sum_nu w_j s_nu sigma_s / sigma_s0 / I_j0
  float *emit_logT;        // n_emit
  double *emit_i0;         // n_emit x 6
  float *emit_m;           // n_emit x 18 (j-major: m[3 j + s])
};
