// mlp.cu -- training data, training and reference evaluation of the
// frequency-integral surrogate (see mlp.cuh).  Everything here is
// hand-written: an exact-quadrature sample generator, the forward and
// backward passes, deterministic weight-gradient reductions and Adam.
#include <cmath>
#include <mutex>
#include <vector>

#include "mlp.cuh"

namespace argot {

// ------------------------------------------------------------- tables
struct MlpTables {
  double cs[3][kNu];      // sigma_s(nu)
  double shat[3][kNu];    // sigma_s(nu) / sigma_s(first absorbing bin)
  double w[kMlpOut][kNu]; // output weights w_j(nu)
  double sig0[3];
};
__constant__ MlpTables c_mt;

static void host_mlp_tables(MlpTables &t) {
  double nu[kNu];
  float cs3[3 * kNu];
  host_tables(nu, cs3);
  const double thr[3] = {kThrHI, kThrHeI, kThrHeII};
  for (int s = 0; s < 3; s++) {
    t.sig0[s] = 0.0;
    for (int k = 0; k < kNu && t.sig0[s] == 0.0; k++) t.sig0[s] = cs3[3 * k + s];
  }
  for (int k = 0; k < kNu; k++) {
    const double nf = (double)(float)nu[k];
    for (int s = 0; s < 3; s++) {
      const double c = cs3[3 * k + s];
      t.cs[s][k] = c;
      t.shat[s][k] = c / t.sig0[s];
      t.w[s][k] = c;
      t.w[3 + s][k] = c * (nf > thr[s] ? nf - thr[s] : 0.0);
    }
  }
}

static int ensure_mlp_tables(int dev) {
  static std::mutex mu;
  static bool done[64] = {false};
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 0 || dev >= 64) return ARGOT_B200_EINVAL;
  if (done[dev]) return 0;
  MlpTables t;
  host_mlp_tables(t);
  ARGOT_CUDA_TRY(cudaMemcpyToSymbol(c_mt, &t, sizeof(t)));
  done[dev] = true;
  return 0;
}

// ---------------------------------------------------------- random numbers
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ double u01(uint64_t x) { return (double)(x >> 11) * (1.0 / 9007199254740992.0); }

// -------------------------------------------------------- training samples
// x = (log10 tau_HI, log10 tau_HeI, log10 tau_HeII) uniform in [-6, 3],
// log10 T on the grid of the given spectra; y = q_j = ln(y_j / ylin_j)
// (mlp.cuh) from the exact 256-bin sums in FP64.
__global__ void k_mlp_samples(const double *__restrict__ spec, const double *__restrict__ i0, int nT,
                              uint64_t n, uint64_t seed, float *__restrict__ X, float *__restrict__ Y) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t base = splitmix64(seed ^ (i * 0x632be59bd9b4e019ull));
    double lt[3];
    for (int s = 0; s < 3; s++) lt[s] = kTauLo + (kTauHi - kTauLo) * u01(splitmix64(base + s + 1));
    const int it = min(nT - 1, (int)(u01(splitmix64(base + 7)) * nT));
    const double tau[3] = {exp10(lt[0]), exp10(lt[1]), exp10(lt[2])};
    const double *sp = spec + (size_t)it * kNu;
    double I[kMlpOut] = {0, 0, 0, 0, 0, 0};
    double lin[kMlpOut] = {0, 0, 0, 0, 0, 0};  // sum_nu w_j s_nu (tau . shat)
    for (int k = 0; k < kNu; k++) {
      const double ts = tau[0] * c_mt.shat[0][k] + tau[1] * c_mt.shat[1][k] + tau[2] * c_mt.shat[2][k];
      const double a = exp(-ts) * sp[k];
#pragma unroll
      for (int j = 0; j < kMlpOut; j++) {
        I[j] = fma(c_mt.w[j][k], a, I[j]);
        lin[j] = fma(c_mt.w[j][k] * sp[k], ts, lin[j]);
      }
    }
    X[4 * i + 0] = (float)lt[0];
    X[4 * i + 1] = (float)lt[1];
    X[4 * i + 2] = (float)lt[2];
    X[4 * i + 3] = (float)(kTLo + (kTHi - kTLo) * (double)it / (double)(nT - 1));
#pragma unroll
    for (int j = 0; j < kMlpOut; j++) {
      const double z = i0[(size_t)it * kMlpOut + j];
      const double y = (I[j] > 0.0 && z > 0.0) ? log(I[j] / z) : -700.0;
      const double ylin = -lin[j] / z;
      Y[kMlpOut * i + j] = (float)log(y / ylin);
    }
  }
}

// ----------------------------------------------------- forward / backward
__device__ __forceinline__ float norm_in(int c, float v) {
  return c < 3 ? (v - 0.5f * (kTauLo + kTauHi)) * (2.f / (kTauHi - kTauLo))
               : (v - 0.5f * (kTLo + kTHi)) * (2.f / (kTHi - kTLo));
}
__device__ __forceinline__ float sigmoidf_(float z) { return 1.f / (1.f + __expf(-z)); }
__device__ __forceinline__ float silu_ref(float z) { return z * sigmoidf_(z); }

// Weights rounded to BF16 (what the tensor cores see) in shared memory.
struct SmemW {
  float w1[kMlpH * kMlpIn], b1[kMlpH], w2[kMlpH * kMlpH], b2[kMlpH], w3[kMlpH * kMlpH], b3[kMlpH],
      w4[kMlpOut * kMlpH], b4[kMlpOut];
};

__device__ void load_weights(SmemW &s, const float *__restrict__ p) {
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) {
    const float v = p[i];
    float *dst;
    int off;
    if (i < kOffB1) { dst = s.w1; off = i - kOffW1; }
    else if (i < kOffW2) { dst = s.b1; off = i - kOffB1; }
    else if (i < kOffB2) { dst = s.w2; off = i - kOffW2; }
    else if (i < kOffW3) { dst = s.b2; off = i - kOffB2; }
    else if (i < kOffB3) { dst = s.w3; off = i - kOffW3; }
    else if (i < kOffW4) { dst = s.b3; off = i - kOffB3; }
    else if (i < kOffB4) { dst = s.w4; off = i - kOffW4; }
    else { dst = s.b4; off = i - kOffB4; }
    const bool is_bias = (dst == s.b1 || dst == s.b2 || dst == s.b3 || dst == s.b4);
    dst[off] = is_bias ? v : bf16_round(v);
  }
}

// One thread per sample.  Stores the pre-activations z1..z3 and the
// activations a1..a3 (FP32: the tensor-core inference carries every
// activation as a BF16 pair hi + lo) in [unit][sample] layout for the
// backward pass, and the normalised outputs o.
template <bool kStore>
__global__ void __launch_bounds__(128) k_mlp_fwd(const float *__restrict__ p, const float *__restrict__ X,
                                                 int nb, float *__restrict__ Z, float *__restrict__ A,
                                                 float *__restrict__ O) {
  __shared__ SmemW s;
  load_weights(s, p);
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  float x[kMlpIn];
#pragma unroll
  for (int c = 0; c < kMlpIn; c++) x[c] = norm_in(c, X[4 * (size_t)i + c]);
  float a[kMlpH], h[kMlpH];
#pragma unroll
  for (int j = 0; j < kMlpH; j++) {
    float z = s.b1[j];
#pragma unroll
    for (int c = 0; c < kMlpIn; c++) z = fmaf(s.w1[j * kMlpIn + c], x[c], z);
    a[j] = silu_ref(z);
    if (kStore) { Z[(size_t)j * nb + i] = z; A[(size_t)j * nb + i] = a[j]; }
  }
#pragma unroll 4
  for (int j = 0; j < kMlpH; j++) {
    float z = s.b2[j];
#pragma unroll
    for (int k = 0; k < kMlpH; k++) z = fmaf(s.w2[j * kMlpH + k], a[k], z);
    h[j] = silu_ref(z);
    if (kStore) { Z[(size_t)(kMlpH + j) * nb + i] = z; A[(size_t)(kMlpH + j) * nb + i] = h[j]; }
  }
#pragma unroll 4
  for (int j = 0; j < kMlpH; j++) {
    float z = s.b3[j];
#pragma unroll
    for (int k = 0; k < kMlpH; k++) z = fmaf(s.w3[j * kMlpH + k], h[k], z);
    a[j] = silu_ref(z);
    if (kStore) { Z[(size_t)(2 * kMlpH + j) * nb + i] = z; A[(size_t)(2 * kMlpH + j) * nb + i] = a[j]; }
  }
#pragma unroll
  for (int j = 0; j < kMlpOut; j++) {
    float z = s.b4[j];
#pragma unroll
    for (int k = 0; k < kMlpH; k++) z = fmaf(s.w4[j * kMlpH + k], a[k], z);
    O[(size_t)j * nb + i] = z;
  }
}

__device__ __forceinline__ float silu_grad(float z) {
  const float sg = sigmoidf_(z);
  return sg * (1.f + z * (1.f - sg));
}

// dO = 2 (o - target_norm) / (nb * 6); back through the layers (straight
// through the BF16 rounding of the weights).  Writes dZ4 (= dO), dZ3, dZ2, dZ1 in
// [unit][sample] layout and each sample's squared error.
__global__ void __launch_bounds__(128) k_mlp_bwd(const float *__restrict__ p, const float *__restrict__ Yt,
                                                 int nb, const float *__restrict__ Z, const float *__restrict__ O,
                                                 float *__restrict__ dZ, float *__restrict__ sqerr) {
  __shared__ SmemW s;
  load_weights(s, p);
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  float d4[kMlpOut];
  float se = 0.f;
  const float sc = 2.f / ((float)nb * (float)kMlpOut);
#pragma unroll
  for (int j = 0; j < kMlpOut; j++) {
    const float tgt = (Yt[kMlpOut * (size_t)i + j] - kOutShift) / kOutScale;
    const float e = O[(size_t)j * nb + i] - tgt;
    se += e * e;
    d4[j] = sc * e;
    dZ[(size_t)(3 * kMlpH + j) * nb + i] = d4[j];
  }
  sqerr[i] = se;
  float d[kMlpH], e[kMlpH];
#pragma unroll
  for (int k = 0; k < kMlpH; k++) {
    float g = 0.f;
#pragma unroll
    for (int j = 0; j < kMlpOut; j++) g = fmaf(s.w4[j * kMlpH + k], d4[j], g);
    d[k] = g * silu_grad(Z[(size_t)(2 * kMlpH + k) * nb + i]);
    dZ[(size_t)(2 * kMlpH + k) * nb + i] = d[k];
  }
#pragma unroll 4
  for (int k = 0; k < kMlpH; k++) {
    float g = 0.f;
#pragma unroll
    for (int j = 0; j < kMlpH; j++) g = fmaf(s.w3[j * kMlpH + k], d[j], g);
    e[k] = g * silu_grad(Z[(size_t)(kMlpH + k) * nb + i]);
    dZ[(size_t)(kMlpH + k) * nb + i] = e[k];
  }
#pragma unroll 4
  for (int k = 0; k < kMlpH; k++) {
    float g = 0.f;
#pragma unroll
    for (int j = 0; j < kMlpH; j++) g = fmaf(s.w2[j * kMlpH + k], e[j], g);
    dZ[(size_t)k * nb + i] = g * silu_grad(Z[(size_t)k * nb + i]);
  }
}

// Weight gradients, deterministic: partial sums over slices of the batch
// into part[slice][param], then a fixed-order sum over slices.
//   layer 1: dW1[j][c] = sum_b dZ1[j][b] x[c][b];  db1[j] = sum_b dZ1[j][b]
//   layer l>1: dWl[j][k] = sum_b dZl[j][b] A_{l-1}[k][b]
constexpr int kGradSlices = 64;

__global__ void __launch_bounds__(256) k_mlp_wgrad(const float *__restrict__ X, int nb, const float *__restrict__ A,
                                                   const float *__restrict__ dZ, float *__restrict__ part) {
  const int slice = blockIdx.x;
  const int per = (nb + kGradSlices - 1) / kGradSlices;
  const int b0 = slice * per, b1 = min(nb, b0 + per);
  float *out = part + (size_t)slice * kMlpParams;
  for (int q = threadIdx.x; q < kMlpParams; q += blockDim.x) {
    float acc = 0.f;
    if (q < kOffB1) {
      const int j = q / kMlpIn, c = q % kMlpIn;
      for (int b = b0; b < b1; b++) acc = fmaf(dZ[(size_t)j * nb + b], norm_in(c, X[4 * (size_t)b + c]), acc);
    } else if (q < kOffW2) {
      const int j = q - kOffB1;
      for (int b = b0; b < b1; b++) acc += dZ[(size_t)j * nb + b];
    } else if (q < kOffB2) {
      const int j = (q - kOffW2) / kMlpH, k = (q - kOffW2) % kMlpH;
      for (int b = b0; b < b1; b++) acc = fmaf(dZ[(size_t)(kMlpH + j) * nb + b], A[(size_t)k * nb + b], acc);
    } else if (q < kOffW3) {
      const int j = q - kOffB2;
      for (int b = b0; b < b1; b++) acc += dZ[(size_t)(kMlpH + j) * nb + b];
    } else if (q < kOffB3) {
      const int j = (q - kOffW3) / kMlpH, k = (q - kOffW3) % kMlpH;
      for (int b = b0; b < b1; b++) acc = fmaf(dZ[(size_t)(2 * kMlpH + j) * nb + b], A[(size_t)(kMlpH + k) * nb + b], acc);
    } else if (q < kOffW4) {
      const int j = q - kOffB3;
      for (int b = b0; b < b1; b++) acc += dZ[(size_t)(2 * kMlpH + j) * nb + b];
    } else if (q < kOffB4) {
      const int j = (q - kOffW4) / kMlpH, k = (q - kOffW4) % kMlpH;
      for (int b = b0; b < b1; b++) acc = fmaf(dZ[(size_t)(3 * kMlpH + j) * nb + b], A[(size_t)(2 * kMlpH + k) * nb + b], acc);
    } else {
      const int j = q - kOffB4;
      for (int b = b0; b < b1; b++) acc += dZ[(size_t)(3 * kMlpH + j) * nb + b];
    }
    out[q] = acc;
  }
}

__global__ void k_mlp_adam(float *__restrict__ p, float *__restrict__ m, float *__restrict__ v,
                           const float *__restrict__ part, float *__restrict__ grad_out, float lr, float b1,
                           float b2, float eps, float bc1, float bc2) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= kMlpParams) return;
  float g = 0.f;
  for (int s = 0; s < kGradSlices; s++) g += part[(size_t)s * kMlpParams + q];
  if (grad_out) grad_out[q] = g;
  if (lr == 0.f) return;  // gradient only
  const float mm = b1 * m[q] + (1.f - b1) * g;
  const float vv = b2 * v[q] + (1.f - b2) * g * g;
  m[q] = mm;
  v[q] = vv;
  p[q] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
}

__global__ void k_sum_sq(const float *__restrict__ x, int n, double *__restrict__ out) {
  __shared__ double red[256];
  double s = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += x[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

}  // namespace argot

using namespace argot;

extern "C" {

int argot_b200_mlp_num_params(void) { return kMlpParams; }

// Normalised blackbody spectra on a grid of nT temperatures,
// log10 T = 4 + 1.5 k / (nT - 1), and their six thin-limit integrals
// I_j0 = sum_nu w_j(nu) s_nu.  spec: nT x 256, i0: nT x 6 (host).
int argot_b200_mlp_spectra(int nT, double *spec, double *i0) {
  if (nT < 2 || !spec || !i0) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  MlpTables t;
  host_mlp_tables(t);
  std::vector<double> c(kNu);
  for (int k = 0; k < nT; k++) {
    const double lT = kTLo + (kTHi - kTLo) * (double)k / (double)(nT - 1);
    double norm;
    argot_b200_photon_counts(0, (float)std::pow(10.0, lT), c.data(), &norm);
    double tot = 0.0;
    for (int b = 0; b < kNu; b++) tot += c[b];
    for (int b = 0; b < kNu; b++) spec[(size_t)k * kNu + b] = c[b] / tot;
    for (int j = 0; j < kMlpOut; j++) {
      double s = 0.0;
      for (int b = 0; b < kNu; b++) s += t.w[j][b] * spec[(size_t)k * kNu + b];
      i0[(size_t)k * kMlpOut + j] = s;
    }
  }
  set_status(0);
  return 0;
}

int argot_b200_mlp_samples(const double *spec_dev, const double *i0_dev, int nT, uint64_t n, uint64_t seed,
                           float *X, float *Y, void *stream) {
  if (!spec_dev || !i0_dev || nT < 2 || (n && (!X || !Y))) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  int dev = 0;
  ARGOT_CUDA_TRY(cudaGetDevice(&dev));
  int rc = ensure_mlp_tables(dev);
  if (rc) return rc;
  if (n) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (n + 127) / 128;
    const int blocks = (int)(want < (uint64_t)sms * 32 ? want : (uint64_t)sms * 32);
    k_mlp_samples<<<blocks, 128, 0, (cudaStream_t)stream>>>(spec_dev, i0_dev, nT, n, seed, X, Y);
    ARGOT_CUDA_TRY(cudaGetLastError());
  }
  set_status(0);
  return 0;
}

// Workspace floats needed by a training step on a batch of nb samples.
uint64_t argot_b200_mlp_workspace(int nb) {
  return (uint64_t)nb * (3 * kMlpH) * 2 + (uint64_t)nb * (3 * kMlpH + kMlpOut) + (uint64_t)nb * kMlpOut +
         (uint64_t)kGradSlices * kMlpParams + (uint64_t)nb + 2;
}

// Forward only: normalised outputs O (6 x n, [output][sample]).
int argot_b200_mlp_forward(const float *params, const float *X, int n, float *O, void *stream) {
  if (!params || (n && (!X || !O))) { set_status(ARGOT_B200_EINVAL); return ARGOT_B200_EINVAL; }
  if (n) {
    k_mlp_fwd<false><<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(params, X, n, nullptr, nullptr, O);
    ARGOT_CUDA_TRY(cudaGetLastError());
  }
  set_status(0);
  return 0;
}

// One training step on the batch (X: nb x 4, Y: nb x 6 targets q_j):
// forward, backward, deterministic gradient reduction, Adam (lr > 0) or
// gradient only (lr == 0; grad_out receives the gradient if non-NULL).
// m, v: Adam moments (kMlpParams each); step: 1-based Adam step;
// loss_out (device double, optional): sum of squared normalised errors.
int argot_b200_mlp_train_step(float *params, float *m, float *v, const float *X, const float *Y, int nb,
                              float lr, int step, float *work, float *grad_out, double *loss_out, void *stream) {
  if (!params || !m || !v || !X || !Y || nb <= 0 || !work || step < 1) {
    set_status(ARGOT_B200_EINVAL);
    return ARGOT_B200_EINVAL;
  }
  cudaStream_t st = (cudaStream_t)stream;
  float *Z = work;
  float *A = Z + (size_t)nb * 3 * kMlpH;
  float *dZ = A + (size_t)nb * 3 * kMlpH;
  float *O = dZ + (size_t)nb * (3 * kMlpH + kMlpOut);
  float *part = O + (size_t)nb * kMlpOut;
  float *sq = part + (size_t)kGradSlices * kMlpParams;
  const int blocks = (nb + 127) / 128;
  k_mlp_fwd<true><<<blocks, 128, 0, st>>>(params, X, nb, Z, A, O);
  k_mlp_bwd<<<blocks, 128, 0, st>>>(params, Y, nb, Z, O, dZ, sq);
  k_mlp_wgrad<<<kGradSlices, 256, 0, st>>>(X, nb, A, dZ, part);
  const float b1 = 0.9f, b2 = 0.999f;
  const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
  k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(params, m, v, part, grad_out, lr, b1, b2, 1e-8f, bc1, bc2);
  if (loss_out) k_sum_sq<<<1, 256, 0, st>>>(sq, nb, loss_out);
  ARGOT_CUDA_TRY(cudaGetLastError());
  set_status(0);
  return 0;
}

}  // extern "C"
