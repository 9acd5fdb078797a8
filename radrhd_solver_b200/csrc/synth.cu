// Seeded synthetic intensity fields generated on the device (benchmark inputs;
// the reference reads its fields from files, so these have no counterpart there).
// Normal variates come from Box-Muller on the counter-based RNG of rng.h, so
// each element is a pure function of (seed, row, direction).
#include <cuda_runtime.h>

#include "rng.h"
#include "rrhd_internal.h"

namespace {

template <class T>
__global__ void k_fill(T *I, int64_t rows, int M, int groups, int kind, double sigma, const double *centers,
                       uint64_t seed) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= rows * M) return;
  const int64_t r = i / M;
  const int64_t k = i - r * M;
  const double u1 = rrhd_u01(seed, (uint64_t)r, 2 * (uint64_t)k) + 0x1.0p-54;  // (0, 1]
  const double u2 = rrhd_u01(seed, (uint64_t)r, 2 * (uint64_t)k + 1);
  const double z = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
  double v = exp(sigma * z);
  if (kind == 0) {
    if (centers) {
      const double *c = centers + 3 * (r / groups);
      v *= exp(-(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]) / 0.2);
    }
  } else {
    const int g = (int)(r % groups);
    v *= exp10(-6.0 + 6.0 * g / (double)(groups > 1 ? groups - 1 : 1));
  }
  I[i] = (T)v;
}

// Config-3 primitive states: rho log-uniform [1e-4, 1e2], p/rho log-uniform
// [1e-6, 1e2], Lorentz factor log-uniform [1, 50], isotropic velocity direction.
__global__ void k_fill_states(double *W, int64_t n, uint64_t seed) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double u0 = rrhd_u01(seed, 101, (uint64_t)i), u1 = rrhd_u01(seed, 102, (uint64_t)i);
  const double u2 = rrhd_u01(seed, 103, (uint64_t)i), u3 = rrhd_u01(seed, 104, (uint64_t)i);
  const double u4 = rrhd_u01(seed, 105, (uint64_t)i);
  const double rho = exp10(-4.0 + 6.0 * u0);
  const double p = rho * exp10(-6.0 + 8.0 * u1);
  const double lor = exp10(u2 * log10(50.0));
  const double v = sqrt(1.0 - 1.0 / (lor * lor));
  const double mu = 2.0 * u3 - 1.0, s = sqrt(fmax(0.0, 1.0 - mu * mu));
  const double ph = 2.0 * u4;  // in units of pi
  double *w = W + 5 * i;
  w[0] = rho;
  w[1] = v * s * cospi(ph);
  w[2] = v * s * sinpi(ph);
  w[3] = v * mu;
  w[4] = p;
}

}  // namespace

extern "C" rrhd_status rrhd_fill_c2p_states(double *W, int64_t n, uint64_t seed, void *stream) {
  RRHD_CHECK_ARG(n >= 0 && (W || n == 0), "bad arguments");
  if (n == 0) return RRHD_OK;
  k_fill_states<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(W, n, seed);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

template <class T>
static rrhd_status fill(T *I, int64_t rows, int32_t M, int32_t groups, int32_t kind, double sigma,
                        const double *centers, uint64_t seed, void *stream) {
  RRHD_CHECK_ARG(I && rows >= 0 && M > 0 && groups > 0 && (kind == 0 || kind == 1), "bad arguments");
  const int64_t n = rows * (int64_t)M;
  if (n == 0) return RRHD_OK;
  k_fill<T><<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(I, rows, M, groups, kind, sigma,
                                                                            centers, seed);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_fill_intensity_f32(float *I, int64_t rows, int32_t M, int32_t groups, int32_t kind,
                                               double sigma, const double *centers, uint64_t seed, void *stream) {
  return fill<float>(I, rows, M, groups, kind, sigma, centers, seed, stream);
}

extern "C" rrhd_status rrhd_fill_intensity_f64(double *I, int64_t rows, int32_t M, int32_t groups, int32_t kind,
                                               double sigma, const double *centers, uint64_t seed, void *stream) {
  return fill<double>(I, rows, M, groups, kind, sigma, centers, seed, stream);
}
