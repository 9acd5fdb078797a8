// FP64 radiation kernels: scattering integral, direction moments, 4-force.
//
// Compiled with --fmad=false: the "exact" kernels perform the reference's
// operations in the reference's order (one rounding each) and reproduce it bit
// for bit; the FMA variant of the scattering uses explicit fma() on a
// precomputed kernel matrix K[d][k] = Gamma(d,k) a_d / full_area.
//
// Scattering is a [rows x M] x [M x M] contraction with rows = cells x groups.
// Tiles: a CTA of 256 threads computes 64 rows x 64 output directions, each
// thread a 4 x 4 register block; I and K tiles of 32 directions are staged in
// shared memory (I rows padded to break bank conflicts).
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "rrhd_internal.h"

#include "dirs.h"
#include "coupled.h"
#include "rad_phys.cuh"

namespace {

constexpr int TR = 64, TK = 64, TD = 32;

// (3 (1 + mu^2)) / 4 with mu = (x0 + x1) + x2: cuda_integrator.cu:10-13
__global__ void k_build_gamma(int M, const double *w, const double *a, double A, double *G,
                              double *K) {
  const int d = blockIdx.y, k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= M) return;
  const double mu = (w[3 * d] * w[3 * k] + w[3 * d + 1] * w[3 * k + 1]) + w[3 * d + 2] * w[3 * k + 2];
  const double g = (3. * (1. + mu * mu)) / 4.;
  G[(size_t)d * M + k] = g;
  K[(size_t)d * M + k] = g * a[d] / A;
}

// Element (row r, direction d) of a [rows][M] array (lg < 0) or of a
// cell-direction-group array [rows >> lg][M][1 << lg] (row r = cell * 2^lg + group).
__device__ __forceinline__ int64_t elem(int64_t r, int d, int M, int lg) {
  return lg >= 0 ? (((r >> lg) * M + d) << lg) + (r & ((1 << lg) - 1)) : r * M + d;
}

// Tile element t of a (rows) x (nd directions) tile in memory order: row r, direction d.
__device__ __forceinline__ void tile_rd(int t, int nd, int lg, int &r, int &d) {
  if (lg >= 0) {
    const int g = t & ((1 << lg) - 1), q = t >> lg;
    d = q % nd;
    r = ((q / nd) << lg) + g;
  } else {
    r = t / nd;
    d = t % nd;
  }
}

template <bool EXACT>
__global__ void __launch_bounds__(256) k_scatter(int64_t rows, int M, int lg, const double *__restrict__ I,
                                                 const double *__restrict__ G,
                                                 const double *__restrict__ a, double A,
                                                 double *__restrict__ S) {
  // the input tiles, then (after the loop) the output tile staged for coalesced stores
  __shared__ double buf[TR * (TD + 1) + TD * TK];
  static_assert(TR * (TD + 1) + TD * TK >= TR * (TK + 1), "output tile must fit");
  double(*sI)[TD + 1] = reinterpret_cast<double(*)[TD + 1]>(buf);
  double(*sG)[TK] = reinterpret_cast<double(*)[TK]>(buf + TR * (TD + 1));
  __shared__ double sa[TD];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int64_t r0 = (int64_t)blockIdx.x * TR;
  const int k0 = blockIdx.y * TK;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0.0;

  for (int d0 = 0; d0 < M; d0 += TD) {
    // I tile: 64 rows x 32 directions
    for (int t = threadIdx.x; t < TR * TD; t += 256) {
      int r, d;
      tile_rd(t, TD, lg, r, d);
      const int64_t gr = r0 + r;
      sI[r][d] = (gr < rows && d0 + d < M) ? I[elem(gr, d0 + d, M, lg)] : 0.0;
    }
    for (int t = threadIdx.x; t < TD * TK; t += 256) {
      const int d = t / TK, k = t % TK;
      sG[d][k] = (d0 + d < M && k0 + k < M) ? G[(size_t)(d0 + d) * M + k0 + k] : 0.0;
    }
    if (threadIdx.x < TD) sa[threadIdx.x] = (d0 + threadIdx.x < M) ? a[d0 + threadIdx.x] : 0.0;
    __syncthreads();
    const int dn = min(TD, M - d0);
    for (int d = 0; d < dn; d++) {
      double iv[4], gv[4];
#pragma unroll
      for (int i = 0; i < 4; i++) iv[i] = sI[ty + 16 * i][d];
#pragma unroll
      for (int j = 0; j < 4; j++) gv[j] = sG[d][tx + 16 * j];
      if (EXACT) {
        const double ad = sa[d];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) {
            double t = gv[j] * iv[i];
            t = t * ad;
            acc[i][j] = acc[i][j] + t;
          }
      } else {
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) acc[i][j] = fma(iv[i], gv[j], acc[i][j]);
      }
    }
    __syncthreads();
  }
  double(*sO)[TK + 1] = reinterpret_cast<double(*)[TK + 1]>(buf);
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) sO[ty + 16 * i][tx + 16 * j] = EXACT ? acc[i][j] / A : acc[i][j];
  __syncthreads();
  // stores in memory order of the layout (consecutive threads, consecutive addresses)
  for (int t = threadIdx.x; t < TR * TK; t += 256) {
    int r, k;
    tile_rd(t, TK, lg, r, k);
    const int64_t gr = r0 + r;
    if (gr < rows && k0 + k < M) S[elem(gr, k0 + k, M, lg)] = sO[r][k];
  }
}

// cuda_sep::device::MakeEnergy / MakeStream / MakeImpuls
// (cuda_illum_sep_param.cu:9-69), one thread per row.
constexpr int MR = 128, MD = 32;
__global__ void __launch_bounds__(MR) k_moments(int64_t rows, int M, int lg, const double *__restrict__ I,
                                                const double *__restrict__ w,
                                                const double *__restrict__ a, double A,
                                                double *__restrict__ E, double *__restrict__ Fo,
                                                double *__restrict__ To) {
  __shared__ double sI[MR][MD + 1];
  __shared__ double sw[MD][3];
  __shared__ double sa[MD];
  const int64_t r0 = (int64_t)blockIdx.x * MR;
  const int64_t r = r0 + threadIdx.x;
  double e = 0, s0 = 0, s1 = 0, s2 = 0;
  double t[9];
#pragma unroll
  for (int i = 0; i < 9; i++) t[i] = 0;
  for (int d0 = 0; d0 < M; d0 += MD) {
    for (int q = threadIdx.x; q < MR * MD; q += MR) {
      int rr, d;
      tile_rd(q, MD, lg, rr, d);
      sI[rr][d] = (r0 + rr < rows && d0 + d < M) ? I[elem(r0 + rr, d0 + d, M, lg)] : 0.0;
    }
    if (threadIdx.x < MD) {
      const int d = d0 + threadIdx.x;
      sa[threadIdx.x] = d < M ? a[d] : 0.0;
      for (int x = 0; x < 3; x++) sw[threadIdx.x][x] = d < M ? w[3 * d + x] : 0.0;
    }
    __syncthreads();
    const int dn = min(MD, M - d0);
    for (int d = 0; d < dn; d++) {
      const double iv = sI[threadIdx.x][d];
      const double ad = sa[d];
      const double w0 = sw[d][0], w1 = sw[d][1], w2 = sw[d][2];
      e = e + iv * ad;
      const double Ia = iv * ad;
      s0 = s0 + w0 * Ia;
      s1 = s1 + w1 * Ia;
      s2 = s2 + w2 * Ia;
      const double ww[3] = {w0, w1, w2};
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int k = 0; k < 3; k++) t[3 * i + k] = t[3 * i + k] + ww[i] * ww[k] * Ia;
    }
    __syncthreads();
  }
  if (r < rows) {
    E[r] = e / A;
    Fo[3 * r + 0] = s0 / A;
    Fo[3 * r + 1] = s1 / A;
    Fo[3 * r + 2] = s2 / A;
#pragma unroll
    for (int i = 0; i < 9; i++) To[9 * r + i] = t[i] / A;
  }
}

// rad_rhd::GetRadSource, solvers/RadRHD/src/radRHD_utils.cpp:44-101
__global__ void k_rad_source(int64_t n, rrhd::Emission em, const double *__restrict__ W,
                             const double *__restrict__ alpha, const double *__restrict__ sigma,
                             const double *__restrict__ E, const double *__restrict__ F,
                             const double *__restrict__ T, double *__restrict__ G) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  double w[5], Fr[3], Tr[9], g[4];
#pragma unroll
  for (int i = 0; i < 5; i++) w[i] = W[5 * c + i];
#pragma unroll
  for (int i = 0; i < 3; i++) Fr[i] = F[3 * c + i];
#pragma unroll
  for (int i = 0; i < 9; i++) Tr[i] = T[9 * c + i];
  rrhd::rad_source_cell(em, w, alpha[c], sigma[c], E[c], Fr, Tr, g);
#pragma unroll
  for (int i = 0; i < 4; i++) G[4 * c + i] = g[i];
}

}  // namespace

extern "C" rrhd_status rrhd_dirs_create(int32_t M, const double *dirs, const double *areas,
                                        double full_area, int32_t device, rrhd_dirs **out) {
  RRHD_CHECK_ARG(out && dirs && areas && M > 0 && M <= 4096 && full_area > 0, "bad direction set");
  *out = nullptr;
  RRHD_CUDA(cudaSetDevice(device));
  rrhd_dirs *d = new rrhd_dirs();
  d->device = device;
  d->M = M;
  d->full_area = full_area;
  d->h_w.assign(dirs, dirs + 3 * M);
  d->h_a.assign(areas, areas + M);
  const size_t mm = sizeof(double) * (size_t)M * M;
  if (cudaMalloc(&d->d_w, sizeof(double) * 3 * M) || cudaMalloc(&d->d_a, sizeof(double) * M) ||
      cudaMalloc(&d->d_G, mm) || cudaMalloc(&d->d_K, mm)) {
    rrhd_dirs_destroy(d);
    return rrhd_fail(RRHD_ERR_OOM, "direction set allocation failed");
  }
  cudaMemcpy(d->d_w, dirs, sizeof(double) * 3 * M, cudaMemcpyHostToDevice);
  cudaMemcpy(d->d_a, areas, sizeof(double) * M, cudaMemcpyHostToDevice);
  k_build_gamma<<<dim3((M + 127) / 128, M), 128>>>(M, d->d_w, d->d_a, full_area, d->d_G, d->d_K);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    rrhd_dirs_destroy(d);
    return rrhd_fail(RRHD_ERR_CUDA, "building the phase matrix failed");
  }
  *out = d;
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_dirs_destroy(rrhd_dirs *d) {
  if (!d) return RRHD_OK;
  cudaSetDevice(d->device);
  cudaFree(d->d_w);
  cudaFree(d->d_a);
  cudaFree(d->d_G);
  cudaFree(d->d_K);
  delete d;
  return RRHD_OK;
}

extern "C" int32_t rrhd_dirs_count(const rrhd_dirs *d) { return d ? d->M : 0; }
extern "C" const double *rrhd_dirs_device_kernel(const rrhd_dirs *d) { return d ? d->d_K : nullptr; }

extern "C" rrhd_status rrhd_scatter_fp64(const rrhd_dirs *d, const double *I, double *S, int64_t rows,
                                         void *stream) {
  RRHD_CHECK_ARG(d && I && S && rows >= 0, "bad arguments");
  if (rows == 0) return RRHD_OK;
  dim3 grid((unsigned)((rows + TR - 1) / TR), (d->M + TK - 1) / TK);
  k_scatter<true><<<grid, 256, 0, (cudaStream_t)stream>>>(rows, d->M, -1, I, d->d_G, d->d_a, d->full_area, S);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

// Same contraction with one FMA per term on K = Gamma a / full_area (rounding
// differs from the reference's three roundings by a few ulp per term).
extern "C" rrhd_status rrhd_scatter_fp64_fma(const rrhd_dirs *d, const double *I, double *S, int64_t rows,
                                             void *stream) {
  RRHD_CHECK_ARG(d && I && S && rows >= 0, "bad arguments");
  if (rows == 0) return RRHD_OK;
  dim3 grid((unsigned)((rows + TR - 1) / TR), (d->M + TK - 1) / TK);
  k_scatter<false><<<grid, 256, 0, (cudaStream_t)stream>>>(rows, d->M, -1, I, d->d_K, d->d_a, d->full_area, S);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_moments_fp64(const rrhd_dirs *d, const double *I, double *E, double *F,
                                         double *T, int64_t rows, void *stream) {
  RRHD_CHECK_ARG(d && I && E && F && T && rows >= 0, "bad arguments");
  if (rows == 0) return RRHD_OK;
  k_moments<<<(unsigned)((rows + MR - 1) / MR), MR, 0, (cudaStream_t)stream>>>(rows, d->M, -1, I, d->d_w, d->d_a,
                                                                               d->full_area, E, F, T);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

rrhd_status rrhd::scatter_fp64_cdg(const rrhd_dirs *d, const double *I, double *S, int64_t cells, int ng, bool exact,
                                   cudaStream_t st) {
  RRHD_CHECK_ARG(d && I && S && cells >= 0 && ng > 0 && TR % ng == 0, "bad arguments");
  const int64_t rows = cells * ng;
  if (rows == 0) return RRHD_OK;
  int lg = 0;
  while ((1 << lg) < ng) lg++;
  dim3 grid((unsigned)((rows + TR - 1) / TR), (d->M + TK - 1) / TK);
  if (exact)
    k_scatter<true><<<grid, 256, 0, st>>>(rows, d->M, lg, I, d->d_G, d->d_a, d->full_area, S);
  else
    k_scatter<false><<<grid, 256, 0, st>>>(rows, d->M, lg, I, d->d_K, d->d_a, d->full_area, S);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

rrhd_status rrhd::moments_fp64_cdg(const rrhd_dirs *d, const double *I, double *E, double *F, double *T,
                                   int64_t cells, int ng, cudaStream_t st) {
  RRHD_CHECK_ARG(d && I && E && F && T && cells >= 0 && ng > 0 && MR % ng == 0, "bad arguments");
  const int64_t rows = cells * ng;
  if (rows == 0) return RRHD_OK;
  int lg = 0;
  while ((1 << lg) < ng) lg++;
  k_moments<<<(unsigned)((rows + MR - 1) / MR), MR, 0, st>>>(rows, d->M, lg, I, d->d_w, d->d_a, d->full_area, E, F,
                                                             T);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

extern "C" rrhd_emission rrhd_emission_reference(void) {
  // CGS constants of lib/global_consts.h and the unit system it defines
  const double kC_Light = 3 * 1e10, k_boltzmann = 1.3807 * 1e-16, kM_hydrogen = 1.6735575 * 1e-24;
  const double kStefanBoltzmann = 5.670374419 * 1e-5, kGravity = 6.6726 * 1e-8;
  const double PI = 3.1415926535897932384626433832795;
  const double kDist = 1e13, kVelocity = kC_Light;
  const double kMass = (kVelocity * kVelocity * kDist) / kGravity;
  const double kTime = (kDist / kVelocity);
  const double kDensity = (kMass / (kDist * kDist * kDist));
  const double kPressure = kMass / (kDist * kTime * kTime);
  const double kRadiation = (kMass / (kTime * kTime * kTime));
  rrhd_emission e;
  e.temp_coef = (kM_hydrogen / k_boltzmann) * kPressure / kDensity;
  e.sigma_sb = kStefanBoltzmann;
  e.pi = PI;
  e.rad_unit = kRadiation;
  return e;
}

extern "C" rrhd_status rrhd_rad_source(const rrhd_emission *em, const double *W, const double *alpha,
                                       const double *sigma, const double *E, const double *F, const double *T,
                                       double *G, int64_t n, void *stream) {
  RRHD_CHECK_ARG(em && W && alpha && sigma && E && F && T && G && n >= 0, "bad arguments");
  if (n == 0) return RRHD_OK;
  rrhd::Emission e{em->temp_coef, em->sigma_sb, em->pi, em->rad_unit};
  k_rad_source<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(n, e, W, alpha, sigma, E, F, T, G);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_scatter_fp64_cdg(const rrhd_dirs *d, const double *I, double *S, int64_t cells,
                                             int32_t groups, int32_t exact, void *stream) {
  return rrhd::scatter_fp64_cdg(d, I, S, cells, groups, exact != 0, (cudaStream_t)stream);
}

extern "C" rrhd_status rrhd_moments_fp64_cdg(const rrhd_dirs *d, const double *I, double *E, double *F, double *T,
                                             int64_t cells, int32_t groups, void *stream) {
  return rrhd::moments_fp64_cdg(d, I, E, F, T, cells, groups, (cudaStream_t)stream);
}
