// Scattering integral and moments through the rank-7 structure of the Thomson
// phase function.
//
// The reference's Gamma(w_d, w_k) = 3 (1 + (w_d . w_k)^2) / 4 (solvers/illum/include/
// scattering.h:32-35, cuda/src/short_characteristics/cuda_integrator.cu:10-13) is,
// as a matrix over the directions, of rank 7:
//   (w_d . w_k)^2 = sum_ij w_d,i w_d,j w_k,i w_k,j,
// so the scattering integral S[k] = sum_d Gamma(w_d, w_k) I[d] a_d / A is
//   S[k] = 3/4 (m0 + w_k^T T w_k),   m0 = sum_d a_d I[d] / A,
//                                    T  = sum_d a_d w_d w_d^T I[d] / A,
// the energy and impulse moments of cuda_illum_sep_param.cu:9-69.  One pass over
// I gives the 10 moments (E, F, T) and S follows from them: O(M) work per row
// instead of O(M^2).  All arithmetic is FP64; I and S are FP64 or FP32.
//
// A warp takes 4 rows with 8 lanes each: the lanes of a row take every 8th
// direction, accumulate its 10 moments in FP64 with per-direction coefficients
// kept in shared memory (one column per coefficient), reduce them over the 8
// lanes with butterfly shuffles, then expand S for their directions.  Blocks loop
// over rows so that the coefficient tables are built once per block.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "coupled.h"
#include "dirs.h"
#include "rrhd_internal.h"

namespace {

constexpr int kLrThreads = 256;  // 8 warps = 8 cells in flight per block
constexpr int kLrWarps = kLrThreads / 32;
constexpr int kNIn = 10;   // moment coefficients per direction: a/A {1, x, y, z, xx, xy, xz, yy, yz, zz}
constexpr int kNOut = 6;   // expansion coefficients per direction: {xx, yy, zz, 2xy, 2xz, 2yz}

__host__ __device__ constexpr size_t lr_smem(int M) { return sizeof(double) * (size_t)M * (kNIn + kNOut); }

// coefficient tables, [coefficient][direction]
__device__ void lr_tables(int M, const double *w, const double *a, double inv_area, double *cin, double *cout) {
  for (int d = threadIdx.x; d < M; d += blockDim.x) {
    const double x = w[3 * d], y = w[3 * d + 1], z = w[3 * d + 2], s = a[d] * inv_area;
    cin[0 * M + d] = s;
    cin[1 * M + d] = s * x;
    cin[2 * M + d] = s * y;
    cin[3 * M + d] = s * z;
    cin[4 * M + d] = s * (x * x);
    cin[5 * M + d] = s * (x * y);
    cin[6 * M + d] = s * (x * z);
    cin[7 * M + d] = s * (y * y);
    cin[8 * M + d] = s * (y * z);
    cin[9 * M + d] = s * (z * z);
    cout[0 * M + d] = x * x;
    cout[1 * M + d] = y * y;
    cout[2 * M + d] = z * z;
    cout[3 * M + d] = 2.0 * (x * y);
    cout[4 * M + d] = 2.0 * (x * z);
    cout[5 * M + d] = 2.0 * (y * z);
  }
}

// A warp takes 4 rows (cell * NG + g) at a time, 8 lanes per row: lane = 4 dl + rr
// handles row rr and directions dl, dl + 8, ...  Element (row, d) sits at
// I[(cell * M + d) * NG + g] (NG = 1: the row layout), so one load instruction
// covers 8 consecutive directions of each of the 4 rows.  Every row sums its
// directions in the same order whatever the layout, so the layouts agree bit for bit.
constexpr int kRowsPerWarp = 4, kDirLanes = 8;

__device__ __forceinline__ int64_t lr_at(int64_t row, int d, int M, int NG) {
  return ((row / NG) * M + d) * NG + row % NG;
}

// the 10 moments of this lane's row, summed over its 8 lanes (every one of them gets them)
template <class T>
__device__ __forceinline__ void lr_moments(const T *I, int64_t row, bool live, int M, int NG, int dl,
                                           const double *cin, double (&m)[kNIn]) {
#pragma unroll
  for (int k = 0; k < kNIn; k++) m[k] = 0.0;
  constexpr int U = 8;
  for (int d0 = 0; d0 < M; d0 += kDirLanes * U) {
    double v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int d = d0 + kDirLanes * u + dl;
      v[u] = (live && d < M) ? (double)__ldcs(I + lr_at(row, d, M, NG)) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int d = d0 + kDirLanes * u + dl;
      if (d < M) {
#pragma unroll
        for (int k = 0; k < kNIn; k++) m[k] = fma(cin[k * M + d], v[u], m[k]);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kNIn; k++)
#pragma unroll
    for (int o = 16; o >= kRowsPerWarp; o >>= 1) m[k] += __shfl_xor_sync(0xffffffffu, m[k], o);
}

// S of direction d from the moments of one row
__device__ __forceinline__ double lr_expand(const double (&m)[kNIn], const double *cout, int M, int d) {
  const double diag = (cout[0 * M + d] * m[4] + cout[1 * M + d] * m[7]) + cout[2 * M + d] * m[9];
  const double off = (cout[3 * M + d] * m[5] + cout[4 * M + d] * m[6]) + cout[5 * M + d] * m[8];
  return 0.75 * ((m[0] + diag) + off);
}

// MOUT: 0 no moments, 1 [rows][16] in T {E, F, Txx, Txy, Txz, Tyy, Tyz, Tzz, 0...},
// 2 FP64 E [rows], F [rows][3], T [rows][3][3] (the plain coupled step's layout)
template <class T, int MOUT>
__global__ void __launch_bounds__(kLrThreads, 3) k_scatter_lowrank(int M, int NG, const double *w, const double *a,
                                                                 double inv_area, const T *I, T *S, T *mom,
                                                                 double *mE, double *mF, double *mT,
                                                                 int64_t rows) {
  extern __shared__ double lr_sm[];
  double *cin = lr_sm, *cout = lr_sm + kNIn * M;
  lr_tables(M, w, a, inv_area, cin, cout);
  __syncthreads();
  const int lane = threadIdx.x & 31, rr = lane & (kRowsPerWarp - 1), dl = lane >> 2;
  const int64_t step = (int64_t)gridDim.x * kLrWarps * kRowsPerWarp;
  for (int64_t r0 = ((int64_t)blockIdx.x * kLrWarps + (threadIdx.x >> 5)) * kRowsPerWarp; r0 < rows; r0 += step) {
    const int64_t row = r0 + rr;
    const bool live = row < rows;
    double m[kNIn];
    lr_moments<T>(I, row, live, M, NG, dl, cin, m);
    if (!live) continue;
    for (int d = dl; d < M; d += kDirLanes) S[lr_at(row, d, M, NG)] = (T)lr_expand(m, cout, M, d);
    if constexpr (MOUT == 1) {
      for (int col = dl; col < 16; col += kDirLanes) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < kNIn; k++) v = col == k ? m[k] : v;
        mom[row * 16 + col] = (T)v;
      }
    } else if constexpr (MOUT == 2) {
      if (dl == 0) {
        mE[row] = m[0];
        mF[3 * row] = m[1];
        mF[3 * row + 1] = m[2];
        mF[3 * row + 2] = m[3];
        double *t = mT + 9 * row;
        t[0] = m[4], t[1] = m[5], t[2] = m[6];
        t[3] = m[5], t[4] = m[7], t[5] = m[8];
        t[6] = m[6], t[7] = m[8], t[8] = m[9];
      }
    }
  }
}

// 4x4 transpose across a quad of lanes: lane p holds element [p][0..3] and ends
// with [0..3][p] (groups of one direction <-> directions of one group)
__device__ __forceinline__ float4 quad_transpose(float4 v, int lane) {
  const bool b0 = lane & 1, b1 = lane & 2;
  const float ra = __shfl_xor_sync(0xffffffffu, b0 ? v.x : v.y, 1);
  const float rb = __shfl_xor_sync(0xffffffffu, b0 ? v.z : v.w, 1);
  const float y0 = b0 ? ra : v.x, y1 = b0 ? v.y : ra;
  const float y2 = b0 ? rb : v.z, y3 = b0 ? v.w : rb;
  const float sa = __shfl_xor_sync(0xffffffffu, b1 ? y0 : y2, 2);
  const float sb = __shfl_xor_sync(0xffffffffu, b1 ? y1 : y3, 2);
  return make_float4(b1 ? sa : y0, b1 ? sb : y1, b1 ? y2 : sa, b1 ? y3 : sb);
}

// FP32, 4 groups: one warp per cell.  Each lane loads the 4 groups of one direction
// (16 bytes, consecutive lanes on consecutive directions), a quad transpose gives
// lane 4q + p group p of directions 4q..4q+3, and the 8 lanes of a group reduce
// its moments.  S goes back through the inverse transpose as 16-byte stores.  The
// per-row summation order differs from the generic kernel's (a few ulp of FP64).
template <int MOUT>
__global__ void __launch_bounds__(kLrThreads, 3) k_scatter_lowrank_f32g4(int M, const double *w, const double *a,
                                                                         double inv_area, const float *I, float *S,
                                                                         float *mom, int64_t cells) {
  extern __shared__ double lr_sm[];
  double *cin = lr_sm, *cout = lr_sm + kNIn * M;
  lr_tables(M, w, a, inv_area, cin, cout);
  __syncthreads();
  const int lane = threadIdx.x & 31, p = lane & 3, q = lane >> 2;
  for (int64_t c = (int64_t)blockIdx.x * kLrWarps + (threadIdx.x >> 5); c < cells; c += (int64_t)gridDim.x * kLrWarps) {
    const float4 *Ic = reinterpret_cast<const float4 *>(I) + c * M;
    double m[kNIn];
#pragma unroll
    for (int k = 0; k < kNIn; k++) m[k] = 0.0;
    for (int d0 = 0; d0 < M; d0 += 64) {
      float4 v[2];
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const int d = d0 + 32 * u + lane;
        v[u] = d < M ? __ldcs(Ic + d) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const float4 t = quad_transpose(v[u], lane);
        const float x[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const int d = d0 + 32 * u + 4 * q + i;
          if (d < M) {
#pragma unroll
            for (int k = 0; k < kNIn; k++) m[k] = fma(cin[k * M + d], (double)x[i], m[k]);
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kNIn; k++)
#pragma unroll
      for (int o = 16; o >= 4; o >>= 1) m[k] += __shfl_xor_sync(0xffffffffu, m[k], o);
    float4 *Sc = reinterpret_cast<float4 *>(S) + c * M;
    for (int d0 = 0; d0 < M; d0 += 32) {
      float x[4];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int d = d0 + 4 * q + i;
        x[i] = d < M ? (float)lr_expand(m, cout, M, d) : 0.f;
      }
      const float4 t = quad_transpose(make_float4(x[0], x[1], x[2], x[3]), lane);
      if (d0 + lane < M) __stcs(Sc + d0 + lane, t);
    }
    if constexpr (MOUT == 1) {
      for (int col = q; col < 16; col += 8) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < kNIn; k++) v = col == k ? m[k] : v;
        mom[(c * 4 + p) * 16 + col] = (float)v;
      }
    }
  }
}

// Error of another S (FP32, same layout) against the low-rank FP64 values, over every
// row-direction: acc_max = max relative error (the bits of a non-negative double,
// ordered like the values), acc_sq = sum of squared relative errors.
__global__ void __launch_bounds__(kLrThreads, 3) k_lowrank_error(int M, int NG, const double *w, const double *a,
                                                               double inv_area, const float *I, const float *St,
                                                               int64_t rows, unsigned long long *acc_max,
                                                               double *acc_sq) {
  extern __shared__ double lr_sm[];
  double *cin = lr_sm, *cout = lr_sm + kNIn * M;
  lr_tables(M, w, a, inv_area, cin, cout);
  __syncthreads();
  const int lane = threadIdx.x & 31, rr = lane & (kRowsPerWarp - 1), dl = lane >> 2;
  const int64_t step = (int64_t)gridDim.x * kLrWarps * kRowsPerWarp;
  double mx = 0.0, sq = 0.0;
  for (int64_t r0 = ((int64_t)blockIdx.x * kLrWarps + (threadIdx.x >> 5)) * kRowsPerWarp; r0 < rows; r0 += step) {
    const int64_t row = r0 + rr;
    const bool live = row < rows;
    double m[kNIn];
    lr_moments<float>(I, row, live, M, NG, dl, cin, m);
    if (!live) continue;
    for (int d = dl; d < M; d += kDirLanes) {
      const double ref = lr_expand(m, cout, M, d);
      const double rel = fabs((double)__ldcs(St + lr_at(row, d, M, NG)) - ref) / fabs(ref);
      mx = fmax(mx, rel);
      sq += rel * rel;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    sq += __shfl_xor_sync(0xffffffffu, sq, o);
  }
  if (lane == 0) {
    atomicMax(acc_max, (unsigned long long)__double_as_longlong(mx));
    atomicAdd(acc_sq, sq);
  }
}

unsigned lr_grid(int64_t rows, int device) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int64_t want = (rows + kLrWarps * kRowsPerWarp - 1) / (kLrWarps * kRowsPerWarp);
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * 8));
}

template <class T, int MOUT>
rrhd_status launch_lr(const rrhd_dirs *d, const T *I, T *S, T *mom, double *mE, double *mF, double *mT,
                      int64_t cells, int ng, cudaStream_t st) {
  const size_t sm = lr_smem(d->M);
  if (sm > 48 * 1024)
    RRHD_CUDA(cudaFuncSetAttribute(k_scatter_lowrank<T, MOUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const int64_t rows = cells * ng;
  k_scatter_lowrank<T, MOUT><<<lr_grid(rows, d->device), kLrThreads, sm, st>>>(
      d->M, ng, d->d_w, d->d_a, 1.0 / d->full_area, I, S, mom, mE, mF, mT, rows);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

template <int MOUT>
rrhd_status launch_lr_f32g4(const rrhd_dirs *d, const float *I, float *S, float *mom, int64_t cells,
                            cudaStream_t st) {
  const size_t sm = lr_smem(d->M);
  if (sm > 48 * 1024)
    RRHD_CUDA(cudaFuncSetAttribute(k_scatter_lowrank_f32g4<MOUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  k_scatter_lowrank_f32g4<MOUT><<<lr_grid(cells * kRowsPerWarp, d->device), kLrThreads, sm, st>>>(
      d->M, d->d_w, d->d_a, 1.0 / d->full_area, I, S, mom, cells);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

template <class T>
rrhd_status run_lr(const rrhd_dirs *d, const T *I, T *S, T *mom, double *mE, double *mF, double *mT,
                   int64_t cells, int ng, cudaStream_t st) {
  RRHD_CHECK_ARG(ng == 1 || ng == 2 || ng == 4, "low-rank scattering: groups must be 1, 2 or 4");
  if constexpr (sizeof(T) == 4) {
    if (ng == 4 && !mE && ((uintptr_t)I & 15) == 0 && ((uintptr_t)S & 15) == 0)
      return mom ? launch_lr_f32g4<1>(d, I, S, mom, cells, st) : launch_lr_f32g4<0>(d, I, S, mom, cells, st);
  }
  if (mom) return launch_lr<T, 1>(d, I, S, mom, mE, mF, mT, cells, ng, st);
  if (mE) return launch_lr<T, 2>(d, I, S, mom, mE, mF, mT, cells, ng, st);
  return launch_lr<T, 0>(d, I, S, mom, mE, mF, mT, cells, ng, st);
}

}  // namespace

rrhd_status rrhd::scatter_lowrank_fp64(const rrhd_dirs *d, const double *I, double *S, double *mE, double *mF,
                                       double *mT, int64_t cells, int G, cudaStream_t st) {
  RRHD_CHECK_ARG(d && I && S && cells >= 0, "bad arguments");
  if (cells == 0) return RRHD_OK;
  return run_lr<double>(d, I, S, nullptr, mE, mF, mT, cells, G, st);
}

rrhd_status rrhd::scatter_lowrank_fp32(const rrhd_dirs *d, const float *I, float *S, float *mom, int64_t cells,
                                       int G, cudaStream_t st) {
  RRHD_CHECK_ARG(d && I && S && cells >= 0, "bad arguments");
  if (cells == 0) return RRHD_OK;
  return run_lr<float>(d, I, S, mom, nullptr, nullptr, nullptr, cells, G, st);
}

extern "C" rrhd_status rrhd_scatter_lowrank(const rrhd_dirs *d, const void *I, void *S, void *moments,
                                            int64_t cells, int32_t groups, int32_t precision, void *stream) {
  RRHD_CHECK_ARG(d && cells >= 0, "bad arguments");
  RRHD_CHECK_ARG(precision == RRHD_RAD_FP64 || precision == RRHD_RAD_FP32, "precision must be RRHD_RAD_FP64 or FP32");
  RRHD_CHECK_ARG(groups == 1 || groups == 2 || groups == 4, "groups must be 1, 2 or 4");
  if (cells == 0) return RRHD_OK;
  RRHD_CHECK_ARG(I && S, "null I or S");
  const size_t al = precision == RRHD_RAD_FP64 ? 8 : 4;
  RRHD_CHECK_ARG(((uintptr_t)I % al) == 0 && ((uintptr_t)S % al) == 0 && ((uintptr_t)moments % al) == 0,
                 "I, S and moments must be aligned to their element size");
  RRHD_CUDA(cudaSetDevice(d->device));
  const cudaStream_t st = (cudaStream_t)stream;
  if (precision == RRHD_RAD_FP64)
    return run_lr<double>(d, (const double *)I, (double *)S, (double *)moments, nullptr, nullptr, nullptr, cells,
                          groups, st);
  return run_lr<float>(d, (const float *)I, (float *)S, (float *)moments, nullptr, nullptr, nullptr, cells, groups, st);
}

extern "C" rrhd_status rrhd_scatter_lowrank_error(const rrhd_dirs *d, const float *I, const float *S_test,
                                                  int64_t cells, int32_t groups, double *max_rel, double *rms_rel,
                                                  void *stream) {
  RRHD_CHECK_ARG(d && I && S_test && max_rel && rms_rel && cells > 0, "bad arguments");
  RRHD_CHECK_ARG(groups == 1 || groups == 2 || groups == 4, "groups must be 1, 2 or 4");
  RRHD_CHECK_ARG(((uintptr_t)I % 4) == 0 && ((uintptr_t)S_test % 4) == 0, "I and S must be 4-byte aligned");
  RRHD_CUDA(cudaSetDevice(d->device));
  const cudaStream_t st = (cudaStream_t)stream;
  void *buf = nullptr;
  RRHD_CUDA(cudaMalloc(&buf, 16));
  RRHD_CUDA(cudaMemsetAsync(buf, 0, 16, st));
  unsigned long long *amax = (unsigned long long *)buf;
  double *asq = (double *)buf + 1;
  const size_t sm = lr_smem(d->M);
  const unsigned grid = lr_grid(cells * groups, d->device);
  cudaError_t e = cudaSuccess;
  if (sm > 48 * 1024) e = cudaFuncSetAttribute(k_lowrank_error, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e == cudaSuccess)
    k_lowrank_error<<<grid, kLrThreads, sm, st>>>(d->M, groups, d->d_w, d->d_a, 1.0 / d->full_area, I, S_test,
                                                  cells * groups, amax, asq);
  if (e == cudaSuccess) e = cudaGetLastError();
  double h[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, buf, 16, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(buf);
  if (e != cudaSuccess) return rrhd_fail(RRHD_ERR_CUDA, "low-rank error pass: %s", cudaGetErrorString(e));
  *max_rel = h[0];  // the bits of the maximum, stored as an unsigned integer, are those of the double
  *rms_rel = sqrt(h[1] / ((double)cells * groups * d->M));
  return RRHD_OK;
}
