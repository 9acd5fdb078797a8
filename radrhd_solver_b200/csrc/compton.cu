// Frequency-coupled Compton scattering over the full 100-bin spectrum.
//
// For every cell i, output direction k and frequency bin f the reference
// (cuda/src/short_characteristics/separate_gpu/spectrum/cuda_scat_full_spectrum.cu:61-118,
// Get_full_spectrum_multi_device) sums over the M incoming directions d
//   S[i][k][f] = sum_d GammaC(k, d, f) I[i][d][bin(frq1)] a_d / A,
// where frq1 is the Doppler- and recoil-shifted frequency of bin centre frq_f
// (get_compton_frq, :8-20), GammaC the Klein-Nishina weight (:22-44) and bin() the
// log-spaced bin of frq1 (get_frq_idx, :50-53), with intensity below the first bin
// centre or above get_frq(99) cut to zero (:101-106).  Work is cells x K x 100 x M
// FP64 terms, a gather over shifted bins rather than a contraction, so this runs on
// the FP64 pipe, not the tensor cores.
//
// Restated per term (same quantities as the reference, regrouped):
//   el_f = hmc frq_f / lorenz,  A_k = 1 - v cosf_k,  C = 1 - cosTh,
//   den = (1 + el_f C) - v cosf1_d,  r = frq1 / frq = A_k / den,  frq1 = frq_f r,
//   GammaC a_d / A = (coef a_d / A) r (r + 1/r + cosTh^2 - 1) = (coef a_d / A) (r (r + cosTh^2 - 1) + 1),
// evaluated as h = y (A^2 y + A (cosTh^2 - 1)) + 1 with y = 1/den, frq1 = (frq_f A) y; the
// staged intensity rows carry the factor coef a_d / A.
// Cells with v^2 <= 1/c (kC_LightInv) take the recoil-only branch: A = 1, v = 0, lorenz = 1,
// and a pair with cosTh > 0.99999999 scatters without shift with weight 2 coef (:32-35),
// i.e. C = 0 and cosTh^2 - 1 = 0 above.
//
// The bin: the reference's idx = N - clamp(floor(sqrt(-betta ln(frq1/frq0)) + 1), 0, N)
// equals the number of edges get_frq(j), j = 1..99, strictly below frq1, and with the
// cut-offs folded in, c = #{edges E_0 < ... < E_99 below frq1} with E_0 the largest double
// below the low cut-off (so that frq1 == cut-off is kept, as `frq1 < cut` keeps it) selects
// slot c of a padded row [0, I_0 .. I_98, 0, 0].  An FP32 estimate t of sqrt(-betta ln(.))
// (error below 0.1) rounded to the nearest integer gives c or c - 1 as 100 - rint(t); one
// exact comparison with the edge table settles it.  Only a frq1 within rounding of a bin
// edge can land in the neighbouring bin relative to the reference's log / sqrt evaluation.
//
// The quantities the shift is made of -- v^2, lorenz, v cosf, v cosf1, cosTh and den -- are
// rounded as the reference's host build rounds them (one rounding per operation, no
// contraction, IEEE division and square root): in ultra-relativistic cells den = (1 + el C)
// - v cosf1 cancels to ~(1 - v), and any other grouping would move its last bits by up to
// 1/(1 - v) ulps of 1.  One decision is a knife edge by construction: the low cut-off
// equals the centre of bin 0, so in a Doppler cell the forward pair (k = d, shift ratio
// exactly 1) keeps or loses its bin-0 term on the last bit of frq1 = frq (1 - v cosf) / den;
// for bin 0 frq1 is therefore the IEEE quotient itself.  Elsewhere 1/den is a Newton-
// Raphson reciprocal (cubically convergent step e + e^2 from the hardware approximation).
//
// Layout: I [cells][M][100] and S [cells][out_stride][100] FP64 as in the reference;
// velocity [cells][3] in units of c.  One block per cell at a time (persistent over
// cells): the cell's intensity rows are staged into shared memory as padded rows, then
// each warp takes (32 output directions) x (FC frequency bins) items, a lane one output
// direction with FC accumulators, and runs over the staged directions.  More directions
// than fit in shared memory are taken in chunks, the partial sums kept in S.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "dirs.h"
#include "rrhd_internal.h"

namespace {

constexpr int kNFrq = 100;           // N_Frq, cuda_scat_full_spectrum.cu:47
constexpr double kFrq0 = 1e24;       // :48
constexpr double kBetta = 350;       // :49
constexpr int kRow = 102;            // padded row: slot 0 and slots 100, 101 are zero
constexpr int kThreads = 384;
constexpr int kWarps = kThreads / 32;
constexpr int kFC = 10;              // frequency bins per item
constexpr int kNfc = kNFrq / kFC;
static_assert(kNFrq % kFC == 0, "bins per item must divide the spectrum");
static_assert(kFC % 2 == 0, "items are read and written as pairs of bins (16-byte accesses)");

// CGS constants of lib/global_consts.h:34-44 as the same products
constexpr double kCLight = 3 * 1e10;
constexpr double kCLightInv = 1.0 / kCLight;
constexpr double kHmc = (6.62 * 1e-27) / (((9.109383701528 * 1e-28) * kCLight) * kCLight);
constexpr double kCoef = ((2 * 3.1415926535897932384626433832795) * (2.8179403 * 1e-13)) * (2.8179403 * 1e-13);
constexpr double kForward = 0.99999999;  // :32

// FP32 estimate of t^2 = -betta ln(x / frq0) = betta ln2 (log2 frq0 - log2 x)
constexpr float kBLn2 = (float)(kBetta * 0.69314718055994530942);
constexpr float kBLnF0 = (float)(kBetta * 55.262042231857095);  // betta ln(1e24)

struct CmpTables {
  double frq[kNFrq];   // bin centres 0.5 (get_frq(f + 1) + get_frq(f))
  double eps[kNFrq];   // hmc frq
  double edge[kNFrq + 1];  // E_0 .. E_99, +inf
};

double host_get_frq(int idx) {
  if (idx <= 0) return 0;
  const double x = kNFrq - idx;
  return kFrq0 * std::exp((-x * x) / kBetta);
}

const CmpTables &tables() {
  static const CmpTables t = [] {
    CmpTables h;
    for (int f = 0; f < kNFrq; f++) {
      h.frq[f] = 0.5 * (host_get_frq(f + 1) + host_get_frq(f));
      h.eps[f] = kHmc * h.frq[f];
    }
    h.edge[0] = std::nextafter(0.5 * (host_get_frq(1) + host_get_frq(0)), -INFINITY);
    for (int j = 1; j < kNFrq; j++) h.edge[j] = host_get_frq(j);
    h.edge[kNFrq] = INFINITY;
    return h;
  }();
  return t;
}

struct Smem {
  double el[kNFrq];
  double frq[kNFrq];
  long long edge[kNFrq + 1];
};

__host__ __device__ constexpr size_t cmp_smem(int dch) {
  return sizeof(Smem) + sizeof(double) * (size_t)dch * (kRow + 4);
}

// Vector3 dot product as the reference's host build rounds it: (x0 + x1) + x2, no FMA
__device__ __forceinline__ double dot_rn(double ax, double ay, double az, double bx, double by, double bz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(ax, bx), __dmul_rn(ay, by)), __dmul_rn(az, bz));
}

// 1/d for normal positive d: hardware approximation y (relative error e) refined by one
// Newton-Raphson step of cubic order, y (1 + e + e^2), e = 1 - d y.
__device__ __forceinline__ double rcp_nr(double d) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
  const double e = fma(-d, y, 1.0);
  return fma(y, fma(e, e, e), y);
}

// slot of the padded row that frq1 = x reads (0, 100 and 101 give zero).  The FP32
// estimate takes x's exponent and top 20 mantissa bits; invalid x (NaN, inf, <= 0) still
// gives a slot in 0 .. 101.
__device__ __forceinline__ int frq_slot(double x, const long long *edge) {
  const float xf = __uint_as_float(((unsigned)__double2hiint(x) - (896u << 20)) << 3);
  float lg, t;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(lg) : "f"(xf));
  const float t2 = fmaxf(fmaf(-kBLn2, lg, kBLnF0), 0.f);
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(t) : "f"(t2));
  int c = (0x4B400000 + kNFrq) - __float_as_int(t + 12582912.f);  // 100 - rint(t), t < 2^22
  c = max(c, 0);
  return c + (__double_as_longlong(x) > edge[c]);
}

__global__ void __launch_bounds__(kThreads, 1)
    k_compton_full(const double *__restrict__ I, const double *__restrict__ vel, const double *__restrict__ w,
                   const double *__restrict__ a, double inv_area, double *__restrict__ S, long long cells, int M,
                   int dir_disp, int dir_count, int out_stride, int dch, const CmpTables tab) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem &sm = *reinterpret_cast<Smem *>(smem_raw);
  double *sI = reinterpret_cast<double *>(smem_raw + sizeof(Smem));  // [dch][kRow]
  double *sWx = sI + (size_t)dch * kRow, *sWy = sWx + dch, *sWz = sWy + dch, *sVc1 = sWz + dch;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int j = tid; j <= kNFrq; j += kThreads) {
    sm.edge[j] = __double_as_longlong(tab.edge[j]);
    if (j < kNFrq) sm.frq[j] = tab.frq[j];
  }
  const int nkb = (dir_count + 31) / 32;
  const int items = nkb * kNfc;

  for (long long cell = blockIdx.x; cell < cells; cell += gridDim.x) {
    const double vx = vel[3 * cell], vy = vel[3 * cell + 1], vz = vel[3 * cell + 2];
    const double v2 = dot_rn(vx, vy, vz, vx, vy, vz);
    const bool doppler = v2 > kCLightInv;  // :84
    const double lorenz = doppler ? __ddiv_rn(1., __dsqrt_rn(__dadd_rn(1., -v2))) : 1.0;
    const double v = doppler ? __dsqrt_rn(v2) : 0.0;
    __syncthreads();  // the previous cell's readers are done with shared memory
    for (int j = tid; j < kNFrq; j += kThreads) sm.el[j] = __ddiv_rn(tab.eps[j], lorenz);

    for (int d0 = 0; d0 < M; d0 += dch) {
      const int nd = min(dch, M - d0);
      if (d0 > 0) __syncthreads();
      const double2 *src = reinterpret_cast<const double2 *>(I + ((size_t)cell * M + d0) * kNFrq);
      for (int e = tid; e < nd * (kNFrq / 2); e += kThreads) {
        const double2 p = __ldcs(src + e);
        const int dd = e / (kNFrq / 2), f = 2 * (e - dd * (kNFrq / 2));
        const double ca = kCoef * a[d0 + dd] * inv_area;
        double *row = sI + dd * kRow + 1 + f;
        row[0] = ca * p.x;
        row[1] = (f + 1 < kNFrq - 1) ? ca * p.y : 0.0;  // I_99 is never selected: its slot is a zero
      }
      for (int dd = tid; dd < nd; dd += kThreads) {
        double *row = sI + dd * kRow;
        row[0] = 0.0;
        row[kRow - 1] = 0.0;
        const double x = w[3 * (d0 + dd)], y = w[3 * (d0 + dd) + 1], z = w[3 * (d0 + dd) + 2];
        sWx[dd] = x;
        sWy[dd] = y;
        sWz[dd] = z;
        // v cosf1, cosf1 = vel . w_d / v (:27-28)
        sVc1[dd] = doppler ? __dmul_rn(v, __ddiv_rn(dot_rn(vx, vy, vz, x, y, z), v)) : 0.0;
      }
      __syncthreads();

      for (int it = warp; it < items; it += kWarps) {
        const int kb = it / kNfc, fc = it - kb * kNfc;
        const int k = kb * 32 + lane;
        const bool valid = k < dir_count;
        const int kk = dir_disp + (valid ? k : dir_count - 1);
        const double kx = w[3 * kk], ky = w[3 * kk + 1], kz = w[3 * kk + 2];
        // A_k = 1 - v cosf, cosf = vel . w_k / v (:85-87)
        const double A = doppler ? __dadd_rn(1., -__dmul_rn(v, __ddiv_rn(dot_rn(vx, vy, vz, kx, ky, kz), v))) : 1.0;
        const bool exact0 = doppler && fc == 0;  // this item holds bin 0 of a Doppler cell
        const double num0 = __dmul_rn(sm.frq[0], A), A2 = A * A;
        double el[kFC], fqA[kFC], acc[kFC];
        double *out = S + ((size_t)cell * out_stride + (valid ? k : 0)) * kNFrq + fc * kFC;
#pragma unroll
        for (int j = 0; j < kFC; j++) {
          el[j] = sm.el[fc * kFC + j];
          fqA[j] = sm.frq[fc * kFC + j] * A;
          acc[j] = 0.0;
        }
        if (d0 > 0 && valid) {
#pragma unroll
          for (int j = 0; j < kFC; j += 2) {
            const double2 p = *reinterpret_cast<const double2 *>(out + j);
            acc[j] = p.x;
            acc[j + 1] = p.y;
          }
        }
        for (int dd = 0; dd < nd; dd++) {
          const double cosTh = dot_rn(kx, ky, kz, sWx[dd], sWy[dd], sWz[dd]);
          double C = __dadd_rn(1.0, -cosTh), c2m1 = fma(cosTh, cosTh, -1.0);
          if (!doppler && cosTh > kForward) C = c2m1 = 0.0;  // :32-35: frq1 = frq, weight 2 coef
          const double vc1 = sVc1[dd], Ac = A * c2m1;
          const double *row = sI + dd * kRow;
#pragma unroll
          for (int j = 0; j < kFC; j++) {
            // den as get_compton_frq (:8-20) rounds it: (1 + el C) - v cosf1
            const double den = __dadd_rn(__dadd_rn(1.0, __dmul_rn(el[j], C)), -vc1);
            const double y = rcp_nr(den);
            const double x = (j == 0 && exact0) ? __ddiv_rn(num0, den) : fqA[j] * y;
            acc[j] = fma(fma(y, fma(A2, y, Ac), 1.0), row[frq_slot(x, sm.edge)], acc[j]);
          }
        }
        if (valid) {
#pragma unroll
          for (int j = 0; j < kFC; j += 2) *reinterpret_cast<double2 *>(out + j) = make_double2(acc[j], acc[j + 1]);
        }
      }
    }
  }
}

// Compton-shifted scattering integral at one frequency (cuda_scat_spectrum.cu:41-83,
// Get_spectrum_multi_device): S[i][k] = 0.25 sum_d GammaC(k, d, frq) I[i][d] a_d / A with
// the same weight as above but no forward special case (its GammaC, :22-39) and no bins.
// One block per cell at a time; the cell's directions, v cosf1 and 0.25 coef a_d I_d / A are
// staged in shared memory and each thread sums one output direction over all of them.
constexpr int kOneThreads = 256;
constexpr double kOneCfl = 0.25;  // :79

__global__ void __launch_bounds__(kOneThreads)
    k_compton_one(const double *__restrict__ I, const double *__restrict__ vel, const double *__restrict__ w,
                  const double *__restrict__ a, double scale, double eps, double *__restrict__ S, long long cells,
                  int M, int dir_disp, int dir_count, int out_stride) {
  extern __shared__ __align__(16) double sh1[];
  double *sWx = sh1, *sWy = sWx + M, *sWz = sWy + M, *sVc1 = sWz + M, *sIa = sVc1 + M;
  for (long long cell = blockIdx.x; cell < cells; cell += gridDim.x) {
    const double vx = vel[3 * cell], vy = vel[3 * cell + 1], vz = vel[3 * cell + 2];
    const double v2 = dot_rn(vx, vy, vz, vx, vy, vz);
    const bool doppler = v2 > kCLightInv;  // :63-68
    const double lorenz = doppler ? __ddiv_rn(1., __dsqrt_rn(__dadd_rn(1., -v2))) : 1.0;
    const double v = doppler ? __dsqrt_rn(v2) : 0.0;
    const double el = __ddiv_rn(eps, lorenz);
    __syncthreads();  // the previous cell's readers are done with shared memory
    for (int d = threadIdx.x; d < M; d += kOneThreads) {
      const double x = w[3 * d], y = w[3 * d + 1], z = w[3 * d + 2];
      sWx[d] = x;
      sWy[d] = y;
      sWz[d] = z;
      sVc1[d] = doppler ? __dmul_rn(v, __ddiv_rn(dot_rn(vx, vy, vz, x, y, z), v)) : 0.0;
      sIa[d] = scale * a[d] * I[cell * M + d];
    }
    __syncthreads();
    for (int k = threadIdx.x; k < dir_count; k += kOneThreads) {
      const int kk = dir_disp + k;
      const double kx = w[3 * kk], ky = w[3 * kk + 1], kz = w[3 * kk + 2];
      const double A = doppler ? __dadd_rn(1., -__dmul_rn(v, __ddiv_rn(dot_rn(vx, vy, vz, kx, ky, kz), v))) : 1.0;
      const double A2 = A * A;
      double acc0 = 0.0, acc1 = 0.0;
#pragma unroll 2
      for (int d = 0; d < M; d++) {
        const double cosTh = dot_rn(kx, ky, kz, sWx[d], sWy[d], sWz[d]);
        const double C = __dadd_rn(1.0, -cosTh), c2m1 = fma(cosTh, cosTh, -1.0);
        const double den = __dadd_rn(__dadd_rn(1.0, __dmul_rn(el, C)), -sVc1[d]);
        const double y = rcp_nr(den);
        const double t = fma(fma(y, fma(A2, y, A * c2m1), 1.0), sIa[d], (d & 1) ? acc1 : acc0);
        if (d & 1) acc1 = t; else acc0 = t;
      }
      S[cell * out_stride + k] = acc0 + acc1;
    }
  }
}

}  // namespace

extern "C" rrhd_status rrhd_compton_full_spectrum(const rrhd_dirs *d, const double *I, const double *velocity,
                                                  double *S, int64_t cells, int32_t dir_disp, int32_t dir_count,
                                                  int32_t out_stride, void *stream) {
  RRHD_CHECK_ARG(d && cells >= 0, "bad arguments");
  RRHD_CHECK_ARG(dir_disp >= 0 && dir_count >= 0 && (int64_t)dir_disp + dir_count <= d->M,
                 "directions dir_disp .. dir_disp + dir_count - 1 must lie in 0 .. M - 1");
  RRHD_CHECK_ARG(out_stride >= dir_count, "out_stride must be at least dir_count");
  if (cells == 0 || dir_count == 0) return RRHD_OK;
  RRHD_CHECK_ARG(I && velocity && S, "null I, velocity or S");
  RRHD_CHECK_ARG(((uintptr_t)I % 16) == 0 && ((uintptr_t)S % 16) == 0 && ((uintptr_t)velocity % 8) == 0,
                 "I and S must be 16-byte aligned, velocity 8-byte aligned");
  RRHD_CUDA(cudaSetDevice(d->device));
  int dev = 0, sms = 0, optin = 0;
  RRHD_CUDA(cudaGetDevice(&dev));
  RRHD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  RRHD_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  int dch = d->M;
  while (dch > 1 && cmp_smem(dch) > (size_t)optin) dch = (dch + 1) / 2;
  RRHD_CHECK_ARG(cmp_smem(dch) <= (size_t)optin, "no direction chunk fits in shared memory");
  const size_t sm = cmp_smem(dch);
  RRHD_CUDA(cudaFuncSetAttribute(k_compton_full, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const long long grid = std::min<long long>(cells, sms);
  k_compton_full<<<(unsigned)grid, kThreads, sm, (cudaStream_t)stream>>>(
      I, velocity, d->d_w, d->d_a, 1.0 / d->full_area, S, cells, d->M, dir_disp, dir_count, out_stride, dch,
      tables());
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_compton_spectrum(const rrhd_dirs *d, const double *I, const double *velocity, double *S,
                                             int64_t cells, double frq, int32_t dir_disp, int32_t dir_count,
                                             int32_t out_stride, void *stream) {
  RRHD_CHECK_ARG(d && cells >= 0, "bad arguments");
  RRHD_CHECK_ARG(frq > 0 && std::isfinite(frq), "frq must be positive and finite");
  RRHD_CHECK_ARG(dir_disp >= 0 && dir_count >= 0 && (int64_t)dir_disp + dir_count <= d->M,
                 "directions dir_disp .. dir_disp + dir_count - 1 must lie in 0 .. M - 1");
  RRHD_CHECK_ARG(out_stride >= dir_count, "out_stride must be at least dir_count");
  if (cells == 0 || dir_count == 0) return RRHD_OK;
  RRHD_CHECK_ARG(I && velocity && S, "null I, velocity or S");
  RRHD_CHECK_ARG(((uintptr_t)I % 8) == 0 && ((uintptr_t)S % 8) == 0 && ((uintptr_t)velocity % 8) == 0,
                 "I, S and velocity must be 8-byte aligned");
  RRHD_CUDA(cudaSetDevice(d->device));
  int dev = 0, sms = 0, optin = 0, per_sm = 0;
  RRHD_CUDA(cudaGetDevice(&dev));
  RRHD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  RRHD_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const size_t sm = sizeof(double) * 5 * (size_t)d->M;
  RRHD_CHECK_ARG(sm <= (size_t)optin, "too many directions for shared memory");
  if (sm > 48 * 1024)
    RRHD_CUDA(cudaFuncSetAttribute(k_compton_one, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  RRHD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_compton_one, kOneThreads, sm));
  const long long grid = std::min<long long>(cells, (long long)sms * std::max(per_sm, 1));
  // 0.25 coef / A (cfl, :79; the weight's 2 pi r_e^2, :35) folded into the staged intensity
  const double scale = kOneCfl * kCoef / d->full_area;
  k_compton_one<<<(unsigned)grid, kOneThreads, sm, (cudaStream_t)stream>>>(
      I, velocity, d->d_w, d->d_a, scale, kHmc * frq, S, cells, d->M, dir_disp, dir_count, out_stride);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}
