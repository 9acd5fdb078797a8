// Learned initial guess for con2prim: a 3-64-64-1 ReLU network trained on the
// device with hand-written kernels, and the con2prim batch kernel that runs it
// before the Newton solve of rhllc::GetPhysValueStab
// (solvers/rhllc/src/rhllc_flux_stab.cpp:123-220).  The reference has no
// learned part; its plain guess p = max(m - E, 0, pmin) is the fallback.
//
// Features of U = (D, S, E), tau = E - D, Q = E - sqrt(|S|^2 + D^2) (the quantity
// of rhllc_flux_stab.cpp:133, which carries the thermal energy of cold fast
// flows that |S|/tau alone loses to cancellation), all built in FP64 from D,
// |S|/tau and tau/D:
//   f = (log(Q/tau), log max(|S|/tau, 1e-30), log(tau/D)), normalised (f - mu)/sigma;
// output y predicts (log(p/tau) - mu_t)/sigma_t, guess p0 = tau exp(y sigma_t + mu_t).
// Parameters (4481 floats): W1 [64][3], b1 [64], W2 [64][64] (row = output), b2,
// W3 [64], b3.
//
// Training (FP32, deterministic): one CTA of 128 threads per 128 samples runs the
// forward and backward pass with activations in shared memory, then forms its
// partial gradient with fixed-order loops; a second kernel sums the partials
// over CTAs in order; Adam updates the parameters.
//
// Inference, two kernels: k_mlp_guess evaluates the network for tiles of 128 states (the
// 64 x 64 hidden layer as one tcgen05 MMA with f16 operands and an FP32 accumulator in
// tensor memory, the first and last layers in FP32; the guess only seeds Newton, so f16
// is enough) and writes the initial pressures; k_c2p_guess runs Newton from them with the
// plain con2prim kernel's structure.  If Newton has not converged after `k_stall`
// iterations the state is solved again from the reference guess, so the result is always a
// converged reference Newton solve.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "hydro_phys.cuh"
#include "rng.h"
#include "coupled.h"
#include "rrhd_internal.h"
#include "umma.cuh"

using namespace rrhd;

namespace {

constexpr int H = 64;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + H * 3, OFF_W2 = OFF_B1 + H, OFF_B2 = OFF_W2 + H * H,
              OFF_W3 = OFF_B2 + H, OFF_B3 = OFF_W3 + H, NPARAM = OFF_B3 + 1;  // 4481
constexpr int TB = 128;  // training samples per CTA

struct Norm {
  float mu[3], sig[3], mu_t, sig_t;
};

// tau and Q are formed in FP64 (both are differences that cancel: Q carries the thermal
// energy of cold fast flows); the ratios and logarithms only feed a BF16 network and are
// taken in FP32 with the fast hardware approximations, so that the features cost a few
// FP32 instructions rather than three FP64 logarithms and divisions.
__device__ __forceinline__ bool features(const double *U, float *f, double &tau) {
  const double D = U[0], E = U[4];
  tau = E - D;
  const double m2 = (U[1] * U[1] + U[2] * U[2]) + U[3] * U[3];
  const double Q = E - sqrt(m2 + D * D);
  if (!(D > 0.0) || !(tau > 0.0) || !(Q > 0.0)) return false;
  const float tf = (float)tau;
  const float S = sqrtf((float)m2);
  f[0] = __logf(__fdividef((float)Q, tf));
  f[1] = __logf(fmaxf(__fdividef(S, tf), 1e-30f));
  f[2] = __logf(__fdividef(tf, (float)D));
  return isfinite(f[0]) && isfinite(f[1]) && isfinite(f[2]);
}

// raw features and targets of labelled states (U, p)
__global__ void k_prepare(const double *U, const double *p, int64_t n, float *x, float *t, uint8_t *ok) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float f[3];
  double tau;
  const bool good = features(U + 5 * i, f, tau) && p[i] > 0.0;
  x[3 * i] = good ? f[0] : 0.f;
  x[3 * i + 1] = good ? f[1] : 0.f;
  x[3 * i + 2] = good ? f[2] : 0.f;
  t[i] = good ? (float)log(p[i] / tau) : 0.f;
  ok[i] = good ? 1 : 0;
}

// forward + backward of one CTA's 128 samples; writes the CTA's partial gradient
// (sum over its samples of d(loss)/d(theta)) and its partial sum of squared residuals
__global__ void __launch_bounds__(TB) k_mlp_grad(const float *__restrict__ theta, const float *__restrict__ x,
                                                 const float *__restrict__ t, const int32_t *__restrict__ idx,
                                                 int64_t nb, Norm nm, float inv_n, float *__restrict__ gpart,
                                                 float *__restrict__ lpart) {
  extern __shared__ float sm[];
  float *sth = sm;                      // [NPARAM]
  float *sx = sth + NPARAM + 3;         // [TB][3]
  float *sh1 = sx + TB * 3;             // [TB][H+1]
  float *sh2 = sh1 + TB * (H + 1);      // [TB][H+1]
  float *sd2 = sh2 + TB * (H + 1);      // [TB][H+1] dL/da2
  float *sd1 = sd2 + TB * (H + 1);      // [TB][H+1] dL/da1
  float *sdy = sd1 + TB * (H + 1);      // [TB]
  float *sr2 = sdy + TB;                // [TB]
  const int s = threadIdx.x;
  for (int q = s; q < NPARAM; q += TB) sth[q] = theta[q];
  const int64_t j = (int64_t)blockIdx.x * TB + s;
  const bool live = j < nb;
  float xi[3] = {0.f, 0.f, 0.f}, ti = 0.f;
  if (live) {
    const int64_t i = idx ? idx[j] : j;
    for (int a = 0; a < 3; a++) xi[a] = (x[3 * i + a] - nm.mu[a]) / nm.sig[a];
    ti = (t[i] - nm.mu_t) / nm.sig_t;
  }
  for (int a = 0; a < 3; a++) sx[3 * s + a] = xi[a];
  __syncthreads();
  const float *W1 = sth + OFF_W1, *b1 = sth + OFF_B1, *W2 = sth + OFF_W2, *b2 = sth + OFF_B2, *W3 = sth + OFF_W3;
  float *h1 = sh1 + s * (H + 1), *h2 = sh2 + s * (H + 1), *d2 = sd2 + s * (H + 1), *d1 = sd1 + s * (H + 1);
  for (int k = 0; k < H; k++) h1[k] = fmaxf(fmaf(W1[3 * k + 2], xi[2], fmaf(W1[3 * k + 1], xi[1], fmaf(W1[3 * k], xi[0], b1[k]))), 0.f);
  float y = sth[OFF_B3];
  for (int o = 0; o < H; o++) {
    float a = b2[o];
    for (int k = 0; k < H; k++) a = fmaf(W2[o * H + k], h1[k], a);
    h2[o] = fmaxf(a, 0.f);
    y = fmaf(W3[o], h2[o], y);
  }
  const float r = live ? y - ti : 0.f;
  const float dy = 2.f * r * inv_n;
  sdy[s] = dy;
  sr2[s] = r * r;
  for (int o = 0; o < H; o++) d2[o] = h2[o] > 0.f ? dy * W3[o] : 0.f;
  for (int k = 0; k < H; k++) {
    float g = 0.f;
    for (int o = 0; o < H; o++) g = fmaf(W2[o * H + k], d2[o], g);
    d1[k] = h1[k] > 0.f ? g : 0.f;
  }
  __syncthreads();
  float *gp = gpart + (int64_t)blockIdx.x * NPARAM;
  // dW2[o][k] = sum_s d2[s][o] h1[s][k]
  for (int e = s; e < H * H; e += TB) {
    const int o = e / H, k = e % H;
    float g = 0.f;
    for (int q = 0; q < TB; q++) g = fmaf(sd2[q * (H + 1) + o], sh1[q * (H + 1) + k], g);
    gp[OFF_W2 + e] = g;
  }
  for (int e = s; e < H; e += TB) {
    float gb2 = 0.f, gw3 = 0.f, gb1 = 0.f, gw1[3] = {0.f, 0.f, 0.f};
    for (int q = 0; q < TB; q++) {
      gb2 += sd2[q * (H + 1) + e];
      gw3 = fmaf(sdy[q], sh2[q * (H + 1) + e], gw3);
      const float dd = sd1[q * (H + 1) + e];
      gb1 += dd;
      for (int a = 0; a < 3; a++) gw1[a] = fmaf(dd, sx[3 * q + a], gw1[a]);
    }
    gp[OFF_B2 + e] = gb2;
    gp[OFF_W3 + e] = gw3;
    gp[OFF_B1 + e] = gb1;
    for (int a = 0; a < 3; a++) gp[OFF_W1 + 3 * e + a] = gw1[a];
  }
  if (s == 0) {
    float gb3 = 0.f, l = 0.f;
    for (int q = 0; q < TB; q++) {
      gb3 += sdy[q];
      l += sr2[q];
    }
    gp[OFF_B3] = gb3;
    lpart[blockIdx.x] = l;
  }
}

__global__ void k_sum_parts(const float *__restrict__ part, int nblk, int width, float *__restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= width) return;
  float g = 0.f;
  for (int b = 0; b < nblk; b++) g += part[(int64_t)b * width + p];
  out[p] = g;
}

__global__ void k_adam(float *theta, float *m, float *v, const float *g, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NPARAM) return;
  const float gg = g[p];
  const float mm = b1 * m[p] + (1.f - b1) * gg;
  const float vv = b2 * v[p] + (1.f - b2) * gg * gg;
  m[p] = mm;
  v[p] = vv;
  theta[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
}

__device__ __forceinline__ uint32_t pack_f16(float lo, float hi) {
  return (uint32_t)__half_as_ushort(__float2half_rn(lo)) | ((uint32_t)__half_as_ushort(__float2half_rn(hi)) << 16);
}

// ---------------------------------------------------------------- inference
// The guess kernel: one CTA of 128 threads per tile of 128 states (thread t = state t = row t
// of both layer products = TMEM lane t), persistent over tiles.  Per tile:
//   the features (FP32 from FP64 differences), normalised, and a constant 1 as row t of the
//   f16 A tile (K = 16, columns 4-15 zero);
//   layer 1 as one 128 x 64 x 16 tcgen05 MMA against [W1 | b1] (f16, FP32 accumulator in 64
//   TMEM columns); the thread reads its row back and writes ReLU(h1) as f16 into row t of
//   the same A tile (K = 64);
//   layer 2 as four 128 x 64 x 16 MMAs against W2 into the same TMEM columns;
//   b2, ReLU and layer 3 (64 -> 1) in FP32 from the thread's TMEM row, with b2, W3 and b3
//   taken from the kernel's parameter (constant bank).
// A and B tiles are K-major, 128-byte swizzled.  Output p0 = tau exp(y sigma_t + mu_t), or 0
// where the state has no usable features or the network gives a non-finite y (the Newton
// kernel then uses the reference guess).
constexpr int GT = 128;
constexpr int G_SMEM = 1024 /*alignment*/ + GT * 128 /*A*/ + 2 * H * 128 /*B1, B2*/ + 64 /*barrier, TMEM slot*/;

// [W1 | b1] (k 0-2 the weights, k 3 the bias, k 4-63 zero) and W2 as the f16 B operands of
// the two MMAs: K-major, 64 rows each, 128-byte swizzled, 8 KiB each.
__global__ void k_pack_b(const float *theta, __half *b1t, __half *w2t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= H * H) return;
  const int nrow = i / H, k = i - nrow * H;
  w2t[rrhd_umma::sw128_offset(nrow, k) / 2] = __float2half_rn(theta[OFF_W2 + i]);
  const float v = k < 3 ? theta[OFF_W1 + 3 * nrow + k] : k == 3 ? theta[OFF_B1 + nrow] : 0.f;
  b1t[rrhd_umma::sw128_offset(nrow, k) / 2] = __float2half_rn(v);
}

struct MlpPartial {
  unsigned long long ok, guess_fallback, fallback, failed, iters, max_iters, err;
};

// the last layer's parameters, passed by value: the kernel's FP32 multiply-adds take them
// from the constant bank, with no load instructions
struct MlpOuter {
  float b2w3[H][2];  // b2[j], W3[j]
  float b3;
};

// ReLU of two FP32 values packed as f16x2 (lo in the low half) in one conversion
__device__ __forceinline__ uint32_t relu_f16x2(float lo, float hi) {
  uint32_t d;
  asm("cvt.rn.relu.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}

// 16 TMEM columns of the warp's 32 lanes (this thread's row) from column c0
__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
}

__global__ void __launch_bounds__(GT) k_mlp_guess(const double *__restrict__ U, int64_t stride,
                                                  const double *__restrict__ G4, double tau_src, int64_t n,
                                                  const __grid_constant__ MlpOuter pw, const uint4 *__restrict__ b1t,
                                                  const uint4 *__restrict__ w2t, Norm nm, double *__restrict__ p0_out,
                                                  int *err) {
  using namespace rrhd_umma;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *sm = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t *sA = sm;               // [128 states][64] f16: the features, then h1
  uint8_t *sB1 = sm + GT * 128;   // [64 hidden][64] f16: [W1 | b1 | 0]
  uint8_t *sB2 = sB1 + H * 128;   // [64 out][64 in] f16: W2
  uint64_t *bar = reinterpret_cast<uint64_t *>(sB2 + H * 128);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
  const int t = threadIdx.x, warp = t >> 5;
  for (int q = t; q < H * 128 / 16; q += GT) {
    reinterpret_cast<uint4 *>(sB1)[q] = b1t[q];
    reinterpret_cast<uint4 *>(sB2)[q] = w2t[q];
  }
  if (t == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;\n" ::"r"(smem_u32(tslot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's TMEM lanes
  const uint64_t adesc = umma_desc(smem_u32(sA)), b1desc = umma_desc(smem_u32(sB1)), b2desc = umma_desc(smem_u32(sB2));
  constexpr uint32_t idesc = umma_idesc(0, H, GT);
  const float isig[3] = {1.f / nm.sig[0], 1.f / nm.sig[1], 1.f / nm.sig[2]};
  const int64_t ntiles = (n + GT - 1) / GT;
  uint32_t phase = 0;
  bool ok = true;
  // one MMA group and its completion (bounded waits; false after a timeout)
  auto mma_sync = [&](uint64_t bdesc, int ksteps) -> bool {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // A writes -> async proxy
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (t == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      for (int kk = 0; kk < ksteps; kk++) umma(tmem, adesc + 2 * kk, bdesc + 2 * kk, idesc, kk > 0 ? 1u : 0u);
      umma_commit(bar);
    }
    bool got = mbar_wait(bar, phase);
    if (!got) got = mbar_wait(bar, phase);  // a second bounded wait before giving up
    phase ^= 1u;
    if (__syncthreads_or(!got)) {
      if (t == 0) atomicOr(err, 1);
      return false;
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    return true;
  };
  // the state of the thread's next tile is loaded one tile ahead (with the source added)
  double un[5];
  auto load_state = [&](int64_t rt) {
    const int64_t i = rt * GT + t;
    if (rt < ntiles && i < n) {
#pragma unroll
      for (int q = 0; q < 5; q++) un[q] = U[stride * i + q];
      if (G4) {
        un[4] += tau_src * G4[4 * i];
        un[1] += tau_src * G4[4 * i + 1];
        un[2] += tau_src * G4[4 * i + 2];
        un[3] += tau_src * G4[4 * i + 3];
      }
    }
  };
  load_state(blockIdx.x);
  for (int64_t rt = blockIdx.x; rt < ntiles && ok; rt += gridDim.x) {  // CTA-uniform
    const int64_t i = rt * GT + t;
    double u[5];
#pragma unroll
    for (int q = 0; q < 5; q++) u[q] = un[q];
    load_state(rt + gridDim.x);
    float x[3] = {0.f, 0.f, 0.f};
    double tau = 0.0;
    bool feat = false;
    if (i < n) {
      float f[3];
      feat = features(u, f, tau);
      if (feat)
#pragma unroll
        for (int a = 0; a < 3; a++) x[a] = (f[a] - nm.mu[a]) * isig[a];
    }
    // row t, k 0-15: the features, 1 (the bias), zeros
    *reinterpret_cast<uint4 *>(sA + sw128_offset(t, 0)) =
        make_uint4(pack_f16(x[0], x[1]), pack_f16(x[2], 1.f), 0u, 0u);
    *reinterpret_cast<uint4 *>(sA + sw128_offset(t, 8)) = make_uint4(0u, 0u, 0u, 0u);
    if (!mma_sync(b1desc, 1)) {
      ok = false;
      break;
    }
    // ReLU(h1) as f16 into row t (the MMA has read the features)
#pragma unroll
    for (int c0 = 0; c0 < H; c0 += 16) {
      uint32_t r[16];
      tmem_ld16(trow + (uint32_t)c0, r);
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
      for (int h = 0; h < 2; h++)
        *reinterpret_cast<uint4 *>(sA + sw128_offset(t, c0 + 8 * h)) = make_uint4(
            relu_f16x2(__uint_as_float(r[8 * h]), __uint_as_float(r[8 * h + 1])),
            relu_f16x2(__uint_as_float(r[8 * h + 2]), __uint_as_float(r[8 * h + 3])),
            relu_f16x2(__uint_as_float(r[8 * h + 4]), __uint_as_float(r[8 * h + 5])),
            relu_f16x2(__uint_as_float(r[8 * h + 6]), __uint_as_float(r[8 * h + 7])));
    }
    if (!mma_sync(b2desc, H / 16)) {
      ok = false;
      break;
    }
    float ys[4] = {pw.b3, 0.f, 0.f, 0.f};  // four partial sums: short dependency chains
#pragma unroll
    for (int c0 = 0; c0 < H; c0 += 16) {
      uint32_t r[16];
      tmem_ld16(trow + (uint32_t)c0, r);
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
      for (int q = 0; q < 16; q++)
        ys[q & 3] = fmaf(pw.b2w3[c0 + q][1], fmaxf(__uint_as_float(r[q]) + pw.b2w3[c0 + q][0], 0.f), ys[q & 3]);
    }
    const float y = (ys[0] + ys[1]) + (ys[2] + ys[3]);
    if (i < n) p0_out[i] = (feat && isfinite(y)) ? tau * (double)__expf(y * nm.sig_t + nm.mu_t) : 0.0;
    // this tile's TMEM reads and A reads are ordered before the next tile's writes and MMA
    // by the next barrier
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  }
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;\n" ::"r"(tmem));
  }
}

// PhysPressureFix out of line: the rare fallback does not add to the registers of the
// kernel's main path.
// The state goes in and out by value: a pointer to the kernel's own arrays would put them in
// local memory for the whole loop, not only for this call.
struct FixState {
  double u[5], w[5];
  int code;
};
__device__ __noinline__ FixState pressure_fix_call(Eos eos, FixState s) {
  s.code = pressure_fix(eos, s.u, s.w);
  return s;
}

// The Newton kernel (the structure of the plain k_c2p_stats: 8 states per thread, the
// states that fail set aside in shared memory for a second pass).  States i live at
// U + stride*i and W + stride*i (stride 5 for separate arrays, 10 for a solver state
// [n][10] = U, W).  With G4 != NULL the radiation source is added first, U.E += tau G0 and
// U.S += tau G[1..3] (radRHD_main.cpp:117-126), and U is written back.  Per state: Newton
// from the learned guess p0[i] for at most k_stall iterations; if that stalls, or p0[i] is
// not a usable guess, the reference solve from its own guess; then (second pass)
// PhysPressureFix when fallback != 0.
constexpr int kGThreads = 256;
constexpr int kGPerThread = 8;
constexpr int kGPerBlock = kGThreads * kGPerThread;
#ifndef RRHD_MLP_MIN_BLOCKS
#define RRHD_MLP_MIN_BLOCKS 3  // CTAs per SM the register budget of k_c2p_guess is sized for
#endif
__global__ void __launch_bounds__(kGThreads, RRHD_MLP_MIN_BLOCKS)
    k_c2p_guess(Eos eos, double *U, double *W, int64_t stride, const double *G4, double tau_src,
                const double *__restrict__ p0s, uint8_t *status, int64_t n, int fallback, int k_stall,
                MlpPartial *scratch) {
  __shared__ unsigned short s_fail[kGPerBlock];  // local index | code << 12
  __shared__ int s_nfail;
  __shared__ unsigned long long red[6][kGThreads / 32];
  if (threadIdx.x == 0) s_nfail = 0;
  __syncthreads();
  unsigned ok = 0, gfb = 0, fb = 0, failed = 0, iters = 0, mx = 0;
  const int64_t base = (int64_t)blockIdx.x * kGPerBlock;
  for (int k = 0; k < kGPerThread; k++) {
    const int loc = k * kGThreads + threadIdx.x;
    const int64_t i = base + loc;
    if (i >= n) break;
    double u[5], w[5];  // w: the solve's output (the Newton solve reads no old W)
    for (int q = 0; q < 5; q++) u[q] = U[stride * i + q];
    if (G4) {
      u[4] += tau_src * G4[4 * i];
      u[1] += tau_src * G4[4 * i + 1];
      u[2] += tau_src * G4[4 * i + 2];
      u[3] += tau_src * G4[4 * i + 3];
      for (int q = 0; q < 5; q++) U[stride * i + q] = u[q];
    }
    const double p0 = p0s[i];
    const bool usable = p0 > 0.0;
    int code = 1, itn = 0;
    if (!usable) gfb++;
    for (int attempt = usable ? 0 : 1; attempt < 2; attempt++) {
      int it = 0;
      code = c2p_from(eos, u, w, p0, attempt == 0, &it, attempt == 0 ? k_stall : RRHD_MAX_ITER);
      itn += it;
      if (code == 0) break;
      if (attempt == 0) gfb++;
    }
    iters += (unsigned)itn;
    mx = (unsigned)itn > mx ? (unsigned)itn : mx;
    if (code == 0) {
      ok++;
      for (int q = 0; q < 5; q++) W[stride * i + q] = w[q];
      if (status) status[i] = 0;
    } else {
      s_fail[atomicAdd(&s_nfail, 1)] = (unsigned short)(loc | (code << 12));
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < s_nfail; q += kGThreads) {
    const int64_t i = base + (s_fail[q] & 0xfff);
    int code = s_fail[q] >> 12;
    FixState fs;
    for (int r = 0; r < 5; r++) {
      fs.u[r] = U[stride * i + r];
      fs.w[r] = W[stride * i + r];
    }
    if (fallback) {
      fs = pressure_fix_call(eos, fs);
      code = code | 0x10 | (fs.code ? 0x20 : 0);
      fb++;
      failed += fs.code ? 1 : 0;
      for (int r = 0; r < 5; r++) U[stride * i + r] = fs.u[r];
    } else {
      failed++;
    }
    for (int r = 0; r < 5; r++) W[stride * i + r] = fs.w[r];
    if (status) status[i] = (uint8_t)code;
  }
  unsigned long long okl = ok, gfbl = gfb, fbl = fb, failedl = failed, itl = iters, mxl = mx;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    okl += __shfl_xor_sync(0xffffffffu, okl, o);
    gfbl += __shfl_xor_sync(0xffffffffu, gfbl, o);
    fbl += __shfl_xor_sync(0xffffffffu, fbl, o);
    failedl += __shfl_xor_sync(0xffffffffu, failedl, o);
    itl += __shfl_xor_sync(0xffffffffu, itl, o);
    const unsigned long long m2 = __shfl_xor_sync(0xffffffffu, mxl, o);
    mxl = m2 > mxl ? m2 : mxl;
  }
  const int wid = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][wid] = okl;
    red[1][wid] = gfbl;
    red[2][wid] = fbl;
    red[3][wid] = failedl;
    red[4][wid] = itl;
    red[5][wid] = mxl;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    MlpPartial p = {0, 0, 0, 0, 0, 0, 0};
    for (int q = 0; q < kGThreads / 32; q++) {
      p.ok += red[0][q];
      p.guess_fallback += red[1][q];
      p.fallback += red[2][q];
      p.failed += red[3][q];
      p.iters += red[4][q];
      p.max_iters = red[5][q] > p.max_iters ? red[5][q] : p.max_iters;
    }
    scratch[blockIdx.x] = p;
  }
}

// Sums the per-CTA partials into scratch[nblocks] (integer counts: exact in any order) and
// moves the guess kernel's error word into it (err reset for the next call).
__global__ void __launch_bounds__(256) k_mlp_stats_reduce(MlpPartial *scratch, int nblocks, int *err) {
  __shared__ MlpPartial red[256];
  MlpPartial t = {0, 0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += 256) {
    const MlpPartial q = scratch[b];
    t.ok += q.ok;
    t.guess_fallback += q.guess_fallback;
    t.fallback += q.fallback;
    t.failed += q.failed;
    t.iters += q.iters;
    t.max_iters = q.max_iters > t.max_iters ? q.max_iters : t.max_iters;
  }
  red[threadIdx.x] = t;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      MlpPartial &a = red[threadIdx.x];
      const MlpPartial b = red[threadIdx.x + o];
      a.ok += b.ok;
      a.guess_fallback += b.guess_fallback;
      a.fallback += b.fallback;
      a.failed += b.failed;
      a.iters += b.iters;
      a.max_iters = b.max_iters > a.max_iters ? b.max_iters : a.max_iters;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    red[0].err = (unsigned long long)*err;
    *err = 0;
    scratch[nblocks] = red[0];
  }
}

Eos make_eos(int eos, double gamma) {
  Eos e;
  e.eos = eos;
  e.g1 = gamma;
  e.gg = gamma / (gamma - 1.0);
  return e;
}

}  // namespace

struct rrhd_mlp {
  int device = 0;
  float *d_theta = nullptr, *d_m = nullptr, *d_v = nullptr, *d_grad = nullptr;
  __half *d_b1t = nullptr, *d_w2t = nullptr;  // [W1 | b1] and W2 as the f16 UMMA operands
  MlpOuter outer{};         // b2, W3, b3 for the guess kernel's parameter
  MlpPartial *d_stats = nullptr;
  int stats_cap = 0;
  double *d_guess = nullptr;  // initial pressures when the caller passes no array
  int64_t guess_cap = 0;
  int *d_err = nullptr;  // a wait of the guess kernel that timed out
  Norm norm{{0, 0, 0}, {1, 1, 1}, 0, 1};
  int adam_t = 0;
  int num_sms = 148;
};

// the inference copies of the parameters (after every change of d_theta)
static rrhd_status mlp_refresh(rrhd_mlp *m, cudaStream_t st) {
  k_pack_b<<<H * H / 256, 256, 0, st>>>(m->d_theta, m->d_b1t, m->d_w2t);
  RRHD_CUDA(cudaGetLastError());
  std::vector<float> th(NPARAM);
  RRHD_CUDA(cudaMemcpyAsync(th.data(), m->d_theta, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, st));
  RRHD_CUDA(cudaStreamSynchronize(st));
  for (int j = 0; j < H; j++) {
    m->outer.b2w3[j][0] = th[OFF_B2 + j];
    m->outer.b2w3[j][1] = th[OFF_W3 + j];
  }
  m->outer.b3 = th[OFF_B3];
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_mlp_create(int32_t device, uint64_t seed, rrhd_mlp **out) {
  RRHD_CHECK_ARG(out, "null argument");
  *out = nullptr;
  RRHD_CUDA(cudaSetDevice(device));
  rrhd_mlp *m = new rrhd_mlp();
  m->device = device;
  cudaDeviceGetAttribute(&m->num_sms, cudaDevAttrMultiProcessorCount, device);
  // He-normal weights from the counter RNG, zero biases
  std::vector<float> th(NPARAM, 0.f);
  auto normal = [&](uint64_t i) {
    const double u1 = rrhd_u01(seed, 77, 2 * i) + 0x1.0p-54, u2 = rrhd_u01(seed, 77, 2 * i + 1);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * 3.141592653589793 * u2);
  };
  for (int q = 0; q < H * 3; q++) th[OFF_W1 + q] = (float)(normal(q) * std::sqrt(2.0 / 3.0));
  for (int q = 0; q < H * H; q++) th[OFF_W2 + q] = (float)(normal(1000 + q) * std::sqrt(2.0 / H));
  for (int q = 0; q < H; q++) th[OFF_W3 + q] = (float)(normal(9000 + q) * std::sqrt(1.0 / H));
  if (cudaMalloc(&m->d_theta, NPARAM * 4) || cudaMalloc(&m->d_m, NPARAM * 4) || cudaMalloc(&m->d_v, NPARAM * 4) ||
      cudaMalloc(&m->d_grad, NPARAM * 4) || cudaMalloc(&m->d_b1t, H * H * 2) || cudaMalloc(&m->d_w2t, H * H * 2) ||
      cudaMalloc(&m->d_err, sizeof(int))) {
    rrhd_mlp_destroy(m);
    return rrhd_fail(RRHD_ERR_OOM, "network allocation failed");
  }
  cudaMemcpy(m->d_theta, th.data(), NPARAM * 4, cudaMemcpyHostToDevice);
  cudaMemset(m->d_m, 0, NPARAM * 4);
  cudaMemset(m->d_v, 0, NPARAM * 4);
  cudaMemset(m->d_err, 0, sizeof(int));
  rrhd_status s = mlp_refresh(m, 0);
  if (s) {
    rrhd_mlp_destroy(m);
    return s;
  }
  RRHD_CUDA(cudaDeviceSynchronize());
  *out = m;
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_mlp_destroy(rrhd_mlp *m) {
  if (!m) return RRHD_OK;
  cudaSetDevice(m->device);
  cudaFree(m->d_theta);
  cudaFree(m->d_m);
  cudaFree(m->d_v);
  cudaFree(m->d_grad);
  cudaFree(m->d_b1t);
  cudaFree(m->d_w2t);
  cudaFree(m->d_guess);
  cudaFree(m->d_err);
  cudaFree(m->d_stats);
  delete m;
  return RRHD_OK;
}

extern "C" int32_t rrhd_mlp_num_params(void) { return NPARAM; }

// theta: host [4481]; norm: host [8] = mu[3], sigma[3], mu_t, sigma_t (either may be NULL)
extern "C" rrhd_status rrhd_mlp_set(rrhd_mlp *m, const float *theta, const float *norm) {
  RRHD_CHECK_ARG(m, "null network");
  RRHD_CUDA(cudaSetDevice(m->device));
  if (theta) RRHD_CUDA(cudaMemcpy(m->d_theta, theta, NPARAM * 4, cudaMemcpyHostToDevice));
  if (norm) {
    for (int a = 0; a < 3; a++) {
      m->norm.mu[a] = norm[a];
      m->norm.sig[a] = norm[3 + a];
    }
    m->norm.mu_t = norm[6];
    m->norm.sig_t = norm[7];
  }
  rrhd_status s = mlp_refresh(m, 0);
  if (s) return s;
  RRHD_CUDA(cudaDeviceSynchronize());
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_mlp_get(const rrhd_mlp *m, float *theta, float *norm) {
  RRHD_CHECK_ARG(m, "null network");
  RRHD_CUDA(cudaSetDevice(m->device));
  if (theta) RRHD_CUDA(cudaMemcpy(theta, m->d_theta, NPARAM * 4, cudaMemcpyDeviceToHost));
  if (norm) {
    for (int a = 0; a < 3; a++) {
      norm[a] = m->norm.mu[a];
      norm[3 + a] = m->norm.sig[a];
    }
    norm[6] = m->norm.mu_t;
    norm[7] = m->norm.sig_t;
  }
  return RRHD_OK;
}

// Loss and gradient of the current parameters over the labelled states
// (U [n][5], p [n], device).  grad: device [4481] (may be NULL); loss: host.
// One CTA per 128 samples; the gradient is of the mean squared error over n.
static rrhd_status grad_batch(rrhd_mlp *m, const float *x, const float *t, const int32_t *idx, int64_t nb,
                              float *gpart, float *lpart, float *grad, float *loss, cudaStream_t st) {
  const int nblk = (int)((nb + TB - 1) / TB);
  const size_t smem = sizeof(float) * (NPARAM + 3 + TB * 3 + 4 * TB * (H + 1) + 2 * TB);
  static bool attr = false;
  if (!attr) {
    RRHD_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  k_mlp_grad<<<nblk, TB, smem, st>>>(m->d_theta, x, t, idx, nb, m->norm, 1.f / (float)nb, gpart, lpart);
  RRHD_CUDA(cudaGetLastError());
  k_sum_parts<<<(NPARAM + 255) / 256, 256, 0, st>>>(gpart, nblk, NPARAM, grad);
  RRHD_CUDA(cudaGetLastError());
  if (loss) {
    k_sum_parts<<<1, 32, 0, st>>>(lpart, nblk, 1, grad + NPARAM);
    RRHD_CUDA(cudaGetLastError());
  }
  return RRHD_OK;
}

static void compute_norm(const std::vector<float> &x, const std::vector<float> &t, const std::vector<uint8_t> &ok,
                         Norm &nm) {
  double s[4] = {0, 0, 0, 0}, s2[4] = {0, 0, 0, 0};
  int64_t c = 0;
  for (size_t i = 0; i < ok.size(); i++) {
    if (!ok[i]) continue;
    c++;
    for (int a = 0; a < 3; a++) {
      s[a] += x[3 * i + a];
      s2[a] += (double)x[3 * i + a] * x[3 * i + a];
    }
    s[3] += t[i];
    s2[3] += (double)t[i] * t[i];
  }
  c = std::max<int64_t>(c, 1);
  for (int a = 0; a < 4; a++) {
    const double mu = s[a] / c, var = std::max(s2[a] / c - mu * mu, 1e-12);
    if (a < 3) {
      nm.mu[a] = (float)mu;
      nm.sig[a] = (float)std::sqrt(var);
    } else {
      nm.mu_t = (float)mu;
      nm.sig_t = (float)std::sqrt(var);
    }
  }
}

// Trains the network on labelled states: U [n][5] (device), p [n] (device) the
// pressures that con2prim should return.  Feature normalisation is set from the
// data when `set_norm` != 0.  Mini-batches of `batch` samples in a seeded random
// order; Adam with learning rate lr (halved at 50 % and 75 % of the epochs).
// loss_hist (host, may be NULL) receives the mean squared normalised error of
// each epoch.
extern "C" rrhd_status rrhd_mlp_train(rrhd_mlp *m, const double *U, const double *p, int64_t n, int32_t epochs,
                                      int32_t batch, float lr, uint64_t seed, int32_t set_norm, float *loss_hist,
                                      void *stream) {
  RRHD_CHECK_ARG(m && U && p && n > 0 && epochs > 0 && batch >= TB && n < (int64_t(1) << 31), "bad arguments");
  RRHD_CUDA(cudaSetDevice(m->device));
  cudaStream_t st = (cudaStream_t)stream;
  float *x = nullptr, *t = nullptr, *gpart = nullptr, *lpart = nullptr, *lsteps = nullptr;
  uint8_t *ok = nullptr;
  int32_t *idx = nullptr;
  const int nblk = (batch + TB - 1) / TB;
  auto cleanup = [&]() {
    cudaFree(lsteps);
    cudaFree(x);
    cudaFree(t);
    cudaFree(ok);
    cudaFree(idx);
    cudaFree(gpart);
    cudaFree(lpart);
  };
  if (cudaMalloc(&x, sizeof(float) * 3 * n) || cudaMalloc(&t, sizeof(float) * n) || cudaMalloc(&ok, n) ||
      cudaMalloc(&idx, sizeof(int32_t) * n) || cudaMalloc(&gpart, sizeof(float) * NPARAM * (size_t)nblk) ||
      cudaMalloc(&lpart, sizeof(float) * nblk) || cudaMalloc(&lsteps, sizeof(float) * (n / batch + 1))) {
    cleanup();
    return rrhd_fail(RRHD_ERR_OOM, "training buffers");
  }
  k_prepare<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(U, p, n, x, t, ok);
  std::vector<float> hx(3 * n), ht(n);
  std::vector<uint8_t> hok(n);
  cudaMemcpyAsync(hx.data(), x, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(ht.data(), t, sizeof(float) * n, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(hok.data(), ok, n, cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) {
    cleanup();
    return rrhd_fail(RRHD_ERR_CUDA, "preparing the training data failed");
  }
  if (set_norm) compute_norm(hx, ht, hok, m->norm);
  std::vector<int32_t> good;
  good.reserve(n);
  for (int64_t i = 0; i < n; i++)
    if (hok[i]) good.push_back((int32_t)i);
  const int64_t ng = (int64_t)good.size();
  if (ng < batch) {
    cleanup();
    return rrhd_fail(RRHD_ERR_INVALID, "fewer usable samples (%lld) than one batch", (long long)ng);
  }
  std::vector<float> lh(epochs, 0.f);
  for (int ep = 0; ep < epochs; ep++) {
    // seeded Fisher-Yates shuffle of the usable samples
    for (int64_t i = ng - 1; i > 0; i--) {
      const int64_t j = (int64_t)(rrhd_u01(seed, 1000 + ep, (uint64_t)i) * (double)(i + 1));
      std::swap(good[i], good[std::min(j, i)]);
    }
    cudaMemcpyAsync(idx, good.data(), sizeof(int32_t) * ng, cudaMemcpyHostToDevice, st);
    const float lr_ep = lr * (ep >= (3 * epochs) / 4 ? 0.25f : ep >= epochs / 2 ? 0.5f : 1.f);
    double esum = 0.0;
    int nsteps = 0;
    for (int64_t b0 = 0; b0 + batch <= ng; b0 += batch) {
      rrhd_status s = grad_batch(m, x, t, idx + b0, batch, gpart, lpart, m->d_grad, nullptr, st);
      if (s) {
        cleanup();
        return s;
      }
      m->adam_t++;
      const float c1 = 1.f - std::pow(0.9f, (float)m->adam_t), c2 = 1.f - std::pow(0.999f, (float)m->adam_t);
      k_adam<<<(NPARAM + 255) / 256, 256, 0, st>>>(m->d_theta, m->d_m, m->d_v, m->d_grad, lr_ep, 0.9f, 0.999f,
                                                   1e-8f, c1, c2);
      // loss of this batch (before the update) into the epoch's step array
      k_sum_parts<<<1, 32, 0, st>>>(lpart, nblk, 1, lsteps + nsteps);
      nsteps++;
    }
    std::vector<float> hl(nsteps);
    cudaMemcpyAsync(hl.data(), lsteps, sizeof(float) * nsteps, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
      cleanup();
      return rrhd_fail(RRHD_ERR_CUDA, "training step failed");
    }
    for (float v : hl) esum += v / batch;
    lh[ep] = (float)(esum / std::max(nsteps, 1));
  }
  rrhd_status s = mlp_refresh(m, st);
  cudaStreamSynchronize(st);
  cleanup();
  if (s) return s;
  if (loss_hist) std::copy(lh.begin(), lh.end(), loss_hist);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

// Gradient of the mean squared normalised error over all n labelled states at
// the current parameters: grad host [4481], loss host.  For checking the
// backward kernels against a reference implementation.
extern "C" rrhd_status rrhd_mlp_gradient(rrhd_mlp *m, const double *U, const double *p, int64_t n, float *grad,
                                         float *loss) {
  RRHD_CHECK_ARG(m && U && p && n > 0 && grad, "bad arguments");
  RRHD_CUDA(cudaSetDevice(m->device));
  float *x = nullptr, *t = nullptr, *gpart = nullptr, *lpart = nullptr, *g = nullptr;
  uint8_t *ok = nullptr;
  const int nblk = (int)((n + TB - 1) / TB);
  cudaMalloc(&x, sizeof(float) * 3 * n);
  cudaMalloc(&t, sizeof(float) * n);
  cudaMalloc(&ok, n);
  cudaMalloc(&gpart, sizeof(float) * NPARAM * (size_t)nblk);
  cudaMalloc(&lpart, sizeof(float) * nblk);
  cudaMalloc(&g, sizeof(float) * (NPARAM + 1));
  k_prepare<<<(unsigned)((n + 255) / 256), 256>>>(U, p, n, x, t, ok);
  rrhd_status s = grad_batch(m, x, t, nullptr, n, gpart, lpart, g, loss, 0);
  if (!s) {
    cudaMemcpy(grad, g, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost);
    if (loss) {
      float l;
      cudaMemcpy(&l, g + NPARAM, sizeof(float), cudaMemcpyDeviceToHost);
      *loss = l / (float)n;
    }
  }
  cudaFree(x);
  cudaFree(t);
  cudaFree(ok);
  cudaFree(gpart);
  cudaFree(lpart);
  cudaFree(g);
  RRHD_CUDA(cudaGetLastError());
  return s;
}

rrhd_status rrhd::mlp_c2p(const rrhd_mlp *m, int eos, double gamma, double *U, double *W, int64_t stride,
                          const double *G4, double tau_src, uint8_t *status, int64_t n, int fallback, int k_stall,
                          rrhd_c2p_stats *stats, int64_t *n_guess_fallback, double *guess, cudaStream_t st) {
  rrhd_mlp *mm = const_cast<rrhd_mlp *>(m);
  const int nblk = (int)std::max<int64_t>(1, (n + kGPerBlock - 1) / kGPerBlock);
  if (mm->stats_cap < nblk + 1 || (!guess && mm->guess_cap < n)) {
    RRHD_CUDA(cudaStreamSynchronize(st));
    if (mm->stats_cap < nblk + 1) {
      cudaFree(mm->d_stats);
      mm->d_stats = nullptr;
      RRHD_CUDA(cudaMalloc(&mm->d_stats, sizeof(MlpPartial) * (nblk + 1)));
      mm->stats_cap = nblk + 1;
    }
    if (!guess && mm->guess_cap < n) {
      cudaFree(mm->d_guess);
      mm->d_guess = nullptr;
      RRHD_CUDA(cudaMalloc(&mm->d_guess, sizeof(double) * n));
      mm->guess_cap = n;
    }
  }
  double *p0 = guess ? guess : mm->d_guess;
  if (n > 0) {
    // persistent CTAs: as many as are resident at once, from the kernel's registers and
    // shared memory (the occupancy calculator counts one CTA per SM for a kernel that
    // allocates tensor memory) and the 512 TMEM columns (64 per CTA)
    static int per_sm = 0;
    if (per_sm == 0) {
      RRHD_CUDA(cudaFuncSetAttribute(k_mlp_guess, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     (int)cudaSharedmemCarveoutMaxShared));
      cudaFuncAttributes fa;
      RRHD_CUDA(cudaFuncGetAttributes(&fa, k_mlp_guess));
      int smem_sm = 0;
      RRHD_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, m->device));
      const int by_regs = 65536 / (((fa.numRegs + 7) & ~7) * GT);
      const int by_smem = smem_sm / (G_SMEM + 1024);
      per_sm = std::max(1, std::min(std::min(by_regs, by_smem), 512 / 64));
    }
    const int64_t tiles = (n + GT - 1) / GT;
    const unsigned gblk = (unsigned)std::min<int64_t>(tiles, (int64_t)per_sm * m->num_sms);
    k_mlp_guess<<<gblk, GT, G_SMEM, st>>>(U, stride, G4, tau_src, n, m->outer,
                                          reinterpret_cast<const uint4 *>(m->d_b1t),
                                          reinterpret_cast<const uint4 *>(m->d_w2t), m->norm, p0, mm->d_err);
    RRHD_CUDA(cudaGetLastError());
    k_c2p_guess<<<nblk, kGThreads, 0, st>>>(make_eos(eos, gamma), U, W, stride, G4, tau_src, p0, status, n, fallback,
                                            k_stall, mm->d_stats);
    RRHD_CUDA(cudaGetLastError());
  } else {
    RRHD_CUDA(cudaMemsetAsync(mm->d_stats, 0, sizeof(MlpPartial), st));
  }
  k_mlp_stats_reduce<<<1, 256, 0, st>>>(mm->d_stats, nblk, mm->d_err);
  RRHD_CUDA(cudaGetLastError());
  if (stats || n_guess_fallback) {
    MlpPartial t;
    RRHD_CUDA(cudaMemcpyAsync(&t, mm->d_stats + nblk, sizeof t, cudaMemcpyDeviceToHost, st));
    RRHD_CUDA(cudaStreamSynchronize(st));
    if (stats) {
      stats->n_ok = (int64_t)t.ok;
      stats->n_fallback = (int64_t)t.fallback;
      stats->n_failed = (int64_t)t.failed;
      stats->newton_iters = (int64_t)t.iters;
      stats->max_iters = (int32_t)t.max_iters;
    }
    if (n_guess_fallback) *n_guess_fallback = (int64_t)t.guess_fallback;
    if (t.err) return rrhd_fail(RRHD_ERR_CUDA, "learned-guess kernel: a tensor-core completion wait timed out");
  }
  return RRHD_OK;
}

// con2prim batch seeded by the network: Newton from the learned guess for at
// most k_stall iterations, then (if needed) the reference solve from its own
// guess, then PhysPressureFix when fallback != 0.  stats (host, may be NULL).
// guess (device [n], may be NULL) receives the learned initial pressures (0 where the
// network gives no usable guess).
extern "C" rrhd_status rrhd_con2prim_batch_mlp(const rrhd_mlp *m, int32_t eos, double gamma, double *U, double *W,
                                               uint8_t *status, int64_t n, int32_t fallback, int32_t k_stall,
                                               rrhd_c2p_stats *stats, int64_t *n_guess_fallback, double *guess,
                                               void *stream) {
  RRHD_CHECK_ARG(m && n >= 0 && ((U && W) || n == 0) && k_stall > 0 && k_stall <= 40, "bad arguments");
  RRHD_CHECK_ARG(eos == RRHD_EOS_IDEAL || eos == RRHD_EOS_TAUB, "bad eos");
  return rrhd::mlp_c2p(m, eos, gamma, U, W, 5, nullptr, 0.0, status, n, fallback, k_stall, stats, n_guess_fallback,
                       guess, (cudaStream_t)stream);
}
