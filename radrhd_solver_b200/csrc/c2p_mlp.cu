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
// Inference: each warp evaluates 32 states at once, all three layers on the
// tensor cores as warp-level mma.sync (f16 operands, FP32 accumulation; the
// guess only seeds Newton, so f16 is enough).  Newton then starts from the guess; if it has
// not converged after `k_stall` iterations the state is solved again from the
// reference guess, so the result is always a converged reference Newton solve.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "hydro_phys.cuh"
#include "rng.h"
#include "coupled.h"
#include "rrhd_internal.h"

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

// B fragments of the three layers for mma.sync (f16 operands, FP32 accumulation), in
// uint32 words, each holding two f16 (the lower k index in the low half):
//   FR_W2 [n-tile 8][k-step 4][lane 32][2]  W2^T for m16n8k16 (k = hidden input, n = output)
//   FR_W1 [n-tile 8][lane 32]               [W1 | b1]^T for m16n8k8: k 0-2 the features,
//                                           k 3 the bias (its A column is 1), k 4-7 zero
//   FR_W3 [k-step 4][lane 32][2]            W3 as column 0 of an m16n8k16 B tile, the
//                                           other 7 columns zero
// Lane l of a B fragment holds column n = l / 4 and rows k = 2 (l % 4) + {0, 1} (+8 for
// the second word of a k16 fragment).
constexpr int FR_W2 = 0, FR_W1 = FR_W2 + 8 * 4 * 32 * 2, FR_W3 = FR_W1 + 8 * 32, NFRAG = FR_W3 + 4 * 32 * 2;  // 2560

__device__ __forceinline__ uint32_t pack_f16(float lo, float hi) {
  return (uint32_t)__half_as_ushort(__float2half_rn(lo)) | ((uint32_t)__half_as_ushort(__float2half_rn(hi)) << 16);
}

__global__ void k_pack_frags(const float *theta, uint32_t *frag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const float *W1 = theta + OFF_W1, *b1 = theta + OFF_B1, *W2 = theta + OFF_W2, *W3 = theta + OFF_W3;
  if (i < 8 * 4 * 32) {
    const int lane = i & 31, ks = (i >> 5) & 3, nt = i >> 7;
    const int n = 8 * nt + (lane >> 2), k0 = 16 * ks + 2 * (lane & 3);
    frag[FR_W2 + 2 * i] = pack_f16(W2[n * H + k0], W2[n * H + k0 + 1]);
    frag[FR_W2 + 2 * i + 1] = pack_f16(W2[n * H + k0 + 8], W2[n * H + k0 + 9]);
  } else if (i < 8 * 4 * 32 + 8 * 32) {
    const int j = i - 8 * 4 * 32, lane = j & 31, nt = j >> 5;
    const int n = 8 * nt + (lane >> 2), c = lane & 3;
    frag[FR_W1 + j] = c == 0 ? pack_f16(W1[3 * n], W1[3 * n + 1]) : c == 1 ? pack_f16(W1[3 * n + 2], b1[n]) : 0u;
  } else if (i < 8 * 4 * 32 + 8 * 32 + 4 * 32) {
    const int j = i - 8 * 4 * 32 - 8 * 32, lane = j & 31, ks = j >> 5;
    const int k0 = 16 * ks + 2 * (lane & 3);
    const bool col0 = (lane >> 2) == 0;
    frag[FR_W3 + 2 * j] = col0 ? pack_f16(W3[k0], W3[k0 + 1]) : 0u;
    frag[FR_W3 + 2 * j + 1] = col0 ? pack_f16(W3[k0 + 8], W3[k0 + 9]) : 0u;
  }
}

struct MlpPartial {
  unsigned long long ok, guess_fallback, fallback, failed, iters, max_iters;
};

constexpr int IT = 128;  // inference threads per CTA

// ReLU of two FP32 accumulators packed as f16x2 (lo in the low half) in one conversion
__device__ __forceinline__ uint32_t relu_f16x2(float lo, float hi) {
  uint32_t d;
  asm("cvt.rn.relu.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}

__device__ __forceinline__ void mma_k16(float *d, const uint32_t *a, uint2 b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

// Warp-cooperative guess for the 32 states of a warp (lane = state); returns this lane's
// y.  All three layers run on the tensor cores, one m16 tile (16 states) at a time:
// layer 1 as m16n8k8 over the features and a constant 1 (the bias), whose FP32 output
// fragments are, after ReLU and packing to f16, the A fragments of layer 2 as they are
// (the accumulator of n-tiles 2k, 2k+1 is the A operand of k-step k); the same for
// layer 3, whose B tile holds W3 in column 0.
__device__ __forceinline__ float mlp_warp(const float *xs, const float *sb2, float b3, const uint32_t *sfrag) {
  const int lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
  // A columns of layer 1 held by a lane: c = 0 features 0, 1; c = 1 feature 2 and the 1
  const uint32_t p01 = pack_f16(xs[0], xs[1]), p2 = pack_f16(xs[2], 1.f);
  float y = 0.f;
#pragma unroll 1
  for (int mt = 0; mt < 2; mt++) {
    const int r0 = 16 * mt + g;  // the states of rows g and g + 8 of this tile
    const uint32_t x0a = __shfl_sync(0xffffffffu, p01, r0), x0b = __shfl_sync(0xffffffffu, p2, r0);
    const uint32_t x1a = __shfl_sync(0xffffffffu, p01, r0 + 8), x1b = __shfl_sync(0xffffffffu, p2, r0 + 8);
    const uint32_t a10 = c == 0 ? x0a : c == 1 ? x0b : 0u, a11 = c == 0 ? x1a : c == 1 ? x1b : 0u;
    uint32_t a2[4][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      float h[4] = {0.f, 0.f, 0.f, 0.f};
      asm volatile(
          "mma.sync.aligned.m16n8k8.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
          : "+f"(h[0]), "+f"(h[1]), "+f"(h[2]), "+f"(h[3])
          : "r"(a10), "r"(a11), "r"(sfrag[FR_W1 + 32 * nt + lane]));
      a2[nt >> 1][2 * (nt & 1)] = relu_f16x2(h[0], h[1]);
      a2[nt >> 1][2 * (nt & 1) + 1] = relu_f16x2(h[2], h[3]);
    }
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      const float2 bb = *reinterpret_cast<const float2 *>(sb2 + 8 * nt + 2 * c);
      acc[nt][0] = bb.x;
      acc[nt][1] = bb.y;
      acc[nt][2] = bb.x;
      acc[nt][3] = bb.y;
    }
#pragma unroll
    for (int ks = 0; ks < 4; ks++)
#pragma unroll
      for (int nt = 0; nt < 8; nt++)
        mma_k16(acc[nt], a2[ks], *reinterpret_cast<const uint2 *>(sfrag + FR_W2 + 2 * ((nt * 4 + ks) * 32 + lane)));
    float o[4] = {b3, 0.f, b3, 0.f};
#pragma unroll
    for (int ks = 0; ks < 4; ks++) {
      const uint32_t a3[4] = {relu_f16x2(acc[2 * ks][0], acc[2 * ks][1]), relu_f16x2(acc[2 * ks][2], acc[2 * ks][3]),
                              relu_f16x2(acc[2 * ks + 1][0], acc[2 * ks + 1][1]),
                              relu_f16x2(acc[2 * ks + 1][2], acc[2 * ks + 1][3])};
      mma_k16(o, a3, *reinterpret_cast<const uint2 *>(sfrag + FR_W3 + 2 * (ks * 32 + lane)));
    }
    // column 0: row g in o[0], row g + 8 in o[2] of lane 4 g
    const float v0 = __shfl_sync(0xffffffffu, o[0], 4 * (lane & 7));
    const float v1 = __shfl_sync(0xffffffffu, o[2], 4 * (lane & 7));
    if ((lane >> 4) == mt) y = (lane & 8) ? v1 : v0;
  }
  return y;
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

// States i live at U + stride*i and W + stride*i (stride 5 for separate arrays,
// 10 for a solver state [n][10] = U, W).  With G4 != NULL the radiation source
// is added first, U.E += tau G0 and U.S += tau G[1..3] (radRHD_main.cpp:117-126).
#ifndef RRHD_MLP_MIN_BLOCKS
#define RRHD_MLP_MIN_BLOCKS 4  // CTAs per SM the register budget of k_c2p_mlp is sized for
#endif
__global__ void __launch_bounds__(IT, RRHD_MLP_MIN_BLOCKS) k_c2p_mlp(Eos eos, double *U, double *W, int64_t stride, const double *G4,
                                                double tau_src, uint8_t *status, int64_t n, int fallback,
                                                int k_stall, const float *__restrict__ theta,
                                                const uint32_t *__restrict__ frag, Norm nm, MlpPartial *scratch,
                                                double *guess_out) {
  __shared__ __align__(16) float sb2[H];
  __shared__ __align__(16) uint32_t sfrag[NFRAG];
  __shared__ unsigned long long red[6][IT / 32];
  for (int q = threadIdx.x; q < H; q += IT) sb2[q] = theta[OFF_B2 + q];
  for (int q = threadIdx.x; q < NFRAG; q += IT) sfrag[q] = frag[q];
  const float b3 = theta[OFF_B3];
  __syncthreads();
  unsigned ok = 0, gfb = 0, fb = 0, failed = 0, iters = 0, mx = 0;  // per thread (u32: a thread sees few states)
  const int lane = threadIdx.x & 31;
  const int64_t nwarps_total = (int64_t)gridDim.x * (IT / 32);
  for (int64_t w = (int64_t)blockIdx.x * (IT / 32) + (threadIdx.x >> 5); w * 32 < n; w += nwarps_total) {
    const int64_t i = w * 32 + lane;
    const bool live = i < n;
    // the state (with the radiation source added) is read twice: for the features, and
    // again after the network, so that it is not held in registers across the network
    auto load_u = [&](double *u) {
      for (int q = 0; q < 5; q++) u[q] = U[stride * i + q];
      if (G4) {
        u[4] += tau_src * G4[4 * i];
        u[1] += tau_src * G4[4 * i + 1];
        u[2] += tau_src * G4[4 * i + 2];
        u[3] += tau_src * G4[4 * i + 3];
      }
    };
    float f[3] = {0.f, 0.f, 0.f};
    double tau = 0.0;
    bool feat = false;
    if (live) {
      double u0[5];
      load_u(u0);
      feat = features(u0, f, tau);
    }
    float xs[3];
#pragma unroll
    for (int a = 0; a < 3; a++) xs[a] = feat ? (f[a] - nm.mu[a]) / nm.sig[a] : 0.f;
    const float y = mlp_warp(xs, sb2, b3, sfrag);
    double u[5] = {0, 0, 0, 0, 0}, wv[5] = {0, 0, 0, 0, 0};
    if (live) {
      load_u(u);
      for (int q = 0; q < 5; q++) wv[q] = W[stride * i + q];
    }
    if (!live) continue;
    bool u_dirty = G4 != nullptr;
    feat = feat && isfinite(y);  // an f16 overflow inside the network: the reference guess
    const double p0 = feat ? tau * (double)__expf(y * nm.sig_t + nm.mu_t) : 0.0;
    if (feat && guess_out) guess_out[i] = p0;
    // attempt 0: Newton from the learned guess for at most k_stall iterations; attempt 1
    // (a stalled or unusable guess): the reference solve from its own guess
    int code = 1, itn = 0;
    if (!feat) gfb++;
    for (int attempt = feat ? 0 : 1; attempt < 2; attempt++) {
      int it = 0;
      code = c2p_from(eos, u, wv, p0, attempt == 0, &it, attempt == 0 ? k_stall : RRHD_MAX_ITER);
      itn += it;
      if (code == 0) break;
      if (attempt == 0) gfb++;
    }
    if (code == 0) ok++;
    iters += (unsigned)itn;
    mx = (unsigned)itn > mx ? (unsigned)itn : mx;
    if (code) {
      if (fallback) {
        FixState fs;
#pragma unroll
        for (int q = 0; q < 5; q++) {
          fs.u[q] = u[q];
          fs.w[q] = wv[q];
        }
        fs = pressure_fix_call(eos, fs);
#pragma unroll
        for (int q = 0; q < 5; q++) {
          u[q] = fs.u[q];
          wv[q] = fs.w[q];
        }
        const int fix = fs.code;
        code = code | 0x10 | (fix ? 0x20 : 0);
        fb++;
        failed += fix ? 1 : 0;
        u_dirty = true;
      } else {
        failed++;
      }
    }
    if (u_dirty)
      for (int q = 0; q < 5; q++) U[stride * i + q] = u[q];
    for (int q = 0; q < 5; q++) W[stride * i + q] = wv[q];
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
  if (lane == 0) {
    red[0][wid] = okl;
    red[1][wid] = gfbl;
    red[2][wid] = fbl;
    red[3][wid] = failedl;
    red[4][wid] = itl;
    red[5][wid] = mxl;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    MlpPartial p = {0, 0, 0, 0, 0, 0};
    for (int q = 0; q < IT / 32; q++) {
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

__global__ void k_mlp_stats_reduce(MlpPartial *scratch, int nblocks) {
  if (threadIdx.x != 0) return;
  MlpPartial t = {0, 0, 0, 0, 0, 0};
  for (int b = 0; b < nblocks; b++) {
    const MlpPartial q = scratch[b];
    t.ok += q.ok;
    t.guess_fallback += q.guess_fallback;
    t.fallback += q.fallback;
    t.failed += q.failed;
    t.iters += q.iters;
    t.max_iters = q.max_iters > t.max_iters ? q.max_iters : t.max_iters;
  }
  scratch[nblocks] = t;
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
  uint32_t *d_frag = nullptr;
  MlpPartial *d_stats = nullptr;
  int stats_cap = 0;
  Norm norm{{0, 0, 0}, {1, 1, 1}, 0, 1};
  int adam_t = 0;
  int num_sms = 148;
};

static rrhd_status mlp_refresh(rrhd_mlp *m, cudaStream_t st) {
  k_pack_frags<<<6, 256, 0, st>>>(m->d_theta, m->d_frag);
  RRHD_CUDA(cudaGetLastError());
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
      cudaMalloc(&m->d_grad, NPARAM * 4) || cudaMalloc(&m->d_frag, NFRAG * 4)) {
    rrhd_mlp_destroy(m);
    return rrhd_fail(RRHD_ERR_OOM, "network allocation failed");
  }
  cudaMemcpy(m->d_theta, th.data(), NPARAM * 4, cudaMemcpyHostToDevice);
  cudaMemset(m->d_m, 0, NPARAM * 4);
  cudaMemset(m->d_v, 0, NPARAM * 4);
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
  cudaFree(m->d_frag);
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
  const int64_t warps = (n + 31) / 32;
  const int nblk = (int)std::max<int64_t>(1, std::min<int64_t>((warps + IT / 32 - 1) / (IT / 32), 8 * m->num_sms));
  if (mm->stats_cap < nblk + 1) {
    RRHD_CUDA(cudaStreamSynchronize(st));
    cudaFree(mm->d_stats);
    mm->d_stats = nullptr;
    RRHD_CUDA(cudaMalloc(&mm->d_stats, sizeof(MlpPartial) * (nblk + 1)));
    mm->stats_cap = nblk + 1;
  }
  k_c2p_mlp<<<nblk, IT, 0, st>>>(make_eos(eos, gamma), U, W, stride, G4, tau_src, status, n, fallback, k_stall,
                                 m->d_theta, m->d_frag, m->norm, mm->d_stats, guess);
  RRHD_CUDA(cudaGetLastError());
  k_mlp_stats_reduce<<<1, 32, 0, st>>>(mm->d_stats, nblk);
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
  }
  return RRHD_OK;
}

// con2prim batch seeded by the network: Newton from the learned guess for at
// most k_stall iterations, then (if needed) the reference solve from its own
// guess, then PhysPressureFix when fallback != 0.  stats (host, may be NULL).
// guess (device [n], may be NULL) receives the learned initial pressures.
extern "C" rrhd_status rrhd_con2prim_batch_mlp(const rrhd_mlp *m, int32_t eos, double gamma, double *U, double *W,
                                               uint8_t *status, int64_t n, int32_t fallback, int32_t k_stall,
                                               rrhd_c2p_stats *stats, int64_t *n_guess_fallback, double *guess,
                                               void *stream) {
  RRHD_CHECK_ARG(m && n >= 0 && ((U && W) || n == 0) && k_stall > 0 && k_stall <= 40, "bad arguments");
  RRHD_CHECK_ARG(eos == RRHD_EOS_IDEAL || eos == RRHD_EOS_TAUB, "bad eos");
  return rrhd::mlp_c2p(m, eos, gamma, U, W, 5, nullptr, 0.0, status, n, fallback, k_stall, stats, n_guess_fallback,
                       guess, (cudaStream_t)stream);
}
