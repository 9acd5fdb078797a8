// Scattering integral and moments on the 5th-generation tensor cores (tcgen05).
//
// C[r][n] = sum_d I[r][d] B[n][d] with, for n < M, B[n][d] = K[d][n] =
// Gamma(w_d . w_n) a_d / full_area (the FP64 kernel of
// cuda/src/short_characteristics/cuda_scattering.cu:82-105 and
// cuda_integrator.cu:10-13) and, for n = M..M+9, the moment weights
// a_d / full_area * {1, wx, wy, wz, wx^2, wx wy, wx wz, wy^2, wy wz, wz^2}
// (cuda_illum_sep_param.cu:9-69; T is symmetric so 6 columns carry it).
// Rows r are cells x frequency groups; I and the outputs are FP32.
//
// Precision forms (A = I, B = the kernel; FP32 accumulation in TMEM):
//   BF16X3 : A = Ah + Al, B = Bh + Bl in bf16; Ah Bh + Ah Bl + Al Bh
//   F16X3  : per-row power-of-two scale s_r (max |s_r I| in [2^14, 2^15)),
//            the same three products in fp16; B pre-scaled by 2^8
//   F16    : per-row scaled fp16, one product
//   BF16   : bf16, one product
// The scaled forms (F16X3, F16) split the kernel 3 (1 + mu^2) / 4 into its isotropic
// 3/4 and 3 mu^2 / 4: B carries only the second, and the drain adds 3/4 E_r with
// E_r = sum_d (a_d / A) I[r][d] summed in FP64 by the row pre-pass, which also forms
// the ten moments in FP64 (the scaled forms carry no moment columns).  The tensor
// cores' rounding then scales with the anisotropic part, a quarter to a half of S.
//
// The tensor core's FP32 accumulation truncates, so an accumulator that takes
// every MMA of a long K loop drifts by about one ulp per MMA.  Each chunk of
// 64 directions is therefore accumulated in a fresh TMEM accumulator (two,
// alternating), and the chunks are summed in FP32 registers with
// round-to-nearest adds by the accumulator warps.
//
// Persistent CTAs (576 threads, one per SM) loop over tiles of 128 rows x 128
// output directions (plus the 16 moment columns in the first direction tile):
// warp 0 issues the TMA loads of B (bf16/fp16, 128-byte swizzle, no multicast),
// warp 1 owns TMEM and issues the MMAs from one thread, warps 2-9 split the
// FP32 intensity tile (brought in by TMA, two chunks ahead) into hi/lo 16-bit
// tiles written in the UMMA K-major 128B-swizzled layout, warps 10-17 drain
// the chunk accumulators (tcgen05.ld), sum, unscale and store.  Two smem stages
// of K = 64 directions.  The row scales of the FP16 forms come from k_row_prepass.
// Every mbarrier wait is bounded: on a timeout the kernel records an error
// word, skips the remaining work, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "coupled.h"
#include "rrhd_internal.h"

#include "dirs.h"
#include "umma.cuh"

namespace {
using namespace rrhd_umma;

constexpr int kForms = 4;
enum { FORM_BF16X3 = 0, FORM_F16X3 = 1, FORM_F16 = 2, FORM_BF16 = 3 };
// The Thomson kernel 3 (1 + mu^2) / 4 splits into an isotropic 3/4 and 3 mu^2 / 4.  The
// scaled forms put only the second part on the tensor cores and add 3/4 E_r (FP64 row
// integral from the row pre-pass) in the drain: the tensor cores' accumulation error then
// applies to the smaller part of S only.
constexpr double kIsoWeight = 0.75;

constexpr int BM = 128;      // rows per CTA (UMMA M)
constexpr int BK = 64;       // directions per stage (one 128-byte swizzle row of 16-bit values)
constexpr int NT = 128;      // output directions per CTA (UMMA N)
constexpr int NMOM = 16;     // moment columns (10 used)
constexpr int STAGES = 2;
constexpr int A32_STAGES = 2;
constexpr int CONV_WARPS = 8;
constexpr int ACC_WARPS = 8;
constexpr int THREADS = 32 * (2 + CONV_WARPS + ACC_WARPS);  // TMA, MMA, converters, accumulators
constexpr int CONV_THREADS = 32 * CONV_WARPS;
constexpr int CONV_ITERS = BM * BK / 4 / CONV_THREADS;     // float4 per converter thread per chunk
constexpr int A_BYTES = BM * BK * 2;                   // 16 KiB
constexpr int B_ROWS = NT + NMOM;                      // 144
constexpr int B_BYTES = B_ROWS * BK * 2;               // 18 KiB
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES; // hi + lo
constexpr int ACC_STRIDE = 256;                        // TMEM columns between the two chunk accumulators
constexpr int MAX_HALF = (NT + NMOM) / 2;              // accumulator columns per thread
constexpr int A32_BYTES = BM * BK * 4;                  // 32 KiB FP32 intensity tile
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + A32_STAGES * A32_BYTES + 1024 /*align*/ + 256 /*barriers*/;
constexpr float kF16BScale = 256.0f;

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// instruction descriptor of the BM-row tiles
__host__ __device__ constexpr uint32_t umma_idesc(int fmt, int n) { return rrhd_umma::umma_idesc(fmt, n, BM); }

// Four values to packed hi (and lo) 16-bit parts: hi = round-to-nearest 16-bit value, lo =
// the rounded remainder (the three-product forms), two values per conversion instruction.
template <int FORM>
__device__ __forceinline__ void split4(const float (&x)[4], uint2 &hi, uint2 &lo) {
  if constexpr (FORM == FORM_F16X3 || FORM == FORM_F16) {
    const __half2 a = __floats2half2_rn(x[0], x[1]), b = __floats2half2_rn(x[2], x[3]);
    hi = make_uint2(*reinterpret_cast<const uint32_t *>(&a), *reinterpret_cast<const uint32_t *>(&b));
    if constexpr (FORM == FORM_F16X3) {
      const float2 fa = __half22float2(a), fb = __half22float2(b);
      const __half2 c = __floats2half2_rn(x[0] - fa.x, x[1] - fa.y), d = __floats2half2_rn(x[2] - fb.x, x[3] - fb.y);
      lo = make_uint2(*reinterpret_cast<const uint32_t *>(&c), *reinterpret_cast<const uint32_t *>(&d));
    } else {
      lo = make_uint2(0u, 0u);
    }
  } else {
    const __nv_bfloat162 a = __floats2bfloat162_rn(x[0], x[1]), b = __floats2bfloat162_rn(x[2], x[3]);
    hi = make_uint2(*reinterpret_cast<const uint32_t *>(&a), *reinterpret_cast<const uint32_t *>(&b));
    if constexpr (FORM == FORM_BF16X3) {
      const float2 fa = __bfloat1622float2(a), fb = __bfloat1622float2(b);
      const __nv_bfloat162 c = __floats2bfloat162_rn(x[0] - fa.x, x[1] - fa.y),
                           d = __floats2bfloat162_rn(x[2] - fb.x, x[3] - fb.y);
      lo = make_uint2(*reinterpret_cast<const uint32_t *>(&c), *reinterpret_cast<const uint32_t *>(&d));
    } else {
      lo = make_uint2(0u, 0u);
    }
  }
}

struct TcParams {
  const float *I;
  float *S;
  float *mom;          // [rows][16] or null
  const float *scale;  // [rows] power-of-two row scales (scaled forms)
  const double *erow;  // [rows] FP64 isotropic integrals E_r (scaled forms)
  int64_t rows;
  int M;
  float b_unscale;
  int *err;
  int b_copies;  // copies of the kernel matrix in global memory (resident kernel)
};

// Per-row pre-pass of the scaled FP16 forms over a cell-direction-group array [cells][M][NG]
// (NG = 1 is the rows layout [rows][M]):
//   scale  2^(14 - floor(log2(max_d |I[r][d]|))), so that max |s_r I| lies in [2^14, 2^15);
//   erow   E_r = sum_d (a_d / A) I[r][d] in FP64, the isotropic part of the Thomson
//          kernel's integral, which the scaled forms add outside the tensor cores;
//   mom    (MOM) the ten moments in FP64, stored as FP32 [rows][16] (columns 10-15 zero):
//          the scaled forms take them from here, not from the tensor cores.
// mw [10][M] holds (a_d / A) {1, wx, wy, wz, wx^2, wx wy, wx wz, wy^2, wy wz, wz^2}
// (cuda_illum_sep_param.cu:9-69).  A warp takes four cells, eight lanes per cell: a cell's
// values are NV = M NG / 4 float4 vectors (P = 4 / NG directions of NG groups each), lane q
// takes vectors q, q + 8, q + 16, ..., so each load instruction reads a whole 128-byte line
// of each of the four cells.  Each term is one fused multiply-add in FP64; the eight lanes'
// partial sums are combined by a fixed butterfly (reduce-scatter over lane bits 4, 2, 1), the
// same order for every cell.  The weight table sits in shared memory by (sub-direction,
// vector), so the eight lanes of a cell read eight consecutive records (no bank conflicts).
constexpr int kPrepassThreads = 256;
template <int NG, bool MOM>
__global__ void __launch_bounds__(kPrepassThreads, 2) k_row_prepass(const float *__restrict__ I, int64_t rows, int M,
                                                                 const double *__restrict__ mw,
                                                                 float *__restrict__ scale, double *__restrict__ erow,
                                                                 float *__restrict__ mom) {
  constexpr int NM = MOM ? 10 : 1;
  constexpr int P = 4 / NG;                 // directions per float4
  constexpr int V = NG * NM;                // sums per cell
  constexpr int VP = (V + 7) / 8 * 8;       // padded to the reduce-scatter's eight lanes
  extern __shared__ double2 smw2[];         // [P][M / P][NM]
  double *smw = reinterpret_cast<double *>(smw2);
  const int MP = M / P;
  for (int x = threadIdx.x; x < NM * M; x += blockDim.x) {
    const int k = x / M, d = x - k * M;
    smw[((d % P) * MP + d / P) * NM + k] = __ldg(mw + x);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, q = lane & 7;
  const int NV = M * NG / 4;  // float4 per cell, a multiple of 8
  const int64_t cells = rows / NG;
  const int64_t quads = (cells + 3) / 4;
  const int64_t wid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const float4 *I4 = reinterpret_cast<const float4 *>(I);
  // the four cells of a group are contiguous (16 NV bytes each): one lane asks L2 for the
  // warp's next group while the warp works on this one, so that the lanes' loads find it there
  auto prefetch = [&](int64_t g4) {
    if (lane == 0 && g4 < quads) {
      const int64_t n = min((int64_t)4, cells - 4 * g4) * NV * 16;  // bytes, a multiple of 16
      const float4 *src = I4 + 4 * g4 * NV;
      for (int64_t o = 0; o < n; o += 65536)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(reinterpret_cast<const char *>(src) + o),
                     "r"((uint32_t)min((int64_t)65536, n - o))
                     : "memory");
    }
  };
  prefetch(wid);
  for (int64_t c4 = wid; c4 < quads; c4 += nw) {  // warp-uniform
    prefetch(c4 + nw);
    const int64_t c = c4 * 4 + (lane >> 3);
    const bool valid = c < cells;
    double acc[VP];
#pragma unroll
    for (int k = 0; k < VP; k++) acc[k] = 0.0;
    float mx[NG];
#pragma unroll
    for (int g = 0; g < NG; g++) mx[g] = 0.f;
    if (valid) {
      const float4 *row = I4 + c * NV;
#pragma unroll 2
      for (int v = q; v < NV; v += 8) {
        const float4 x = __ldcs(row + v);
        const float e[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
        for (int s = 0; s < P; s++) {
          double w[NM];
          const double2 *wr = smw2 + ((s * MP + v) * NM) / 2;
          if constexpr (MOM) {
#pragma unroll
            for (int j = 0; j < NM / 2; j++) {
              const double2 t = wr[j];
              w[2 * j] = t.x;
              w[2 * j + 1] = t.y;
            }
          } else {
            w[0] = smw[s * MP + v];
          }
#pragma unroll
          for (int g = 0; g < NG; g++) {
            const float val = e[s * NG + g];
            mx[g] = fmaxf(mx[g], fabsf(val));
#pragma unroll
            for (int k = 0; k < NM; k++) acc[g * NM + k] = __fma_rn((double)val, w[k], acc[g * NM + k]);
          }
        }
      }
    }
    // the group maxima to every lane of the cell; the sums reduce-scattered
#pragma unroll
    for (int o = 4; o >= 1; o >>= 1)
#pragma unroll
      for (int g = 0; g < NG; g++) mx[g] = fmaxf(mx[g], __shfl_xor_sync(0xffffffffu, mx[g], o));
#pragma unroll
    for (int o = 4, h = VP / 2; o >= 1; o >>= 1, h >>= 1) {
      const bool up = lane & o;
#pragma unroll
      for (int k = 0; k < VP / 2; k++) {
        if (k < h) {
          const double send = up ? acc[k] : acc[h + k];
          const double keep = up ? acc[h + k] : acc[k];
          acc[k] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
      }
    }
    // this lane now holds sums base .. base + VP/8 - 1 of its cell
    const int base = ((lane >> 2) & 1) * (VP / 2) + ((lane >> 1) & 1) * (VP / 4) + (lane & 1) * (VP / 8);
#pragma unroll
    for (int k = 0; k < VP / 8; k++) {
      const int f = base + k;
      if (valid && f < V) {
        const int g = f / NM, kk = f - g * NM;
        const int64_t r = c * NG + g;
        if (kk == 0) {
          float m = mx[0];
#pragma unroll
          for (int gg = 1; gg < NG; gg++)
            if (g == gg) m = mx[gg];
          scale[r] = (m > 0.f && isfinite(m)) ? ldexpf(1.f, 14 - ilogbf(m)) : 1.f;
          erow[r] = acc[k];
        }
        if (MOM) {
          mom[16 * r + kk] = (float)acc[k];
          if (kk == NM - 1)
#pragma unroll
            for (int z = NM; z < 16; z++) mom[16 * r + z] = 0.f;
        }
      }
    }
  }
}

template <int FORM, int NG>
__global__ void __launch_bounds__(THREADS, 1)
    k_scatter_tc(const __grid_constant__ CUtensorMap tm_bh, const __grid_constant__ CUtensorMap tm_bl,
                 const __grid_constant__ CUtensorMap tm_mh, const __grid_constant__ CUtensorMap tm_ml,
                 const __grid_constant__ CUtensorMap tm_a, const TcParams P) {
  constexpr bool THREE = (FORM == FORM_BF16X3 || FORM == FORM_F16X3);
  constexpr bool SCALED = (FORM == FORM_F16X3 || FORM == FORM_F16);
  constexpr int FMT = (FORM == FORM_BF16X3 || FORM == FORM_BF16) ? 1 : 0;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t *a32 = smem + STAGES * STAGE_BYTES;  // [A32_STAGES][128][64] FP32
  uint64_t *bars = reinterpret_cast<uint64_t *>(a32 + A32_STAGES * A32_BYTES);
  uint64_t *full_a = bars, *full_b = bars + STAGES, *empty = bars + 2 * STAGES;
  uint64_t *acc_full = bars + 3 * STAGES, *acc_empty = bars + 3 * STAGES + 2;
  uint64_t *a32_full = bars + 3 * STAGES + 4, *a32_empty = a32_full + A32_STAGES;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 3 * STAGES + 4 + 2 * A32_STAGES);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nk = P.M / BK;
  const int nS = P.M < NT ? P.M : NT;  // output directions per tile (M <= 128 or M % 128 == 0)
  const int n_nt = P.M / nS;
  const int64_t n_rt = (P.rows + BM - 1) / BM;
  const int64_t tiles = n_rt * n_nt;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; s++) {
      mbar_init(&full_a[s], CONV_THREADS);
      mbar_init(&full_b[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], ACC_WARPS);
    }
    for (int b = 0; b < A32_STAGES; b++) {
      mbar_init(&a32_full[b], 1);
      mbar_init(&a32_empty[b], CONV_THREADS);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;\n" ::"r"(smem_u32(tmem_slot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  auto fail = [&]() {
    *abort_flag = 1;
    atomicOr(P.err, 1);
  };

  if (warp == 0) {
    // ---------------- B producer (TMA)
    if (lane == 0) {
      int issued[STAGES] = {0};
      int64_t g = 0;
      for (int64_t tile = blockIdx.x; tile < tiles && !*abort_flag; tile += gridDim.x) {
        const int nt = (int)(tile % n_nt);
        const bool with_mom = (nt == 0) && P.mom != nullptr;
        const uint32_t bytes = (uint32_t)((THREE ? 2 : 1) * (nS + (with_mom ? NMOM : 0)) * BK * 2);
        for (int k = 0; k < nk; k++, g++) {
          const int s = (int)(g % STAGES);
          if (g >= STAGES && !mbar_wait(&empty[s], (uint32_t)((g / STAGES) - 1) & 1)) {
            fail();
            break;
          }
          if (*abort_flag) break;
          uint8_t *st = smem + s * STAGE_BYTES;
          uint8_t *bh = st + 2 * A_BYTES, *bl = bh + B_BYTES;
          mbar_arrive_expect_tx(&full_b[s], bytes);
          tma_load_2d(bh, &tm_bh, k * BK, nt * NT, &full_b[s]);
          if (THREE) tma_load_2d(bl, &tm_bl, k * BK, nt * NT, &full_b[s]);
          if (with_mom) {
            tma_load_2d(bh + NT * 128, &tm_mh, k * BK, 0, &full_b[s]);
            if (THREE) tma_load_2d(bl + NT * 128, &tm_ml, k * BK, 0, &full_b[s]);
          }
          issued[s]++;
        }
      }
      // no copy may still be in flight when the CTA retires (bounded)
      for (int s = 0; s < STAGES; s++)
        if (issued[s] && !mbar_wait(&full_b[s], (issued[s] - 1) & 1)) fail();
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer: chunk g goes to accumulator g % 2, fresh each chunk
    if (lane == 0) {
      const uint32_t idN = umma_idesc(FMT, nS);
      constexpr uint32_t idM = umma_idesc(FMT, NMOM);
      int64_t g = 0;
      for (int64_t tile = blockIdx.x; tile < tiles && !*abort_flag; tile += gridDim.x) {
        const bool with_mom = (tile % n_nt == 0) && P.mom != nullptr;
        for (int k = 0; k < nk; k++, g++) {
          const int s = (int)(g % STAGES), ab = (int)(g & 1);
          const uint32_t par = (uint32_t)(g / STAGES) & 1;
          if (!mbar_wait(&full_a[s], par) || !mbar_wait(&full_b[s], par) ||
              (g >= 2 && !mbar_wait(&acc_empty[ab], (uint32_t)((g >> 1) - 1) & 1))) {
            fail();
            break;
          }
          if (*abort_flag) break;
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          uint8_t *st = smem + s * STAGE_BYTES;
          const uint32_t ah = smem_u32(st), al = ah + A_BYTES;
          const uint32_t bh = al + A_BYTES, bl = bh + B_BYTES;
          const uint32_t acc_s = tmem + ab * ACC_STRIDE, acc_m = acc_s + nS;
          // the split forms add the cross terms first (hi x Bl, lo x Bh) and hi x Bh last,
          // so that only four MMAs add to an accumulator of full size
          const uint32_t bm_h = bh + NT * 128, bm_l = bl + NT * 128;
          if (THREE) {
#pragma unroll
            for (int kk = 0; kk < BK / 16; kk++) {
              const uint32_t o = kk * 32, acc = kk > 0 ? 1u : 0u;
              umma(acc_s, umma_desc(ah + o), umma_desc(bl + o), idN, acc);
              if (with_mom) umma(acc_m, umma_desc(ah + o), umma_desc(bm_l + o), idM, acc);
            }
#pragma unroll
            for (int kk = 0; kk < BK / 16; kk++) {
              const uint32_t o = kk * 32;
              umma(acc_s, umma_desc(al + o), umma_desc(bh + o), idN, 1u);
              if (with_mom) umma(acc_m, umma_desc(al + o), umma_desc(bm_h + o), idM, 1u);
            }
          }
#pragma unroll
          for (int kk = 0; kk < BK / 16; kk++) {
            const uint32_t o = kk * 32, acc = (THREE || kk > 0) ? 1u : 0u;
            umma(acc_s, umma_desc(ah + o), umma_desc(bh + o), idN, acc);
            if (with_mom) umma(acc_m, umma_desc(ah + o), umma_desc(bm_h + o), idM, acc);
          }
          umma_commit(&empty[s]);
          umma_commit(&acc_full[ab]);
        }
      }
    }
  } else if (warp < 2 + CONV_WARPS) {
    // ---------------- A converters: FP32 tile (TMA-staged) -> hi/lo 16-bit tiles in the
    // UMMA K-major 128B-swizzled layout.  Every converter arrives on a32_empty
    // once it has read chunk g; converter thread 0 waits for that (bounded) and
    // issues the TMA of chunk g + 2 into the same staging slot, so the intensity
    // stream runs two chunks ahead.
    const int t = threadIdx.x - 64;
    const int64_t my_chunks = (tiles > blockIdx.x ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0) * nk;
    auto issue_a = [&](int64_t gg) {
      const int64_t tile = blockIdx.x + (gg / nk) * gridDim.x;
      const int kk = (int)(gg % nk);
      const int sa = (int)(gg % A32_STAGES);
      mbar_arrive_expect_tx(&a32_full[sa], A32_BYTES);
      // NG > 1: box {BK * NG, BM / NG} of the [cells][M * NG] view
      tma_load_2d(a32 + sa * A32_BYTES, &tm_a, kk * BK * NG, (int)((tile / n_nt) * (BM / NG)), &a32_full[sa]);
    };
    if (t == 0)
      for (int64_t gg = 0; gg < A32_STAGES && gg < my_chunks; gg++) issue_a(gg);
    int64_t g = 0;
    for (int64_t tile = blockIdx.x; tile < tiles && !*abort_flag; tile += gridDim.x) {
      const int64_t r0 = (tile / n_nt) * BM;
      for (int k = 0; k < nk; k++, g++) {
        const int s = (int)(g % STAGES), sa = (int)(g % A32_STAGES);
        if (!mbar_wait(&a32_full[sa], (uint32_t)(g / A32_STAGES) & 1)) {
          fail();
          break;
        }
        float4 v[CONV_ITERS];
        const float4 *src = reinterpret_cast<const float4 *>(a32 + sa * A32_BYTES);
        // rows layout: float4 i*CONV_THREADS + t; [cells][64][ng]: the ng float4s of unit i/ng*CONV_THREADS + t
        constexpr int ush = NG == 4 ? 2 : (NG == 2 ? 1 : 0);
#pragma unroll
        for (int i = 0; i < CONV_ITERS; i++)
          v[i] = src[((((i >> ush) * CONV_THREADS) + t) << ush) + (i & ((1 << ush) - 1))];
        // the next TMA into this slot (async proxy) must not overtake these generic-proxy reads
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_arrive(&a32_empty[sa]);
        if (t == 0 && g + A32_STAGES < my_chunks) {
          if (!mbar_wait(&a32_empty[sa], (uint32_t)(g / A32_STAGES) & 1)) {
            fail();
            break;
          }
          issue_a(g + A32_STAGES);
        }
        if (g >= STAGES && !mbar_wait(&empty[s], (uint32_t)((g / STAGES) - 1) & 1)) {
          fail();
          break;
        }
        if (*abort_flag) break;
        uint8_t *ah = smem + s * STAGE_BYTES, *al = ah + A_BYTES;
        // (row, c4) of the unit each converted quad belongs to, and its 4 values
        auto put = [&](int row, int c4, float x0, float x1, float x2, float x3) {
          float x[4] = {x0, x1, x2, x3};
          if (SCALED) {
            const int64_t gr = r0 + row;
            const float sc = gr < P.rows ? __ldg(P.scale + gr) : 1.f;
#pragma unroll
            for (int q = 0; q < 4; q++) x[q] *= sc;
          }
          uint2 hv, lv;
          split4<FORM>(x, hv, lv);
          const uint32_t off = row * 128 + ((((c4 >> 1) ^ (row & 7))) << 4) + ((c4 & 1) << 3);
          *reinterpret_cast<uint2 *>(ah + off) = hv;
          if (THREE) *reinterpret_cast<uint2 *>(al + off) = lv;
        };
        if constexpr (NG == 4) {
          // staged tile [32 cells][64 directions][4 groups]: unit (cell, c4) = float4s 4u..4u+3, one per direction
#pragma unroll
          for (int iu = 0; iu < CONV_ITERS / 4; iu++) {
            const int u = iu * CONV_THREADS + t, cl = u >> 4, c4 = u & 15;
            const float4 d0 = v[4 * iu], d1 = v[4 * iu + 1], d2 = v[4 * iu + 2], d3 = v[4 * iu + 3];
            put(cl * 4 + 0, c4, d0.x, d1.x, d2.x, d3.x);
            put(cl * 4 + 1, c4, d0.y, d1.y, d2.y, d3.y);
            put(cl * 4 + 2, c4, d0.z, d1.z, d2.z, d3.z);
            put(cl * 4 + 3, c4, d0.w, d1.w, d2.w, d3.w);
          }
        } else if constexpr (NG == 2) {
          // [64 cells][64 directions][2 groups]: unit (cell, c4) = 2 float4s {d0 g0, d0 g1, d1 g0, d1 g1}, {d2 .., d3 ..}
#pragma unroll
          for (int iu = 0; iu < CONV_ITERS / 2; iu++) {
            const int u = iu * CONV_THREADS + t, cl = u >> 4, c4 = u & 15;
            const float4 a = v[2 * iu], b = v[2 * iu + 1];
            put(cl * 2 + 0, c4, a.x, a.z, b.x, b.z);
            put(cl * 2 + 1, c4, a.y, a.w, b.y, b.w);
          }
        } else {
#pragma unroll
          for (int i = 0; i < CONV_ITERS; i++) {
            const int e = i * CONV_THREADS + t;
            put(e >> 4, e & 15, v[i].x, v[i].y, v[i].z, v[i].w);
          }
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_arrive(&full_a[s]);
      }
    }
    // drain: every issued intensity copy has landed before the CTA retires (bounded)
    if (t == 0)
      for (int64_t gg = g; gg < my_chunks && gg < g + A32_STAGES; gg++)
        if (!mbar_wait(&a32_full[gg % A32_STAGES], (uint32_t)(gg / A32_STAGES) & 1)) fail();
  } else {
    // ---------------- accumulator warps: warp w reads TMEM lanes 32*(w%4)..+31 (one row
    // per thread); the first four take the first half of the columns, the others the second
    const int q = warp & 3, hf = (warp - 2 - CONV_WARPS) >> 2;
    const int row = q * 32 + lane;
    int64_t g = 0;
    bool ok = true;
    for (int64_t tile = blockIdx.x; tile < tiles && ok && !*abort_flag; tile += gridDim.x) {
      const int nt = (int)(tile % n_nt);
      const bool with_mom = (nt == 0) && P.mom != nullptr;
      const int64_t gr = (tile / n_nt) * BM + row;
      const int half = (nS + (with_mom ? NMOM : 0)) >> 1;  // multiple of 8
      const int c0 = hf * half;
      float run[MAX_HALF];
#pragma unroll
      for (int j = 0; j < MAX_HALF; j++) run[j] = 0.f;
      for (int k = 0; k < nk; k++, g++) {
        const int ab = (int)(g & 1);
        if (!mbar_wait(&acc_full[ab], (uint32_t)(g >> 1) & 1)) {
          fail();
          ok = false;
          break;
        }
        if (*abort_flag) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * ACC_STRIDE + c0);
#pragma unroll
        for (int j = 0; j < MAX_HALF / 8; j++) {
          if (j * 8 < half) {
            uint32_t r[8];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7])
                         : "r"(base + j * 8));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
            for (int i = 0; i < 8; i++) run[j * 8 + i] = __fadd_rn(run[j * 8 + i], __uint_as_float(r[i]));
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[ab]);
      }
      if (ok && gr < P.rows) {
        const float inv = (SCALED ? 1.f / __ldg(P.scale + gr) : 1.f) * P.b_unscale;
        const double eiso = SCALED ? __ldg(P.erow + gr) : 0.0;  // the isotropic part, added in FP64
#pragma unroll
        for (int j = 0; j < MAX_HALF / 4; j++) {
          const int col = c0 + 4 * j;
          if (4 * j < half) {
            float4 v = make_float4(run[4 * j] * inv, run[4 * j + 1] * inv, run[4 * j + 2] * inv,
                                   run[4 * j + 3] * inv);
            if (SCALED && col < nS) {
              v.x = (float)((double)v.x + kIsoWeight * eiso);
              v.y = (float)((double)v.y + kIsoWeight * eiso);
              v.z = (float)((double)v.z + kIsoWeight * eiso);
              v.w = (float)((double)v.w + kIsoWeight * eiso);
            }
            if (col < nS) {
              if constexpr (NG > 1) {
                float *o = P.S + ((gr / NG) * P.M + nt * NT + col) * NG + gr % NG;
                o[0] = v.x;
                o[NG] = v.y;
                o[2 * NG] = v.z;
                o[3 * NG] = v.w;
              } else {
                *reinterpret_cast<float4 *>(P.S + gr * P.M + nt * NT + col) = v;
              }
            } else
              *reinterpret_cast<float4 *>(P.mom + gr * NMOM + (col - nS)) = v;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;\n" ::"r"(tmem));
  }
}

// ---------------------------------------------------------------------------
// Resident-tile kernel for M = 128 or 256 output directions.
//
// A CTA takes a tile of 128 rows and every output column.  The converter warps
// split the tile's intensities once into hi/lo 16-bit K-major tiles that stay
// in shared memory for the whole tile (M/64 chunks of 2 x 16 KiB); the MMA warp
// then runs the output halves (128 directions each; the first carries the 16
// moment columns in the same N = 144 product) over those chunks, so a row tile
// is read and converted once whatever M is.  The intensities come straight
// from global memory: 16-byte loads in which consecutive lanes read consecutive
// addresses, one chunk prefetched in registers, then regrouped into rows with
// lane shuffles (cell-direction-group layouts); the drain regroups the sums the
// same way so that S leaves as 16-byte stores.  The kernel matrix streams
// through a ring of 18 KiB stages, one 16-bit part per stage, and three TMEM
// accumulators rotate between the MMA and the drain.  Per chunk and output half
// the three products are issued cross terms first (hi x Bl, then lo x Bh) and
// hi x Bh last into a fresh accumulator, so only the last four MMAs of a chunk
// add to a sum of full size.
//
// Warp roles are whole warpgroups so that registers can move between them
// (setmaxnreg): warpgroup 0 = TMA producer (warp 0), MMA issuer (warp 1) and two
// idle warps, shrunk to R_REG_CTRL registers; warpgroups 1-2 = converters,
// grown to R_REG_CONV; warpgroups 3-4 = accumulator drain, grown to R_REG_DRAIN.
// The launcher checks the compiled register count against the sum first.
constexpr int R_BST = 4;                     // kernel-matrix stages
constexpr int R_KG = 1;                      // 64-direction chunks per accumulator group (2 measured slower,
                                             // and its longer full-size sums less accurate)
constexpr int R_BSTAGE = B_ROWS * BK * 2;    // 18 KiB: one 16-bit part, 144 rows x 64 directions
constexpr int R_NACC = 3;                    // TMEM accumulators
constexpr int R_ACC_STRIDE = 160;            // TMEM columns between accumulators (144 used)
constexpr int R_GROUP = 2;                   // TMEM loads (x8) in flight per wait in the drain
constexpr int R_THREADS = 640;               // 5 warpgroups
constexpr int R_CONV0 = 4, R_DRAIN0 = 12;    // first converter / drain warp
constexpr int R_REG_CTRL = 56, R_REG_CONV = 104, R_REG_DRAIN = 104;
constexpr int R_COPIES = 1;                  // kernel-matrix copies in global memory (16 measured no faster)
// registers the five warpgroups hold after the setmaxnreg split
constexpr int R_REG_TOTAL = 128 * R_REG_CTRL + 256 * R_REG_CONV + 256 * R_REG_DRAIN;

__host__ __device__ constexpr int r_smem_bytes(int nk) {
  return 2 * nk * A_BYTES + R_BST * R_BSTAGE + 1024 /*align*/ + 256 /*barriers*/;
}

// Regroups the float4 a lane holds between quads (NG = 4) or pairs (NG = 2) of
// lanes.  NG = 4 is a 4x4 transpose across the quad: lane p holds element
// [p][0..3] and ends with [0..3][p] (groups of one direction -> directions of
// one group, and back).  NG = 2: lane pairs hold {d g0, d g1, d+1 g0, d+1 g1};
// the even lane ends with group 0, the odd with group 1 of directions 4m..4m+3.
// NG = 1: rows are already direction-major.
template <int NG>
__device__ __forceinline__ void regroup(const float4 v, int lane, float (&x)[4]) {
  if constexpr (NG == 1) {
    x[0] = v.x;
    x[1] = v.y;
    x[2] = v.z;
    x[3] = v.w;
  } else if constexpr (NG == 2) {
    const bool odd = lane & 1;
    const float ra = __shfl_xor_sync(0xffffffffu, odd ? v.x : v.y, 1);
    const float rb = __shfl_xor_sync(0xffffffffu, odd ? v.z : v.w, 1);
    x[0] = odd ? ra : v.x;
    x[1] = odd ? rb : v.z;
    x[2] = odd ? v.y : ra;
    x[3] = odd ? v.w : rb;
  } else {
    const bool b0 = lane & 1, b1 = lane & 2;
    // stage 1, partner lane ^ 1: even lanes keep columns 0, 2; odd lanes keep 1, 3
    const float ra = __shfl_xor_sync(0xffffffffu, b0 ? v.x : v.y, 1);
    const float rb = __shfl_xor_sync(0xffffffffu, b0 ? v.z : v.w, 1);
    const float y0 = b0 ? ra : v.x, y1 = b0 ? v.y : ra;
    const float y2 = b0 ? rb : v.z, y3 = b0 ? v.w : rb;
    // stage 2, partner lane ^ 2
    const float sa = __shfl_xor_sync(0xffffffffu, b1 ? y0 : y2, 2);
    const float sb = __shfl_xor_sync(0xffffffffu, b1 ? y1 : y3, 2);
    x[0] = b1 ? sa : y0;
    x[1] = b1 ? sb : y1;
    x[2] = b1 ? y2 : sa;
    x[3] = b1 ? y3 : sb;
  }
}

// The inverse for the drain at NG = 2: the even lane holds group 0, the odd lane
// group 1 of directions c..c+3; the even lane ends with {c g0, c g1, c+1 g0,
// c+1 g1}, the odd one with directions c+2, c+3.
__device__ __forceinline__ void ungroup2(const float (&v)[4], int lane, float (&x)[4]) {
  const bool odd = lane & 1;
  const float ra = __shfl_xor_sync(0xffffffffu, odd ? v[0] : v[2], 1);
  const float rb = __shfl_xor_sync(0xffffffffu, odd ? v[1] : v[3], 1);
  x[0] = odd ? ra : v[0];
  x[1] = odd ? v[2] : ra;
  x[2] = odd ? rb : v[1];
  x[3] = odd ? v[3] : rb;
}

template <int FORM, int NG>
__global__ void __launch_bounds__(R_THREADS, 1)
    k_scatter_tc_res(const __grid_constant__ CUtensorMap tm_bh, const __grid_constant__ CUtensorMap tm_bl,
                     const __grid_constant__ CUtensorMap tm_mh, const __grid_constant__ CUtensorMap tm_ml,
                     const TcParams P) {
  constexpr bool THREE = (FORM == FORM_BF16X3 || FORM == FORM_F16X3);
  constexpr bool SCALED = (FORM == FORM_F16X3 || FORM == FORM_F16);
  constexpr int FMT = (FORM == FORM_BF16X3 || FORM == FORM_BF16) ? 1 : 0;
  constexpr int NPART = THREE ? 2 : 1;
  constexpr int FPC = 16 * NG;   // float4 per cell and 64-direction chunk
  constexpr int CPT = 128 / NG;  // cells per 128-row tile
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int nk = P.M / BK;  // 2 or 4 chunks
  const int nS = NT;        // output directions per half
  // the kernel-matrix copy this CTA reads (rows copy * (M + 16) .. of the replicated maps)
  const int brow = (int)(blockIdx.x % (unsigned)P.b_copies) * (P.M + NMOM);
  const int n_h = P.M / NT;
  const bool mom = P.mom != nullptr;
  uint8_t *a16 = smem;                         // [hi, lo][chunk][128 rows][128 B]
  uint8_t *bst = smem + 2 * nk * A_BYTES;      // [R_BST][144 rows][128 B]
  uint64_t *bars = reinterpret_cast<uint64_t *>(bst + R_BST * R_BSTAGE);
  uint64_t *a_full = bars, *a_empty = bars + 4;
  uint64_t *b_full = bars + 8, *b_empty = bars + 8 + R_BST;
  uint64_t *acc_full = bars + 8 + 2 * R_BST, *acc_empty = acc_full + R_NACC;
  uint64_t *mma_done = acc_empty + R_NACC;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mma_done + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t n_rt = (P.rows + BM - 1) / BM;

  if (threadIdx.x == 0) {
    for (int k = 0; k < 4; k++) {
      mbar_init(&a_full[k], CONV_WARPS);
      mbar_init(&a_empty[k], 1);
    }
    for (int s = 0; s < R_BST; s++) {
      mbar_init(&b_full[s], 1);
      mbar_init(&b_empty[s], 1);
    }
    for (int b = 0; b < R_NACC; b++) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], ACC_WARPS);
    }
    mbar_init(mma_done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;\n" ::"r"(smem_u32(tmem_slot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  auto fail = [&]() {
    *abort_flag = 1;
    atomicOr(P.err, 1);
  };

  if (warp < R_CONV0) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(R_REG_CTRL));
    if (warp == 0 && lane == 0) {
      // ---------------- kernel-matrix producer (TMA, one 16-bit part per stage)
      int issued[R_BST] = {0};
      int64_t s = 0;
      bool ok = true;
      // stage order per group: the R_KG chunks' lo parts, then their hi parts
      for (int64_t rt = blockIdx.x; rt < n_rt && ok && !*abort_flag; rt += gridDim.x)
        for (int h = 0; h < n_h && ok; h++)
          for (int m = 0; m < nk / R_KG && ok; m++)
            for (int pc = 0; pc < NPART * R_KG; pc++, s++) {
              const int part = pc / R_KG, k = m * R_KG + pc % R_KG;
              const int sb = (int)(s % R_BST);
              if (s >= R_BST && !mbar_wait(&b_empty[sb], (uint32_t)((s / R_BST) - 1) & 1)) {
                fail();
                ok = false;
                break;
              }
              if (*abort_flag) {
                ok = false;
                break;
              }
              const bool lo = THREE && part == 0;
              const bool wm = (h == 0) && mom;
              uint8_t *dst = bst + sb * R_BSTAGE;
              mbar_arrive_expect_tx(&b_full[sb], (uint32_t)((nS + (wm ? NMOM : 0)) * BK * 2));
              tma_load_2d(dst, lo ? &tm_bl : &tm_bh, k * BK, brow + h * nS, &b_full[sb]);
              if (wm) tma_load_2d(dst + nS * 128, lo ? &tm_ml : &tm_mh, k * BK, brow + P.M, &b_full[sb]);
              issued[sb]++;
            }
      // no copy may still be in flight when the CTA retires (bounded)
      for (int sb = 0; sb < R_BST; sb++)
        if (issued[sb] && !mbar_wait(&b_full[sb], (issued[sb] - 1) & 1)) fail();
    } else if (warp == 1 && lane == 0) {
      // ---------------- MMA issuer: group (tile, half, chunk) -> accumulator g % R_NACC, fresh each group
      const uint64_t ddesc = umma_desc(0);
      const uint32_t a16_u32 = smem_u32(a16), bst_u32 = smem_u32(bst);
      int64_t s = 0, g = 0, ti = 0;
      bool ok = true;
      for (int64_t rt = blockIdx.x; rt < n_rt && ok && !*abort_flag; rt += gridDim.x, ti++)
        for (int h = 0; h < n_h && ok; h++) {
          const uint32_t idesc = umma_idesc(FMT, nS + ((h == 0 && mom) ? NMOM : 0));
          for (int m = 0; m < nk / R_KG && ok; m++, g++) {
            const int ab = (int)(g % R_NACC);
            bool got = true;
            if (h == 0)
              for (int c = 0; c < R_KG; c++) got = got && mbar_wait(&a_full[m * R_KG + c], (uint32_t)(ti & 1));
            if (!got || (g >= R_NACC && !mbar_wait(&acc_empty[ab], (uint32_t)((g / R_NACC) - 1) & 1))) {
              fail();
              ok = false;
              break;
            }
            if (*abort_flag) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t acc = tmem + ab * R_ACC_STRIDE;
            // descriptors: constant fields | (address >> 4); the K step of 16 elements
            // (32 bytes) adds 2 to the address field inside a 1 KiB-aligned tile
            auto a_hi = [&](int c) { return ddesc | (uint64_t)((a16_u32 + (m * R_KG + c) * A_BYTES) >> 4); };
            auto a_lo = [&](int c) { return ddesc | (uint64_t)((a16_u32 + (nk + m * R_KG + c) * A_BYTES) >> 4); };
            auto b_at = [&](int64_t ss) { return ddesc | (uint64_t)((bst_u32 + (int)(ss % R_BST) * R_BSTAGE) >> 4); };
            auto b_wait = [&](int64_t ss) {
              if (!mbar_wait(&b_full[ss % R_BST], (uint32_t)(ss / R_BST) & 1)) {
                fail();
                ok = false;
                return false;
              }
              asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
              return true;
            };
            const int64_t s0 = s;
            if (THREE) {
              // cross terms of every chunk of the group first (hi x Bl, lo x Bh), hi x Bh last
              for (int c = 0; c < R_KG && ok; c++) {
                if (!b_wait(s0 + c)) break;
#pragma unroll
                for (int kk = 0; kk < BK / 16; kk++)
                  umma(acc, a_hi(c) + 2 * kk, b_at(s0 + c) + 2 * kk, idesc,
                       (c > 0 || kk > 0) ? 1u : 0u);
              }
              if (!ok) break;
              for (int c = 0; c < R_KG; c++) umma_commit(&b_empty[(s0 + c) % R_BST]);
              for (int c = 0; c < R_KG && ok; c++) {
                if (!b_wait(s0 + R_KG + c)) break;
#pragma unroll
                for (int kk = 0; kk < BK / 16; kk++)
                  umma(acc, a_lo(c) + 2 * kk, b_at(s0 + R_KG + c) + 2 * kk, idesc, 1u);
              }
              if (!ok) break;
              for (int c = 0; c < R_KG; c++)
#pragma unroll
                for (int kk = 0; kk < BK / 16; kk++)
                  umma(acc, a_hi(c) + 2 * kk, b_at(s0 + R_KG + c) + 2 * kk, idesc, 1u);
              for (int c = 0; c < R_KG; c++) umma_commit(&b_empty[(s0 + R_KG + c) % R_BST]);
              s += 2 * R_KG;
            } else {
              for (int c = 0; c < R_KG && ok; c++) {
                if (!b_wait(s0 + c)) break;
#pragma unroll
                for (int kk = 0; kk < BK / 16; kk++)
                  umma(acc, a_hi(c) + 2 * kk, b_at(s0 + c) + 2 * kk, idesc,
                       (c > 0 || kk > 0) ? 1u : 0u);
                umma_commit(&b_empty[(s0 + c) % R_BST]);
              }
              if (!ok) break;
              s += R_KG;
            }
            umma_commit(&acc_full[ab]);
            if (h == n_h - 1)
              for (int c = 0; c < R_KG; c++) umma_commit(&a_empty[m * R_KG + c]);
          }
        }
      // every issued MMA has completed before TMEM is released (bounded)
      if (s > 0) {
        umma_commit(mma_done);
        if (!mbar_wait(mma_done, 0)) fail();
      }
    }
  } else if (warp < R_DRAIN0) {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(R_REG_CONV));
    // ---------------- converters: chunk (tile, k) from global memory -> hi/lo tiles in smem
    const int t = threadIdx.x - 32 * R_CONV0;
    const int off = t % FPC;                  // float4 within a cell's chunk
    const int c4 = off / NG;                  // direction quad of the row after regrouping
    const int gsel = t & (NG - 1);            // group of the row after regrouping
    const int64_t ncell = P.rows / NG;
    const int64_t cstride = (int64_t)P.M * NG / 4;  // float4 per cell
    const float4 *I4 = reinterpret_cast<const float4 *>(P.I);
    const int64_t my_tiles = n_rt > blockIdx.x ? (n_rt - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const int64_t nchunks = my_tiles * nk;
    auto cellrel = [&](int j) { return j * (256 / FPC) + t / FPC; };
    // tiles start on even chunk numbers (nk is 2 or 4), so the scales of a tile
    // always arrive with buffer A; row scales are powers of two, kept as their
    // 8-bit biased exponents, four per word
    float4 bufA[8], bufB[8];
    uint32_t scA[2], sc[2];
    auto scale_of = [&](const uint32_t (&e)[2], int j) {
      return __uint_as_float(((e[j >> 2] >> (8 * (j & 3))) & 0xffu) << 23);
    };
    // a tile's rows are contiguous: CPT cells x M x NG floats (128 rows of M); when a tile's
    // first chunk is loaded, one thread asks L2 for the CTA's next tile, so that the
    // converters' loads of it find it there
    const int64_t tile_bytes = (int64_t)BM * P.M * 4;
    auto prefetch_tile = [&](int64_t rt) {
      if (t != 0 || rt >= n_rt) return;
      const char *src = reinterpret_cast<const char *>(P.I) + rt * tile_bytes;
      const int64_t n = std::min(tile_bytes, (int64_t)P.rows * P.M * 4 - rt * tile_bytes);
      for (int64_t o = 0; o < n; o += 65536)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(src + o),
                     "r"((uint32_t)std::min((int64_t)65536, n - o))
                     : "memory");
    };
    auto load = [&](int64_t gc, float4 (&buf)[8], bool with_scales) {
      const int64_t rt = blockIdx.x + (gc / nk) * gridDim.x;
      const int k = (int)(gc % nk);
      const int64_t cell0 = rt * CPT;
      if (k == 0) prefetch_tile(rt + gridDim.x);
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int64_t c = cell0 + cellrel(j);
        buf[j] = c < ncell ? __ldcs(I4 + c * cstride + k * FPC + off) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
      if (SCALED && with_scales && k == 0) {
        scA[0] = scA[1] = 0u;
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const int64_t r = (cell0 + cellrel(j)) * NG + gsel;
          const float v = r < P.rows ? __ldg(P.scale + r) : 1.f;
          scA[j >> 2] |= ((__float_as_uint(v) >> 23) & 0xffu) << (8 * (j & 3));
        }
      }
    };
    auto process = [&](int64_t gc, const float4 (&buf)[8]) -> bool {
      const int64_t ti = gc / nk;
      const int k = (int)(gc % nk);
      if (SCALED && k == 0) {
        sc[0] = scA[0];
        sc[1] = scA[1];
      }
      // decisions stay warp-uniform: the regrouping below shuffles across lanes
      const bool waited = ti == 0 || mbar_wait(&a_empty[k], (uint32_t)((ti - 1) & 1));
      if (!__all_sync(0xffffffffu, waited)) {
        fail();
        return false;
      }
      if (__any_sync(0xffffffffu, *abort_flag != 0)) return false;
      uint8_t *ah = a16 + k * A_BYTES, *al = a16 + (nk + k) * A_BYTES;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        float x[4];
        regroup<NG>(buf[j], lane, x);
        if (SCALED) {
          const float f = scale_of(sc, j);
#pragma unroll
          for (int q = 0; q < 4; q++) x[q] *= f;
        }
        uint2 hv, lv;
        split4<FORM>(x, hv, lv);
        const int row = cellrel(j) * NG + gsel;
        const uint32_t o = row * 128 + ((((c4 >> 1) ^ (row & 7))) << 4) + ((c4 & 1) << 3);
        *reinterpret_cast<uint2 *>(ah + o) = hv;
        if (THREE) *reinterpret_cast<uint2 *>(al + o) = lv;
      }
      // every lane's generic-proxy writes become visible to the MMA (async proxy)
      // before the warp's one arrival
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&a_full[k]);
      return true;
    };
    prefetch_tile(blockIdx.x);
    if (nchunks > 0) load(0, bufA, true);
    for (int64_t gc = 0; gc < nchunks; gc += 2) {
      if (gc + 1 < nchunks) load(gc + 1, bufB, false);
      if (!process(gc, bufA)) break;
      if (gc + 2 < nchunks) load(gc + 2, bufA, true);
      if (gc + 1 < nchunks && !process(gc + 1, bufB)) break;
    }
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(R_REG_DRAIN));
    // ---------------- accumulator warps: warp w reads TMEM lanes 32*(w%4)..+31 (one row
    // per thread); the first four take the first half of the columns, the others the second
    const int q = warp & 3, hf = (warp - R_DRAIN0) >> 2;
    const int row = q * 32 + lane;
    const int64_t ncell = P.rows / NG;
    int64_t g = 0;
    bool ok = true;
    for (int64_t rt = blockIdx.x; rt < n_rt && ok && !*abort_flag; rt += gridDim.x) {
      const int64_t gr = rt * BM + row;
      const int64_t cell = gr / NG;  // the quad (pair) of lanes holding one cell's groups
      // the row's unscale factor, loaded before the sums arrive
      const float inv = (SCALED ? 1.f / (gr < P.rows ? __ldg(P.scale + gr) : 1.f) : 1.f) * P.b_unscale;
      const double eiso = (SCALED && gr < P.rows) ? __ldg(P.erow + gr) : 0.0;  // the isotropic part, in FP64
      for (int h = 0; h < n_h && ok; h++) {
        const bool with_mom = (h == 0) && mom;
        const int half = (nS + (with_mom ? NMOM : 0)) >> 1;  // multiple of 8
        const int c0 = hf * half;
        float run[MAX_HALF];
#pragma unroll
        for (int j = 0; j < MAX_HALF; j++) run[j] = 0.f;
        for (int m = 0; m < nk / R_KG; m++, g++) {
          const int ab = (int)(g % R_NACC);
          const bool got = mbar_wait(&acc_full[ab], (uint32_t)(g / R_NACC) & 1);
          if (!__all_sync(0xffffffffu, got)) {
            fail();
            ok = false;
            break;
          }
          if (__any_sync(0xffffffffu, *abort_flag != 0)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * R_ACC_STRIDE + c0);
#pragma unroll
          for (int j0 = 0; j0 < MAX_HALF / 8; j0 += R_GROUP) {
            uint32_t r[R_GROUP][8];
#pragma unroll
            for (int jj = 0; jj < R_GROUP; jj++)
              if ((j0 + jj) * 8 < half)
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                             : "=r"(r[jj][0]), "=r"(r[jj][1]), "=r"(r[jj][2]), "=r"(r[jj][3]), "=r"(r[jj][4]),
                               "=r"(r[jj][5]), "=r"(r[jj][6]), "=r"(r[jj][7])
                             : "r"(base + (j0 + jj) * 8));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
            for (int jj = 0; jj < R_GROUP; jj++)
              if ((j0 + jj) * 8 < half)
#pragma unroll
                for (int i = 0; i < 8; i++)
                  run[(j0 + jj) * 8 + i] = __fadd_rn(run[(j0 + jj) * 8 + i], __uint_as_float(r[jj][i]));
          }
          asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
          __syncwarp();
          if (lane == 0) mbar_arrive(&acc_empty[ab]);
        }
        if (!ok) break;
        // every lane takes part in the regrouping shuffles; stores are guarded per cell.
        // so: this lane's first output (direction h*nS + c0 + its quad / pair slot)
        float *so = P.S + (NG == 4 ? (cell * P.M + h * nS + c0 + (lane & 3)) * 4
                                   : NG == 2 ? (cell * P.M + h * nS + c0 + 2 * (lane & 1)) * 2
                                             : gr * P.M + h * nS + c0);
        const bool row_ok = NG > 1 ? cell < ncell : gr < P.rows;
#pragma unroll
        for (int j = 0; j < MAX_HALF / 4; j++) {
          const int col = c0 + 4 * j;
          if (4 * j < half) {
            float v[4] = {run[4 * j] * inv, run[4 * j + 1] * inv, run[4 * j + 2] * inv, run[4 * j + 3] * inv};
            if (SCALED && col < nS) {
#pragma unroll
              for (int i = 0; i < 4; i++) v[i] = (float)((double)v[i] + kIsoWeight * eiso);
            }
            if (col < nS) {
              if constexpr (NG == 4) {
                // lane (cell, g) holds group g of directions n..n+3 -> lane (cell, p): direction n+p, groups 0..3
                float x[4];
                regroup<4>(make_float4(v[0], v[1], v[2], v[3]), lane, x);
                if (row_ok) __stcs(reinterpret_cast<float4 *>(so + 16 * j), make_float4(x[0], x[1], x[2], x[3]));
              } else if constexpr (NG == 2) {
                float x[4];
                ungroup2(v, lane, x);
                if (row_ok) __stcs(reinterpret_cast<float4 *>(so + 8 * j), make_float4(x[0], x[1], x[2], x[3]));
              } else {
                if (row_ok) __stcs(reinterpret_cast<float4 *>(so + 4 * j), make_float4(v[0], v[1], v[2], v[3]));
              }
            } else if (gr < P.rows) {
              *reinterpret_cast<float4 *>(P.mom + gr * NMOM + (col - nS)) = make_float4(v[0], v[1], v[2], v[3]);
            }
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;\n" ::"r"(tmem));
  }
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void *p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

}  // namespace

struct rrhd_scatter_tc {
  int device = 0;
  int form = 0;
  int M = 0;
  // [copies][M + 16][M] 16-bit, row n = output column n.  The resident kernel
  // reads copy blockIdx % copies (R_COPIES, one by default: spreading the CTAs
  // over 16 copies measured no faster).
  uint16_t *d_bh = nullptr, *d_bl = nullptr;
  int copies = 1;
  CUtensorMap tm_bh, tm_bl, tm_mh, tm_ml;          // copy 0 (two-pass kernel)
  CUtensorMap tr_bh, tr_bl, tr_mh, tr_ml;          // all copies (resident kernel)
  float b_unscale = 1.f;
  int *d_err = nullptr;
  float *d_scale = nullptr;  // row scales of the FP16 forms (grown on demand)
  double *d_erow = nullptr;  // their FP64 isotropic row integrals (grown with d_scale)
  int64_t scale_cap = 0;
  double *d_mw = nullptr;    // [10][M] (a_d / A) times the moment weights (pre-pass)
  int num_sms = 148;
};

static uint16_t to_bf16(double x) {
  const __nv_bfloat16 b = __float2bfloat16_rn((float)x);  // x is representable in float range here
  return __bfloat16_as_ushort(b);
}

extern "C" rrhd_status rrhd_scatter_tc_create(const rrhd_dirs *d, int32_t form, rrhd_scatter_tc **out) {
  RRHD_CHECK_ARG(d && out, "null argument");
  RRHD_CHECK_ARG(form >= 0 && form < kForms, "unknown tensor-core form %d", form);
  RRHD_CHECK_ARG(d->M % BK == 0 && d->M >= BK && d->M <= 1024 && (d->M <= NT || d->M % NT == 0),
                 "tensor-core scattering needs M = 64 or a multiple of 128 (<= 1024)");
  *out = nullptr;
  auto enc = get_encode();
  if (!enc) return rrhd_fail(RRHD_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  RRHD_CUDA(cudaSetDevice(d->device));
  const int M = d->M, NB = M + NMOM;
  const double A = d->full_area;
  const bool f16 = (form == FORM_F16X3 || form == FORM_F16);
  const double bscale = f16 ? kF16BScale : 1.0;
  std::vector<uint16_t> bh((size_t)NB * M), bl((size_t)NB * M);
  for (int n = 0; n < NB; n++)
    for (int dd = 0; dd < M; dd++) {
      const double *w = &d->h_w[3 * dd];
      double v = 0.0;
      if (n < M) {
        const double *wn = &d->h_w[3 * n];
        const double mu = (w[0] * wn[0] + w[1] * wn[1]) + w[2] * wn[2];
        // the scaled forms take the anisotropic part only (kIsoWeight E_r is added in FP64)
        v = (f16 ? 3. * (mu * mu) : 3. * (1. + mu * mu)) / 4. * d->h_a[dd] / A;
      } else {
        const double f[10] = {1.0, w[0], w[1], w[2], w[0] * w[0], w[0] * w[1], w[0] * w[2], w[1] * w[1], w[1] * w[2], w[2] * w[2]};
        const int j = n - M;
        v = j < 10 ? f[j] * d->h_a[dd] / A : 0.0;
      }
      v *= bscale;
      uint16_t h, l;
      if (f16) {
        const __half a = __float2half_rn((float)v);
        const __half b = __float2half_rn((float)(v - (double)__half2float(a)));
        h = __half_as_ushort(a);
        l = __half_as_ushort(b);
      } else {
        h = to_bf16(v);
        const double hv = (double)__bfloat162float(__ushort_as_bfloat16(h));
        l = to_bf16(v - hv);
      }
      bh[(size_t)n * M + dd] = h;
      bl[(size_t)n * M + dd] = l;
    }
  rrhd_scatter_tc *t = new rrhd_scatter_tc();
  t->device = d->device;
  t->form = form;
  t->M = M;
  t->b_unscale = (float)(1.0 / bscale);
  cudaDeviceGetAttribute(&t->num_sms, cudaDevAttrMultiProcessorCount, d->device);
  t->copies = (M == 128 || M == 256) ? R_COPIES : 1;
  const size_t bytes = sizeof(uint16_t) * bh.size();
  if (cudaMalloc(&t->d_bh, bytes * t->copies) != cudaSuccess || cudaMalloc(&t->d_bl, bytes * t->copies) != cudaSuccess ||
      cudaMalloc(&t->d_err, sizeof(int)) != cudaSuccess || cudaMalloc(&t->d_mw, sizeof(double) * 10 * M) != cudaSuccess) {
    cudaFree(t->d_bh);
    cudaFree(t->d_bl);
    cudaFree(t->d_mw);
    cudaFree(t->d_err);
    delete t;
    return rrhd_fail(RRHD_ERR_OOM, "tensor-core operand allocation failed");
  }
  for (int c = 0; c < t->copies; c++) {
    cudaMemcpy(t->d_bh + (size_t)c * bh.size(), bh.data(), bytes, cudaMemcpyHostToDevice);
    cudaMemcpy(t->d_bl + (size_t)c * bl.size(), bl.data(), bytes, cudaMemcpyHostToDevice);
  }
  cudaMemset(t->d_err, 0, sizeof(int));
  {
    std::vector<double> mw(10 * (size_t)M);
    for (int dd = 0; dd < M; dd++) {
      const double aw = d->h_a[dd] / A, x = d->h_w[3 * dd], y = d->h_w[3 * dd + 1], z = d->h_w[3 * dd + 2];
      const double f[10] = {1.0, x, y, z, x * x, x * y, x * z, y * y, y * z, z * z};
      for (int k = 0; k < 10; k++) mw[(size_t)k * M + dd] = aw * f[k];
    }
    cudaMemcpy(t->d_mw, mw.data(), sizeof(double) * mw.size(), cudaMemcpyHostToDevice);
  }
  const CUtensorMapDataType dt = f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  auto make = [&](CUtensorMap *m, uint16_t *base, int rows_total, int box_rows, int row0) -> bool {
    cuuint64_t dims[2] = {(cuuint64_t)M, (cuuint64_t)rows_total};
    cuuint64_t strides[1] = {(cuuint64_t)M * 2};
    cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1, 1};
    return enc(m, dt, 2, base + (size_t)row0 * M, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  const int box_n = M < NT ? M : NT;
  if (!make(&t->tm_bh, t->d_bh, M, box_n, 0) || !make(&t->tm_bl, t->d_bl, M, box_n, 0) ||
      !make(&t->tm_mh, t->d_bh, NMOM, NMOM, M) || !make(&t->tm_ml, t->d_bl, NMOM, NMOM, M) ||
      !make(&t->tr_bh, t->d_bh, t->copies * NB, box_n, 0) || !make(&t->tr_bl, t->d_bl, t->copies * NB, box_n, 0) ||
      !make(&t->tr_mh, t->d_bh, t->copies * NB, NMOM, 0) || !make(&t->tr_ml, t->d_bl, t->copies * NB, NMOM, 0)) {
    cudaFree(t->d_bh);
    cudaFree(t->d_bl);
    cudaFree(t->d_err);
    delete t;
    cudaFree(t->d_mw);
    return rrhd_fail(RRHD_ERR_CUDA, "tensor map encoding failed");
  }
  *out = t;
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_scatter_tc_destroy(rrhd_scatter_tc *t) {
  if (!t) return RRHD_OK;
  cudaSetDevice(t->device);
  cudaFree(t->d_bh);
  cudaFree(t->d_bl);
  cudaFree(t->d_err);
  cudaFree(t->d_scale);
  cudaFree(t->d_erow);
  cudaFree(t->d_mw);
  delete t;
  return RRHD_OK;
}

// NG = 1: I, S are [rows][M]; NG = 2, 4: [rows / NG][M][NG] (row = cell * NG + group)
template <int FORM, int NG>
static rrhd_status launch_tc(const rrhd_scatter_tc *t, const float *I, float *S, float *mom, int64_t rows,
                             cudaStream_t st) {
  constexpr int ng = NG;
  static bool attr = false;
  if (!attr) {
    RRHD_CUDA(cudaFuncSetAttribute(k_scatter_tc<FORM, NG>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
    attr = true;
  }
  constexpr bool SCALED = (FORM == FORM_F16X3 || FORM == FORM_F16);
  if (SCALED) {
    // a warp per four cells
    const unsigned nb = (unsigned)std::min<int64_t>((rows / ng + 4 * (kPrepassThreads / 32) - 1) /
                                                        (4 * (kPrepassThreads / 32)), 8 * t->num_sms);
    const size_t wbytes = sizeof(double) * (mom ? 10 : 1) * t->M;  // <= 80 KiB (M <= 1024)
    if (mom) {
      static bool attr = false;
      if (!attr) {
        RRHD_CUDA(cudaFuncSetAttribute(k_row_prepass<NG, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(sizeof(double) * 10 * 1024)));
        attr = true;
      }
      k_row_prepass<NG, true><<<nb, kPrepassThreads, wbytes, st>>>(I, rows, t->M, t->d_mw, t->d_scale, t->d_erow, mom);
    } else {
      k_row_prepass<NG, false><<<nb, kPrepassThreads, wbytes, st>>>(I, rows, t->M, t->d_mw, t->d_scale, t->d_erow, nullptr);
    }
    RRHD_CUDA(cudaGetLastError());
  }
  // the scaled forms' moments come from the pre-pass, in FP64
  TcParams P{I, S, SCALED ? nullptr : mom, t->d_scale, t->d_erow, rows, t->M, t->b_unscale, t->d_err, t->copies};
  // M = 128 or 256: one CTA per 128-row tile and all output columns, converted
  // intensity resident.  Its warpgroups move registers between them (setmaxnreg);
  // the kernel is used only if the registers it is launched with cover the split.
  static int res_ok = -1;
  if (res_ok < 0) {
    cudaFuncAttributes fa;
    res_ok = cudaFuncGetAttributes(&fa, k_scatter_tc_res<FORM, NG>) == cudaSuccess &&
             fa.numRegs * R_THREADS >= R_REG_TOTAL &&
             cudaFuncSetAttribute(k_scatter_tc_res<FORM, NG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  r_smem_bytes(4)) == cudaSuccess;
    cudaGetLastError();
  }
  if (res_ok && (t->M == 128 || t->M == 256)) {
    const unsigned grid = (unsigned)std::min<int64_t>((rows + BM - 1) / BM, t->num_sms);
    k_scatter_tc_res<FORM, NG><<<grid, R_THREADS, r_smem_bytes(t->M / BK), st>>>(t->tr_bh, t->tr_bl, t->tr_mh,
                                                                                t->tr_ml, P);
    RRHD_CUDA(cudaGetLastError());
    return RRHD_OK;
  }
  CUtensorMap tm_a;
  {
    auto enc = get_encode();
    // rows layout: [rows][M], box {BK, BM}; cell-direction-group: [cells][M * ng], box {BK * ng, BM / ng}
    const int u = ng > 1 ? ng : 1;
    cuuint64_t dims[2] = {(cuuint64_t)t->M * u, (cuuint64_t)(rows / u)};
    cuuint64_t strides[1] = {(cuuint64_t)t->M * u * 4};
    cuuint32_t box[2] = {(cuuint32_t)(BK * u), (cuuint32_t)(BM / u)};
    cuuint32_t es[2] = {1, 1};
    if (!enc || enc(&tm_a, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(I), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return rrhd_fail(RRHD_ERR_CUDA, "tensor map encoding for the intensity failed");
  }
  const int64_t tiles = ((rows + BM - 1) / BM) * (int64_t)(t->M < NT ? 1 : t->M / NT);
  const unsigned grid = (unsigned)std::min<int64_t>(tiles, t->num_sms);
  k_scatter_tc<FORM, NG><<<grid, THREADS, SMEM_BYTES, st>>>(t->tm_bh, t->tm_bl, t->tm_mh, t->tm_ml, tm_a, P);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

static rrhd_status run_tc(const rrhd_scatter_tc *t, const float *I, float *S, float *mom, int64_t rows, int ng,
                          cudaStream_t st) {
  const bool scaled = t->form == FORM_F16X3 || t->form == FORM_F16;
  if (scaled && t->scale_cap < rows) {
    rrhd_scatter_tc *tm = const_cast<rrhd_scatter_tc *>(t);
    RRHD_CUDA(cudaStreamSynchronize(st));
    cudaFree(tm->d_scale);
    cudaFree(tm->d_erow);
    tm->d_scale = nullptr;
    tm->d_erow = nullptr;
    tm->scale_cap = 0;
    RRHD_CUDA(cudaMalloc(&tm->d_scale, sizeof(float) * rows));
    RRHD_CUDA(cudaMalloc(&tm->d_erow, sizeof(double) * rows));
    tm->scale_cap = rows;
  }
  RRHD_CHECK_ARG(((uintptr_t)I & 15) == 0 && ((uintptr_t)S & 15) == 0 && ((uintptr_t)mom & 15) == 0,
                 "I, S and moments must be 16-byte aligned");
  switch (t->form * 3 + (ng == 4 ? 2 : ng == 2 ? 1 : 0)) {
#define RRHD_TC_CASE(F)                                                        \
  case 3 * F + 0: return launch_tc<F, 1>(t, I, S, mom, rows, st);   \
  case 3 * F + 1: return launch_tc<F, 2>(t, I, S, mom, rows, st);   \
  case 3 * F + 2: return launch_tc<F, 4>(t, I, S, mom, rows, st);
    RRHD_TC_CASE(FORM_BF16X3)
    RRHD_TC_CASE(FORM_F16X3)
    RRHD_TC_CASE(FORM_F16)
    RRHD_TC_CASE(FORM_BF16)
#undef RRHD_TC_CASE
    default: return rrhd_fail(RRHD_ERR_INVALID, "bad tensor-core form");
  }
}

rrhd_status rrhd::scatter_tc_cdg(const rrhd_scatter_tc *t, const float *I, float *S, float *mom, int64_t cells,
                                 int ng, cudaStream_t st) {
  RRHD_CHECK_ARG(t && cells >= 0 && (ng == 1 || ng == 2 || ng == 4), "bad arguments");
  if (cells == 0) return RRHD_OK;
  RRHD_CHECK_ARG(I && S, "null I or S");
  return run_tc(t, I, S, mom, cells * ng, ng, st);
}


extern "C" rrhd_status rrhd_scatter_tc_run(const rrhd_scatter_tc *t, const float *I, float *S, float *mom,
                                           int64_t rows, void *stream) {
  RRHD_CHECK_ARG(t && rows >= 0, "bad arguments");
  if (rows == 0) return RRHD_OK;
  RRHD_CHECK_ARG(I && S, "null I or S");
  return run_tc(t, I, S, mom, rows, 0, (cudaStream_t)stream);
}

extern "C" rrhd_status rrhd_scatter_tc_run_cdg(const rrhd_scatter_tc *t, const float *I, float *S, float *mom,
                                               int64_t cells, int32_t groups, void *stream) {
  return rrhd::scatter_tc_cdg(t, I, S, mom, cells, groups, (cudaStream_t)stream);
}

// Error word of the tensor-core kernels (non-zero after a bounded wait timed
// out); reading it synchronises the stream, clear resets it.
extern "C" rrhd_status rrhd_scatter_tc_check(const rrhd_scatter_tc *t, void *stream, int32_t clear) {
  RRHD_CHECK_ARG(t, "null argument");
  int e = 0;
  RRHD_CUDA(cudaMemcpyAsync(&e, t->d_err, sizeof e, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  RRHD_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  if (clear) RRHD_CUDA(cudaMemsetAsync(t->d_err, 0, sizeof(int), (cudaStream_t)stream));
  if (e) return rrhd_fail(RRHD_ERR_CUDA, "tensor-core scattering: a pipeline wait timed out");
  return RRHD_OK;
}
