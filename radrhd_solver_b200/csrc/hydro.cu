// Context, device-resident mesh/state and the fused RHLLC step.
//
// Layout in HBM (all in a renumbered cell order: Morton order of cell centres,
// so that a CTA's cells and their neighbours are close in memory):
//   state  [N][10] doubles = U(5) | W(5) per cell, 80 B, loaded as 5 x double2;
//          two buffers (read one, write the other) so that no CTA overwrites a
//          neighbour state another CTA still reads.
//   per CTA (cells_per_block consecutive cells) a list of every face touching
//   one of its cells as 40-byte records {n0, n1, n2, area, l, r} (l, r the
//   CTA-local state slots, r < 0 a boundary code), padded to an even count so
//   that every CTA's list starts on a 16-byte boundary; and a halo list of the
//   neighbour cells owned by other CTAs.  A face between two CTAs sits in both
//   lists and is computed by both, bit-identically.  Per cell a 16-byte record
//   {4 local face slots with the cell's sign bit in bit 15, volume}.
// One kernel does the whole step:
//   phase 0  cp.async stages the CTA's own states (one contiguous range), its
//            halo states, its face records and its cell records into shared
//            memory, all requests in flight at once;
//   then     the squared sound speed of every staged cell (a function of its rho
//            and p alone), once per cell rather than once per face side;
//   phase 1  face fluxes from the staged states; each thread overwrites the
//            face record it has read with that face's flux;
//   phase 2  each cell sums its 4 faces in the reference's order (id_faces
//            j = 0..3 with sign_n), updates U, runs con2prim with the
//            PhysPressureFix fallback and writes U, W and a status byte.
// No atomics touch the state; the max signal speed and the fallback counts are
// reduced per CTA and combined with one atomic per CTA.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <vector>

#include <cuda.h>

#include "ctx.h"
#include "hydro_phys.cuh"
#include "rrhd_internal.h"

using namespace rrhd;

namespace {

struct StepParams {
  Eos eos;
  int N;
  int cpb;
  int b0;  // first CTA block of this launch (the rank's range under a split)
  const int32_t *__restrict__ off;
  const int32_t *__restrict__ halo_off;
  const int32_t *__restrict__ halo_ids;
  int max_halo;
  const FaceRec *__restrict__ face;
  const int32_t *__restrict__ gid;
  const CellRec *__restrict__ cell;
  const double *__restrict__ sin;
  double *__restrict__ sout;
  uint8_t *__restrict__ status;
  double *__restrict__ face_flux;
  const StepScalars *prev;
  StepScalars *out;
  double tau;
  int device_tau;
  double cfl_hmin;
  BcTable bc;
};

__device__ __forceinline__ void store_state(double *s, int c, const double *U, const double *W) {
  double2 *p = reinterpret_cast<double2 *>(s + 10 * (size_t)c);
  p[0] = make_double2(U[0], U[1]);
  p[1] = make_double2(U[2], U[3]);
  p[2] = make_double2(U[4], W[0]);
  p[3] = make_double2(W[1], W[2]);
  p[4] = make_double2(W[3], W[4]);
}

// rhllc::BoundConditions (solvers/rhllc/src/rhllc_utils.cpp:45-133) from the table.
// R is the face's rotation (GetRotationMatrix of its normal).  UR/WR may alias UL/WL.
__device__ __forceinline__ void boundary(const BcTable &bc, int code, const Rot &R, const double *UL,
                                         const double *WL, double *UR, double *WR) {
  const int k = -code - 1;
  const int kind = (k < 8) ? bc.kind[k] : 0;
  if (kind == RRHD_BC_FIXED) {
#pragma unroll
    for (int i = 0; i < 5; i++) {
      UR[i] = bc.U[k][i];
      WR[i] = bc.W[k][i];
    }
    return;
  }
#pragma unroll
  for (int i = 0; i < 5; i++) {
    UR[i] = UL[i];
    WR[i] = WL[i];
  }
  if (kind == RRHD_BC_REFLECT) {
    // v -> T^T diag(-1, 1, 1) T v, with T^T formed as a matrix (Matrix3 * Vector3 order)
    double r[3];
    matvec(R, UR + 1, r);
    r[0] = -r[0];
    matvec_transposed(R, r, UR + 1);
    matvec(R, WR + 1, r);
    r[0] = -r[0];
    matvec_transposed(R, r, WR + 1);
  }
}

#ifndef RRHD_STEP_THREADS
#define RRHD_STEP_THREADS 256  // threads per CTA of the step kernel
#endif
constexpr int kStepThreads = RRHD_STEP_THREADS;
constexpr int kMaxCellsPerBlock = 1024;  // local cell index fits 12 bits

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

__device__ __forceinline__ void load_state_smem(const double *s, int slot, double *U, double *W) {
  const double2 *p = reinterpret_cast<const double2 *>(s + 10 * slot);
  const double2 a = p[0], b = p[1], d = p[2], e = p[3], f = p[4];
  U[0] = a.x;
  U[1] = a.y;
  U[2] = b.x;
  U[3] = b.y;
  U[4] = d.x;
  W[0] = d.y;
  W[1] = e.x;
  W[2] = e.y;
  W[3] = f.x;
  W[4] = f.y;
}

#ifndef RRHD_STEP_MIN_BLOCKS
#define RRHD_STEP_MIN_BLOCKS 3  // CTAs per SM the register budget is sized for
#endif
// kFaceFlux: also write every face's flux to P.face_flux (caller numbering), for
// rrhd_keep_face_flux; a separate instantiation keeps the common one lean.
template <bool kFaceFlux>
__global__ void __launch_bounds__(kStepThreads, RRHD_STEP_MIN_BLOCKS) k_hydro_step(const StepParams P) {
  extern __shared__ double2 smem_raw[];
  double *sstate = reinterpret_cast<double *>(smem_raw);      // [cpb + max_halo][10]
  double *sface = sstate + 10 * (P.cpb + P.max_halo);         // [entries][5]: record, then flux
  const int b = P.b0 + blockIdx.x;
  const int e0 = P.off[b], e1 = P.off[b + 1];
  CellRec *scell = reinterpret_cast<CellRec *>(sface + 5 * (e1 - e0));  // [cpb]
  double *scs2 = reinterpret_cast<double *>(scell + P.cpb);              // [cpb + max_halo] sound speeds^2
  __shared__ double s_red[kStepThreads / 32];
  __shared__ unsigned long long s_cnt[2];
  __shared__ unsigned short s_fail[kMaxCellsPerBlock];
  __shared__ int s_nfail;
  const int c0 = b * P.cpb;
  const int nc = min(P.cpb, P.N - c0);
  const int h0 = P.halo_off[b], h1 = P.halo_off[b + 1];
  double tau = P.tau;
  if (P.device_tau) tau = P.cfl_hmin / P.prev->max_speed;
  if (threadIdx.x < 2) s_cnt[threadIdx.x] = 0;
  if (threadIdx.x == 0) s_nfail = 0;

  // phase 0: stage own (contiguous) and halo states, the face records and the
  // cell records, 16 bytes per request.  Each CTA's face list starts on a
  // 16-byte boundary and holds an even number of 40-byte records.
  {
    const char *g = reinterpret_cast<const char *>(P.sin);
    char *sm = reinterpret_cast<char *>(sstate);
    for (int q = threadIdx.x; q < nc * 5; q += kStepThreads)
      cp_async16(sm + 16 * q, g + 80 * (size_t)c0 + 16 * q);
    for (int q = threadIdx.x; q < (h1 - h0) * 5; q += kStepThreads) {
      const int h = q / 5, k = q - 5 * h;
      cp_async16(sm + 80 * (P.cpb + h) + 16 * k, g + 80 * (size_t)P.halo_ids[h0 + h] + 16 * k);
    }
    const char *gf = reinterpret_cast<const char *>(P.face + e0);
    char *sf = reinterpret_cast<char *>(sface);
    for (int q = threadIdx.x; q < (e1 - e0) * 40 / 16; q += kStepThreads) cp_async16(sf + 16 * q, gf + 16 * q);
    const char *gc = reinterpret_cast<const char *>(P.cell + c0);
    char *sc = reinterpret_cast<char *>(scell);
    for (int q = threadIdx.x; q < nc; q += kStepThreads) cp_async16(sc + 16 * q, gc + 16 * q);
    cp_async_wait_all();
  }
  __syncthreads();
  // the squared sound speed of every staged cell (GetFluxStab's cs^2, rhllc_flux_stab.cpp:276-291,
  // depends on the cell's rho and p alone): once per cell instead of once per face side
  for (int q = threadIdx.x; q < nc + (h1 - h0); q += kStepThreads) {
    const int slot = q < nc ? q : P.cpb + (q - nc);
    const double *st = sstate + 10 * slot;
    scs2[slot] = sound_speed2(P.eos, st[5], st[9]);
  }
  __syncthreads();

  // phase 1: every face touching this CTA's cells; the flux replaces the record
  double vmax = 0.0;
  for (int e = threadIdx.x; e < e1 - e0; e += kStepThreads) {
    double *rec = sface + 5 * e;
    const double n0 = rec[0], n1 = rec[1], n2 = rec[2], area = rec[3];
    const int2 lr = *reinterpret_cast<const int2 *>(rec + 4);
    if (lr.y == kFacePad) continue;
    Rot R;
    rotation(n0, n1, n2, R);
    double U[5], W[5], Fl[5];
    load_state_smem(sstate, lr.x, U, W);
    const FaceSide sl = face_side(R, U, W, scs2[lr.x]);
    double cs2r;
    if (lr.y >= 0) {
      load_state_smem(sstate, lr.y, U, W);
      cs2r = scs2[lr.y];
    } else {
      boundary(P.bc, lr.y, R, U, W, U, W);  // ghost state from the left one, in place
      cs2r = sound_speed2(P.eos, W[0], W[4]);
    }
    const FaceSide sr = face_side(R, U, W, cs2r);
    const FaceStar fs = face_star(sl, sr);
    vmax = smax(vmax, fs.vmax);
    // the selected side's conservative state again (registers are the scarce resource)
    load_state_smem(sstate, (fs.right && lr.y >= 0) ? lr.y : lr.x, U, W);
    if (fs.right && lr.y < 0) boundary(P.bc, lr.y, R, U, W, U, W);
    face_flux(R, U, fs.right ? sr : sl, fs, area, Fl);
#pragma unroll
    for (int i = 0; i < 5; i++) rec[i] = Fl[i];
    if (kFaceFlux) {
      const int gf = P.gid[e0 + e];
      if (gf >= 0) {
#pragma unroll
        for (int i = 0; i < 5; i++) P.face_flux[5 * (size_t)gf + i] = Fl[i];
      }
    }
  }
  __syncthreads();

  // phase 2: gather, update, con2prim.  Cells whose con2prim fails keep their
  // updated U and old W in the staging slot for the fallback pass below.
  unsigned n_fb = 0, n_fail = 0;
  for (int cl = threadIdx.x; cl < nc; cl += kStepThreads) {
    const int c = c0 + cl;
    const CellRec cr = scell[cl];
    double sum[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const double *f = sface + 5 * (cr.s[j] & 0x7fff);
      if (cr.s[j] & 0x8000) {
#pragma unroll
        for (int i = 0; i < 5; i++) sum[i] += f[i];
      } else {
#pragma unroll
        for (int i = 0; i < 5; i++) sum[i] -= f[i];
      }
    }
    const double sc = (tau / cr.V);
    double U[5], W[5];
    load_state_smem(sstate, cl, U, W);
#pragma unroll
    for (int i = 0; i < 5; i++) U[i] -= sum[i] * sc;
    const int code = c2p(P.eos, U, W);
    if (code) {
      store_state(sstate, cl, U, W);
      s_fail[atomicAdd(&s_nfail, 1)] = (unsigned short)(cl | (code << 12));
    } else {
      store_state(P.sout, c, U, W);
      P.status[c] = 0;
    }
  }
  __syncthreads();
  // fallback pass: rhllc::PhysPressureFix where con2prim failed (rare)
  for (int i = threadIdx.x; i < s_nfail; i += kStepThreads) {
    const int cl = s_fail[i] & 0xfff, code = s_fail[i] >> 12;
    double U[5], W[5];
    load_state_smem(sstate, cl, U, W);
    const int fix = pressure_fix(P.eos, U, W);
    store_state(P.sout, c0 + cl, U, W);
    P.status[c0 + cl] = (uint8_t)(code | RRHD_STATUS_FALLBACK | (fix ? RRHD_STATUS_FAILED : 0));
    n_fb += 1;
    n_fail += fix ? 1u : 0u;
  }

  // CTA reduction of the max speed and the counters
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) vmax = smax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = vmax;
  if (n_fb) atomicAdd(&s_cnt[0], (unsigned long long)n_fb);
  if (n_fail) atomicAdd(&s_cnt[1], (unsigned long long)n_fail);
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < kStepThreads / 32; w++) m = smax(m, s_red[w]);
    // non-negative doubles order like their bit patterns
    atomicMax(reinterpret_cast<unsigned long long *>(&P.out->max_speed),
              (unsigned long long)__double_as_longlong(m));
    if (s_cnt[0]) atomicAdd(&P.out->n_fallback, s_cnt[0]);
    if (s_cnt[1]) atomicAdd(&P.out->n_failed, s_cnt[1]);
    if (blockIdx.x == 0) P.out->tau = tau;
  }
}

// caller order <-> context order
__global__ void k_set_state(int64_t N, const double *W, int64_t sw, const double *U, int64_t su,
                            const int32_t *iperm, double *state) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= N) return;
  double *dst = state + 10 * (size_t)iperm[i];
  if (U)
    for (int k = 0; k < 5; k++) dst[k] = U[i * su + k];
  if (W)
    for (int k = 0; k < 5; k++) dst[5 + k] = W[i * sw + k];
}

__global__ void k_get_state(int64_t N, double *W, int64_t sw, double *U, int64_t su,
                            const int32_t *iperm, const double *state) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double *src = state + 10 * (size_t)iperm[i];
  if (U)
    for (int k = 0; k < 5; k++) U[i * su + k] = src[k];
  if (W)
    for (int k = 0; k < 5; k++) W[i * sw + k] = src[5 + k];
}

__global__ void k_prim2con_state(int64_t N, Eos eos, double *state) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= N) return;
  double *s = state + 10 * (size_t)c;
  double U[5], W[5];
  for (int k = 0; k < 5; k++) W[k] = s[5 + k];
  p2c(eos, W, U);
  for (int k = 0; k < 5; k++) {
    s[k] = U[k];
    s[5 + k] = W[k];
  }
}

__global__ void k_get_status(int64_t N, const int32_t *iperm, const uint8_t *st, uint8_t *out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < N) out[i] = st[iperm[i]];
}

__global__ void k_c2p_batch(Eos eos, double *U, double *W, uint8_t *status, int64_t n,
                            int fallback) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double u[5], w[5];
  for (int k = 0; k < 5; k++) {
    u[k] = U[5 * i + k];
    w[k] = W[5 * i + k];
  }
  int code = c2p(eos, u, w);
  if (code && fallback) {
    const int fix = pressure_fix(eos, u, w);
    code = code | 0x10 | (fix ? 0x20 : 0);
    for (int k = 0; k < 5; k++) U[5 * i + k] = u[k];
  }
  for (int k = 0; k < 5; k++) W[5 * i + k] = w[k];
  if (status) status[i] = (uint8_t)code;
}

// con2prim with per-CTA statistics.  Each CTA handles kC2pPerBlock states and
// writes one partial record (ok, fallback, failed, Newton iterations, max
// iterations) to scratch[blockIdx.x]; k_c2p_stats_reduce sums the partials in a
// fixed order into scratch[nblocks], so the totals do not depend on scheduling.
constexpr int kC2pThreads = 256;
constexpr int kC2pPerThread = 8;
constexpr int kC2pPerBlock = kC2pThreads * kC2pPerThread;

struct C2pPartial {
  unsigned long long ok, fallback, failed, iters, max_iters;
};

#ifndef RRHD_C2P_MIN_BLOCKS
#define RRHD_C2P_MIN_BLOCKS 3  // CTAs per SM the register budget of k_c2p_stats is sized for
#endif
__global__ void __launch_bounds__(kC2pThreads, RRHD_C2P_MIN_BLOCKS) k_c2p_stats(Eos eos, double *U, double *W, uint8_t *status,
                                                          int64_t n, int fallback, C2pPartial *scratch) {
  // the states whose Newton solve fails go to a second pass (PhysPressureFix), so that the
  // main loop keeps few registers live: local index | code << 12
  __shared__ unsigned short s_fail[kC2pPerBlock];
  __shared__ int s_nfail;
  if (threadIdx.x == 0) s_nfail = 0;
  __syncthreads();
  unsigned ok = 0, it_sum = 0, it_max = 0;
  const int64_t base = (int64_t)blockIdx.x * kC2pPerBlock;
  for (int k = 0; k < kC2pPerThread; k++) {
    const int loc = k * kC2pThreads + threadIdx.x;
    const int64_t i = base + loc;
    if (i >= n) break;
    double u[5], w[5];  // w: the solve's output (the Newton solve reads no old W)
    for (int q = 0; q < 5; q++) u[q] = U[5 * i + q];
    int it = 0;
    const int code = c2p_from(eos, u, w, 0.0, false, &it);
    it_sum += (unsigned)it;
    it_max = (unsigned)it > it_max ? (unsigned)it : it_max;
    if (code == 0) {
      ok++;
      for (int q = 0; q < 5; q++) W[5 * i + q] = w[q];
      if (status) status[i] = 0;
    } else {
      s_fail[atomicAdd(&s_nfail, 1)] = (unsigned short)(loc | (code << 12));
    }
  }
  __syncthreads();
  unsigned fb = 0, failed = 0;
  for (int q = threadIdx.x; q < s_nfail; q += kC2pThreads) {
    const int64_t i = base + (s_fail[q] & 0xfff);
    int code = s_fail[q] >> 12;
    double u[5], w[5];
    for (int r = 0; r < 5; r++) {
      u[r] = U[5 * i + r];
      w[r] = W[5 * i + r];
    }
    if (fallback) {
      const int fix = pressure_fix(eos, u, w);
      code = code | 0x10 | (fix ? 0x20 : 0);
      fb++;
      failed += fix ? 1 : 0;
      for (int r = 0; r < 5; r++) U[5 * i + r] = u[r];
    } else {
      failed++;
    }
    for (int r = 0; r < 5; r++) W[5 * i + r] = w[r];
    if (status) status[i] = (uint8_t)code;
  }
  unsigned long long okl = ok, fbl = fb, failedl = failed, iters = it_sum, mx = it_max;
  __shared__ unsigned long long red[5][kC2pThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    okl += __shfl_xor_sync(0xffffffffu, okl, o);
    fbl += __shfl_xor_sync(0xffffffffu, fbl, o);
    failedl += __shfl_xor_sync(0xffffffffu, failedl, o);
    iters += __shfl_xor_sync(0xffffffffu, iters, o);
    const unsigned long long m2 = __shfl_xor_sync(0xffffffffu, mx, o);
    mx = m2 > mx ? m2 : mx;
  }
  const int wid = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][wid] = okl;
    red[1][wid] = fbl;
    red[2][wid] = failedl;
    red[3][wid] = iters;
    red[4][wid] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    C2pPartial p = {0, 0, 0, 0, 0};
    for (int w2 = 0; w2 < kC2pThreads / 32; w2++) {
      p.ok += red[0][w2];
      p.fallback += red[1][w2];
      p.failed += red[2][w2];
      p.iters += red[3][w2];
      p.max_iters = red[4][w2] > p.max_iters ? red[4][w2] : p.max_iters;
    }
    scratch[blockIdx.x] = p;
  }
}

__global__ void k_c2p_stats_reduce(C2pPartial *scratch, int nblocks) {
  __shared__ C2pPartial red[256];
  C2pPartial p = {0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += 256) {
    const C2pPartial q = scratch[b];
    p.ok += q.ok;
    p.fallback += q.fallback;
    p.failed += q.failed;
    p.iters += q.iters;
    p.max_iters = q.max_iters > p.max_iters ? q.max_iters : p.max_iters;
  }
  red[threadIdx.x] = p;
  __syncthreads();
  if (threadIdx.x == 0) {
    C2pPartial t = {0, 0, 0, 0, 0};
    for (int k = 0; k < 256; k++) {
      t.ok += red[k].ok;
      t.fallback += red[k].fallback;
      t.failed += red[k].failed;
      t.iters += red[k].iters;
      t.max_iters = red[k].max_iters > t.max_iters ? red[k].max_iters : t.max_iters;
    }
    scratch[nblocks] = t;
  }
}

__global__ void k_p2c_batch(Eos eos, double *W, double *U, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double u[5], w[5];
  for (int k = 0; k < 5; k++) w[k] = W[5 * i + k];
  p2c(eos, w, u);
  for (int k = 0; k < 5; k++) {
    U[5 * i + k] = u[k];
    W[5 * i + k] = w[k];
  }
}

inline unsigned grid1d(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

Eos make_eos(int eos, double gamma) {
  Eos e;
  e.eos = eos;
  e.g1 = gamma;
  e.gg = gamma / (gamma - 1.0);
  return e;
}

template <class T>
rrhd_status upload(T **dst, const std::vector<T> &src) {
  RRHD_CUDA(cudaMalloc((void **)dst, sizeof(T) * std::max<size_t>(src.size(), 1)));
  RRHD_CUDA(cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice));
  return RRHD_OK;
}

void free_ctx(rrhd_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  rrhd_rad_release(c);
  void *ptrs[] = {c->d_perm, c->d_iperm, c->d_bface_off, c->d_bface_rec, c->d_halo_off, c->d_halo_ids,
                  c->d_bface_gid, c->d_cell_rec, c->d_state[0],
                  c->d_state[1], c->d_status, c->d_scal, c->d_face_flux, c->d_scratch_io,
                  c->d_send_ids, c->d_recv_ids};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (c->h_pinned) cudaFreeHost(c->h_pinned);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

}  // namespace

extern "C" rrhd_status rrhd_create(const rrhd_mesh_desc *m, const rrhd_opts *opts, rrhd_ctx **out) {
  RRHD_CHECK_ARG(m && out, "null argument");
  *out = nullptr;
  RRHD_CHECK_ARG(m->n_cells > 0 && m->n_faces > 0 && m->n_cells < (int64_t(1) << 30) &&
                     m->n_faces < (int64_t(1) << 31),
                 "bad mesh sizes");
  RRHD_CHECK_ARG(m->face_id_l && m->face_id_r && m->face_n && m->face_area && m->cell_faces &&
                     m->cell_sign && m->cell_volume && m->cell_center,
                 "null mesh array");
  const int64_t N = m->n_cells, F = m->n_faces;
  for (int64_t f = 0; f < F; f++) {
    RRHD_CHECK_ARG(m->face_id_l[f] >= 0 && m->face_id_l[f] < N, "face %lld: bad id_l", (long long)f);
    RRHD_CHECK_ARG(m->face_id_r[f] < N && m->face_id_r[f] >= -8, "face %lld: bad id_r", (long long)f);
  }
  for (int64_t c = 0; c < 4 * N; c++)
    RRHD_CHECK_ARG(m->cell_faces[c] >= 0 && m->cell_faces[c] < F, "cell %lld: bad face id", (long long)(c / 4));

  rrhd_ctx *c = new rrhd_ctx();
  rrhd_status st = RRHD_OK;
  auto fail = [&](rrhd_status s) {
    free_ctx(c);
    return s;
  };
  c->device = opts ? opts->device : 0;
  c->eos = (opts && opts->eos) ? opts->eos : RRHD_EOS_IDEAL;
  c->gamma = (opts && opts->gamma > 0) ? opts->gamma : 5.0 / 3.0;
  c->cpb = (opts && opts->cells_per_block > 0) ? opts->cells_per_block : 256;
  if (c->eos != RRHD_EOS_IDEAL && c->eos != RRHD_EOS_TAUB) return fail(rrhd_fail(RRHD_ERR_INVALID, "bad eos"));
  if (c->cpb > 1024 || c->cpb < 32) return fail(rrhd_fail(RRHD_ERR_INVALID, "cells_per_block out of [32,1024]"));
  c->N = N;
  c->F = F;
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(rrhd_fail(RRHD_ERR_CUDA, "cudaSetDevice(%d) failed", c->device));
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(rrhd_fail(RRHD_ERR_CUDA, "stream creation failed"));

  // renumbering: Morton order of cell centres (rrhd_cell_order)
  std::vector<int32_t> perm(N), iperm(N);
  if ((st = rrhd_cell_order(m, opts ? opts->renumber : 0, perm.data()))) return fail(st);
  for (int64_t i = 0; i < N; i++) iperm[perm[i]] = (int32_t)i;

  // per-CTA face lists
  const int cpb = c->cpb;
  const int nb = (int)((N + cpb - 1) / cpb);
  c->nblocks = nb;
  c->part_b1 = nb;
  c->part_c1 = N;
  std::vector<int32_t> off(nb + 1, 0);
  std::vector<FaceRec> frec;
  std::vector<int32_t> gid;
  frec.reserve((size_t)(F * 1.3));
  gid.reserve((size_t)(F * 1.3));
  std::vector<CellRec> crec(N);
  std::vector<int32_t> stamp(F, -1), local(F, 0);
  std::vector<int32_t> hstamp(N, -1), hlocal(N, 0);
  std::vector<int32_t> hoff(nb + 1, 0), hids;
  hids.reserve((size_t)(N / 2));
  int max_e = 0, max_h = 0;
  for (int b = 0; b < nb; b++) {
    int ne = 0, nh = 0;
    const int64_t c0 = (int64_t)b * cpb, c1 = std::min<int64_t>(N, c0 + cpb);
    // CTA-local state slot of a cell: own cells first, then the halo
    auto slot_of = [&](int32_t x) -> int32_t {
      if (x >= c0 && x < c1) return (int32_t)(x - c0);
      if (hstamp[x] != b) {
        hstamp[x] = b;
        hlocal[x] = nh++;
        hids.push_back(x);
      }
      return cpb + hlocal[x];
    };
    for (int64_t cn = c0; cn < c1; cn++) {
      const int32_t co = perm[cn];
      unsigned short s4[4];
      for (int j = 0; j < 4; j++) {
        const int32_t f = m->cell_faces[4 * co + j];
        if (stamp[f] != b) {
          stamp[f] = b;
          local[f] = ne++;
          const int32_t l = iperm[m->face_id_l[f]];
          const int32_t r = m->face_id_r[f] >= 0 ? iperm[m->face_id_r[f]] : m->face_id_r[f];
          const int32_t ls = slot_of(l);
          const int32_t rs = r >= 0 ? slot_of(r) : r;
          frec.push_back(FaceRec{m->face_n[3 * f], m->face_n[3 * f + 1], m->face_n[3 * f + 2], m->face_area[f],
                                 ls, rs});
          gid.push_back((l / cpb == b) ? f : -1);
        }
        s4[j] = (unsigned short)local[f];
      }
      CellRec &cr = crec[cn];
      for (int j = 0; j < 4; j++)
        cr.s[j] = (uint16_t)(s4[j] | (((m->cell_sign[co] >> j) & 1u) << 15));
      cr.V = m->cell_volume[co];
    }
    if (ne & 1) {  // pad to an even count: every CTA's list then starts on a 16-byte boundary
      frec.push_back(FaceRec{0.0, 0.0, 0.0, 0.0, 0, kFacePad});
      gid.push_back(-1);
      ne++;
    }
    if (ne > 32767) return fail(rrhd_fail(RRHD_ERR_LIMIT, "CTA face list too long"));
    max_e = std::max(max_e, ne);
    max_h = std::max(max_h, nh);
    off[b + 1] = off[b] + ne;
    hoff[b + 1] = hoff[b] + nh;
  }
  c->max_halo = max_h;
  c->h_cell_faces.assign(m->cell_faces, m->cell_faces + 4 * N);
  c->h_cell_sign.assign(m->cell_sign, m->cell_sign + N);
  c->h_face_l.assign(m->face_id_l, m->face_id_l + F);
  c->h_face_r.assign(m->face_id_r, m->face_id_r + F);
  c->h_face_n.assign(m->face_n, m->face_n + 3 * F);
  c->h_face_area.assign(m->face_area, m->face_area + F);
  c->h_cell_V.assign(m->cell_volume, m->cell_volume + N);
  c->max_entries = max_e;
  c->n_entries = off[nb];
  c->h_perm = perm;
  if ((st = upload(&c->d_perm, perm)) || (st = upload(&c->d_iperm, iperm)) ||
      (st = upload(&c->d_bface_off, off)) || (st = upload(&c->d_bface_rec, frec)) ||
      (st = upload(&c->d_bface_gid, gid)) || (st = upload(&c->d_cell_rec, crec)) || (st = upload(&c->d_halo_off, hoff)) ||
      (st = upload(&c->d_halo_ids, hids)))
    return fail(st);
  const size_t ssz = sizeof(double) * 10 * N;
  if (cudaMalloc(&c->d_state[0], ssz) != cudaSuccess || cudaMalloc(&c->d_state[1], ssz) != cudaSuccess ||
      cudaMalloc(&c->d_status, N) != cudaSuccess || cudaMalloc(&c->d_scal, 2 * sizeof(StepScalars)) != cudaSuccess ||
      cudaMalloc(&c->d_scratch_io, ssz) != cudaSuccess)
    return fail(rrhd_fail(RRHD_ERR_OOM, "device allocation of the state failed"));
  cudaMemset(c->d_state[0], 0, ssz);
  cudaMemset(c->d_state[1], 0, ssz);
  cudaMemset(c->d_status, 0, N);
  StepScalars init[2] = {{0, 0, 0, 0}, {1.0, 0, 0, 0}};  // rhllc::max_signal_speed = 1 initially
  cudaMemcpy(c->d_scal, init, sizeof init, cudaMemcpyHostToDevice);
  c->scal_cur = 0;
  for (int k = 0; k < 8; k++) c->bc.kind[k] = RRHD_BC_TRANSMISSIVE;
  // staged states (own + halo), the CTA's face records (then fluxes) and cell records
  const size_t smem =
      sizeof(double) * (10 * (size_t)(cpb + max_h) + 5 * (size_t)max_e + (size_t)(cpb + max_h)) + sizeof(CellRec) * cpb;
  c->step_smem = smem;
  if (smem > 227 * 1024)
    return fail(rrhd_fail(RRHD_ERR_LIMIT, "step needs %zu B of shared memory per CTA; lower cells_per_block", smem));
  if (cudaFuncSetAttribute(k_hydro_step<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      cudaFuncSetAttribute(k_hydro_step<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return fail(rrhd_fail(RRHD_ERR_LIMIT, "cannot reserve %zu B of shared memory", smem));
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(rrhd_fail(RRHD_ERR_CUDA, "%s", cudaGetErrorString(cudaGetLastError())));
  *out = c;
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_destroy(rrhd_ctx *c) {
  if (c) {
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    free_ctx(c);
  }
  return RRHD_OK;
}

extern "C" void *rrhd_stream(rrhd_ctx *c) { return c ? (void *)c->stream : nullptr; }

extern "C" rrhd_status rrhd_sync(rrhd_ctx *c) {
  RRHD_CHECK_ARG(c, "null context");
  RRHD_CUDA(cudaStreamSynchronize(c->stream));
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_set_boundary(rrhd_ctx *c, int32_t code, int32_t kind, const double *W) {
  RRHD_CHECK_ARG(c && code <= -1 && code >= -8, "boundary code must be in [-8, -1]");
  RRHD_CHECK_ARG(kind >= 0 && kind <= 2, "bad boundary kind");
  const int k = -code - 1;
  c->bc.kind[k] = kind;
  if (kind == RRHD_BC_FIXED) {
    RRHD_CHECK_ARG(W, "fixed boundary needs a state");
    const double gg = c->gamma / (c->gamma - 1.0);
    for (int i = 0; i < 5; i++) c->bc.W[k][i] = W[i];
    p2c_plain(gg, c->bc.W[k], c->bc.U[k]);
  }
  return RRHD_OK;
}

static rrhd_status state_transfer(rrhd_ctx *c, double *W, double *U, int64_t stride, int32_t where, bool set) {
  RRHD_CHECK_ARG(c, "null context");
  RRHD_CHECK_ARG(stride >= 5, "stride must be >= 5");
  RRHD_CHECK_ARG(where == RRHD_HOST || where == RRHD_DEVICE, "bad `where`");
  RRHD_CUDA(cudaSetDevice(c->device));
  const int64_t N = c->N;
  double *state = c->d_state[c->cur];
  if (where == RRHD_DEVICE) {
    if (set)
      k_set_state<<<grid1d(N, 256), 256, 0, c->stream>>>(N, W, stride, U, stride, c->d_iperm, state);
    else
      k_get_state<<<grid1d(N, 256), 256, 0, c->stream>>>(N, W, stride, U, stride, c->d_iperm, state);
    RRHD_CUDA(cudaGetLastError());
    return RRHD_OK;
  }
  // host: contiguous [N][5] arrays go straight to/from the device staging area
  // (fast when the caller's memory is pinned); strided records are packed
  // through the context's pinned buffer.
  double *dW = c->d_scratch_io, *dU = c->d_scratch_io + 5 * N;
  const size_t bytes = sizeof(double) * 5 * N;
  if (stride != 5 && !c->h_pinned) RRHD_CUDA(cudaMallocHost(&c->h_pinned, 2 * bytes));
  double *hW = c->h_pinned, *hU = c->h_pinned ? c->h_pinned + 5 * N : nullptr;
  if (set) {
    if (stride != 5) {
      for (int64_t i = 0; i < N; i++) {
        if (W) memcpy(hW + 5 * i, W + i * stride, 5 * sizeof(double));
        if (U) memcpy(hU + 5 * i, U + i * stride, 5 * sizeof(double));
      }
    }
    if (W) RRHD_CUDA(cudaMemcpyAsync(dW, stride == 5 ? W : hW, bytes, cudaMemcpyHostToDevice, c->stream));
    if (U) RRHD_CUDA(cudaMemcpyAsync(dU, stride == 5 ? U : hU, bytes, cudaMemcpyHostToDevice, c->stream));
    k_set_state<<<grid1d(N, 256), 256, 0, c->stream>>>(N, W ? dW : nullptr, 5, U ? dU : nullptr, 5,
                                                        c->d_iperm, state);
    RRHD_CUDA(cudaGetLastError());
    if (stride != 5) RRHD_CUDA(cudaStreamSynchronize(c->stream));
  } else {
    k_get_state<<<grid1d(N, 256), 256, 0, c->stream>>>(N, W ? dW : nullptr, 5, U ? dU : nullptr, 5,
                                                        c->d_iperm, state);
    RRHD_CUDA(cudaGetLastError());
    if (W) RRHD_CUDA(cudaMemcpyAsync(stride == 5 ? W : hW, dW, bytes, cudaMemcpyDeviceToHost, c->stream));
    if (U) RRHD_CUDA(cudaMemcpyAsync(stride == 5 ? U : hU, dU, bytes, cudaMemcpyDeviceToHost, c->stream));
    RRHD_CUDA(cudaStreamSynchronize(c->stream));
    if (stride != 5) {
      for (int64_t i = 0; i < N; i++) {
        if (W) memcpy(W + i * stride, hW + 5 * i, 5 * sizeof(double));
        if (U) memcpy(U + i * stride, hU + 5 * i, 5 * sizeof(double));
      }
    }
  }
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_set_state(rrhd_ctx *c, const double *W, const double *U, int64_t stride,
                                      int32_t where) {
  return state_transfer(c, const_cast<double *>(W), const_cast<double *>(U), stride, where, true);
}

extern "C" rrhd_status rrhd_hydro_layout_info(const rrhd_ctx *c, int32_t *cells_per_block, int32_t *blocks,
                                              int64_t *face_entries, int64_t *faces) {
  RRHD_CHECK_ARG(c, "null context");
  if (cells_per_block) *cells_per_block = c->cpb;
  if (blocks) *blocks = c->nblocks;
  if (face_entries) *face_entries = c->n_entries;
  if (faces) *faces = c->F;
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_get_state(rrhd_ctx *c, double *W, double *U, int64_t stride, int32_t where) {
  return state_transfer(c, W, U, stride, where, false);
}

extern "C" rrhd_status rrhd_set_state_prim(rrhd_ctx *c, const double *W, int64_t stride, int32_t where) {
  rrhd_status st = state_transfer(c, const_cast<double *>(W), nullptr, stride, where, true);
  if (st) return st;
  k_prim2con_state<<<grid1d(c->N, 256), 256, 0, c->stream>>>(c->N, make_eos(c->eos, c->gamma),
                                                               c->d_state[c->cur]);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_set_time_step(rrhd_ctx *c, double cfl, double h_min, double initial_max_speed) {
  RRHD_CHECK_ARG(c && cfl > 0 && h_min > 0, "bad time-step parameters");
  c->cfl = cfl;
  c->h_min = h_min;
  if (initial_max_speed > 0) {
    RRHD_CUDA(cudaStreamSynchronize(c->stream));
    StepScalars s = {initial_max_speed, 0, 0, 0};
    RRHD_CUDA(cudaMemcpy(&c->d_scal[c->scal_cur ^ 1], &s, sizeof s, cudaMemcpyHostToDevice));
  }
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_hydro_step(rrhd_ctx *c, double tau, rrhd_step_stats *stats) {
  RRHD_CHECK_ARG(c, "null context");
  if (tau <= 0) RRHD_CHECK_ARG(c->h_min > 0, "tau <= 0 needs rrhd_set_time_step first");
  RRHD_CUDA(cudaSetDevice(c->device));
  if (c->keep_face_flux && !c->d_face_flux) RRHD_CUDA(cudaMalloc(&c->d_face_flux, sizeof(double) * 5 * c->F));
  StepParams P;
  P.eos = make_eos(c->eos, c->gamma);
  P.N = (int)c->N;
  P.cpb = c->cpb;
  P.b0 = c->part_b0;
  P.off = c->d_bface_off;
  P.halo_off = c->d_halo_off;
  P.halo_ids = c->d_halo_ids;
  P.max_halo = c->max_halo;
  P.face = c->d_bface_rec;
  P.gid = c->d_bface_gid;
  P.cell = c->d_cell_rec;
  P.sin = c->d_state[c->cur];
  P.sout = c->d_state[c->cur ^ 1];
  P.status = c->d_status;
  P.face_flux = c->keep_face_flux ? c->d_face_flux : nullptr;
  P.prev = c->d_scal + (c->scal_cur ^ 1);
  P.out = c->d_scal + c->scal_cur;
  P.tau = tau;
  P.device_tau = tau <= 0 ? 1 : 0;
  P.cfl_hmin = c->cfl * c->h_min;
  P.bc = c->bc;
  RRHD_CUDA(cudaMemsetAsync(P.out, 0, sizeof(StepScalars), c->stream));
  if (P.face_flux)
    k_hydro_step<true><<<c->part_b1 - c->part_b0, kStepThreads, c->step_smem, c->stream>>>(P);
  else
    k_hydro_step<false><<<c->part_b1 - c->part_b0, kStepThreads, c->step_smem, c->stream>>>(P);
  RRHD_CUDA(cudaGetLastError());
  c->cur ^= 1;
  c->scal_cur ^= 1;
  if (stats) {
    StepScalars s;
    RRHD_CUDA(cudaMemcpyAsync(&s, P.out, sizeof s, cudaMemcpyDeviceToHost, c->stream));
    RRHD_CUDA(cudaStreamSynchronize(c->stream));
    stats->max_speed = s.max_speed;
    stats->n_fallback = (int64_t)s.n_fallback;
    stats->n_failed = (int64_t)s.n_failed;
    if (s.n_failed) return rrhd_fail(RRHD_ERR_C2P, "con2prim failed in %llu cells after the fallback", s.n_failed);
  }
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_get_step_info(rrhd_ctx *c, double *tau_used, double *max_speed) {
  RRHD_CHECK_ARG(c, "null context");
  StepScalars s;
  RRHD_CUDA(cudaMemcpyAsync(&s, c->d_scal + (c->scal_cur ^ 1), sizeof s, cudaMemcpyDeviceToHost, c->stream));
  RRHD_CUDA(cudaStreamSynchronize(c->stream));
  if (tau_used) *tau_used = s.tau;
  if (max_speed) *max_speed = s.max_speed;
  return RRHD_OK;
}

namespace {

__global__ void k_pack_states(const int32_t *__restrict__ ids, int64_t n, const double2 *__restrict__ state,
                              double2 *__restrict__ buf) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= 5 * n) return;
  const int64_t k = i / 5;
  buf[i] = state[5 * (int64_t)ids[k] + (i - 5 * k)];
}

__global__ void k_unpack_states(const int32_t *__restrict__ ids, int64_t n, const double2 *__restrict__ buf,
                                double2 *__restrict__ state) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= 5 * n) return;
  const int64_t k = i / 5;
  state[5 * (int64_t)ids[k] + (i - 5 * k)] = buf[i];
}

}  // namespace

extern "C" rrhd_status rrhd_hydro_set_part(rrhd_ctx *c, int32_t world, int32_t rank) {
  RRHD_CHECK_ARG(c, "null context");
  RRHD_CUDA(cudaSetDevice(c->device));
  rrhd_mesh_desc m{};
  m.n_cells = c->N;
  m.n_faces = c->F;
  m.face_id_l = c->h_face_l.data();
  m.face_id_r = c->h_face_r.data();
  int64_t range[2];
  std::vector<int64_t> sc(std::max(world, 1)), rc(std::max(world, 1));
  rrhd_status st = rrhd_part_plan(&m, c->h_perm.data(), c->cpb, world, rank, range, sc.data(), rc.data(),
                                  nullptr, nullptr);
  if (st) return st;
  const int64_t ns = std::accumulate(sc.begin(), sc.end(), int64_t(0));
  const int64_t nr = std::accumulate(rc.begin(), rc.end(), int64_t(0));
  std::vector<int32_t> sid(std::max<int64_t>(ns, 1)), rid(std::max<int64_t>(nr, 1));
  if ((st = rrhd_part_plan(&m, c->h_perm.data(), c->cpb, world, rank, range, sc.data(), rc.data(), sid.data(),
                           rid.data())))
    return st;
  RRHD_CUDA(cudaStreamSynchronize(c->stream));
  // upload the new id lists first: on failure the context keeps its previous split
  int32_t *d_sid = nullptr, *d_rid = nullptr;
  if ((st = upload(&d_sid, sid)) || (st = upload(&d_rid, rid))) {
    if (d_sid) cudaFree(d_sid);
    if (d_rid) cudaFree(d_rid);
    return st;
  }
  if (c->d_send_ids) cudaFree(c->d_send_ids);
  if (c->d_recv_ids) cudaFree(c->d_recv_ids);
  c->d_send_ids = d_sid;
  c->d_recv_ids = d_rid;
  c->part_world = world;
  c->part_rank = rank;
  c->part_b0 = (int)(c->nblocks * (int64_t)rank / world);
  c->part_b1 = (int)(c->nblocks * (int64_t)(rank + 1) / world);
  c->part_c0 = range[0];
  c->part_c1 = range[1];
  c->n_send = ns;
  c->n_recv = nr;
  c->send_counts = sc;
  c->recv_counts = rc;
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_hydro_part_info(rrhd_ctx *c, int64_t *cell_range, int64_t *send_counts,
                                            int64_t *recv_counts, int32_t *cells) {
  RRHD_CHECK_ARG(c, "null context");
  if (cell_range) cell_range[0] = c->part_c0, cell_range[1] = c->part_c1;
  for (int q = 0; q < c->part_world; q++) {
    if (send_counts) send_counts[q] = c->part_world > 1 ? c->send_counts[q] : 0;
    if (recv_counts) recv_counts[q] = c->part_world > 1 ? c->recv_counts[q] : 0;
  }
  if (cells)
    for (int64_t k = c->part_c0; k < c->part_c1; k++) cells[k - c->part_c0] = c->h_perm[k];
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_hydro_pack_halo(rrhd_ctx *c, double *send_buf) {
  RRHD_CHECK_ARG(c, "null context");
  if (c->n_send == 0) return RRHD_OK;
  RRHD_CHECK_ARG(send_buf, "null send buffer");
  RRHD_CUDA(cudaSetDevice(c->device));
  k_pack_states<<<grid1d(5 * c->n_send, 256), 256, 0, c->stream>>>(
      c->d_send_ids, c->n_send, reinterpret_cast<const double2 *>(c->d_state[c->cur]),
      reinterpret_cast<double2 *>(send_buf));
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_hydro_unpack_halo(rrhd_ctx *c, const double *recv_buf) {
  RRHD_CHECK_ARG(c, "null context");
  if (c->n_recv == 0) return RRHD_OK;
  RRHD_CHECK_ARG(recv_buf, "null receive buffer");
  RRHD_CUDA(cudaSetDevice(c->device));
  k_unpack_states<<<grid1d(5 * c->n_recv, 256), 256, 0, c->stream>>>(
      c->d_recv_ids, c->n_recv, reinterpret_cast<const double2 *>(recv_buf),
      reinterpret_cast<double2 *>(c->d_state[c->cur]));
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_hydro_max_speed_ptr(rrhd_ctx *c, double **max_speed) {
  RRHD_CHECK_ARG(c && max_speed, "null argument");
  *max_speed = &c->d_scal[c->scal_cur ^ 1].max_speed;
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_hydro_step_host(rrhd_ctx *c, double tau, double *W, double *U, int64_t stride,
                                           rrhd_step_stats *stats) {
  RRHD_CHECK_ARG(c, "null context");
  RRHD_CHECK_ARG(c->part_world == 1, "host-buffer step of a split context: use rrhd_hydro_step");
  rrhd_status st = rrhd_set_state(c, W, U, stride, RRHD_HOST);
  if (st) return st;
  rrhd_status step = rrhd_hydro_step(c, tau, stats);
  if (step && step != RRHD_ERR_C2P) return step;
  st = rrhd_get_state(c, W, U, stride, RRHD_HOST);
  return st ? st : step;
}

extern "C" rrhd_status rrhd_keep_face_flux(rrhd_ctx *c, int32_t on) {
  RRHD_CHECK_ARG(c, "null context");
  c->keep_face_flux = on != 0;
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_get_face_flux(rrhd_ctx *c, double *F) {
  RRHD_CHECK_ARG(c && F, "null argument");
  RRHD_CHECK_ARG(c->keep_face_flux && c->d_face_flux, "call rrhd_keep_face_flux(ctx, 1) before the step");
  RRHD_CUDA(cudaMemcpyAsync(F, c->d_face_flux, sizeof(double) * 5 * c->F, cudaMemcpyDeviceToHost, c->stream));
  RRHD_CUDA(cudaStreamSynchronize(c->stream));
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_get_cell_status(rrhd_ctx *c, uint8_t *status) {
  RRHD_CHECK_ARG(c && status, "null argument");
  uint8_t *d = reinterpret_cast<uint8_t *>(c->d_scratch_io);
  k_get_status<<<grid1d(c->N, 256), 256, 0, c->stream>>>(c->N, c->d_iperm, c->d_status, d);
  RRHD_CUDA(cudaGetLastError());
  RRHD_CUDA(cudaMemcpyAsync(status, d, c->N, cudaMemcpyDeviceToHost, c->stream));
  RRHD_CUDA(cudaStreamSynchronize(c->stream));
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_con2prim_batch(int32_t eos, double gamma, double *U, double *W, uint8_t *status,
                                           int64_t n, int32_t fallback, void *stream) {
  RRHD_CHECK_ARG(n >= 0 && ((U && W) || n == 0), "bad arguments");
  RRHD_CHECK_ARG(eos == RRHD_EOS_IDEAL || eos == RRHD_EOS_TAUB, "bad eos");
  if (n == 0) return RRHD_OK;
  k_c2p_batch<<<grid1d(n, 128), 128, 0, (cudaStream_t)stream>>>(make_eos(eos, gamma), U, W, status, n, fallback);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_prim2con_batch(int32_t eos, double gamma, double *W, double *U, int64_t n,
                                           void *stream) {
  RRHD_CHECK_ARG(n >= 0 && ((U && W) || n == 0), "bad arguments");
  RRHD_CHECK_ARG(eos == RRHD_EOS_IDEAL || eos == RRHD_EOS_TAUB, "bad eos");
  if (n == 0) return RRHD_OK;
  k_p2c_batch<<<grid1d(n, 256), 256, 0, (cudaStream_t)stream>>>(make_eos(eos, gamma), W, U, n);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

// Scratch of rrhd_con2prim_batch_stats: one buffer per (device, stream),
// allocated on first use and grown when a larger batch needs more partial
// records.  Calls on one stream run one after another on the GPU, so they can
// share a buffer; calls on different streams get different buffers and may
// overlap.  The registry lock is held from the lookup until the kernels and the
// read-back of the totals are enqueued, so a call that grows a stream's buffer
// (after synchronising that stream) can never free memory that another thread
// has looked up but not yet used.
namespace {
struct ScratchKey {
  int dev;
  cudaStream_t stream;
  bool operator<(const ScratchKey &o) const { return dev != o.dev ? dev < o.dev : stream < o.stream; }
};
struct ScratchBuf {
  C2pPartial *ptr = nullptr;
  int64_t cap = 0;
};
std::mutex g_c2p_scratch_mu;
std::map<ScratchKey, ScratchBuf> g_c2p_scratch;

// Enqueues the batch and the reduction (and, with stats, the read-back of the
// totals into *total) on `stream`; the caller synchronises before reading it.
rrhd_status c2p_stats_enqueue(Eos eos, double *U, double *W, uint8_t *status, int64_t n, int32_t fallback,
                              C2pPartial *scratch, C2pPartial *total, cudaStream_t stream) {
  const int64_t nb = (n + kC2pPerBlock - 1) / kC2pPerBlock;
  if (nb > 0) {
    k_c2p_stats<<<(unsigned)nb, kC2pThreads, 0, stream>>>(eos, U, W, status, n, fallback, scratch);
    RRHD_CUDA(cudaGetLastError());
  }
  k_c2p_stats_reduce<<<1, 256, 0, stream>>>(scratch, (int)nb);
  RRHD_CUDA(cudaGetLastError());
  if (total) RRHD_CUDA(cudaMemcpyAsync(total, scratch + nb, sizeof *total, cudaMemcpyDeviceToHost, stream));
  return RRHD_OK;
}

rrhd_status c2p_stats_finish(const C2pPartial *total, rrhd_c2p_stats *stats, cudaStream_t stream) {
  if (!stats) return RRHD_OK;
  RRHD_CUDA(cudaStreamSynchronize(stream));
  stats->n_ok = (int64_t)total->ok;
  stats->n_fallback = (int64_t)total->fallback;
  stats->n_failed = (int64_t)total->failed;
  stats->newton_iters = (int64_t)total->iters;
  stats->max_iters = (int32_t)total->max_iters;
  return RRHD_OK;
}
}  // namespace

extern "C" rrhd_status rrhd_con2prim_batch_stats(int32_t eos, double gamma, double *U, double *W,
                                                 uint8_t *status, int64_t n, int32_t fallback,
                                                 rrhd_c2p_stats *stats, void *stream) {
  RRHD_CHECK_ARG(n >= 0 && ((U && W) || n == 0), "bad arguments");
  RRHD_CHECK_ARG(eos == RRHD_EOS_IDEAL || eos == RRHD_EOS_TAUB, "bad eos");
  int dev = 0;
  RRHD_CUDA(cudaGetDevice(&dev));
  const cudaStream_t s = (cudaStream_t)stream;
  const int64_t need = (n + kC2pPerBlock - 1) / kC2pPerBlock + 1;
  C2pPartial total{};
  {
    std::lock_guard<std::mutex> lk(g_c2p_scratch_mu);
    ScratchBuf &buf = g_c2p_scratch[ScratchKey{dev, s}];
    if (buf.cap < need) {
      if (buf.ptr) {
        // every earlier user of this buffer enqueued its work on `stream`
        RRHD_CUDA(cudaStreamSynchronize(s));
        cudaFree(buf.ptr);
        buf.ptr = nullptr;
        buf.cap = 0;
      }
      const int64_t cap = std::max<int64_t>(need, 1024);
      RRHD_CUDA(cudaMalloc(&buf.ptr, sizeof(C2pPartial) * cap));
      buf.cap = cap;
    }
    const rrhd_status st =
        c2p_stats_enqueue(make_eos(eos, gamma), U, W, status, n, fallback, buf.ptr, stats ? &total : nullptr, s);
    if (st) return st;
  }
  return c2p_stats_finish(&total, stats, s);
}

// ---------------------------------------------------------------------------
// Allocation-free variant of rrhd_con2prim_batch_stats.
//
// For callers that must not allocate device memory themselves: hosts whose
// memory pool or arena reserves the whole GPU (a cudaMalloc would fail or
// bypass their accounting), and latency-critical loops that cannot accept
// cudaMalloc's implicit device synchronisation.  The per-CTA partial records
// live in the file-scope array below, which every GPU that loads this library
// holds until the process exits.
//
// Host code cannot use the array's name as a device address (it is a host-side
// stand-in), so the first call on each device looks the address up with
// cudaGetSymbolAddress while that device is current and caches it together with
// the device's current context (a reset device gets a new context, and the
// address is looked up again); make that first call before any stream capture.
// All calls share the array and it keeps
// the last call's contents: every call rewrites all the records it reads (one
// per CTA, then the total), so nothing has to be cleared, but calls that
// overlap on the GPU (concurrent streams) race on it and must be serialised.
constexpr int kNoallocMaxBlocks = 8192;
constexpr int64_t kNoallocMaxStates = (int64_t)kNoallocMaxBlocks * kC2pPerBlock;  // 16,777,216
static __device__ __align__(256) C2pPartial g_c2p_noalloc_scratch[kNoallocMaxBlocks + 1];  // 320 KiB

namespace {
std::mutex g_noalloc_mu;
// device address of the array per device ordinal, with the primary context it
// was looked up in: a reset device (cudaDeviceReset) gets a new context and the
// module is loaded again, so the address is looked up again.
C2pPartial *g_noalloc_addr[64] = {nullptr};
CUcontext g_noalloc_ctx[64] = {nullptr};
}  // namespace

extern "C" rrhd_status rrhd_con2prim_batch_stats_noalloc(int32_t eos, double gamma, double *U, double *W,
                                                         uint8_t *status, int64_t n, int32_t fallback,
                                                         rrhd_c2p_stats *stats, void *stream) {
  RRHD_CHECK_ARG(n >= 0 && ((U && W) || n == 0), "bad arguments");
  RRHD_CHECK_ARG(eos == RRHD_EOS_IDEAL || eos == RRHD_EOS_TAUB, "bad eos");
  if (n > kNoallocMaxStates)
    return rrhd_fail(RRHD_ERR_LIMIT, "rrhd_con2prim_batch_stats_noalloc: %lld states exceed the fixed maximum of %lld",
                     (long long)n, (long long)kNoallocMaxStates);
  int dev = 0;
  RRHD_CUDA(cudaGetDevice(&dev));
  RRHD_CHECK_ARG(dev >= 0 && dev < 64, "device ordinal out of range");
  RRHD_CUDA(cudaSetDevice(dev));  // initialises the device's primary context and makes it current
  // the driver's cuCtxGetCurrent through the runtime, so that the library has no
  // link-time dependency on the driver library
  static CUresult (*ctx_get_current)(CUcontext *) = nullptr;
  if (!ctx_get_current) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      ctx_get_current = reinterpret_cast<CUresult (*)(CUcontext *)>(p);
  }
  CUcontext ctx = nullptr;
  if (!ctx_get_current || ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx)
    return rrhd_fail(RRHD_ERR_CUDA, "rrhd_con2prim_batch_stats_noalloc: no current CUDA context");
  const cudaStream_t s = (cudaStream_t)stream;
  C2pPartial total{};
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev] || g_noalloc_ctx[dev] != ctx) {
      void *addr = nullptr;
      RRHD_CUDA(cudaGetSymbolAddress(&addr, g_c2p_noalloc_scratch));
      g_noalloc_addr[dev] = reinterpret_cast<C2pPartial *>(addr);
      g_noalloc_ctx[dev] = ctx;
    }
    const rrhd_status st = c2p_stats_enqueue(make_eos(eos, gamma), U, W, status, n, fallback, g_noalloc_addr[dev],
                                             stats ? &total : nullptr, s);
    if (st) return st;
  }
  return c2p_stats_finish(&total, stats, s);
}
