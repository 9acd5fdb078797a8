// Transport sweep (short characteristics) and the coupled radiation-hydro step.
//
// The reference sweeps every direction on the CPU in the order of a precomputed
// graph (sorted_graph: (cell, out-face) pairs) with precomputed node distances
// (vec_x0), solvers/illum/src/mpi/multi_gpu/illum_multi_gpu_face_calc.cpp:91-190.
// Here the order is built on the device once per mesh and direction set as
// levels: level 0 holds the (cell, direction) pairs whose in-faces are all on
// the boundary, level L+1 those whose last upwind neighbour is in level L.  All
// pairs of a level are independent, so one level is one kernel launch with one
// thread per pair, and a sweep is one CUDA graph of all level launches.  A batch
// of DB directions is swept together, so the face values of one batch,
// [DB][F][G] (direction-major), are the only scratch.
//
// Per pair the kernel classifies the four faces by the sign of n_j . w, traces
// the three nodes of each out-face back to the in-face they came through (the
// smallest t_h = lam_h H_h / -cos_h, H_h the height of the cell over face h and
// lam_h the node's barycentric weight of the vertex opposite h: no vertex data
// is needed), evaluates GetIllum per group with one set of exponentials shared by
// all groups (the opacity k = alpha + betta does not depend on the group), and
// folds the four face values into the cell value (ReCalcIllumOpt) in the same
// thread, so face values are read once.  Compiled with --fmad=false: in double
// precision every value is the oracle's operation for operation, exp aside.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <cub/device/device_radix_sort.cuh>
#include <type_traits>
#include <vector>

#include "coupled.h"
#include "ctx.h"
#include "dirs.h"
#include "hydro_phys.cuh"
#include "rad_phys.cuh"
#include "rrhd_internal.h"

using namespace rrhd;

namespace {

constexpr int kSweepThreads = 128;

// Per-cell record (RW words): 0-11 outward normals n_j, 12-15 heights H_j, then the
// face-value slots as int32 (4: 2 doubles or 4 floats; bit 31 set where the face has no
// neighbour), then the source record {k, betta/k, alpha Q_g/k} of the step, and in the
// last 16 bytes the neighbours (int32, -1 on the boundary), which only the plan reads.
// RW makes a record a whole number of 128-byte lines (G = 4: 256 B in double, 128 B in
// float); what one level item reads of its cell is 6 sectors (double) or 4 (float).
template <class T>
struct Rec {
  static constexpr int IDS = 16;                       // word offset of the face-value slots
  static constexpr int DYN = sizeof(T) == 8 ? 18 : 20;  // word offset of the source record
  static constexpr int NBRW = 16 / (int)sizeof(T);      // words of the neighbours, at the record's end
  static constexpr int LINE = 128 / (int)sizeof(T);     // words per 128-byte line
};
constexpr int32_t kNoNeighbour = INT32_MIN;  // bit 31 of a face-value slot id

// normals, heights and face-value slot ids (negative: a face without a neighbour)
template <class T>
__device__ __forceinline__ void load_rec(const T *r, T *g, int *fid) {
#pragma unroll
  for (int q = 0; q < 16; q += 16 / (int)sizeof(T)) {
    if constexpr (sizeof(T) == 8) {
      const double2 v = __ldg(reinterpret_cast<const double2 *>(r) + q / 2);
      g[q] = v.x;
      g[q + 1] = v.y;
    } else {
      const float4 v = __ldg(reinterpret_cast<const float4 *>(r) + q / 4);
      g[q] = v.x;
      g[q + 1] = v.y;
      g[q + 2] = v.z;
      g[q + 3] = v.w;
    }
  }
  const int4 f = __ldg(reinterpret_cast<const int4 *>(r + Rec<T>::IDS));
  fid[0] = f.x, fid[1] = f.y, fid[2] = f.z, fid[3] = f.w;
}
// normals and neighbours only (the plan kernels); RW: record words
template <class T>
__device__ __forceinline__ void load_normals(const T *r, int RW, T *g, int *nbr) {
#pragma unroll
  for (int q = 0; q < 12; q++) g[q] = __ldg(r + q);
  const int4 n = __ldg(reinterpret_cast<const int4 *>(r + RW - Rec<T>::NBRW));
  nbr[0] = n.x, nbr[1] = n.y, nbr[2] = n.z, nbr[3] = n.w;
}
__device__ __forceinline__ int64_t slot_of(int fid) { return (int64_t)(fid & 0x7fffffff); }

// T: geometry and source records (directions, per-cell records, face areas); TV: face
// values and the transport arithmetic.
template <class T, class TV>
struct SweepArgs {
  const SweepIO *io;
  const uint32_t *items;
  int64_t n;  // items of this level
  int shift, DB, d0, M, G, RW, GS, nbd;  // item = direction << shift | cell
  int64_t NF;                            // face-value slots
  const T *w;     // [M][3]
  const T *rec;   // [N][RW]
  const T *area;  // [N][4] face areas (cell values)
  TV *fv;         // [DB][NF][GS] face values, direction-major (GS >= G, full 32-byte sectors)
  const uint4 *geo;  // per item of the level (items[i] <-> geo[i]): its geometry, or null
  TV bc;
  int64_t last;
};

__device__ __forceinline__ double ex(double x) { return exp(x); }
__device__ __forceinline__ float ex(float x) { return __expf(x); }
__device__ __forceinline__ double dv(double a, double b) { return a / b; }
__device__ __forceinline__ float dv(float a, float b) { return __fdividef(a, b); }

template <class T>
__device__ __forceinline__ void face_cos(const T *g, T wx, T wy, T wz, T *cosf) {
#pragma unroll
  for (int j = 0; j < 4; j++) cosf[j] = (g[3 * j] * wx + g[3 * j + 1] * wy) + g[3 * j + 2] * wz;
}

// Geometry of one (cell, direction) item from the cell's normals and heights g[16]:
// r[f] = H_f / -cos_f for the in-faces (cos_f < 0), 0 for the others, and the code word
//   bits 0-3   in-faces (cos_f < 0)
//   bits 4-7   out-faces (cos_f > 0)
//   bits 8-23  per vertex v (4 bits at 8 + 4v) the in-face its node is traced to: face
//              index, bit 2 lam = 2/3 (the face opposite v), bit 3 no in-face.
// Node selection: the restatement takes, for each node, the in-face with the smallest
// (t, face index); t = t4 = 2r/3 for the face opposite the node's own vertex, t1 = r/6 for
// the others.  So only the two smallest in-faces by (t1, index) are needed: the node's
// candidate among the other faces is the best unless that is its own opposite face.  The
// choice depends on the node's vertex only, not on the out-face the node belongs to.
template <class T>
__device__ __forceinline__ uint32_t item_geometry(const T *g, T wx, T wy, T wz, T (&r)[4]) {
  T cosf[4], t1[4], t4[4];
  face_cos(g, wx, wy, wz, cosf);
  uint32_t code = 0;
#pragma unroll
  for (int f = 0; f < 4; f++) {
    r[f] = t1[f] = t4[f] = (T)0;
    if (cosf[f] < 0) {
      r[f] = dv(g[12 + f], -cosf[f]);
      t1[f] = (T)(1.0 / 6.0) * r[f];
      t4[f] = (T)(2.0 / 3.0) * r[f];
      code |= 1u << f;
    } else if (cosf[f] > 0) {
      code |= 16u << f;
    }
  }
  int b1 = -1, b2 = -1;
  T tb1 = 0, tb2 = 0;
#pragma unroll
  for (int f = 0; f < 4; f++) {
    if (!(cosf[f] < 0)) continue;
    if (b1 < 0 || t1[f] < tb1) {
      b2 = b1;
      tb2 = tb1;
      b1 = f;
      tb1 = t1[f];
    } else if (b2 < 0 || t1[f] < tb2) {
      b2 = f;
      tb2 = t1[f];
    }
  }
#pragma unroll
  for (int v = 0; v < 4; v++) {
    const int B = b1 != v ? b1 : b2;
    const T tB = b1 != v ? tb1 : tb2;
    uint32_t cv;
    if (cosf[v] < 0 && (B < 0 || t4[v] < tB || (t4[v] == tB && v < B)))
      cv = (uint32_t)v | 4u;
    else
      cv = B < 0 ? 8u : (uint32_t)B;
    code |= cv << (8 + 4 * v);
  }
  return code;
}


// G values at p (contiguous), vectorised for 2 and 4 groups
template <class T, int G>
__device__ __forceinline__ void ld_groups(const T *p, T (&v)[G]) {
  if constexpr (sizeof(T) == 8 && G % 2 == 0) {
#pragma unroll
    for (int q = 0; q < G / 2; q++) {
      const double2 x = reinterpret_cast<const double2 *>(p)[q];
      v[2 * q] = x.x;
      v[2 * q + 1] = x.y;
    }
  } else if constexpr (sizeof(T) == 4 && G == 4) {
    const float4 x = *reinterpret_cast<const float4 *>(p);
    v[0] = x.x, v[1] = x.y, v[2] = x.z, v[3] = x.w;
  } else {
#pragma unroll
    for (int q = 0; q < G; q++) v[q] = p[q];
  }
}
// G values to a face-value slot of GS values; float slots of 4 groups are padded to 8 so
// that every store fills a whole 32-byte sector
template <class T, int G>
__device__ __forceinline__ void st_slot(T *p, const T (&v)[G]) {
  if constexpr (sizeof(T) == 8 && G % 2 == 0) {
#pragma unroll
    for (int q = 0; q < G / 2; q++) reinterpret_cast<double2 *>(p)[q] = make_double2(v[2 * q], v[2 * q + 1]);
  } else if constexpr (sizeof(T) == 4 && G == 4) {
    reinterpret_cast<float4 *>(p)[0] = make_float4(v[0], v[1], v[2], v[3]);
    reinterpret_cast<float4 *>(p)[1] = make_float4(0.f, 0.f, 0.f, 0.f);
  } else {
#pragma unroll
    for (int q = 0; q < G; q++) p[q] = v[q];
  }
}

// One thread per (cell, direction) pair of a level: the out-face values of all
// groups.  GT: compile-time group count (1, 2 or 4), 0 for any other (loop).
//
// Node distances: node q of out-face j is traced to the in-face f with the
// smallest t = lam r_f (r_f = H_f / -cos_f, lam = 2/3 when f is opposite the
// node's own vertex, 1/6 otherwise), compared exactly as in the restatement.
// The attenuations need only one exponential per in-face: E1_f = exp(-k r_f / 6)
// and exp(-k 2 r_f / 3) = E1_f^4 (equal to a few ulp).
template <class T, class TV, class TI, int GT, bool PRE>
__global__ void __launch_bounds__(kSweepThreads) k_sweep_level(SweepArgs<T, TV> a) {
  // Levels after the first of a batch are launched with programmatic stream
  // serialisation: the next level may start while this one drains, and everything up to
  // the first face-value read (item, cell record, source record, S, geometry,
  // exponentials) overlaps the previous level; griddepcontrol.wait then waits for the
  // previous level to complete and its writes to be visible.
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const uint32_t it = a.items[i];
  uint4 gq = make_uint4(0u, 0u, 0u, 0u);
  if constexpr (PRE) gq = __ldcs(a.geo + i);  // read once per sweep, in item order
  const int64_t c = it & ((1u << a.shift) - 1u);
  const int dl = (int)(it >> a.shift);
  const int d = a.d0 + dl;
  int fid[4];
  T r[4];
  uint32_t code;
  const T *rc = a.rec + (int64_t)a.RW * c;
  if constexpr (PRE) {
    // the item's geometry from the stream (item_geometry at setup, the in-face distances
    // in face order, k_plan_geometry's format); of the cell record only the face-value
    // slots and the source record are read
    const int4 f = __ldg(reinterpret_cast<const int4 *>(rc + Rec<T>::IDS));
    fid[0] = f.x, fid[1] = f.y, fid[2] = f.z, fid[3] = f.w;
    code = gq.x;
    int m = 0;
    if constexpr (sizeof(T) == 4) {
#pragma unroll
      for (int f = 0; f < 4; f++) {
        r[f] = (T)0;
        if ((code >> f) & 1u) {
          r[f] = __uint_as_float(m == 0 ? gq.y : m == 1 ? gq.z : gq.w);
          m++;
        }
      }
    } else {
      // 2^(e-32), exact: e in [-127, 127]
      const double down = __hiloint2double((int)((code >> 24) - 128u - 32u + 1023u) << 20, 0);
#pragma unroll
      for (int f = 0; f < 4; f++) {
        r[f] = (T)0;
        if ((code >> f) & 1u) {
          r[f] = (T)((double)(m == 0 ? gq.y : m == 1 ? gq.z : gq.w) * down);
          m++;
        }
      }
    }
  } else {
    T g[16];
    load_rec<T>(rc, g, fid);
    code = item_geometry<T>(g, a.w[3 * d], a.w[3 * d + 1], a.w[3 * d + 2], r);
  }
  const T *dy = rc + Rec<T>::DYN;
  const T k = dy[0], bk = dy[1];
  const SweepIO io = *a.io;
  const TI *Sv = (const TI *)io.S;
  // S element (group gg) of this cell and direction: base + gg * gs
  int64_t base, gs;
  if (io.layout) {
    base = (c * a.M + d) * a.G;
    gs = 1;
  } else {
    base = (int64_t)io.row_of[c] * a.G * a.M + d;
    gs = a.M;
  }
  TV E1[4], E4[4];
#pragma unroll
  for (int f = 0; f < 4; f++) {
    E1[f] = E4[f] = (TV)1;
    if ((code >> f) & 1u) {
      const T t1 = (T)(1.0 / 6.0) * r[f];
      E1[f] = ex((TV)(-k * t1));
      const TV e2 = E1[f] * E1[f];
      E4[f] = e2 * e2;
    }
  }
  // 4 bits per (out-face, node) from the node's vertex code; out-faces compacted into
  // slots (2 bits each in jo)
  uint64_t sel = 0;
  uint32_t jo = 0;
  int nout = 0;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    if (!((code >> (4 + j)) & 1u)) continue;
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const int vq = (j + 1 + q) & 3;
      sel |= (uint64_t)((code >> (8 + 4 * vq)) & 15u) << (12 * nout + 4 * q);
    }
    jo |= (uint32_t)j << (2 * nout);
    nout++;
  }
  if constexpr (GT > 0) {
    // separate per-face arrays (not one [4][GT] array), selected by comparisons, so that
    // no selection turns into an indexed local-memory access
    TV rhs[GT], f0[GT], f1[GT], f2[GT], f3[GT];
    TI sv[GT];
    if (io.layout) {
      ld_groups<TI, GT>(Sv + base, sv);
    } else {
#pragma unroll
      for (int q = 0; q < GT; q++) sv[q] = Sv[base + q * gs];
    }
#pragma unroll
    for (int q = 0; q < GT; q++) rhs[q] = (TV)dy[2 + q] + (TV)bk * (TV)sv[q];
    asm volatile("griddepcontrol.wait;" ::: "memory");
    auto in_face = [&](int j, TV (&fj)[GT]) {
      if (((code >> j) & 1u) && fid[j] >= 0) {
        ld_groups<TV, GT>(a.fv + ((int64_t)dl * a.NF + fid[j]) * a.GS, fj);
      } else {
#pragma unroll
        for (int q = 0; q < GT; q++) fj[q] = a.bc;
      }
    };
    in_face(0, f0);
    in_face(1, f1);
    in_face(2, f2);
    in_face(3, f3);
    const TV E1_0 = E1[0], E1_1 = E1[1], E1_2 = E1[2], E1_3 = E1[3];
    const TV E4_0 = E4[0], E4_1 = E4[1], E4_2 = E4[2], E4_3 = E4[3];
    const int64_t fid0 = slot_of(fid[0]), fid1 = slot_of(fid[1]), fid2 = slot_of(fid[2]), fid3 = slot_of(fid[3]);
    // the (at most three) out-faces, one slot after another
    for (int o = 0; o < nout; o++) {
      const int j = (jo >> (2 * o)) & 3;
      TV e[3];
      int h[3];
#pragma unroll
      for (int n = 0; n < 3; n++) {
        const uint32_t code = (uint32_t)(sel >> (12 * o + 4 * n)) & 15u;
        h[n] = code & 8u ? -1 : (int)(code & 3u);
        const bool four = code & 4u;
        e[n] = h[n] == 0 ? (four ? E4_0 : E1_0)
             : h[n] == 1 ? (four ? E4_1 : E1_1)
             : h[n] == 2 ? (four ? E4_2 : E1_2)
             : h[n] == 3 ? (four ? E4_3 : E1_3) : (TV)1;
      }
      TV out[GT];
#pragma unroll
      for (int q = 0; q < GT; q++) {
        TV I0[3];
#pragma unroll
        for (int n = 0; n < 3; n++)
          I0[n] = h[n] == 0 ? f0[q] : h[n] == 1 ? f1[q] : h[n] == 2 ? f2[q] : h[n] == 3 ? f3[q] : a.bc;
        TV Icur = e[0] * (I0[0] - rhs[q]) + rhs[q];
        Icur += (e[1] * (I0[1] - rhs[q]) + rhs[q]);
        Icur += (e[2] * (I0[2] - rhs[q]) + rhs[q]);
        out[q] = Icur * (TV)0.3333333333333333;
      }
      const int64_t fj = j == 0 ? fid0 : j == 1 ? fid1 : j == 2 ? fid2 : fid3;
      st_slot<TV, GT>(a.fv + ((int64_t)dl * a.NF + fj) * a.GS, out);
    }
  } else {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    for (int gg = 0; gg < a.G; gg++) {
      const TV rhs = (TV)dy[2 + gg] + (TV)bk * (TV)Sv[base + gg * gs];
      TV fvals[4];
#pragma unroll
      for (int j = 0; j < 4; j++)
        fvals[j] = (((code >> j) & 1u) && fid[j] >= 0) ? a.fv[((int64_t)dl * a.NF + fid[j]) * a.GS + gg] : a.bc;
      for (int o = 0; o < nout; o++) {
        const int j = (jo >> (2 * o)) & 3;
        TV I0[3], e[3];
#pragma unroll
        for (int n = 0; n < 3; n++) {
          const uint32_t code = (uint32_t)(sel >> (12 * o + 4 * n)) & 15u;
          const int h = code & 8u ? -1 : (int)(code & 3u);
          I0[n] = a.bc;
          e[n] = (TV)1;
#pragma unroll
          for (int f = 0; f < 4; f++)
            if (h == f) {
              I0[n] = fvals[f];
              e[n] = code & 4u ? E4[f] : E1[f];
            }
        }
        TV Icur = e[0] * (I0[0] - rhs) + rhs;
        Icur += (e[1] * (I0[1] - rhs) + rhs);
        Icur += (e[2] * (I0[2] - rhs) + rhs);
        a.fv[((int64_t)dl * a.NF + slot_of(fid[j])) * a.GS + gg] = Icur * (TV)0.3333333333333333;
      }
    }
  }
}

// Cell values of one direction batch from its face values: ReCalcIllumOpt
// (illum_utils.cpp:377-433), the area-weighted face mean, a plain mean for the caller's
// last cell.  Faces nobody wrote for a direction (inflow boundary, parallel to it) hold
// the boundary value.  A CTA takes 32 cells (lane = cell) x 32 directions of the batch (four
// per warp): the face values of one direction are stored direction-major, so a warp's reads
// of 32 neighbouring cells' face slots fall close together (a face shared by two of them is
// read from L1 the second time), and each cell's record is read once per CTA.  The cell
// values go through a shared-memory tile [direction][cell + 1 pad] and each warp writes four
// cells' rows, lane = direction, so the stores of a cell's 32 directions are contiguous.
constexpr int kRcCells = 32, kRcDirs = 32;
template <class T, class TV, class TI, int GT>
__global__ void __launch_bounds__(256) k_recalc(SweepArgs<T, TV> a, int64_t N) {
  constexpr int GQ = GT > 0 ? GT : 1;
  __shared__ __align__(16) TI tile[kRcDirs][kRcCells + 1][GQ];
  // the tile's cells: outward normals, face areas and face-value slots, read once per CTA
  __shared__ T s_n[kRcCells][12];
  __shared__ T s_area[kRcCells][4];
  __shared__ int s_fid[kRcCells][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t c = (int64_t)blockIdx.x * kRcCells + lane;
  const int dl0 = (int)blockIdx.y * kRcDirs;
  const bool cell_ok = c < N;
  if (warp == 0 && cell_ok) {
    T g[16];
    int f[4];
    load_rec<T>(a.rec + (int64_t)a.RW * c, g, f);
#pragma unroll
    for (int q = 0; q < 12; q++) s_n[lane][q] = g[q];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      s_area[lane][j] = __ldg(a.area + 4 * c + j);
      s_fid[lane][j] = f[j];
    }
  }
  __syncthreads();
  const SweepIO io = *a.io;
  TI *I = (TI *)io.I;
  const bool last = c == a.last;
  auto cell_value = [&](const TV *fv) {
    TV curI = 0;
    if (!last) {
      TV Ssum = 0;
#pragma unroll
      for (int j = 0; j < 4; j++) {
        curI += fv[j] * (TV)s_area[lane][j];
        Ssum += (TV)s_area[lane][j];
      }
      curI /= Ssum;
    } else {
#pragma unroll
      for (int j = 0; j < 4; j++) curI += fv[j];
      curI /= (TV)4;
    }
    return curI;
  };
#pragma unroll 1
  for (int k = 0; k < kRcDirs / 8; k++) {
    const int dd = warp * (kRcDirs / 8) + k;  // direction within the tile
    const int dl = dl0 + dd;
    if (!cell_ok || dl >= a.nbd) continue;
    const int d = a.d0 + dl;
    T cosf[4];
    face_cos(s_n[lane], a.w[3 * d], a.w[3 * d + 1], a.w[3 * d + 2], cosf);
    int fid[4];
    bool have[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      fid[j] = s_fid[lane][j];
      have[j] = cosf[j] > 0 || (cosf[j] < 0 && fid[j] >= 0);
    }
    const TV *fvd = a.fv + (int64_t)dl * a.NF * a.GS;
    if constexpr (GT > 0) {
      // all four face slots in flight at once, vector loads
      TV f0[GT], f1[GT], f2[GT], f3[GT];
      auto slot = [&](int j, TV (&fj)[GT]) {
        if (have[j]) {
          ld_groups<TV, GT>(fvd + slot_of(fid[j]) * a.GS, fj);
        } else {
#pragma unroll
          for (int q = 0; q < GT; q++) fj[q] = a.bc;
        }
      };
      slot(0, f0);
      slot(1, f1);
      slot(2, f2);
      slot(3, f3);
#pragma unroll
      for (int q = 0; q < GT; q++) {
        const TV fv[4] = {f0[q], f1[q], f2[q], f3[q]};
        tile[dd][lane][q] = (TI)cell_value(fv);  // the cell values as stored (float in the mixed form)
      }
    } else {
      int64_t base, gs;
      if (io.layout) {
        base = (c * a.M + d) * a.G;
        gs = 1;
      } else {
        base = (int64_t)io.row_of[c] * a.G * a.M + d;
        gs = a.M;
      }
      for (int gg = 0; gg < a.G; gg++) {
        TV fv[4];
#pragma unroll
        for (int j = 0; j < 4; j++) fv[j] = have[j] ? fvd[slot_of(fid[j]) * a.GS + gg] : a.bc;
        I[base + gg * gs] = (TI)cell_value(fv);
      }
    }
  }
  if constexpr (GT > 0) {
    __syncthreads();
    const int dl = dl0 + lane;
    if (dl < a.nbd) {
      const int d = a.d0 + dl;
#pragma unroll 1
      for (int k = 0; k < kRcCells / 8; k++) {
        const int cl = warp * (kRcCells / 8) + k;
        const int64_t cc = (int64_t)blockIdx.x * kRcCells + cl;
        if (cc >= N) break;
        const TI *v = tile[lane][cl];
        if (io.layout) {
          TI *o = I + (cc * a.M + d) * a.G;
          if constexpr (sizeof(TI) == 8 && GT % 2 == 0) {
#pragma unroll
            for (int q = 0; q < GT / 2; q++) reinterpret_cast<double2 *>(o)[q] = make_double2(v[2 * q], v[2 * q + 1]);
          } else if constexpr (sizeof(TI) == 4 && GT == 4) {
            *reinterpret_cast<float4 *>(o) = make_float4(v[0], v[1], v[2], v[3]);
          } else {
#pragma unroll
            for (int q = 0; q < GT; q++) o[q] = v[q];
          }
        } else {
          const int64_t base = (int64_t)io.row_of[cc] * a.G * a.M + d;
#pragma unroll
          for (int q = 0; q < GT; q++) I[base + (int64_t)q * a.M] = v[q];
        }
      }
    }
  }
}

// ---------------------------------------------------------------- plan
template <class T>
__global__ void k_plan_init(int64_t N, int nbd, int shift, int d0, const T *w, const T *rec, int RW, uint32_t *indeg,
                            uint32_t *plan, unsigned long long *tail) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= N * nbd) return;
  const int64_t c = i / nbd;
  const int dl = (int)(i - c * nbd);
  const int d = d0 + dl;
  T g[12];
  int nbr[4];
  load_normals<T>(rec + (int64_t)RW * c, RW, g, nbr);
  T cosf[4];
  face_cos(g, w[3 * d], w[3 * d + 1], w[3 * d + 2], cosf);
  uint32_t cnt = 0;
#pragma unroll
  for (int j = 0; j < 4; j++) cnt += (cosf[j] < 0 && nbr[j] >= 0) ? 1u : 0u;
  indeg[i] = cnt;
  if (cnt == 0) plan[atomicAdd(tail, 1ull)] = ((uint32_t)dl << shift) | (uint32_t)c;
}

template <class T>
__global__ void k_plan_expand(const uint32_t *cur, int64_t n, int nbd, int shift, int d0, const T *w, const T *rec,
                              int RW, uint32_t *indeg, uint32_t *plan, unsigned long long *tail) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t it = cur[i];
  const int64_t c = it & ((1u << shift) - 1u);
  const int dl = (int)(it >> shift);
  const int d = d0 + dl;
  T g[12];
  int nbr[4];
  load_normals<T>(rec + (int64_t)RW * c, RW, g, nbr);
  T cosf[4];
  face_cos(g, w[3 * d], w[3 * d + 1], w[3 * d + 2], cosf);
#pragma unroll
  for (int j = 0; j < 4; j++) {
    if (!(cosf[j] > 0) || nbr[j] < 0) continue;
    const int64_t q = (int64_t)nbr[j] * nbd + dl;
    if (atomicSub(indeg + q, 1u) == 1u) plan[atomicAdd(tail, 1ull)] = ((uint32_t)dl << shift) | (uint32_t)nbr[j];
  }
}

// The geometry stream: per plan item (in plan order) item_geometry's code word and the
// distances r_f of the in-faces, in face order (at most three in-faces: the four outward
// normals weighted by the face areas sum to zero).
//   T = float: the distances as float, the values the sweep computes anyway.
//   T = double: block floating point.  Only in-faces that some node of an out-face is traced
//   to matter (the others are never read), and for those t = lam r_f is the distance from
//   the node back to where its characteristic enters the cell, so r_f is at most six cell
//   diameters.  With 2^(e-1) <= max r_f < 2^e over those faces, each is stored as
//   round(r_f 2^(32-e)) in 32 bits and e in bits 24-31 of the code word (biased by 128):
//   the error of every used distance is at most max r_f 2^-33, so an attenuation
//   exp(-k t) moves by at most k (6 diameters) 2^-33 relative.
template <class T>
__global__ void k_plan_geometry(const uint32_t *items, int64_t n, int shift, int DB, int d0, const T *w,
                                const T *rec, int RW, uint4 *geo) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t it = items[i];
  const int64_t c = it & ((1u << shift) - 1u);
  const int d = d0 + (int)(it >> shift);
  T g[16];
  int fid[4];
  load_rec<T>(rec + (int64_t)RW * c, g, fid);
  T r[4];
  uint32_t code = item_geometry<T>(g, w[3 * d], w[3 * d + 1], w[3 * d + 2], r);
  uint32_t q[3] = {0u, 0u, 0u};
  if constexpr (sizeof(T) == 4) {
    int m = 0;
#pragma unroll
    for (int f = 0; f < 4; f++)
      if ((code >> f) & 1u) {
        const uint32_t v = __float_as_uint(r[f]);
        if (m == 0) q[0] = v;
        else if (m == 1) q[1] = v;
        else q[2] = v;
        m++;
      }
  } else {
    uint32_t used = 0;  // in-faces some node of an out-face is traced to
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (!((code >> (4 + j)) & 1u)) continue;
#pragma unroll
      for (int qq = 0; qq < 3; qq++) {
        const uint32_t cv = (code >> (8 + 4 * (((j + 1 + qq) & 3)))) & 15u;
        if (!(cv & 8u)) used |= 1u << (cv & 3u);
      }
    }
    double rmax = 0.0;
#pragma unroll
    for (int f = 0; f < 4; f++)
      if ((used >> f) & 1u) rmax = fmax(rmax, (double)r[f]);
    const int e = rmax > 0.0 ? max(-127, min(127, ilogb(rmax) + 1)) : 0;
    const double up = ldexp(1.0, 32 - e);
    int m = 0;
#pragma unroll
    for (int f = 0; f < 4; f++)
      if ((code >> f) & 1u) {
        const uint32_t v = ((used >> f) & 1u) ? (uint32_t)fmin(rint((double)r[f] * up), 4294967295.0) : 0u;
        if (m == 0) q[0] = v;
        else if (m == 1) q[1] = v;
        else q[2] = v;
        m++;
      }
    code |= (uint32_t)(e + 128) << 24;
  }
  geo[i] = make_uint4(code, q[0], q[1], q[2]);
}

// Source record {k = alpha + betta, betta / k, alpha Q_g / k} of each context cell
// (rhs_g = alpha Q_g / k + (betta / k) S_g, GetRhsOpt with the division by k
// distributed) from caller arrays (caller numbering) ...
template <class T, class TA>
__global__ void k_dyn_from_arrays(int64_t N, int G, int RW, const int32_t *perm, const TA *alpha, const TA *betta,
                                  const TA *Q, T *rec) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= N) return;
  const int64_t p = perm[c];
  const T al = (T)alpha[p], be = (T)betta[p];
  T *o = rec + (int64_t)RW * c + Rec<T>::DYN;
  const T k = al + be;
  o[0] = k;
  o[1] = be / k;
  for (int g = 0; g < G; g++) o[2 + g] = (al * (T)Q[p * G + g]) / k;
}

// ... or from the solver state: alpha = a rho, betta = b rho, Q_g = B(T) / kRadiation / G.
template <class T>
__global__ void k_dyn_from_state(int64_t N, int G, int RW, const double *state, double a_coef, double b_coef,
                                 Emission em, T *rec) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= N) return;
  const double rho = state[10 * c + 5], prs = state[10 * c + 9];
  const T al = (T)(a_coef * rho), be = (T)(b_coef * rho);
  const T q = (T)(planck_B(em, rho, prs) / em.rad_unit / (double)G);
  T *o = rec + (int64_t)RW * c + Rec<T>::DYN;
  const T k = al + be;
  o[0] = k;
  o[1] = be / k;
  const T aq = (al * q) / k;
  for (int g = 0; g < G; g++) o[2 + g] = aq;
}

// ---------------------------------------------------------------- coupled step
// 4-force from the moments summed over the groups.  FP64 moments per row: E
// [rows], F [rows][3], T [rows][9]; FP32 moments: [rows][16] = {E, F, Txx, Txy,
// Txz, Tyy, Tyz, Tzz, ...}.
__global__ void k_source(int64_t N, int G, const double *state, double a_coef, double b_coef, Emission em,
                         const double *mE, const double *mF, const double *mT, const float *mom, double *G4) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= N) return;
  double E = 0, F[3] = {0, 0, 0}, Tm[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int g = 0; g < G; g++) {
    const int64_t r = c * G + g;
    if (mom) {
      const float4 *m4 = reinterpret_cast<const float4 *>(mom + 16 * r);
      const float4 a = m4[0], b = m4[1], cc = m4[2];
      const double t9[9] = {b.x, b.y, b.z, b.y, b.w, cc.x, b.z, cc.x, cc.y};
      E += a.x;
      F[0] += a.y;
      F[1] += a.z;
      F[2] += a.w;
#pragma unroll
      for (int q = 0; q < 9; q++) Tm[q] += t9[q];
    } else {
      E += mE[r];
#pragma unroll
      for (int q = 0; q < 3; q++) F[q] += mF[3 * r + q];
#pragma unroll
      for (int q = 0; q < 9; q++) Tm[q] += mT[9 * r + q];
    }
  }
  double w[5];
#pragma unroll
  for (int q = 0; q < 5; q++) w[q] = state[10 * c + 5 + q];
  double out[4];
  rad_source_cell(em, w, a_coef * w[0], b_coef * w[0], E, F, Tm, out);
#pragma unroll
  for (int q = 0; q < 4; q++) G4[4 * c + q] = out[q];
}

// U.E += tau G0, U.S += tau G (radRHD_main.cpp:117-126), then GetPhysValueStab
// from its own guess without fallback (its status is ignored there as well).
// cnt: {ok, failed, newton iterations, max iterations}.
__global__ void k_source_c2p(int64_t N, Eos eos, double *state, const double *G4, double tau,
                             unsigned long long *cnt) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  unsigned long long ok = 0, failed = 0, iters = 0;
  if (c < N) {
    double u[5], w[5];
#pragma unroll
    for (int q = 0; q < 5; q++) {
      u[q] = state[10 * c + q];
      w[q] = state[10 * c + 5 + q];
    }
    u[4] += tau * G4[4 * c];
    u[1] += tau * G4[4 * c + 1];
    u[2] += tau * G4[4 * c + 2];
    u[3] += tau * G4[4 * c + 3];
    int it = 0;
    const int code = c2p_from(eos, u, w, 0.0, false, &it);
    ok = code == 0;
    failed = code != 0;
    iters = (unsigned long long)it;
#pragma unroll
    for (int q = 0; q < 5; q++) {
      state[10 * c + q] = u[q];
      state[10 * c + 5 + q] = w[q];
    }
  }
  unsigned long long mx = iters;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ok += __shfl_xor_sync(0xffffffffu, ok, o);
    failed += __shfl_xor_sync(0xffffffffu, failed, o);
    iters += __shfl_xor_sync(0xffffffffu, iters, o);
    const unsigned long long m2 = __shfl_xor_sync(0xffffffffu, mx, o);
    mx = m2 > mx ? m2 : mx;
  }
  if ((threadIdx.x & 31) == 0 && (ok | failed)) {
    atomicAdd(cnt + 0, ok);
    atomicAdd(cnt + 1, failed);
    atomicAdd(cnt + 2, iters);
    atomicMax(cnt + 3, mx);
  }
}

template <class T>
__global__ void k_rows_to_host_order(int64_t N, int64_t width, const int32_t *perm, const T *src, double *dst) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= N * width) return;
  const int64_t c = i / width, k = i - c * width;
  dst[(int64_t)perm[c] * width + k] = (double)src[i];
}

unsigned grid_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

Eos eos_of(const rrhd_ctx *c) {
  Eos e;
  e.eos = c->eos;
  e.g1 = c->gamma;
  e.gg = c->gamma / (c->gamma - 1.0);
  return e;
}

template <class T>
rrhd_status build_plan(rrhd_ctx *c) {
  RadState &R = c->rad;
  const int64_t N = c->N;
  const int64_t total = N * (int64_t)R.M;
  cudaStream_t st = c->stream;
  uint32_t *indeg = nullptr, *tmp = nullptr;
  unsigned long long *d_tail = nullptr;
  void *sort_tmp = nullptr;
  size_t sort_bytes = 0;
  auto cleanup = [&]() {
    cudaFree(indeg);
    cudaFree(tmp);
    cudaFree(d_tail);
    cudaFree(sort_tmp);
  };
  const int64_t bmax = N * (int64_t)R.DB;
  if (cudaMalloc(&R.d_plan, sizeof(uint32_t) * total) != cudaSuccess ||
      cudaMalloc(&indeg, sizeof(uint32_t) * bmax) != cudaSuccess ||
      cudaMalloc(&tmp, sizeof(uint32_t) * bmax) != cudaSuccess ||
      cudaMalloc(&d_tail, sizeof(unsigned long long)) != cudaSuccess) {
    cleanup();
    return rrhd_fail(RRHD_ERR_OOM, "sweep plan allocation failed");
  }
  int db_bits = 0;
  while ((1 << db_bits) < R.DB) db_bits++;
  const int end_bit = R.shift + db_bits;
  cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, (const uint32_t *)nullptr, (uint32_t *)nullptr, bmax, 0,
                                 end_bit, st);
  if (cudaMalloc(&sort_tmp, sort_bytes) != cudaSuccess) {
    cleanup();
    return rrhd_fail(RRHD_ERR_OOM, "sweep plan allocation failed");
  }
  R.lvl.assign(R.nbatch, {});
  R.levels = 0;
  R.max_level = 0;
  int64_t base = 0;
  for (int b = 0; b < R.nbatch; b++) {
    const int d0 = b * R.DB;
    const int nbd = std::min(R.DB, R.M - d0);
    uint32_t *plan = R.d_plan + base;
    const unsigned long long zero = 0;
    RRHD_CUDA(cudaMemcpyAsync(d_tail, &zero, sizeof zero, cudaMemcpyHostToDevice, st));
    k_plan_init<T><<<grid_for(N * nbd, 256), 256, 0, st>>>(N, nbd, R.shift, d0, (const T *)R.d_w,
                                                            (const T *)R.d_rec, R.RW, indeg, plan, d_tail);
    RRHD_CUDA(cudaGetLastError());
    std::vector<int64_t> &off = R.lvl[b];
    off.assign(1, 0);
    int64_t lo = 0;
    for (;;) {
      unsigned long long hi_u = 0;
      RRHD_CUDA(cudaMemcpyAsync(&hi_u, d_tail, sizeof hi_u, cudaMemcpyDeviceToHost, st));
      RRHD_CUDA(cudaStreamSynchronize(st));
      const int64_t hi = (int64_t)hi_u;
      if (hi == lo) break;
      // items of a level in ascending (direction, cell) order: deterministic launches,
      // and the items of one direction in cell order, so that neighbouring cells' face
      // slots (direction-major) and records are read close together
      cub::DeviceRadixSort::SortKeys(sort_tmp, sort_bytes, plan + lo, tmp, hi - lo, 0, end_bit, st);
      RRHD_CUDA(cudaMemcpyAsync(plan + lo, tmp, sizeof(uint32_t) * (hi - lo), cudaMemcpyDeviceToDevice, st));
      off.push_back(hi);
      R.max_level = std::max(R.max_level, hi - lo);
      k_plan_expand<T><<<grid_for(hi - lo, 256), 256, 0, st>>>(plan + lo, hi - lo, nbd, R.shift, d0,
                                                                (const T *)R.d_w, (const T *)R.d_rec, R.RW,
                                                                indeg, plan, d_tail);
      RRHD_CUDA(cudaGetLastError());
      lo = hi;
    }
    if (lo != N * nbd) {
      cleanup();
      return rrhd_fail(RRHD_ERR_STATE, "sweep dependency cycle: %lld of %lld (cell, direction) pairs of batch %d "
                                       "have an upwind neighbour that depends on them",
                       (long long)(N * nbd - lo), (long long)(N * nbd), b);
    }
    R.levels += (int64_t)off.size() - 1;
    base += N * nbd;
  }
  cleanup();
  return RRHD_OK;
}

template <class T, class TV, class TI, int GT, bool PRE>
cudaError_t launch_level(const SweepArgs<T, TV> &a, unsigned nb, cudaStream_t st, bool pdl) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nb);
  cfg.blockDim = dim3(kSweepThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k_sweep_level<T, TV, TI, GT, PRE>, a);
}

// the geometry stream exists for the float-intensity forms only (its distances are float)
template <class T, class TV, class TI, int GT>
cudaError_t launch_level_any(const SweepArgs<T, TV> &a, unsigned nb, cudaStream_t st, bool pdl) {
  if constexpr (sizeof(TI) == 4) {
    if (a.geo) return launch_level<T, TV, TI, GT, true>(a, nb, st, pdl);
  }
  return launch_level<T, TV, TI, GT, false>(a, nb, st, pdl);
}

template <class T, class TV, class TI>
rrhd_status capture_sweep(rrhd_ctx *c) {
  RadState &R = c->rad;
  cudaStream_t cs = nullptr;
  RRHD_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaGraph_t g = nullptr;
  cudaError_t launch_err = cudaSuccess;
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    SweepArgs<T, TV> a;
    a.io = R.d_io;
    a.shift = R.shift;
    a.DB = R.DB;
    a.M = R.M;
    a.G = R.G;
    a.RW = R.RW;
    a.w = (const T *)R.d_w;
    a.rec = (const T *)R.d_rec;
    a.area = (const T *)R.d_area;
    a.fv = (TV *)R.d_fv;
    a.NF = c->F;
    a.geo = nullptr;
    a.bc = (TV)R.bc;
    a.last = R.last_cell;
    a.GS = R.GS;
    int64_t base = 0;
    for (int b = 0; b < R.nbatch; b++) {
      a.d0 = b * R.DB;
      const int nbd = std::min(R.DB, R.M - a.d0);
      a.nbd = nbd;
      const std::vector<int64_t> &off = R.lvl[b];
      for (size_t L = 0; L + 1 < off.size(); L++) {
        a.items = R.d_plan + base + off[L];
        a.n = off[L + 1] - off[L];
        const unsigned nb = grid_for(a.n, kSweepThreads);
        const bool pdl = L > 0;  // the first level of a batch follows a full dependency
        cudaError_t le;
        a.geo = R.d_geo ? R.d_geo + base + off[L] : nullptr;
        switch (R.G) {
          case 1: le = launch_level_any<T, TV, TI, 1>(a, nb, cs, pdl); break;
          case 2: le = launch_level_any<T, TV, TI, 2>(a, nb, cs, pdl); break;
          case 4: le = launch_level_any<T, TV, TI, 4>(a, nb, cs, pdl); break;
          default: le = launch_level_any<T, TV, TI, 0>(a, nb, cs, pdl); break;
        }
        if (le != cudaSuccess && launch_err == cudaSuccess) launch_err = le;
      }
      const dim3 nr((unsigned)((c->N + kRcCells - 1) / kRcCells), (unsigned)((nbd + kRcDirs - 1) / kRcDirs));
      switch (R.G) {
        case 1: k_recalc<T, TV, TI, 1><<<nr, 256, 0, cs>>>(a, c->N); break;
        case 2: k_recalc<T, TV, TI, 2><<<nr, 256, 0, cs>>>(a, c->N); break;
        case 4: k_recalc<T, TV, TI, 4><<<nr, 256, 0, cs>>>(a, c->N); break;
        default: k_recalc<T, TV, TI, 0><<<nr, 256, 0, cs>>>(a, c->N); break;
      }
      base += c->N * nbd;
    }
    e = cudaStreamEndCapture(cs, &g);
  }
  if (e == cudaSuccess) e = launch_err;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&R.graph, g, 0);
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cs);
  RRHD_CUDA(e);
  return RRHD_OK;
}

}  // namespace

void rrhd_rad_release(rrhd_ctx *c) {
  RadState &R = c->rad;
  if (R.graph) cudaGraphExecDestroy(R.graph);
  void *ptrs[] = {R.d_w, R.d_rec, R.d_area, R.d_plan, R.d_geo, R.d_io, R.d_fv, R.d_I, R.d_S, R.d_G4, R.d_mE, R.d_mF,
                  R.d_mT, R.d_mom, R.d_cnt};
  for (void *p : ptrs) cudaFree(p);
  for (cudaEvent_t e : R.ev)
    if (e) cudaEventDestroy(e);
  if (R.side) cudaStreamDestroy(R.side);
  if (R.tc) rrhd_scatter_tc_destroy(R.tc);
  R = RadState();
}

// T: the records (geometry, opacities and sources) and directions; TV: the face values
// and the transport arithmetic; TI: the intensity and scattering-integral arrays the
// sweep reads and writes.
template <class T, class TV, class TI>
static rrhd_status rad_setup_t(rrhd_ctx *c) {
  RadState &R = c->rad;
  const int64_t N = c->N;
  const int W = ((Rec<T>::DYN + 2 + R.G + Rec<T>::NBRW + Rec<T>::LINE - 1) / Rec<T>::LINE) * Rec<T>::LINE;
  R.RW = W;
  std::vector<T> rec((size_t)W * N, (T)0), area(4 * (size_t)N), w(3 * R.M);
  std::vector<int32_t> iperm(N);
  for (int64_t i = 0; i < N; i++) iperm[c->h_perm[i]] = (int32_t)i;
  // face-value slots numbered in order of first use by context cells, so that the
  // faces of neighbouring cells sit close together
  std::vector<int32_t> fslot(c->F, -1);
  int32_t nslot = 0;
  for (int64_t cn = 0; cn < N; cn++)
    for (int j = 0; j < 4; j++) {
      const int32_t fc = c->h_cell_faces[4 * c->h_perm[cn] + j];
      if (fslot[fc] < 0) fslot[fc] = nslot++;
    }
  for (int64_t cn = 0; cn < N; cn++) {
    const int64_t p = c->h_perm[cn];
    T *r = rec.data() + (size_t)W * cn;
    int32_t ids[8];
    for (int j = 0; j < 4; j++) {
      const int32_t fc = c->h_cell_faces[4 * p + j];
      const bool out = (c->h_cell_sign[p] >> j) & 1;
      for (int x = 0; x < 3; x++) {
        const double v = c->h_face_n[3 * (int64_t)fc + x];
        r[3 * j + x] = (T)(out ? v : -v);
      }
      r[12 + j] = (T)(3.0 * c->h_cell_V[p] / c->h_face_area[fc]);
      area[4 * cn + j] = (T)c->h_face_area[fc];
      const int32_t l = c->h_face_l[fc], rr = c->h_face_r[fc];
      const int32_t o = (l == p) ? rr : l;
      ids[j] = o < 0 ? (fslot[fc] | kNoNeighbour) : fslot[fc];
      ids[4 + j] = o < 0 ? -1 : iperm[o];
    }
    std::memcpy(r + Rec<T>::IDS, ids, 4 * sizeof(int32_t));
    std::memcpy(r + W - Rec<T>::NBRW, ids + 4, 4 * sizeof(int32_t));
  }
  for (int q = 0; q < 3 * R.M; q++) w[q] = (T)R.dirs->h_w[q];
  R.last_cell = iperm[N - 1];
  R.GS = sizeof(TV) == 8 ? ((R.G + 3) & ~3) : ((R.G + 7) & ~7);
  auto up = [&](void **dst, const void *src, size_t bytes) -> rrhd_status {
    if (cudaMalloc(dst, bytes) != cudaSuccess) return rrhd_fail(RRHD_ERR_OOM, "sweep allocation failed");
    RRHD_CUDA(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
    return RRHD_OK;
  };
  rrhd_status s;
  if ((s = up(&R.d_rec, rec.data(), sizeof(T) * rec.size())) || (s = up(&R.d_w, w.data(), sizeof(T) * w.size())) ||
      (s = up(&R.d_area, area.data(), sizeof(T) * area.size())))
    return s;
  if (cudaMalloc(&R.d_io, sizeof(SweepIO)) != cudaSuccess ||
      cudaMalloc(&R.d_fv, sizeof(TV) * (size_t)c->F * R.DB * R.GS) != cudaSuccess)
    return rrhd_fail(RRHD_ERR_OOM, "sweep allocation failed");
  if ((s = build_plan<T>(c))) return s;
  if (R.item_geometry) {
    const int64_t total = N * (int64_t)R.M;
    if (cudaMalloc(&R.d_geo, sizeof(uint4) * total) != cudaSuccess) {
      R.d_geo = nullptr;
      return rrhd_fail(RRHD_ERR_OOM, "sweep geometry stream allocation failed (%lld bytes)",
                       (long long)(sizeof(uint4) * total));
    }
    int64_t base = 0;
    for (int b = 0; b < R.nbatch; b++) {
      const int d0 = b * R.DB;
      const int64_t n = N * std::min(R.DB, R.M - d0);
      k_plan_geometry<T><<<grid_for(n, 256), 256, 0, c->stream>>>(R.d_plan + base, n, R.shift, R.DB, d0,
                                                                  (const T *)R.d_w, (const T *)R.d_rec, R.RW,
                                                                  R.d_geo + base);
      RRHD_CUDA(cudaGetLastError());
      base += n;
    }
    RRHD_CUDA(cudaStreamSynchronize(c->stream));
  }
  return capture_sweep<T, TV, TI>(c);
}

extern "C" rrhd_status rrhd_rad_setup(rrhd_ctx *c, const rrhd_dirs *dirs, const rrhd_rad_opts *o) {
  RRHD_CHECK_ARG(c && dirs && o, "null argument");
  RRHD_CHECK_ARG(o->groups >= 1 && o->groups <= 64, "groups must be in [1, 64]");
  RRHD_CHECK_ARG(o->precision == RRHD_RAD_FP64 || o->precision == RRHD_RAD_FP32 || o->precision == RRHD_RAD_MIXED,
                 "bad precision");
  RRHD_CHECK_ARG(dirs->device == c->device, "direction set lives on another device");
  RRHD_CHECK_ARG(o->item_geometry == 0 || o->item_geometry == 1, "item_geometry: 0 or 1");
  RRHD_CHECK_ARG(o->item_geometry == 0 || o->precision != RRHD_RAD_FP64,
                 "item_geometry needs RRHD_RAD_FP32 or RRHD_RAD_MIXED (its distances are float)");
  int DB = o->dirs_per_batch;
  RRHD_CHECK_ARG(DB == 0 || (DB > 0 && DB <= 256 && (DB & (DB - 1)) == 0), "dirs_per_batch: power of two <= 256");
  RRHD_CUDA(cudaSetDevice(c->device));
  RRHD_CUDA(cudaStreamSynchronize(c->stream));
  rrhd_rad_release(c);
  RadState &R = c->rad;
  R.dirs = dirs;
  R.M = dirs->M;
  R.G = o->groups;
  if (DB == 0) {
    DB = 1;
    while (DB < std::min(R.M, 64)) DB <<= 1;
  }
  R.DB = DB;
  R.shift = 0;  // item = direction << shift | cell
  while ((int64_t(1) << R.shift) < c->N) R.shift++;
  if (R.shift > 31 || ((int64_t)DB << R.shift) > (int64_t)UINT32_MAX + 1)
    return rrhd_fail(RRHD_ERR_LIMIT, "sweep items are 32-bit: dirs_per_batch x 2^ceil(log2 cells) must stay "
                                     "within 2^32");
  R.nbatch = (R.M + DB - 1) / DB;
  R.prec = o->precision;
  R.bc = o->boundary_value;
  R.item_geometry = o->item_geometry != 0;
  const rrhd_status s = R.prec == RRHD_RAD_FP64   ? rad_setup_t<double, double, double>(c)
                        : R.prec == RRHD_RAD_MIXED ? rad_setup_t<double, double, float>(c)
                                                   : rad_setup_t<float, float, float>(c);
  if (s) {
    rrhd_rad_release(c);
    return s;
  }
  R.ready = true;
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_rad_plan_info(const rrhd_ctx *c, int64_t *levels, int64_t *max_level_items) {
  RRHD_CHECK_ARG(c, "null context");
  if (!c->rad.ready) return rrhd_fail(RRHD_ERR_STATE, "rrhd_rad_setup has not run");
  if (levels) *levels = c->rad.levels;
  if (max_level_items) *max_level_items = c->rad.max_level;
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_rad_plan_levels(const rrhd_ctx *c, int32_t *levels) {
  RRHD_CHECK_ARG(c && levels, "null argument");
  const RadState &R = c->rad;
  if (!R.ready) return rrhd_fail(RRHD_ERR_STATE, "rrhd_rad_setup has not run");
  RRHD_CUDA(cudaSetDevice(c->device));
  const int64_t N = c->N, total = N * (int64_t)R.M;
  std::vector<uint32_t> plan((size_t)total);
  RRHD_CUDA(cudaStreamSynchronize(c->stream));
  RRHD_CUDA(cudaMemcpy(plan.data(), R.d_plan, sizeof(uint32_t) * total, cudaMemcpyDeviceToHost));
  for (int64_t i = 0; i < total; i++) levels[i] = -1;
  int64_t base = 0;
  for (int b = 0; b < R.nbatch; b++) {
    const int d0 = b * R.DB;
    const int nbd = std::min(R.DB, R.M - d0);
    const std::vector<int64_t> &off = R.lvl[b];
    for (size_t L = 0; L + 1 < off.size(); L++)
      for (int64_t k = off[L]; k < off[L + 1]; k++) {
        const uint32_t it = plan[(size_t)(base + k)];
        const int64_t cc = it & ((1u << R.shift) - 1u);
        const int d = d0 + (int)(it >> R.shift);
        levels[(int64_t)d * N + c->h_perm[cc]] = (int32_t)L;
      }
    base += N * nbd;
  }
  return RRHD_OK;
}

static rrhd_status launch_sweep(rrhd_ctx *c, const SweepIO &io) {
  RadState &R = c->rad;
  // the graph reads its pointers from d_io; upload only when they change
  if (!R.io_valid || std::memcmp(&io, &R.h_io, sizeof io) != 0) {
    R.h_io = io;
    RRHD_CUDA(cudaMemcpyAsync(R.d_io, &R.h_io, sizeof io, cudaMemcpyHostToDevice, c->stream));
    RRHD_CUDA(cudaStreamSynchronize(c->stream));
    R.io_valid = true;
  }
  RRHD_CUDA(cudaGraphLaunch(R.graph, c->stream));
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_sweep(rrhd_ctx *c, const void *alpha, const void *betta, const void *Q, const void *S,
                                  void *I) {
  RRHD_CHECK_ARG(c && alpha && betta && Q && S && I, "null argument");
  RadState &R = c->rad;
  if (!R.ready) return rrhd_fail(RRHD_ERR_STATE, "rrhd_rad_setup has not run");
  RRHD_CUDA(cudaSetDevice(c->device));
  const int64_t N = c->N;
  if (R.prec == RRHD_RAD_FP64)
    k_dyn_from_arrays<double, double><<<grid_for(N, 256), 256, 0, c->stream>>>(
        N, R.G, R.RW, c->d_perm, (const double *)alpha, (const double *)betta, (const double *)Q, (double *)R.d_rec);
  else if (R.prec == RRHD_RAD_MIXED)  // float arrays, double records
    k_dyn_from_arrays<double, float><<<grid_for(N, 256), 256, 0, c->stream>>>(
        N, R.G, R.RW, c->d_perm, (const float *)alpha, (const float *)betta, (const float *)Q, (double *)R.d_rec);
  else
    k_dyn_from_arrays<float, float><<<grid_for(N, 256), 256, 0, c->stream>>>(
        N, R.G, R.RW, c->d_perm, (const float *)alpha, (const float *)betta, (const float *)Q, (float *)R.d_rec);
  RRHD_CUDA(cudaGetLastError());
  SweepIO io{S, I, c->d_perm, 0};
  return launch_sweep(c, io);
}

// ---------------------------------------------------------------- coupled step
namespace {
template <class T>
__global__ void k_cdg_to_rows(int64_t N, int M, int G, const int32_t *perm, const T *src, double *dst) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t per = (int64_t)M * G;
  if (i >= N * per) return;
  const int64_t c = i / per, rem = i - c * per;
  const int d = (int)(rem / G), g = (int)(rem - (int64_t)d * G);
  dst[((int64_t)perm[c] * G + g) * M + d] = (double)src[i];
}

// Moments of the last scattering per row (cell * G + g), caller order, as
// {E, F0, F1, F2, T00, T01, T02, T11, T12, T22}: from the FP64 arrays (E [rows],
// F [rows][3], T [rows][9] column-major) or the FP32 [rows][16] columns.
__global__ void k_mom_to_rows(int64_t N, int G, const int32_t *perm, const double *mE, const double *mF,
                              const double *mT, const float *mom, double *dst) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= N * G) return;
  const int64_t c = r / G, g = r - c * G;
  double *o = dst + ((int64_t)perm[c] * G + g) * 10;
  if (mom) {
    for (int k = 0; k < 10; k++) o[k] = (double)mom[16 * r + k];
    return;
  }
  o[0] = mE[r];
  for (int k = 0; k < 3; k++) o[1 + k] = mF[3 * r + k];
  const int ij[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  for (int k = 0; k < 6; k++) o[4 + k] = mT[9 * r + 3 * ij[k][1] + ij[k][0]];
}

template <class T>
__global__ void k_rows_to_cdg(int64_t N, int M, int G, const int32_t *perm, const double *src, T *dst) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t per = (int64_t)M * G;
  if (i >= N * per) return;
  const int64_t c = i / per, rem = i - c * per;
  const int d = (int)(rem / G), g = (int)(rem - (int64_t)d * G);
  dst[i] = (T)src[((int64_t)perm[c] * G + g) * M + d];
}
}  // namespace

// T: the element type of the intensity and scattering-integral arrays.
template <class T>
static rrhd_status alloc_coupled(rrhd_ctx *c) {
  RadState &R = c->rad;
  const int64_t N = c->N, rows = N * R.G;
  const size_t big = sizeof(T) * (size_t)rows * R.M;
  if (cudaMalloc(&R.d_I, big) != cudaSuccess || cudaMalloc(&R.d_S, big) != cudaSuccess ||
      cudaMalloc(&R.d_G4, sizeof(double) * 4 * N) != cudaSuccess ||
      cudaMalloc(&R.d_cnt, sizeof(unsigned long long) * 8) != cudaSuccess)
    return rrhd_fail(RRHD_ERR_OOM, "coupled-step allocation failed");
  for (cudaEvent_t &e : R.ev) RRHD_CUDA(cudaEventCreate(&e));
  RRHD_CUDA(cudaStreamCreateWithFlags(&R.side, cudaStreamNonBlocking));
  RRHD_CUDA(cudaMemsetAsync(R.d_I, 0, big, c->stream));
  RRHD_CUDA(cudaMemsetAsync(R.d_S, 0, big, c->stream));
  RRHD_CUDA(cudaMemsetAsync(R.d_G4, 0, sizeof(double) * 4 * N, c->stream));
  if (R.prec == RRHD_RAD_FP64) {
    if (cudaMalloc(&R.d_mE, sizeof(double) * rows) != cudaSuccess ||
        cudaMalloc(&R.d_mF, sizeof(double) * 3 * rows) != cudaSuccess ||
        cudaMalloc(&R.d_mT, sizeof(double) * 9 * rows) != cudaSuccess)
      return rrhd_fail(RRHD_ERR_OOM, "coupled-step allocation failed");
    RRHD_CUDA(cudaMemsetAsync(R.d_mE, 0, sizeof(double) * rows, c->stream));
    RRHD_CUDA(cudaMemsetAsync(R.d_mF, 0, sizeof(double) * 3 * rows, c->stream));
    RRHD_CUDA(cudaMemsetAsync(R.d_mT, 0, sizeof(double) * 9 * rows, c->stream));
  } else {
    if (cudaMalloc(&R.d_mom, sizeof(float) * 16 * rows) != cudaSuccess)
      return rrhd_fail(RRHD_ERR_OOM, "coupled-step allocation failed");
    RRHD_CUDA(cudaMemsetAsync(R.d_mom, 0, sizeof(float) * 16 * rows, c->stream));
  }
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_coupled_step(rrhd_ctx *c, double tau, const rrhd_coupled_opts *o, rrhd_step_stats *hs,
                                         rrhd_c2p_stats *ss) {
  RRHD_CHECK_ARG(c && o, "null argument");
  RRHD_CHECK_ARG(tau > 0, "tau must be > 0");
  RRHD_CHECK_ARG(c->part_world == 1, "the coupled step runs on a whole mesh (no rrhd_hydro_set_part split)");
  RadState &R = c->rad;
  if (!R.ready) return rrhd_fail(RRHD_ERR_STATE, "rrhd_rad_setup has not run");
  const bool fp64 = R.prec == RRHD_RAD_FP64;         // intensity and scattering integral in double
  const bool rec64 = R.prec != RRHD_RAD_FP32;        // records (geometry, opacities, sources) in double
  const bool lowrank = o->scatter == RRHD_SCATTER_LOWRANK;
  RRHD_CHECK_ARG(lowrank || (fp64 ? o->scatter == RRHD_SCATTER_FP64
                                  : (o->scatter >= RRHD_TC_BF16X3 && o->scatter <= RRHD_TC_BF16)),
                 "scatter form does not match the sweep precision");
  RRHD_CHECK_ARG((fp64 && !lowrank) ? (64 % R.G == 0) : (R.G == 1 || R.G == 2 || R.G == 4),
                 "coupled step groups: a divisor of 64 (FP64 direct sum) or 1, 2, 4 (tensor cores, low rank)");
  const int k_stall = o->k_stall ? o->k_stall : 12;
  RRHD_CHECK_ARG(k_stall > 0 && k_stall <= 40, "k_stall must be in [1, 40]");
  RRHD_CUDA(cudaSetDevice(c->device));
  rrhd_status s;
  if (!R.d_I && (s = fp64 ? alloc_coupled<double>(c) : alloc_coupled<float>(c))) return s;
  if (!fp64 && !lowrank && (!R.tc || R.tc_form != o->scatter)) {
    if (R.tc) rrhd_scatter_tc_destroy(R.tc);
    R.tc = nullptr;
    if ((s = rrhd_scatter_tc_create(R.dirs, o->scatter, &R.tc))) return s;
    R.tc_form = o->scatter;
  }
  cudaStream_t st = c->stream;
  const int64_t N = c->N;
  // a previous step that returned early may have left its source term on the side stream
  RRHD_CUDA(cudaStreamWaitEvent(st, R.ev[4], 0));
  RRHD_CUDA(cudaEventRecord(R.ev[0], st));
  // 1. hydro step (flux, update, con2prim with fallback)
  rrhd_step_stats hst;
  const rrhd_status hstat = rrhd_hydro_step(c, tau, hs ? &hst : nullptr);
  if (hstat && hstat != RRHD_ERR_C2P) return hstat;
  if (hs) *hs = hst;
  RRHD_CUDA(cudaEventRecord(R.ev[1], st));
  double *state = c->d_state[c->cur];
  const Emission em{o->emission.temp_coef, o->emission.sigma_sb, o->emission.pi, o->emission.rad_unit};
  // 2. opacities and emission from the new primitives
  if (rec64)
    k_dyn_from_state<double><<<grid_for(N, 256), 256, 0, st>>>(N, R.G, R.RW, state, o->absorption, o->scattering,
                                                                em, (double *)R.d_rec);
  else
    k_dyn_from_state<float><<<grid_for(N, 256), 256, 0, st>>>(N, R.G, R.RW, state, o->absorption, o->scattering, em,
                                                               (float *)R.d_rec);
  RRHD_CUDA(cudaGetLastError());
  // 4. 4-force from the previous intensity's moments and the source con2prim, on the side
  // stream beside the sweep: they read the state after the opacities were taken from it and
  // the previous step's moments, and write the state and G4, none of which the sweep touches.
  RRHD_CUDA(cudaEventRecord(R.ev[3], st));
  RRHD_CUDA(cudaStreamWaitEvent(R.side, R.ev[3], 0));
  const cudaStream_t ss_st = R.side;
  k_source<<<grid_for(N, 128), 128, 0, ss_st>>>(N, R.G, state, o->absorption, o->scattering, em, R.d_mE, R.d_mF,
                                                 R.d_mT, R.d_mom, R.d_G4);
  RRHD_CUDA(cudaGetLastError());
  if (o->guess) {
    if ((s = mlp_c2p(o->guess, c->eos, c->gamma, state, state + 5, 10, R.d_G4, tau, nullptr, N, 0, k_stall, ss,
                     nullptr, nullptr, ss_st)))
      return s;
  } else {
    RRHD_CUDA(cudaMemsetAsync(R.d_cnt, 0, sizeof(unsigned long long) * 8, ss_st));
    k_source_c2p<<<grid_for(N, 256), 256, 0, ss_st>>>(N, eos_of(c), state, R.d_G4, tau, R.d_cnt);
    RRHD_CUDA(cudaGetLastError());
  }
  RRHD_CUDA(cudaEventRecord(R.ev[4], ss_st));
  // 3. sweep with the previous scattering integral
  SweepIO io{R.d_S, R.d_I, nullptr, 1};
  if ((s = launch_sweep(c, io))) return s;
  RRHD_CUDA(cudaEventRecord(R.ev[2], st));
  // the scattering below overwrites the moments the source read, and the next step reads
  // the state the source wrote: join the side stream
  RRHD_CUDA(cudaStreamWaitEvent(st, R.ev[4], 0));
  RRHD_CUDA(cudaEventRecord(R.ev[5], st));
  if (!o->guess && ss) {
    unsigned long long h[8];
    RRHD_CUDA(cudaMemcpyAsync(h, R.d_cnt, sizeof h, cudaMemcpyDeviceToHost, st));
    RRHD_CUDA(cudaStreamSynchronize(st));
    ss->n_ok = (int64_t)h[0];
    ss->n_fallback = 0;
    ss->n_failed = (int64_t)h[1];
    ss->newton_iters = (int64_t)h[2];
    ss->max_iters = (int32_t)h[3];
  }
  // 5. scattering integral and moments of the new intensity, for the next step
  if (lowrank) {
    if (fp64) {
      if ((s = scatter_lowrank_fp64(R.dirs, (const double *)R.d_I, (double *)R.d_S, R.d_mE, R.d_mF, R.d_mT, N, R.G,
                                    st)))
        return s;
    } else if ((s = scatter_lowrank_fp32(R.dirs, (const float *)R.d_I, (float *)R.d_S, R.d_mom, N, R.G, st))) {
      return s;
    }
  } else if (fp64) {
    if ((s = scatter_fp64_cdg(R.dirs, (const double *)R.d_I, (double *)R.d_S, N, R.G, false, st))) return s;
    if ((s = moments_fp64_cdg(R.dirs, (const double *)R.d_I, R.d_mE, R.d_mF, R.d_mT, N, R.G, st))) return s;
  } else {
    if ((s = scatter_tc_cdg(R.tc, (const float *)R.d_I, (float *)R.d_S, R.d_mom, N, R.G, st))) return s;
  }
  RRHD_CUDA(cudaEventRecord(R.ev[6], st));
  return hstat;
}

extern "C" rrhd_status rrhd_coupled_phase_ms(rrhd_ctx *c, float *ms) {
  RRHD_CHECK_ARG(c && ms, "null argument");
  RadState &R = c->rad;
  if (!R.ev[0]) return rrhd_fail(RRHD_ERR_STATE, "no coupled step has run");
  RRHD_CUDA(cudaSetDevice(c->device));
  RRHD_CUDA(cudaEventSynchronize(R.ev[6]));
  // hydro (with the opacities), sweep, source (side stream, beside the sweep), scattering
  RRHD_CUDA(cudaEventElapsedTime(ms + 0, R.ev[0], R.ev[3]));
  RRHD_CUDA(cudaEventElapsedTime(ms + 1, R.ev[3], R.ev[2]));
  RRHD_CUDA(cudaEventElapsedTime(ms + 2, R.ev[3], R.ev[4]));
  RRHD_CUDA(cudaEventElapsedTime(ms + 3, R.ev[5], R.ev[6]));
  return RRHD_OK;
}

namespace {
// The scattering integral and moments the last coupled step left (FP32, cell-direction-group
// layout, moments [rows][16]) against their FP64 values from the same FP32 intensity, on
// every stride-th cell: one thread per (sampled cell, group) loops over the output
// directions (S relative to itself) and forms the ten moments (F and T relative to E).
// err: {max S, sum of squared S errors, count, max moments} as doubles, the maxima as the
// bit patterns of non-negative doubles.
__global__ void k_coupled_scatter_error(int64_t ncell, int64_t stride, int M, int G, const double *__restrict__ K,
                                        const double *__restrict__ w, const double *__restrict__ a, double area,
                                        const float *__restrict__ I, const float *__restrict__ S,
                                        const float *__restrict__ mom, double *err) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= ncell * G) return;
  const int64_t c = (t / G) * stride;
  const int g = (int)(t % G);
  const float *Ic = I + c * (int64_t)M * G + g;
  double emax = 0.0, esq = 0.0;
  for (int o = 0; o < M; o++) {
    double ref = 0.0;
    for (int d = 0; d < M; d++) ref += K[(int64_t)d * M + o] * (double)Ic[(int64_t)d * G];  // K[d][o] = Gamma a_d / A
    const double e = fabs((double)S[(c * M + o) * G + g] - ref) / fabs(ref);
    if (ref != 0.0) {
      emax = fmax(emax, e);
      esq += e * e;
    }
  }
  double m[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int d = 0; d < M; d++) {
    const double wi = a[d] / area * (double)Ic[(int64_t)d * G];
    const double x = w[3 * d], y = w[3 * d + 1], z = w[3 * d + 2];
    const double f[10] = {1.0, x, y, z, x * x, x * y, x * z, y * y, y * z, z * z};
    for (int k = 0; k < 10; k++) m[k] += f[k] * wi;
  }
  double mmax = 0.0;
  if (mom && m[0] != 0.0) {
    const float *mr = mom + 16 * (c * G + g);
    mmax = fabs((double)mr[0] - m[0]) / fabs(m[0]);
    for (int k = 1; k < 10; k++) mmax = fmax(mmax, fabs((double)mr[k] - m[k]) / fabs(m[0]));
  }
  atomicMax(reinterpret_cast<unsigned long long *>(err), (unsigned long long)__double_as_longlong(emax));
  atomicAdd(err + 1, esq);
  atomicAdd(err + 2, (double)M);
  atomicMax(reinterpret_cast<unsigned long long *>(err + 3), (unsigned long long)__double_as_longlong(mmax));
}
}  // namespace

extern "C" rrhd_status rrhd_coupled_scatter_error(rrhd_ctx *c, int64_t sample_cells, double *max_rel, double *rms_rel,
                                                  double *moments_max) {
  RRHD_CHECK_ARG(c && sample_cells > 0, "bad argument");
  RadState &R = c->rad;
  if (!R.ready || !R.d_I) return rrhd_fail(RRHD_ERR_STATE, "no coupled step has run");
  if (R.prec == RRHD_RAD_FP64) return rrhd_fail(RRHD_ERR_STATE, "the FP64 form has no reduced-precision scattering");
  RRHD_CUDA(cudaSetDevice(c->device));
  const int64_t N = c->N;
  const int64_t stride = std::max<int64_t>(1, N / sample_cells);
  const int64_t ncell = (N + stride - 1) / stride;
  double *d_err = nullptr;
  RRHD_CUDA(cudaMalloc(&d_err, 4 * sizeof(double)));
  double h[4] = {0, 0, 0, 0};
  cudaError_t e = cudaMemsetAsync(d_err, 0, 4 * sizeof(double), c->stream);
  if (e == cudaSuccess) {
    k_coupled_scatter_error<<<grid_for(ncell * R.G, 128), 128, 0, c->stream>>>(
        ncell, stride, R.M, R.G, R.dirs->d_K, R.dirs->d_w, R.dirs->d_a, R.dirs->full_area, (const float *)R.d_I,
        (const float *)R.d_S, R.d_mom, d_err);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, d_err, sizeof h, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d_err);
  RRHD_CUDA(e);
  if (max_rel) *max_rel = h[0];
  if (rms_rel) *rms_rel = h[2] > 0 ? std::sqrt(h[1] / h[2]) : 0.0;
  if (moments_max) *moments_max = h[3];
  return RRHD_OK;
}

// ---------------------------------------------------------------- caller-array pieces of the coupled step
// (for a step composed over ranks, where each piece runs on a rank's share of cells or rows)
namespace {
// alpha = a rho, betta = b rho, Q_g = B(T) / kRadiation / G from primitives W [n][stride]
// (the opacity and emission rule of the coupled step, as k_dyn_from_state forms them).
__global__ void k_rad_opacities(int64_t n, int64_t stride, int G, const double *W, double a_coef, double b_coef,
                                Emission em, double *alpha, double *betta, double *Q) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  const double rho = W[stride * c], prs = W[stride * c + 4];
  alpha[c] = a_coef * rho;
  betta[c] = b_coef * rho;
  const double q = planck_B(em, rho, prs) / em.rad_unit / (double)G;
  for (int g = 0; g < G; g++) Q[c * G + g] = q;
}

// 4-force per cell from the FP64 moments of its G rows (E [n G], F [n G][3], T [n G][9]),
// summed over the groups in order as k_source does.
__global__ void k_rad_source_rows(int64_t n, int64_t stride, int G, const double *W, double a_coef, double b_coef,
                                  Emission em, const double *mE, const double *mF, const double *mT, double *G4) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= n) return;
  double E = 0, F[3] = {0, 0, 0}, Tm[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int g = 0; g < G; g++) {
    const int64_t r = c * G + g;
    E += mE[r];
#pragma unroll
    for (int q = 0; q < 3; q++) F[q] += mF[3 * r + q];
#pragma unroll
    for (int q = 0; q < 9; q++) Tm[q] += mT[9 * r + q];
  }
  double w[5];
#pragma unroll
  for (int q = 0; q < 5; q++) w[q] = W[stride * c + q];
  double out[4];
  rad_source_cell(em, w, a_coef * w[0], b_coef * w[0], E, F, Tm, out);
#pragma unroll
  for (int q = 0; q < 4; q++) G4[4 * c + q] = out[q];
}

// U.E += tau G0, U.S += tau G (radRHD_main.cpp:117-126), then GetPhysValueStab from its own
// guess without fallback, on caller arrays; cnt as in k_source_c2p.
__global__ void k_rad_source_c2p(int64_t n, int64_t stride, Eos eos, double *U, double *W, const double *G4,
                                 double tau, unsigned long long *cnt) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  unsigned long long ok = 0, failed = 0, iters = 0;
  if (c < n) {
    double u[5], w[5];
#pragma unroll
    for (int q = 0; q < 5; q++) {
      u[q] = U[stride * c + q];
      w[q] = W[stride * c + q];
    }
    u[4] += tau * G4[4 * c];
    u[1] += tau * G4[4 * c + 1];
    u[2] += tau * G4[4 * c + 2];
    u[3] += tau * G4[4 * c + 3];
    int it = 0;
    const int code = c2p_from(eos, u, w, 0.0, false, &it);
    ok = code == 0;
    failed = code != 0;
    iters = (unsigned long long)it;
#pragma unroll
    for (int q = 0; q < 5; q++) {
      U[stride * c + q] = u[q];
      W[stride * c + q] = w[q];
    }
  }
  unsigned long long mx = iters;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ok += __shfl_xor_sync(0xffffffffu, ok, o);
    failed += __shfl_xor_sync(0xffffffffu, failed, o);
    iters += __shfl_xor_sync(0xffffffffu, iters, o);
    const unsigned long long m2 = __shfl_xor_sync(0xffffffffu, mx, o);
    mx = m2 > mx ? m2 : mx;
  }
  if ((threadIdx.x & 31) == 0 && (ok | failed)) {
    atomicAdd(cnt + 0, ok);
    atomicAdd(cnt + 1, failed);
    atomicAdd(cnt + 2, iters);
    atomicMax(cnt + 3, mx);
  }
}
}  // namespace

extern "C" rrhd_status rrhd_rad_opacities(const rrhd_emission *em, const double *W, int64_t stride, int64_t n,
                                          double absorption, double scattering, int32_t groups, double *alpha,
                                          double *betta, double *Q, void *stream) {
  RRHD_CHECK_ARG(em && W && alpha && betta && Q && n >= 0 && stride >= 5 && groups >= 1, "bad arguments");
  if (n == 0) return RRHD_OK;
  const Emission e{em->temp_coef, em->sigma_sb, em->pi, em->rad_unit};
  k_rad_opacities<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, stride, groups, W, absorption, scattering, e,
                                                                      alpha, betta, Q);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_rad_source_rows(const rrhd_emission *em, const double *W, int64_t stride, int64_t n,
                                            double absorption, double scattering, int32_t groups, const double *E,
                                            const double *F, const double *T, double *G4, void *stream) {
  RRHD_CHECK_ARG(em && W && E && F && T && G4 && n >= 0 && stride >= 5 && groups >= 1, "bad arguments");
  if (n == 0) return RRHD_OK;
  const Emission e{em->temp_coef, em->sigma_sb, em->pi, em->rad_unit};
  k_rad_source_rows<<<grid_for(n, 128), 128, 0, (cudaStream_t)stream>>>(n, stride, groups, W, absorption, scattering,
                                                                        e, E, F, T, G4);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_rad_source_con2prim(int32_t eos, double gamma, double *U, double *W, int64_t stride,
                                                const double *G4, double tau, int64_t n, rrhd_c2p_stats *stats,
                                                void *stream) {
  RRHD_CHECK_ARG(U && W && G4 && n >= 0 && stride >= 5 && (eos == 1 || eos == 2), "bad arguments");
  if (n == 0) {
    if (stats) *stats = rrhd_c2p_stats{0, 0, 0, 0, 0};
    return RRHD_OK;
  }
  cudaStream_t st = (cudaStream_t)stream;
  Eos e;
  e.eos = eos;
  e.g1 = gamma;
  e.gg = gamma / (gamma - 1.0);
  unsigned long long *cnt = nullptr;
  RRHD_CUDA(cudaMallocAsync(&cnt, 4 * sizeof(unsigned long long), st));
  cudaError_t err = cudaMemsetAsync(cnt, 0, 4 * sizeof(unsigned long long), st);
  if (err == cudaSuccess) {
    k_rad_source_c2p<<<grid_for(n, 256), 256, 0, st>>>(n, stride, e, U, W, G4, tau, cnt);
    err = cudaGetLastError();
  }
  unsigned long long h[4] = {0, 0, 0, 0};
  if (err == cudaSuccess && stats) err = cudaMemcpyAsync(h, cnt, sizeof h, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(cnt, st);
  if (err == cudaSuccess && stats) err = cudaStreamSynchronize(st);
  RRHD_CUDA(err);
  if (stats) {
    stats->n_ok = (int64_t)h[0];
    stats->n_fallback = 0;
    stats->n_failed = (int64_t)h[1];
    stats->newton_iters = (int64_t)h[2];
    stats->max_iters = (int32_t)h[3];
  }
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_rad_get(rrhd_ctx *c, int32_t what, double *out) {
  RRHD_CHECK_ARG(c && out, "null argument");
  RadState &R = c->rad;
  RRHD_CHECK_ARG(what == RRHD_RAD_I || what == RRHD_RAD_S || what == RRHD_RAD_G4 || what == RRHD_RAD_MOM,
                 "bad array id");
  if (!R.ready || !R.d_I) return rrhd_fail(RRHD_ERR_STATE, "no coupled step has run");
  RRHD_CUDA(cudaSetDevice(c->device));
  const int64_t N = c->N;
  const int64_t width = what == RRHD_RAD_G4 ? 4 : what == RRHD_RAD_MOM ? 10 * (int64_t)R.G : (int64_t)R.G * R.M;
  double *tmp = nullptr;
  RRHD_CUDA(cudaMalloc(&tmp, sizeof(double) * N * width));
  if (what == RRHD_RAD_MOM)
    k_mom_to_rows<<<grid_for(N * R.G, 256), 256, 0, c->stream>>>(N, R.G, c->d_perm, R.d_mom ? nullptr : R.d_mE,
                                                                  R.d_mF, R.d_mT, R.d_mom, tmp);
  else if (what == RRHD_RAD_G4)
    k_rows_to_host_order<double><<<grid_for(N * width, 256), 256, 0, c->stream>>>(N, width, c->d_perm, R.d_G4, tmp);
  else if (R.prec == RRHD_RAD_FP64)
    k_cdg_to_rows<double><<<grid_for(N * width, 256), 256, 0, c->stream>>>(
        N, R.M, R.G, c->d_perm, (const double *)(what == RRHD_RAD_I ? R.d_I : R.d_S), tmp);
  else
    k_cdg_to_rows<float><<<grid_for(N * width, 256), 256, 0, c->stream>>>(
        N, R.M, R.G, c->d_perm, (const float *)(what == RRHD_RAD_I ? R.d_I : R.d_S), tmp);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, tmp, sizeof(double) * N * width, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(tmp);
  RRHD_CUDA(e);
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_rad_set(rrhd_ctx *c, int32_t what, const double *in) {
  RRHD_CHECK_ARG(c && in, "null argument");
  RadState &R = c->rad;
  RRHD_CHECK_ARG(what == RRHD_RAD_I || what == RRHD_RAD_S, "bad array id");
  if (!R.ready) return rrhd_fail(RRHD_ERR_STATE, "rrhd_rad_setup has not run");
  RRHD_CUDA(cudaSetDevice(c->device));
  rrhd_status s;
  if (!R.d_I && (s = R.prec == RRHD_RAD_FP64 ? alloc_coupled<double>(c) : alloc_coupled<float>(c))) return s;
  const int64_t N = c->N, width = (int64_t)R.G * R.M;
  double *tmp = nullptr;
  RRHD_CUDA(cudaMalloc(&tmp, sizeof(double) * N * width));
  void *dst = what == RRHD_RAD_I ? R.d_I : R.d_S;
  cudaError_t e = cudaMemcpyAsync(tmp, in, sizeof(double) * N * width, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) {
    if (R.prec == RRHD_RAD_FP64)
      k_rows_to_cdg<double><<<grid_for(N * width, 256), 256, 0, c->stream>>>(N, R.M, R.G, c->d_perm, tmp,
                                                                             (double *)dst);
    else
      k_rows_to_cdg<float><<<grid_for(N * width, 256), 256, 0, c->stream>>>(N, R.M, R.G, c->d_perm, tmp,
                                                                            (float *)dst);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(tmp);
  RRHD_CUDA(e);
  return RRHD_OK;
}
