// Image-plane ray tracing: which surface triangle (or analytic body) each ray of the
// picture plane meets first, and the image and light-curve value built from it.
//
// Reference: cuda/src/ray_tracing/cuda_ray_calc.cu (RayTracing, RayTracing_Phl1445,
// InnerRayTracing, RayTracingGrid: for each ray the nearest triangle by Moeller-Trumbore,
// RayIntersectsTriangle :10-44), cuda/src/ray_tracing/cuda_ray_geo_intersect.cu (the
// Roche-lobe root search and the accretor sphere / disk test) as launched by
// cuda/src/ray_tracing/cuda_ray_interface.cu, and the per-frame image and light curve of
// solvers/ray_tracing/src/ray_tracing_calc_illum.cpp (MakeIllumAndCurve / MakeEnergyAndCurve).
//
// Parity: this translation unit is compiled without FMA contraction and every quantity is
// formed in the reference's operation order (Eigen's cross product component by component,
// dot products as (x0 + x1) + x2, IEEE division and square root), so distances are the
// reference's bit for bit and the nearest-hit choice -- strictly closer than the best so
// far, i.e. the first triangle in input order among equal distances -- is the same.
//
// Layout: the surface lives on the device as [n][9] doubles {A, B - A, C - A} plus the
// triangles' ids; rays as the reference's Ray_t records {orig[3], direction[3]}.  A block
// of 256 rays streams the triangles through shared memory in tiles of 256 (a thread
// stages one triangle), every thread testing its ray against each staged triangle
// (broadcast reads).  Work is rays x triangles FP64 tests, most rejected by the
// barycentric u test.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "rrhd_internal.h"

struct rrhd_ray_surface {
  int device = 0;
  int64_t n = 0;
  double *tri = nullptr;  // [n][9] {A, E1 = B - A, E2 = C - A}
  int32_t *ids = nullptr;
  // image-plane bins (one trace call at a time per surface)
  int32_t *bins = nullptr;    // [NB + 1] counts, then offsets
  int32_t *cursor = nullptr;  // [NB]
  int32_t *entries = nullptr; // [kMaxBins * n] triangle indices by bin
  int32_t *glist = nullptr;   // [n] triangles every ray tests
  long long *ctrl = nullptr;  // [8]: uniform flag, global count, ray box keys (x0, x1, y0, y1)
  double *ray2d = nullptr;    // [cap][2]
  int64_t ray_cap = 0;
};

namespace {

constexpr int kRayThreads = 256;
constexpr int kTile = 256;
constexpr double kEps = 1e-10;  // cuda_ray_calc.cu:12
constexpr int kNone = -1, kDisk = -2, kSphere = -3, kRoche = -4;  // ray_tracing_const.h e_ray_intersect_code

__device__ __forceinline__ double dot3(const double *a, const double *b) {
  return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}
__device__ __forceinline__ void cross3(const double *a, const double *b, double *r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}

// FaceCell records {int32 face_id; 4 bytes padding; double A[3], B[3], C[3]} -> {A, B - A, C - A}
__global__ void k_surface_prep(const unsigned char *fc, int64_t n, double *tri, int32_t *ids) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned char *r = fc + 80 * i;
  const double *v = reinterpret_cast<const double *>(r + 8);
  ids[i] = *reinterpret_cast<const int32_t *>(r);
  double *t = tri + 9 * i;
  for (int k = 0; k < 3; k++) {
    t[k] = v[k];
    t[3 + k] = v[3 + k] - v[k];
    t[6 + k] = v[6 + k] - v[k];
  }
}

// Rosh (cuda_ray_geo_intersect.cu:22-42)
__device__ double rosh(const double *o, const double *a, double t) {
  constexpr double max_potential = -1.82547, m = 0.8795180722891566;
  const double x1 = o[0] + a[0] * t;
  const double x2 = (o[1] + a[1] * t) * (o[1] + a[1] * t);
  const double x3 = (o[2] + a[2] * t) * (o[2] + a[2] * t);
  return -max_potential - ((x1 - m) * (x1 - m) + x2 + x3) * 0.5 - m / sqrt((x1 - 1) * (x1 - 1) + x2 + x3) -
         (1 - m) / sqrt(x1 * x1 + x2 + x3);
}

// FindRoshRoots + GetIntersectionWithRosh (:44-86): sign changes of the potential at 1001
// points of t in [-3, 3]; with 4 or 6 of them the second is the entry into the donor's lobe
// if it lies at x < 0.3.  Only the first 6 roots are kept (the reference's array size); the
// roots come out ascending, so the reference's sort leaves them as they are.
__device__ int roche(const double *o, const double *dir, double *dist) {
  constexpr int n = 1001;
  constexpr double a = -3, b = 3;
  const double step = (b - a) / (n - 1);
  double r1 = 0;
  int size = 0;
  double fi_1 = rosh(o, dir, a + 0 * step);
  for (int i = 1; i < n; ++i) {
    const double fi_2 = rosh(o, dir, a + (i)*step);
    if (fi_1 * fi_2 < 0) {
      if (size == 1) r1 = ((2 * a + (2. * i - 1) * step) / 2.);
      size++;
    }
    fi_1 = fi_2;
  }
  if (size == 6 || size == 4) {
    if (o[0] + dir[0] * r1 < 0.3) {
      *dist = r1;
      return kRoche;
    }
  }
  *dist = -1;
  return kNone;
}

// IntersectionWithPlane + GetIntersectionWithSphereOfDisk (:88-169); the reference
// returns "sphere" as soon as the ray meets the accretor sphere.
__device__ int sphere_disk(const double *o, const double *n) {
  const double A[3] = {1, 0, 0}, B[3] = {0, 0.9928768384869221, 0.11914522061843064}, C[3] = {2, 0, 0};
  const double pa = A[1] * (B[2] - C[2]) + B[1] * (C[2] - A[2]) + C[1] * (A[2] - B[2]);
  const double pb = A[0] * (C[2] - B[2]) + B[0] * (A[2] - C[2]) + C[0] * (B[2] - A[2]);
  const double pc = A[0] * (B[1] - C[1]) + B[0] * (C[1] - A[1]) + C[0] * (A[1] - B[1]);
  const double pd = A[0] * (C[1] * B[2] - B[1] * C[2]) + B[0] * (A[1] * C[2] - C[1] * A[2]) +
                    C[0] * (B[1] * A[2] - A[1] * B[2]);
  const double t = -(pa * o[0] + pb * o[1] + pc * o[2] + pd) / (pa * n[0] + pb * n[1] + pc * n[2]);
  const double res[3] = {n[0] * t + o[0], n[1] * t + o[1], n[2] * t + o[2]};
  const double v1[3] = {1, 0, 0}, v2[3] = {0, -0.992877, -0.119145};
  double l0 = 0, l1 = 0;
  for (int k = 0; k < 3; k++) {
    l0 += (res[k]) * v1[k];
    l1 += (res[k]) * v2[k];
  }
  const double lx = l0 - 1, ly = l1 - 0;
  const double lsq = lx * lx + ly * ly;
  const double An = dot3(n, n);
  const double oc[3] = {o[0] - 1, o[1] - 0, o[2] - 0};
  const double proj = dot3(oc, n);
  constexpr double r_s = 0.01, r_in = 0.01, r_ex = 0.06;  // ray_tracing_const.h
  const double radical = 4. * (proj * proj - An * (1 - 2 * o[0] + dot3(o, o) - r_s * r_s));
  if (radical >= 0) return kSphere;
  if (lsq < r_ex * r_ex && (lsq > r_in * r_in)) return kDisk;
  return kNone;
}

// mode 0 RayTracing / 3 RayTracingGrid: nearest triangle; 1 RayTracing_Phl1445: the
// Roche lobe first, triangles only if nearer; 2 InnerRayTracing: accretor sphere or disk,
// else the nearest triangle.
//
// Two savings that leave every decision the reference's:
//  * a block whose rays share one direction (every ray of an image plane does) stages
//    h = dir x (C - A) and det = (B - A) . h once per triangle with the tile instead of once
//    per ray and triangle (the same operations on the same operands, so the same bits);
//  * u = fl(fl(1 / det) (s . h)) is first settled without the division where it is
//    certain: u < 0 exactly when s . h is non-zero with the sign opposite to det, and
//    u > 1 certainly when |s . h| > |det| (1 + 2^-48) (two roundings move it by less than
//    2^-52); only the remaining tests divide, and then exactly as the reference does.
constexpr int kRec = 16;  // doubles per staged triangle: A, B - A, C - A, h, det, padding
__global__ void __launch_bounds__(kRayThreads)
    k_ray_trace(const double *__restrict__ rays, int64_t M, const double *__restrict__ tri,
                const int32_t *__restrict__ ids, int64_t n, int mode, int32_t *__restrict__ out,
                const long long *__restrict__ binned) {
  if (binned && binned[0] != 0) return;  // every ray shares one direction: the image-plane bins answered
  __shared__ __align__(16) double st[kTile * kRec];
  __shared__ int32_t sid[kTile];
  __shared__ double dir0[3];
  const int64_t r0 = blockIdx.x * (int64_t)kRayThreads;
  const int64_t r = r0 + threadIdx.x;
  const bool live = r < M;
  double o[3] = {0, 0, 0}, dir[3] = {0, 0, 1};
  if (live)
    for (int k = 0; k < 3; k++) {
      o[k] = rays[6 * r + k];
      dir[k] = rays[6 * r + 3 + k];
    }
  if (threadIdx.x == 0)
    for (int k = 0; k < 3; k++) dir0[k] = dir[k];
  __syncthreads();
  const bool uni = __syncthreads_and(!live || (__double_as_longlong(dir[0]) == __double_as_longlong(dir0[0]) &&
                                               __double_as_longlong(dir[1]) == __double_as_longlong(dir0[1]) &&
                                               __double_as_longlong(dir[2]) == __double_as_longlong(dir0[2])));
  int32_t best_id = kNone;
  double best = 1e10;
  bool done = !live;
  if (live && mode == 1) {
    double rd;
    if (roche(o, dir, &rd) != kNone) {
      best = rd;
      best_id = kRoche;
    }
  } else if (live && mode == 2) {
    const int code = sphere_disk(o, dir);
    if (code != kNone) {
      best_id = code;
      done = true;
    }
  }
  constexpr double kHi = 1.0 + 3.552713678800501e-15;  // 1 + 2^-48
  for (int64_t t0 = 0; t0 < n; t0 += kTile) {
    const int nt = n - t0 < kTile ? (int)(n - t0) : kTile;
    __syncthreads();
    if (threadIdx.x < nt) {
      const double *g = tri + 9 * (t0 + threadIdx.x);
      double *T = st + kRec * threadIdx.x;
      for (int k = 0; k < 9; k++) T[k] = g[k];
      if (uni) {
        double h[3];
        cross3(dir0, T + 6, h);
        T[9] = h[0], T[10] = h[1], T[11] = h[2];
        T[12] = dot3(T + 3, h);
      }
      sid[threadIdx.x] = ids[t0 + threadIdx.x];
    }
    __syncthreads();
    if (done) continue;
    for (int j = 0; j < nt; j++) {
      const double *A = st + kRec * j, *e1 = A + 3, *e2 = A + 6;
      double h[3], det;
      if (uni) {
        h[0] = A[9], h[1] = A[10], h[2] = A[11];
        det = A[12];
      } else {
        cross3(dir, e2, h);
        det = dot3(e1, h);
      }
      if (det > -kEps && det < kEps) continue;
      const double s[3] = {o[0] - A[0], o[1] - A[1], o[2] - A[2]};
      const double un = dot3(s, h);
      if (un != 0.0 && ((un < 0.0) != (det < 0.0))) continue;  // u < 0
      if (fabs(un) > fabs(det) * kHi) continue;                // u > 1
      const double inv_det = 1.0 / det;
      const double u = inv_det * un;
      if (u < 0.0 || u > 1.0) continue;
      double q[3];
      cross3(s, e1, q);
      const double v = inv_det * dot3(dir, q);
      if (v < 0.0 || u + v > 1.0) continue;
      const double d = inv_det * dot3(e2, q);
      if (d > 0.0 && d < best) {
        best = d;
        best_id = sid[j];
      }
    }
  }
  if (live) out[r] = best_id;
}

// ---------------------------------------------------------------- image-plane bins
// When every ray of a call has the same direction (an image plane), each ray tests only the
// triangles whose projection onto the plane normal to that direction can contain the ray's
// projected origin, instead of all of them; the test itself is unchanged, so the answer is
// the brute-force one.  Soundness: a triangle the reference accepts for a ray contains the
// ray's projected origin up to the rounding of its u, v (a few 1e-16 relative, amplified by
// at most 1e6 for triangles neither sliver-shaped nor seen edge-on), and its projected box is
// widened by 1e-7 of the scene size; slivers (sin of the corner angle < 1e-3), triangles seen
// within 1e-3 of edge-on and triangles covering more than kMaxBins bins go to a list every ray
// tests; triangles with |det| < 1e-10 never hit (the reference rejects them as parallel).  The
// nearest hit is the smallest (distance, input index), which is what the reference's strictly-
// closer loop in input order returns, so the bins need no order.
constexpr int kGX = 256, kGY = 128, kNB = kGX * kGY;
constexpr int kMaxBins = 128;
constexpr int64_t kMaxBinnedTriangles = 0x7fffffff / kMaxBins;  // bin offsets stay within int32
constexpr double kMargin = 1e-7;

__device__ __forceinline__ long long dkey(double x) {  // order-preserving double -> int64
  const long long b = __double_as_longlong(x);
  return b >= 0 ? b : b ^ 0x7fffffffffffffffll;
}
__device__ __forceinline__ double dval(long long k) {
  return __longlong_as_double(k >= 0 ? k : k ^ 0x7fffffffffffffffll);
}

// orthonormal u, v spanning the plane normal to d
__device__ void plane_basis(const double *d, double *u, double *v) {
  const double ax = fabs(d[0]), ay = fabs(d[1]), az = fabs(d[2]);
  const double e[3] = {(ax <= ay && ax <= az) ? 1.0 : 0.0, (!(ax <= ay && ax <= az) && ay <= az) ? 1.0 : 0.0,
                       (!(ax <= ay && ax <= az) && !(ay <= az)) ? 1.0 : 0.0};
  cross3(d, e, u);
  const double nu = sqrt(dot3(u, u));
  for (int k = 0; k < 3; k++) u[k] /= nu;
  cross3(d, u, v);
  const double nv = sqrt(dot3(v, v));
  for (int k = 0; k < 3; k++) v[k] /= nv;
}

struct Box {
  double x0, x1, y0, y1, ix, iy, margin;
};
__device__ Box ray_box(const long long *ctrl) {
  Box b;
  b.x0 = dval(ctrl[2]), b.x1 = dval(ctrl[3]), b.y0 = dval(ctrl[4]), b.y1 = dval(ctrl[5]);
  b.ix = b.x1 > b.x0 ? kGX / (b.x1 - b.x0) : 0.0;
  b.iy = b.y1 > b.y0 ? kGY / (b.y1 - b.y0) : 0.0;
  b.margin = kMargin * (1.0 + fmax(fmax(fabs(b.x0), fabs(b.x1)), fmax(fabs(b.y0), fabs(b.y1))));
  return b;
}
__device__ __forceinline__ int bin_x(const Box &b, double x) {
  const double f = floor((x - b.x0) * b.ix);
  return f < 0 ? 0 : f > kGX - 1 ? kGX - 1 : (int)f;
}
__device__ __forceinline__ int bin_y(const Box &b, double y) {
  const double f = floor((y - b.y0) * b.iy);
  return f < 0 ? 0 : f > kGY - 1 ? kGY - 1 : (int)f;
}

__global__ void k_bins_reset(int32_t *bins, long long *ctrl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= kNB) bins[i] = 0;
  if (i == 0) {
    ctrl[0] = 1;  // uniform until a ray says otherwise
    ctrl[1] = 0;
    ctrl[2] = ctrl[4] = 0x7fffffffffffffffll;
    ctrl[3] = ctrl[5] = -0x7fffffffffffffffll - 1;
  }
}

// projected ray origins, their box, and whether all directions equal ray 0's
__global__ void __launch_bounds__(256) k_rays_project(const double *__restrict__ rays, int64_t M, double *ray2d,
                                                      long long *ctrl) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const double d0[3] = {rays[3], rays[4], rays[5]};
  double u[3], v[3];
  plane_basis(d0, u, v);
  long long kx0 = 0x7fffffffffffffffll, ky0 = kx0, kx1 = -kx0 - 1, ky1 = kx1;
  bool same = true;
  if (r < M) {
    const double *ry = rays + 6 * r;
    same = __double_as_longlong(ry[3]) == __double_as_longlong(d0[0]) &&
           __double_as_longlong(ry[4]) == __double_as_longlong(d0[1]) &&
           __double_as_longlong(ry[5]) == __double_as_longlong(d0[2]);
    const double x = dot3(ry, u), y = dot3(ry, v);
    ray2d[2 * r] = x;
    ray2d[2 * r + 1] = y;
    kx0 = kx1 = dkey(x);
    ky0 = ky1 = dkey(y);
  }
  for (int o = 16; o > 0; o >>= 1) {
    kx0 = min(kx0, __shfl_xor_sync(0xffffffffu, kx0, o));
    kx1 = max(kx1, __shfl_xor_sync(0xffffffffu, kx1, o));
    ky0 = min(ky0, __shfl_xor_sync(0xffffffffu, ky0, o));
    ky1 = max(ky1, __shfl_xor_sync(0xffffffffu, ky1, o));
  }
  const bool all_same = __all_sync(0xffffffffu, same);
  if ((threadIdx.x & 31) == 0) {
    if (!all_same) atomicExch((unsigned long long *)&ctrl[0], 0ull);
    atomicMin(&ctrl[2], kx0);
    atomicMax(&ctrl[3], kx1);
    atomicMin(&ctrl[4], ky0);
    atomicMax(&ctrl[5], ky1);
  }
}

// classification of triangle t for direction d0: -1 skip, 0 every-ray list, 1 binned (range out)
__device__ int classify(const double *T, const double *d0, const double *u, const double *v, const Box &b,
                        int *bx0, int *bx1, int *by0, int *by1) {
  const double *e1 = T + 3, *e2 = T + 6;
  double h[3];
  cross3(d0, e2, h);
  const double det = dot3(e1, h);
  if (det > -kEps && det < kEps) return -1;  // rejected as parallel by the reference, whatever the ray
  double n[3];
  cross3(e1, e2, n);
  const double nn = dot3(n, n), l1 = dot3(e1, e1), l2 = dot3(e2, e2), dd = dot3(d0, d0);
  const double nd = dot3(n, d0);
  if (!(nn >= 1e-6 * l1 * l2) || !(nd * nd >= 1e-6 * nn * dd)) return 0;
  double xs[3], ys[3];
  for (int k = 0; k < 3; k++) {
    const double p[3] = {T[0] + (k == 1 ? e1[0] : k == 2 ? e2[0] : 0.0), T[1] + (k == 1 ? e1[1] : k == 2 ? e2[1] : 0.0),
                         T[2] + (k == 1 ? e1[2] : k == 2 ? e2[2] : 0.0)};
    xs[k] = dot3(p, u);
    ys[k] = dot3(p, v);
  }
  const double m = b.margin + kMargin * fmax(fmax(fabs(xs[0]), fabs(ys[0])), fmax(fabs(T[0]), fabs(T[1])));
  const double xmin = fmin(fmin(xs[0], xs[1]), xs[2]) - m, xmax = fmax(fmax(xs[0], xs[1]), xs[2]) + m;
  const double ymin = fmin(fmin(ys[0], ys[1]), ys[2]) - m, ymax = fmax(fmax(ys[0], ys[1]), ys[2]) + m;
  if (xmax < b.x0 || xmin > b.x1 || ymax < b.y0 || ymin > b.y1) return -1;  // no ray projects there
  *bx0 = bin_x(b, xmin), *bx1 = bin_x(b, xmax), *by0 = bin_y(b, ymin), *by1 = bin_y(b, ymax);
  return (*bx1 - *bx0 + 1) * (*by1 - *by0 + 1) > kMaxBins ? 0 : 1;
}

template <bool FILL>
__global__ void __launch_bounds__(256) k_tri_bin(const double *__restrict__ rays, const double *__restrict__ tri,
                                                 int64_t n, int32_t *bins, int32_t *cursor, int32_t *entries,
                                                 int32_t *glist, long long *ctrl) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n || ctrl[0] == 0) return;
  const double d0[3] = {rays[3], rays[4], rays[5]};
  double u[3], v[3];
  plane_basis(d0, u, v);
  const Box b = ray_box(ctrl);
  int bx0, bx1, by0, by1;
  const int c = classify(tri + 9 * t, d0, u, v, b, &bx0, &bx1, &by0, &by1);
  if (c < 0) return;
  if (c == 0) {
    if (!FILL) glist[atomicAdd((unsigned long long *)&ctrl[1], 1ull)] = (int32_t)t;
    return;
  }
  for (int y = by0; y <= by1; y++)
    for (int x = bx0; x <= bx1; x++) {
      const int k = y * kGX + x;
      if (FILL)
        entries[atomicAdd(&cursor[k], 1)] = (int32_t)t;
      else
        atomicAdd(&bins[k], 1);
    }
}

// exclusive scan of the kNB counts into offsets (bins[kNB] = total), cursor = offsets: a thread
// owns 32 consecutive bins (vector loads, all in flight), warp shuffles scan the thread sums
__global__ void __launch_bounds__(1024) k_bins_scan(int32_t *bins, int32_t *cursor) {
  constexpr int per = kNB / 1024;
  static_assert(per % 4 == 0, "bins per thread must be whole int4s");
  __shared__ int32_t wsum[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int4 *b4 = reinterpret_cast<int4 *>(bins + per * threadIdx.x);
  int4 *c4 = reinterpret_cast<int4 *>(cursor + per * threadIdx.x);
  int32_t v[per];
#pragma unroll
  for (int i = 0; i < per / 4; i++) {
    const int4 x = b4[i];
    v[4 * i] = x.x, v[4 * i + 1] = x.y, v[4 * i + 2] = x.z, v[4 * i + 3] = x.w;
  }
  int32_t sum = 0;
#pragma unroll
  for (int i = 0; i < per; i++) sum += v[i];
  int32_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int32_t w = wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    wsum[lane] = w;
  }
  __syncthreads();
  int32_t run = incl - sum + (warp > 0 ? wsum[warp - 1] : 0);
#pragma unroll
  for (int i = 0; i < per / 4; i++) {
    int4 x;
    x.x = run, run += v[4 * i];
    x.y = run, run += v[4 * i + 1];
    x.z = run, run += v[4 * i + 2];
    x.w = run, run += v[4 * i + 3];
    b4[i] = x;
    c4[i] = x;
  }
  if (threadIdx.x == 1023) bins[kNB] = run;
}

// one thread per ray: its bin's triangles and the every-ray list, smallest (distance, index)
__global__ void __launch_bounds__(256)
    k_ray_trace_binned(const double *__restrict__ rays, int64_t M, const double *__restrict__ ray2d,
                       const double *__restrict__ tri, const int32_t *__restrict__ ids, const int32_t *bins,
                       const int32_t *entries, const int32_t *glist, const long long *ctrl, int mode,
                       int32_t *__restrict__ out) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= M || ctrl[0] == 0) return;
  const double o[3] = {rays[6 * r], rays[6 * r + 1], rays[6 * r + 2]};
  const double dir[3] = {rays[6 * r + 3], rays[6 * r + 4], rays[6 * r + 5]};
  int32_t code = kNone;
  double best = 1e10;
  int64_t best_t = -1;
  if (mode == 1) {
    double rd;
    if (roche(o, dir, &rd) != kNone) {
      best = rd;
      code = kRoche;
    }
  } else if (mode == 2) {
    const int c = sphere_disk(o, dir);
    if (c != kNone) {
      out[r] = c;
      return;
    }
  }
  auto test = [&](int64_t t) {
    const double *A = tri + 9 * t, *e1 = A + 3, *e2 = A + 6;
    double h[3];
    cross3(dir, e2, h);
    const double det = dot3(e1, h);
    if (det > -kEps && det < kEps) return;
    const double inv_det = 1.0 / det;
    const double s[3] = {o[0] - A[0], o[1] - A[1], o[2] - A[2]};
    const double u = inv_det * dot3(s, h);
    if (u < 0.0 || u > 1.0) return;
    double q[3];
    cross3(s, e1, q);
    const double v = inv_det * dot3(dir, q);
    if (v < 0.0 || u + v > 1.0) return;
    const double d = inv_det * dot3(e2, q);
    if (d > 0.0 && (d < best || (d == best && best_t >= 0 && t < best_t))) {
      best = d;
      best_t = t;
    }
  };
  const Box b = ray_box(ctrl);
  const int k = bin_y(b, ray2d[2 * r + 1]) * kGX + bin_x(b, ray2d[2 * r]);
  const int e0 = bins[k], e1 = bins[k + 1];
  int e = e0;
  for (; e + 1 < e1; e += 2) {  // two candidates' loads in flight at once
    const int t0 = entries[e], t1 = entries[e + 1];
    test(t0);
    test(t1);
  }
  if (e < e1) test(entries[e]);
  const int ng = (int)ctrl[1];
  for (int g = 0; g < ng; g++) test(glist[g]);
  out[r] = best_t >= 0 ? ids[best_t] : code;
}

// MakeIllumAndCurve / MakeEnergyAndCurve (ray_tracing_calc_illum.cpp): pixel value by
// intersection code, curve = sum of value * pixel_factor.  One block: each thread sums a
// strided slice, then a fixed-order tree, so the curve is deterministic.
constexpr int kImgThreads = 1024;
__global__ void __launch_bounds__(kImgThreads)
    k_ray_image(const int32_t *__restrict__ codes, int64_t M, const double *__restrict__ value, int cell_size,
                double pixel_factor, double *__restrict__ image, double *__restrict__ curve, int *__restrict__ bad) {
  __shared__ double part[kImgThreads];
  double acc = 0;
  for (int64_t i = threadIdx.x; i < M; i += kImgThreads) {
    const int c = codes[i];
    double x;
    switch (c) {
      case kNone: x = 0; break;
      case kRoche: x = 0.00001; break;  // k_rosh_energy
      case kDisk: x = 5; break;         // k_disk_energy
      case kSphere: x = 10; break;      // k_accretion_energy
      default:
        if (c < 0) {
          atomicOr(bad, 1);
          x = 0;
        } else {
          x = value[c / cell_size];
        }
    }
    image[i] = x;
    acc += x * pixel_factor;
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kImgThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *curve = part[0];
}

}  // namespace

extern "C" rrhd_status rrhd_ray_surface_create(const void *face_cells, int64_t n, int32_t device,
                                               rrhd_ray_surface **out) {
  RRHD_CHECK_ARG(out && n >= 0 && (face_cells || n == 0), "bad arguments");
  RRHD_CUDA(cudaSetDevice(device));
  auto *s = new rrhd_ray_surface;
  s->device = device;
  s->n = n;
  if (n > 0) {
    unsigned char *d_fc = nullptr;
    cudaError_t e = cudaMalloc(&d_fc, 80 * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&s->tri, 72 * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&s->ids, 4 * (size_t)n);
    if (e == cudaSuccess) e = cudaMemcpy(d_fc, face_cells, 80 * (size_t)n, cudaMemcpyDefault);
    if (e == cudaSuccess) {
      k_surface_prep<<<(unsigned)((n + 255) / 256), 256>>>(d_fc, n, s->tri, s->ids);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(d_fc);
    if (e != cudaSuccess) {
      cudaFree(s->tri);
      cudaFree(s->ids);
      delete s;
      return rrhd_fail(e == cudaErrorMemoryAllocation ? RRHD_ERR_OOM : RRHD_ERR_CUDA, "ray surface: %s",
                       cudaGetErrorString(e));
    }
  }
  *out = s;
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_ray_surface_destroy(rrhd_ray_surface *s) {
  if (!s) return RRHD_OK;
  cudaSetDevice(s->device);
  cudaFree(s->tri);
  cudaFree(s->ids);
  cudaFree(s->bins);
  cudaFree(s->cursor);
  cudaFree(s->entries);
  cudaFree(s->glist);
  cudaFree(s->ctrl);
  cudaFree(s->ray2d);
  delete s;
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_ray_trace(const rrhd_ray_surface *s, const double *rays, int64_t M, int32_t mode,
                                      int32_t *codes, void *stream) {
  RRHD_CHECK_ARG(s && M >= 0, "bad arguments");
  RRHD_CHECK_ARG(mode >= 0 && mode <= 3, "mode must be 0 (surface), 1 (Roche lobe), 2 (inner) or 3 (grid)");
  if (M == 0) return RRHD_OK;
  RRHD_CHECK_ARG(rays && codes, "null rays or codes");
  RRHD_CUDA(cudaSetDevice(s->device));
  cudaStream_t st = (cudaStream_t)stream;
  if (s->n > kMaxBinnedTriangles) {
    // bin offsets are 32-bit: a surface this large takes the every-triangle kernel
    k_ray_trace<<<(unsigned)((M + kRayThreads - 1) / kRayThreads), kRayThreads, 0, st>>>(rays, M, s->tri, s->ids,
                                                                                          s->n, mode, codes, nullptr);
    RRHD_CUDA(cudaGetLastError());
    return RRHD_OK;
  }
  rrhd_ray_surface *sm = const_cast<rrhd_ray_surface *>(s);
  if (!sm->bins) {
    RRHD_CUDA(cudaMalloc(&sm->bins, sizeof(int32_t) * (kNB + 1)));
    RRHD_CUDA(cudaMalloc(&sm->cursor, sizeof(int32_t) * kNB));
    RRHD_CUDA(cudaMalloc(&sm->ctrl, sizeof(long long) * 8));
    if (s->n > 0) {
      RRHD_CUDA(cudaMalloc(&sm->entries, sizeof(int32_t) * kMaxBins * (size_t)s->n));
      RRHD_CUDA(cudaMalloc(&sm->glist, sizeof(int32_t) * (size_t)s->n));
    }
  }
  if (sm->ray_cap < M) {
    RRHD_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    cudaFree(sm->ray2d);
    sm->ray2d = nullptr;
    sm->ray_cap = 0;
    RRHD_CUDA(cudaMalloc(&sm->ray2d, sizeof(double) * 2 * (size_t)M));
    sm->ray_cap = M;
  }
  const unsigned rb = (unsigned)((M + 255) / 256), tb = (unsigned)((s->n + 255) / 256);
  k_bins_reset<<<(kNB + 1 + 255) / 256, 256, 0, st>>>(sm->bins, sm->ctrl);
  k_rays_project<<<rb, 256, 0, st>>>(rays, M, sm->ray2d, sm->ctrl);
  if (s->n > 0) {
    k_tri_bin<false><<<tb, 256, 0, st>>>(rays, s->tri, s->n, sm->bins, sm->cursor, sm->entries, sm->glist, sm->ctrl);
    k_bins_scan<<<1, 1024, 0, st>>>(sm->bins, sm->cursor);
    k_tri_bin<true><<<tb, 256, 0, st>>>(rays, s->tri, s->n, sm->bins, sm->cursor, sm->entries, sm->glist, sm->ctrl);
  }
  k_ray_trace_binned<<<rb, 256, 0, st>>>(rays, M, sm->ray2d, s->tri, s->ids, sm->bins, sm->entries, sm->glist,
                                         sm->ctrl, mode, codes);
  // rays of several directions: every ray against every triangle
  k_ray_trace<<<(unsigned)((M + kRayThreads - 1) / kRayThreads), kRayThreads, 0, st>>>(rays, M, s->tri, s->ids, s->n,
                                                                                        mode, codes, sm->ctrl);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_ray_image(const int32_t *codes, int64_t M, const double *value, int32_t cell_size,
                                      double pixel_factor, double *image, double *curve, int32_t *bad,
                                      void *stream) {
  RRHD_CHECK_ARG(M >= 0 && cell_size > 0, "bad arguments");
  RRHD_CHECK_ARG(codes && image && curve && bad && (value || M == 0), "null argument");
  k_ray_image<<<1, kImgThreads, 0, (cudaStream_t)stream>>>(codes, M, value, cell_size, pixel_factor, image, curve,
                                                          bad);
  RRHD_CUDA(cudaGetLastError());
  return RRHD_OK;
}

// MakeRays(num_frame) of ray_tracing_build_plane.cpp on the host (constants of
// ray_tracing_const.h, GRB_TASK plane): [600 * 300][6] rays, ray i * 300 + j for pixel (i, j).
namespace {
void host_cross(const double *a, const double *b, double *r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}
double host_dot(const double *a, const double *b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }
void host_normalize(double *v) {
  const double z = host_dot(v, v);
  if (z > 0) {
    const double s = std::sqrt(z);
    for (int k = 0; k < 3; k++) v[k] = v[k] / s;
  }
}
}  // namespace

extern "C" rrhd_status rrhd_ray_make_rays(int32_t frame, double *rays) {
  RRHD_CHECK_ARG(rays, "null rays");
  const double PIv = 3.1415926535897932384626433832795, com[3] = {0.879518, 0, 0};
  constexpr int nw = 600, nh = 300, nframes = 120;
  const double width = 1.2, height = 0.6, above = 0.1;
  const double start_angle = 2 * PIv / nframes * frame;
  const double start[3] = {std::cos(start_angle) + com[0], std::sin(start_angle) + com[1], above + com[2]};
  double dir[3] = {com[0] - start[0], com[1] - start[1], com[2] - start[2]};
  host_normalize(dir);
  // intersection::SetBasis (lib/geometry/src/intersections.cpp:3-40): rows v2, v1, normal
  double v1[3], v2[3];
  if (std::fabs(dir[1]) < 1e-20) {
    v1[0] = 0, v1[1] = 1, v1[2] = 0;
  } else {
    v1[0] = 1, v1[2] = 0;
    v1[1] = -(dir[0] * v1[0] + dir[2] * v1[2]) / dir[1];
  }
  if (dir[1] < 0)
    for (int k = 0; k < 3; k++) v1[k] = -v1[k];
  host_cross(dir, v1, v2);
  host_normalize(v1);
  host_normalize(v2);
  const double ap0 = -(width / 2), ap1 = -(height / 2);
  const double step_x = width / nw, step_y = height / nh;
  for (int i = 0; i < nw; ++i)
    for (int j = 0; j < nh; ++j) {
      const double x = ap0 + i * step_x, y = ap1 + j * step_y, z = 0;
      double *r = rays + 6 * ((int64_t)i * nh + j);
      // basis.transpose() * (x, y, z): row k = (v2[k] x + v1[k] y) + dir[k] z
      const double o3[3] = {(v2[0] * x + v1[0] * y) + dir[0] * z, (v2[1] * x + v1[1] * y) + dir[1] * z,
                            (v2[2] * x + v1[2] * y) + dir[2] * z};
      for (int k = 0; k < 3; k++) {
        r[k] = o3[k] + start[k];
        r[3 + k] = dir[k];
      }
    }
  return RRHD_OK;
}
