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
                const int32_t *__restrict__ ids, int64_t n, int mode, int32_t *__restrict__ out) {
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
  k_ray_trace<<<(unsigned)((M + kRayThreads - 1) / kRayThreads), kRayThreads, 0, (cudaStream_t)stream>>>(
      rays, M, s->tri, s->ids, s->n, mode, codes);
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
