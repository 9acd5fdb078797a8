// Test infrastructure, not product code: the checker, never the thing measured.
//
// Runs the reference's own ray-tracing kernels on the CPU.  The device sources
// cuda/src/ray_tracing/cuda_ray_calc.cu (RayTracing, RayTracing_Phl1445, InnerRayTracing,
// RayTracingGrid) and cuda/src/ray_tracing/cuda_ray_geo_intersect.cu (the Roche-lobe and
// accretor sphere / disk intersections) are compiled in place by g++ with the host
// stand-ins of <cuda_runtime.h> / <device_launch_parameters.h> under oracle/host_cuda/,
// and so is the host code that builds the image-plane rays
// (solvers/ray_tracing/src/ray_tracing_build_plane.cpp MakeRays,
// lib/geometry/src/intersections.cpp SetBasis).  One call of a kernel body with
// blockIdx.x = ray, blockDim.x = 1 is one thread of the reference launch.
#include <omp.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "cuda_ray_calc.h"
#include "cuda_ray_geo_intersect.h"
#include "ray_tracing_build_plane.h"
#include "ray_tracing_const.h"

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;

namespace rt = cuda::ray_tracing;

// rays [M][6] = {orig, dir}; faces [N] {id, A[3], B[3], C[3]}; mode 0 RayTracing,
// 1 RayTracing_Phl1445, 2 InnerRayTracing, 3 RayTracingGrid.
extern "C" int ref_ray_trace(int32_t mode, const double *rays, int32_t M, const int32_t *ids, const double *abc,
                             int32_t N, int32_t *out, int nthreads) {
  std::vector<rt::Ray> r(M);
  for (int i = 0; i < M; i++) {
    r[i].orig = Vector3(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]);
    r[i].dir = Vector3(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]);
  }
  std::vector<rt::Face> f(N);
  for (int j = 0; j < N; j++) {
    f[j].id = ids[j];
    f[j].A = Vector3(abc[9 * j], abc[9 * j + 1], abc[9 * j + 2]);
    f[j].B = Vector3(abc[9 * j + 3], abc[9 * j + 4], abc[9 * j + 5]);
    f[j].C = Vector3(abc[9 * j + 6], abc[9 * j + 7], abc[9 * j + 8]);
  }
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
  for (int i = 0; i < M; i++) {
    blockDim = dim3{1, 1, 1};
    threadIdx = uint3{0, 0, 0};
    blockIdx = uint3{(unsigned)i, 0, 0};
    switch (mode) {
      case 0: rt::RayTracing(M, r.data(), N, f.data(), out); break;
      case 1: rt::RayTracing_Phl1445(M, r.data(), N, f.data(), out); break;
      case 2: rt::InnerRayTracing(M, r.data(), N, f.data(), out); break;
      default: rt::RayTracingGrid(M, r.data(), N, f.data(), out); break;
    }
  }
  return 0;
}

// RayIntersectsTriangle for one ray and one triangle: the distance (or -1).
extern "C" double ref_ray_triangle(const double *ray, const double *abc) {
  rt::Ray r;
  r.orig = Vector3(ray[0], ray[1], ray[2]);
  r.dir = Vector3(ray[3], ray[4], ray[5]);
  rt::Face f;
  f.id = 0;
  f.A = Vector3(abc[0], abc[1], abc[2]);
  f.B = Vector3(abc[3], abc[4], abc[5]);
  f.C = Vector3(abc[6], abc[7], abc[8]);
  Vector3 p;
  return rt::RayIntersectsTriangle(r, f, p);
}

// GetIntersectionWithRosh: the code, the distance through *dist.
extern "C" int ref_ray_roche(const double *ray, double *dist) {
  rt::Ray r;
  r.orig = Vector3(ray[0], ray[1], ray[2]);
  r.dir = Vector3(ray[3], ray[4], ray[5]);
  return rt::GetIntersectionWithRosh(r, dist);
}

// The image-plane rays of frame `frame` (MakeRays): [600 * 300][6], ray i * 300 + j.
extern "C" int ref_ray_make_rays(int frame, double *rays) {
  std::vector<Ray_t> r;
  ray_tracing::MakeRays(frame, r);
  for (size_t i = 0; i < r.size(); i++)
    for (int a = 0; a < 3; a++) {
      rays[6 * i + a] = r[i].orig[a];
      rays[6 * i + 3 + a] = r[i].direction[a];
    }
  return (int)r.size();
}
