// Drop-in replacement for cuda/src/ray_tracing/cuda_ray_interface.cu (with cuda_ray_init.cu and
// the kernels of cuda_ray_calc.cu / cuda_ray_geo_intersect.cu): the functions
// cuda::ray_tracing::interface::{InitDevice, ClearDevice, StartTracing, StartTracingGrid,
// FindInnerIntersection, TracingGrid} (cuda/include/interface/cuda_ray_interface.h) on the B200
// library's C ABI.  Link it, with radrhd_solver_b200/librrhd.so and the CUDA runtime, in place of
// those files; ray_tracing::RunRayTracing and the light-curve code stay unchanged.
//
// The reference's mapping of calls to kernels is kept: StartTracing runs RayTracing_Phl1445 (the
// donor's Roche lobe, then nearer triangles), StartTracingGrid RayTracing, FindInnerIntersection
// InnerRayTracing (accretor sphere / disk first), TracingGrid RayTracingGrid.  FaceCell and Ray_t
// records go to the device as they are.  Intersection codes are the reference's, ray for ray.
#if defined USE_CUDA
#include "cuda_ray_interface.h"

#include "rrhd.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

namespace {
rrhd_ray_surface *g_surf = nullptr;
double *d_rays = nullptr;
int32_t *d_codes = nullptr;
size_t g_cap = 0;

void die(const char *what, const char *msg) {
  std::fprintf(stderr, "ray tracing interface (B200): %s: %s\n", what, msg);
  std::abort();
}

int trace(const std::vector<Ray_t> &rays, std::vector<int> &out, int mode) {
  static_assert(sizeof(Ray_t) == 6 * sizeof(double), "Ray_t must be {orig[3], direction[3]}");
  const size_t M = rays.size();
  out.resize(M);
  if (M == 0) return e_completion_success;
  if (M > g_cap) {
    cudaFree(d_rays);
    cudaFree(d_codes);
    d_rays = nullptr;
    d_codes = nullptr;
    g_cap = 0;
    if (cudaMalloc(&d_rays, sizeof(Ray_t) * M) != cudaSuccess || cudaMalloc(&d_codes, sizeof(int32_t) * M) != cudaSuccess)
      die("cudaMalloc", "out of device memory");
    g_cap = M;
  }
  if (cudaMemcpy(d_rays, rays.data(), sizeof(Ray_t) * M, cudaMemcpyHostToDevice) != cudaSuccess)
    die("cudaMemcpy", "rays");
  if (rrhd_ray_trace(g_surf, d_rays, (int64_t)M, mode, d_codes, nullptr) != RRHD_OK)
    die("rrhd_ray_trace", rrhd_last_error());
  if (cudaMemcpy(out.data(), d_codes, sizeof(int32_t) * M, cudaMemcpyDeviceToHost) != cudaSuccess)
    die("cudaMemcpy", "intersections");
  return e_completion_success;
}
}  // namespace

void cuda::ray_tracing::interface::InitDevice(const std::vector<FaceCell> &faces_host,
                                              const std::vector<Ray_t> &rays_host) {
  static_assert(sizeof(FaceCell) == 80, "FaceCell must be {int face_id; Face{A, B, C}}");
  (void)rays_host;
  if (g_surf) rrhd_ray_surface_destroy(g_surf);
  if (rrhd_ray_surface_create(faces_host.data(), (int64_t)faces_host.size(), 0, &g_surf) != RRHD_OK)
    die("rrhd_ray_surface_create", rrhd_last_error());
}

void cuda::ray_tracing::interface::ClearDevice() {
  rrhd_ray_surface_destroy(g_surf);
  g_surf = nullptr;
  cudaFree(d_rays);
  cudaFree(d_codes);
  d_rays = nullptr;
  d_codes = nullptr;
  g_cap = 0;
}

int cuda::ray_tracing::interface::StartTracing(const std::vector<Ray_t> &rays, std::vector<IntId> &out) {
  return trace(rays, out, RRHD_RAY_ROCHE);
}
int cuda::ray_tracing::interface::StartTracingGrid(const std::vector<Ray_t> &rays, std::vector<int> &out) {
  return trace(rays, out, RRHD_RAY_SURFACE);
}
int cuda::ray_tracing::interface::FindInnerIntersection(const std::vector<Ray_t> &rays, std::vector<IntId> &out) {
  return trace(rays, out, RRHD_RAY_INNER);
}
int cuda::ray_tracing::interface::TracingGrid(const std::vector<Ray_t> &rays, std::vector<IntId> &out) {
  return trace(rays, out, RRHD_RAY_GRID);
}
#endif
