// Test infrastructure, not product code.
//
// Drives the ray-tracing drop-in adapter (adapter/cuda_ray_interface_b200.cpp) through the
// reference's own interface and types: std::vector<FaceCell> and std::vector<Ray_t> handed to
// cuda::ray_tracing::interface::InitDevice / StartTracing / StartTracingGrid /
// FindInnerIntersection / TracingGrid / ClearDevice, as ray_tracing::RunRayTracing does.
#include <cstdint>
#include <vector>

#include "cuda_ray_interface.h"

namespace ri = cuda::ray_tracing::interface;

// ids [n], abc [n][9]; rays [M][6]; call 0 StartTracing, 1 StartTracingGrid,
// 2 FindInnerIntersection, 3 TracingGrid; out [M]
extern "C" int rayad_run(const int32_t *ids, const double *abc, int64_t n, const double *rays, int64_t M, int call,
                         int32_t *out) {
  std::vector<FaceCell> faces;
  faces.reserve(n);
  for (int64_t i = 0; i < n; i++) {
    Face f;
    f.A = Vector3(abc[9 * i], abc[9 * i + 1], abc[9 * i + 2]);
    f.B = Vector3(abc[9 * i + 3], abc[9 * i + 4], abc[9 * i + 5]);
    f.C = Vector3(abc[9 * i + 6], abc[9 * i + 7], abc[9 * i + 8]);
    faces.push_back(FaceCell(ids[i], f));
  }
  std::vector<Ray_t> r(M);
  for (int64_t i = 0; i < M; i++)
    r[i] = Ray_t(Vector3(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]),
                 Vector3(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]));
  ri::InitDevice(faces, r);
  std::vector<IntId> res;
  std::vector<int> res_grid;
  int rc;
  switch (call) {
    case 0: rc = ri::StartTracing(r, res); break;
    case 1: rc = ri::StartTracingGrid(r, res_grid); break;
    case 2: rc = ri::FindInnerIntersection(r, res); break;
    default: rc = ri::TracingGrid(r, res); break;
  }
  const std::vector<int> &o = call == 1 ? res_grid : res;
  for (int64_t i = 0; i < M; i++) out[i] = o[i];
  ri::ClearDevice();
  return rc;
}
