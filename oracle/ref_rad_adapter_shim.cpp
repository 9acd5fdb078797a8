// Test infrastructure, not product code.
//
// Drives the radiation drop-in adapter (adapter/cuda_interface_sep_b200.cpp) through the
// reference's own interface and types: a grid_t and a grid_directions_t as the illum drivers
// hold them, then cuda::interface::separate_device::InitDevice / CalculateIntScatteringAsync /
// ClearHost / ClearDevice exactly as those drivers call them.
#include <cstdint>
#include <cstring>

#include "cuda_interface.h"
#include "cuda_multi_interface.h"
#include "cuda_struct.h"

namespace sep = cuda::interface::separate_device;

namespace {
struct RadAdapter {
  grid_t *grid;
  grid_directions_t *dirs;
};
}  // namespace

extern "C" void *radad_create(int64_t N, int32_t M, const double *w, const double *areas, double full_area) {
  RadAdapter *r = new RadAdapter;
  r->grid = new grid_t();  // kept for the process: its destructor lives in the reference's grid module
  r->grid->size = N;
  r->dirs = new grid_directions_t(M);
  for (int k = 0; k < M; k++) {
    r->dirs->directions[k].dir = Vector3(w[3 * k], w[3 * k + 1], w[3 * k + 2]);
    r->dirs->directions[k].area = areas[k];
  }
  r->dirs->full_area = full_area;
  if (sep::InitDevice(*r->dirs, *r->grid) != e_completion_success) return nullptr;
  return r;
}

// I [N][M] in; S [N][end - start], E [N], F [N][3], T [N][9] out
extern "C" int radad_scatter(void *p, const double *I, int32_t start, int32_t end, double *S, double *E, double *F,
                             double *T) {
  RadAdapter *r = (RadAdapter *)p;
  grid_t &g = *r->grid;
  const int64_t N = g.size, M = r->dirs->size;
  std::memcpy(g.Illum, I, sizeof(double) * N * M);
  const int rc = sep::CalculateIntScatteringAsync(*r->dirs, g, start, end, cuda::e_cuda_scattering_1);
  if (rc != e_completion_success) return rc;
  std::memcpy(S, g.scattering, sizeof(double) * N * (end - start));
  std::memcpy(E, g.energy, sizeof(double) * N);
  std::memcpy(F, g.stream, sizeof(double) * 3 * N);
  std::memcpy(T, g.impuls, sizeof(double) * 9 * N);
  return 0;
}

extern "C" void radad_destroy(void *p) {
  RadAdapter *r = (RadAdapter *)p;
  sep::ClearHost(*r->grid);
  sep::ClearDevice();
  delete r->dirs;
  delete r;
}
