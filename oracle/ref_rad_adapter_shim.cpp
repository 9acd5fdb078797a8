// Test infrastructure, not product code.
//
// Drives the radiation drop-in adapter (adapter/cuda_interface_sep_b200.cpp) through the
// reference's own interface and types: a grid_t and a grid_directions_t as the illum drivers
// hold them, then cuda::interface::separate_device::InitDevice / CalculateIntScatteringAsync /
// ClearHost / ClearDevice exactly as those drivers call them.  Compiled a second time with
// SPECTRUM it drives SendVelocity / CalculateFullSpectrumIntScattering /
// CalculateSpectrumIntScattering the same way.
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
#ifdef SPECTRUM
  r->grid->size_frq = 100;  // N_Frq of the full-spectrum kernel
  r->grid->cells.resize(N);
  r->grid->frq_grid.assign(2, 0.0);
  r->grid->cur_frq_id = 0;
#endif
  r->dirs = new grid_directions_t(M);
  for (int k = 0; k < M; k++) {
    r->dirs->directions[k].dir = Vector3(w[3 * k], w[3 * k + 1], w[3 * k + 2]);
    r->dirs->directions[k].area = areas[k];
  }
  r->dirs->full_area = full_area;
  if (sep::InitDevice(*r->dirs, *r->grid) != e_completion_success) return nullptr;
  return r;
}

#ifdef ON_FULL_ILLUM_ARRAYS
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
#endif

#ifdef SPECTRUM
static void send_velocity(RadAdapter *r, const double *vel) {
  grid_t &g = *r->grid;
  for (int64_t i = 0; i < g.size; i++) g.cells[i].phys_val.v = Vector3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
  sep::SendVelocity(g);
}

// I [N][M][100], vel [N][3] in; S [N][end - start][100] out
extern "C" int radad_full_spectrum(void *p, const double *I, const double *vel, int32_t start, int32_t end, double *S) {
  RadAdapter *r = (RadAdapter *)p;
  grid_t &g = *r->grid;
  const int64_t N = g.size, M = r->dirs->size;
  send_velocity(r, vel);
  std::memcpy(g.Illum, I, sizeof(double) * N * M * 100);
  const int rc = sep::CalculateFullSpectrumIntScattering(*r->dirs, g, start, end, cuda::e_cuda_scattering_1);
  if (rc != e_completion_success) return rc;
  std::memcpy(S, g.scattering, sizeof(double) * N * (end - start) * 100);
  return 0;
}

// I [N][M] at the frequency 0.5 (lo + hi) (frq_grid = {lo, hi}, cur_frq_id = 0); S [N][end - start]
extern "C" int radad_spectrum(void *p, const double *I, const double *vel, double lo, double hi, int32_t start,
                              int32_t end, double *S) {
  RadAdapter *r = (RadAdapter *)p;
  grid_t &g = *r->grid;
  const int64_t N = g.size, M = r->dirs->size;
  g.frq_grid[0] = lo;
  g.frq_grid[1] = hi;
  send_velocity(r, vel);
  std::memcpy(g.Illum, I, sizeof(double) * N * M);
  const int rc = sep::CalculateSpectrumIntScattering(*r->dirs, g, start, end, cuda::e_cuda_scattering_1);
  if (rc != e_completion_success) return rc;
  std::memcpy(S, g.scattering, sizeof(double) * N * (end - start));
  return 0;
}
#endif

extern "C" void radad_destroy(void *p) {
  RadAdapter *r = (RadAdapter *)p;
  sep::ClearHost(*r->grid);
  sep::ClearDevice();
  delete r->dirs;
  delete r;
}
