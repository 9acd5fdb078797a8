// Test infrastructure, not product code: the checker, never the thing measured.
//
// Runs the reference's own Compton scattering kernels on the CPU: the frequency-coupled
// full-spectrum one, and (this file compiled a second time with RRHD_SHIM_ONE) the
// single-frequency one of cuda_scat_spectrum.cu:41-83, Get_spectrum_multi_device.
// The device source (cuda/src/short_characteristics/separate_gpu/spectrum/
// cuda_scat_full_spectrum.cu:61-118, Get_full_spectrum_multi_device) is included from
// its place in the reference tree and compiled by g++ with this file, with the host
// stand-ins of <cuda_runtime.h>
// and <device_launch_parameters.h> under oracle/host_cuda/: the CUDA qualifiers are
// no-ops and blockIdx / blockDim / threadIdx are per-thread host variables.  One call
// of the kernel body per (cell, direction, frequency), with blockDim = (1,1,1) and
// blockIdx = (cell, direction, frequency), is one thread of the reference launch.
//
// The reference's kernel reads one element past a row of the intensity when the
// shifted frequency lies above the spectrum (get_frq_idx returns N_Frq there; the
// value read is then replaced by zero).  The intensity is therefore copied into a
// buffer with a zero pad behind it, so that this read stays inside the allocation.
#ifndef RRHD_SHIM_ONE
#include "cuda_scat_full_spectrum.cu"
#else
#include "cuda_scat_spectrum.cu"
#endif

#include <omp.h>

#include <cstdint>
#include <cstring>
#include <vector>

#ifndef RRHD_SHIM_ONE
thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;

namespace {
constexpr int kFrq = 100; // N_Frq, cuda_scat_full_spectrum.cu:47
constexpr int kPad = 128;
} // namespace

// S[(i * out_stride + k) * 100 + f], k < dir_count, out direction dir_disp + k;
// I[(i * M + d) * 100 + f]; vel[3 * i]; dirs[3 * d]; areas[d].
extern "C" int ref_compton_full_spectrum(int32_t M, const double *dirs, const double *areas, double full_area,
                                         int64_t cells, const double *I, const double *vel, int32_t dir_disp,
                                         int32_t dir_count, int32_t out_stride, double *S, int nthreads) {
  using namespace cuda::geo;
  if (M <= 0 || cells < 0 || dir_count < 0 || dir_disp < 0 || dir_disp + dir_count > M || out_stride < dir_count)
    return -1;
  std::vector<direction_device_t> dd(M);
  for (int d = 0; d < M; d++) {
    dd[d].dir = Vector3(dirs[3 * d], dirs[3 * d + 1], dirs[3 * d + 2]);
    dd[d].area = areas[d];
  }
  grid_directions_device_t gd;
  gd.size = M;
  gd.directions = dd.data();
  gd.full_area = full_area;

  const size_t n_in = (size_t)cells * M * kFrq;
  std::vector<double> illum(n_in + kPad, 0.0);
  std::memcpy(illum.data(), I, n_in * sizeof(double));
  std::vector<Vector3> v(cells);
  for (int64_t i = 0; i < cells; i++) v[i] = Vector3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);

  grid_device_t g;
  g.size = cells;
  g.loc_size_gpu = cells;
  g.shift_gpu = 0;
  g.loc_size_params = cells;
  g.shift_params = 0;
  g.local_scattering_size = out_stride;
  g.local_scattering_disp = dir_disp;
  g.illum = illum.data();
  g.int_scattering = S;
  g.velocity = v.data();

  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (int64_t i = 0; i < cells; i++) {
    blockDim = dim3{1, 1, 1};
    threadIdx = uint3{0, 0, 0};
    for (int k = 0; k < dir_count; k++)
      for (int f = 0; f < kFrq; f++) {
        blockIdx = uint3{(unsigned)i, (unsigned)k, (unsigned)f};
        cuda::kernel::Get_full_spectrum_multi_device(&gd, &g, dir_count);
      }
  }
  return 0;
}

// N_Frq of the compiled kernel (cuda_scat_full_spectrum.cu:47).
extern "C" int ref_compton_n_frq() { return N_Frq; }

// The kernel's frequency grid (get_frq, :54-59) and bin search (get_frq_idx, :50-53).
extern "C" double ref_compton_get_frq(int idx) { return get_frq(idx); }
extern "C" int ref_compton_get_frq_idx(double frq) { return get_frq_idx(frq); }

// GammaC (:22-44) for one pair of directions; returns the weight, frq1 through *frq1.
extern "C" double ref_compton_gamma(double cosf, double v, const double *vel, double frq, double lorenz,
                                    const double *main_dir, const double *scat_dir, double *frq1) {
  return GammaC(cosf, v, Vector3(vel[0], vel[1], vel[2]), frq, lorenz, Vector3(main_dir[0], main_dir[1], main_dir[2]),
                Vector3(scat_dir[0], scat_dir[1], scat_dir[2]), *frq1);
}

#else  // RRHD_SHIM_ONE

// S[i * out_stride + k], I[i * M + d] at the single frequency frq.
extern "C" int ref_compton_spectrum(int32_t M, const double *dirs, const double *areas, double full_area,
                                    int64_t cells, const double *I, const double *vel, double frq, int32_t dir_disp,
                                    int32_t dir_count, int32_t out_stride, double *S, int nthreads) {
  using namespace cuda::geo;
  if (M <= 0 || cells < 0 || dir_count < 0 || dir_disp < 0 || dir_disp + dir_count > M || out_stride < dir_count)
    return -1;
  std::vector<direction_device_t> dd(M);
  for (int d = 0; d < M; d++) {
    dd[d].dir = Vector3(dirs[3 * d], dirs[3 * d + 1], dirs[3 * d + 2]);
    dd[d].area = areas[d];
  }
  grid_directions_device_t gd;
  gd.size = M;
  gd.directions = dd.data();
  gd.full_area = full_area;
  std::vector<Vector3> v(cells);
  for (int64_t i = 0; i < cells; i++) v[i] = Vector3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
  grid_device_t g;
  g.size = cells;
  g.loc_size_gpu = cells;
  g.shift_gpu = 0;
  g.loc_size_params = cells;
  g.shift_params = 0;
  g.local_scattering_size = out_stride;
  g.local_scattering_disp = dir_disp;
  g.illum = const_cast<double *>(I);
  g.int_scattering = S;
  g.velocity = v.data();
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (int64_t i = 0; i < cells; i++) {
    blockDim = dim3{1, 1, 1};
    threadIdx = uint3{0, 0, 0};
    for (int k = 0; k < dir_count; k++) {
      blockIdx = uint3{(unsigned)i, (unsigned)k, 0};
      cuda::kernel::Get_spectrum_multi_device(&gd, &g, frq, dir_count);
    }
  }
  return 0;
}
#endif
