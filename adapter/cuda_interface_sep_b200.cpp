// Drop-in replacement for the reference's single-GPU radiation interface
// (cuda/src/short_characteristics/separate_gpu/cuda_interface_sep_mem.cu, cuda_interface_sep_solve.cu,
// cuda_multi_init.cu and cuda/src/interface/cuda_interface_stream.cu): the functions the illum
// and RadRHD drivers call -- cuda::interface::separate_device::{InitDevice, ClearDevice,
// ClearHost, CalculateIntScatteringAsync, CalculateAllParamAsync} and
// cuda::interface::{SetStreams, CudaWait, CudaSyncStream, CudaSendIllumAsync}
// (declared in cuda/include/short_characteristics/separate_gpu/cuda_multi_interface.h:35-57 and
// cuda/include/interface/cuda_interface.h:114-136) -- implemented on the B200 library's C ABI.
// Link it, with radrhd_solver_b200/librrhd.so and the CUDA runtime, in place of those files.
//
// As in the reference (SINGLE_GPU, one part): InitDevice allocates the pinned host arrays
// grid.Illum [N][M], grid.scattering [N][M], grid.energy, grid.stream, grid.impuls and the
// device copies; CalculateIntScatteringAsync sends Illum, computes the scattering integral of
// the output directions start_dir .. end_dir - 1 into grid.scattering [N][end - start] and, when
// grid.energy is allocated, the energy / stream / impulse moments; it returns with the results
// in host memory (the reference synchronises its streams before returning).  The scattering is
// the FP64 O(M^2) sum in the reference kernel's order (GetS_MPI_multi_device,
// cuda_scattering.cu:82-105) and the moments those of MakeIllumParam (cuda_illum_sep_param.cu),
// bit for bit.  The tensor a cell's impulse moment is symmetric, so Eigen's column-major Matrix3
// and the library's row-major [3][3] hold the same numbers.
//
// In a SPECTRUM build the same file also stands behind separate_device::{SendVelocity,
// CalculateSpectrumIntScattering, CalculateFullSpectrumIntScattering}
// (cuda/src/short_characteristics/separate_gpu/spectrum/cuda_interface_spectrum.cu): Illum holds
// [N][M][size_frq] values (SAVE_FULL_SPECTRUM), the scattering the Compton integral of the
// reference's kernels (rrhd_compton_full_spectrum / rrhd_compton_spectrum).
#if defined USE_CUDA && defined SOLVERS && defined ILLUM
#include "cuda_interface.h"
#include "cuda_multi_interface.h"
#include "cuda_struct.h"

#include "rrhd.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

cudaStream_t cuda_streams[cuda::e_cuda_streams_count];  // cuda_interface_stream.cu:11

namespace {
rrhd_dirs *g_dirs = nullptr;
double *d_I = nullptr, *d_S = nullptr, *d_E = nullptr, *d_F = nullptr, *d_T = nullptr, *d_vel = nullptr;
int64_t g_N = 0, g_M = 0, g_frq = 1;
bool g_streams = false;

void die(const char *what, const char *msg) {
  std::fprintf(stderr, "radiation interface (B200): %s: %s\n", what, msg);
  std::abort();
}
void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) die(what, cudaGetErrorString(e));
}
void check(rrhd_status s, const char *what) {
  if (s != RRHD_OK) die(what, rrhd_last_error());
}
}  // namespace

void cuda::interface::CudaWait() { check(cudaDeviceSynchronize(), "cudaDeviceSynchronize"); }

void cuda::interface::CudaSyncStream(const e_cuda_stream_id_t stream_id) {
  check(cudaStreamSynchronize(cuda_streams[stream_id]), "cudaStreamSynchronize");
}

// the reference's three streams with their priorities (cuda_interface_stream.cu:17-26)
void cuda::interface::SetStreams() {
  if (g_streams) return;
  int lo = 0, hi = 0;
  cudaDeviceGetStreamPriorityRange(&lo, &hi);
  check(cudaStreamCreateWithPriority(&cuda_streams[e_cuda_scattering_1], cudaStreamNonBlocking, hi), "streams");
  check(cudaStreamCreateWithPriority(&cuda_streams[e_cuda_scattering_2], cudaStreamNonBlocking, (hi + lo) / 2),
        "streams");
  check(cudaStreamCreateWithPriority(&cuda_streams[e_cuda_params], cudaStreamNonBlocking, lo), "streams");
  g_streams = true;
}

// part of Illum (size values from shift) to the device (cuda_interface_stream.cu:28-32)
void cuda::interface::CudaSendIllumAsync(const IdType size, const IdType shift, const Type *Illum_host) {
  check(cudaMemcpyAsync(d_I + shift, Illum_host + shift, size * sizeof(Type), cudaMemcpyHostToDevice,
                        cuda_streams[e_cuda_scattering_1]),
        "CudaSendIllumAsync");
}

int cuda::interface::separate_device::InitDevice(const grid_directions_t &grid_dir, grid_t &grid) {
  SetStreams();
  g_N = grid.size;
  g_M = grid_dir.size;
  std::vector<double> w(3 * g_M), a(g_M);
  for (int64_t k = 0; k < g_M; k++) {
    a[k] = grid_dir.directions[k].area;
    for (int x = 0; x < 3; x++) w[3 * k + x] = grid_dir.directions[k].dir[x];
  }
  check(rrhd_dirs_create((int32_t)g_M, w.data(), a.data(), grid_dir.full_area, 0, &g_dirs), "rrhd_dirs_create");
  g_frq = 1;
#ifdef SAVE_FULL_SPECTRUM
  g_frq = grid.size_frq;
#endif
  // host arrays as the reference's InitDevice sizes them (cuda_interface_sep_mem.cu:91-108)
  const size_t nm = sizeof(double) * g_N * g_M * g_frq;
  check(cudaMallocHost(&grid.Illum, nm), "cudaMallocHost");
  check(cudaMallocHost(&grid.scattering, sizeof(double) * grid_dir.loc_size * g_N * g_frq), "cudaMallocHost");
#ifdef ON_FULL_ILLUM_ARRAYS
  check(cudaMallocHost(&grid.energy, sizeof(Type) * g_N), "cudaMallocHost");
  check(cudaMallocHost(&grid.stream, sizeof(Vector3) * g_N), "cudaMallocHost");
  check(cudaMallocHost(&grid.impuls, sizeof(Matrix3) * g_N), "cudaMallocHost");
#endif
#ifdef SPECTRUM
  check(cudaMalloc(&d_vel, sizeof(double) * 3 * g_N), "cudaMalloc");
#endif
  check(cudaMalloc(&d_I, nm), "cudaMalloc");
  check(cudaMalloc(&d_S, nm), "cudaMalloc");
  return e_completion_success;
}

void cuda::interface::separate_device::ClearDevice() {
  cudaFree(d_I), cudaFree(d_S), cudaFree(d_E), cudaFree(d_F), cudaFree(d_T), cudaFree(d_vel);
  d_I = d_S = d_E = d_F = d_T = d_vel = nullptr;
  if (g_dirs) rrhd_dirs_destroy(g_dirs);
  g_dirs = nullptr;
}

void cuda::interface::separate_device::ClearHost(grid_t &grid) {
  cudaFreeHost(grid.Illum), cudaFreeHost(grid.scattering);
  grid.Illum = grid.scattering = nullptr;
#ifdef ON_FULL_ILLUM_ARRAYS
  cudaFreeHost(grid.energy), cudaFreeHost(grid.stream), cudaFreeHost(grid.impuls);
  grid.energy = nullptr;
  grid.stream = nullptr;
  grid.impuls = nullptr;
#endif
}

// E, F, T of the Illum on the device (the reference's MakeIllumParam) into grid.energy /
// stream / impuls; id_dev and im_dev select the device part (one here)
int cuda::interface::separate_device::CalculateAllParamAsync(const int id_dev, const int im_dev,
                                                             const grid_directions_t &grid_dir, grid_t &grid,
                                                             e_cuda_stream_id_t st) {
  (void)id_dev, (void)im_dev, (void)grid_dir, (void)grid, (void)st;
#ifdef ON_FULL_ILLUM_ARRAYS
  cudaStream_t s = cuda_streams[st];
  if (!d_E) {
    check(cudaMalloc(&d_E, sizeof(double) * g_N), "cudaMalloc");
    check(cudaMalloc(&d_F, sizeof(double) * 3 * g_N), "cudaMalloc");
    check(cudaMalloc(&d_T, sizeof(double) * 9 * g_N), "cudaMalloc");
  }
  check(rrhd_moments_fp64(g_dirs, d_I, d_E, d_F, d_T, g_N, s), "rrhd_moments_fp64");
  check(cudaMemcpyAsync(grid.energy, d_E, sizeof(double) * g_N, cudaMemcpyDeviceToHost, s), "energy");
  check(cudaMemcpyAsync(grid.stream, d_F, sizeof(double) * 3 * g_N, cudaMemcpyDeviceToHost, s), "stream");
  check(cudaMemcpyAsync(grid.impuls, d_T, sizeof(double) * 9 * g_N, cudaMemcpyDeviceToHost, s), "impuls");
#endif
  return e_completion_success;
}

int cuda::interface::separate_device::CalculateIntScatteringAsync(const grid_directions_t &grid_dir, grid_t &grid,
                                                                  const IdType start_dir, const IdType end_dir,
                                                                  const e_cuda_stream_id_t stream) {
  const int64_t M_loc = end_dir - start_dir;
  if (M_loc <= 0 || start_dir < 0 || end_dir > g_M) return e_completion_fail;
  cudaStream_t s = cuda_streams[stream];
  check(cudaMemcpyAsync(d_I, grid.Illum, sizeof(double) * g_N * g_M, cudaMemcpyHostToDevice, s), "Illum");
  check(rrhd_scatter_fp64(g_dirs, d_I, d_S, g_N, s), "rrhd_scatter_fp64");
  // columns start_dir .. end_dir - 1 of S [N][M] into scattering [N][M_loc]
  check(cudaMemcpy2DAsync(grid.scattering, sizeof(double) * M_loc, d_S + start_dir, sizeof(double) * g_M,
                          sizeof(double) * M_loc, g_N, cudaMemcpyDeviceToHost, s),
        "scattering");
  check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
#ifdef ON_FULL_ILLUM_ARRAYS
  if (grid.energy != nullptr) {
    CalculateAllParamAsync(0, 0, grid_dir, grid, e_cuda_params);
    CudaSyncStream(e_cuda_params);
  }
#endif
  return e_completion_success;
}

#ifdef SPECTRUM
// cells' velocities (units of c) to the device (cuda_interface_spectrum.cu:20-37)
void cuda::interface::separate_device::SendVelocity(const grid_t &grid) {
  std::vector<double> v(3 * g_N);
  for (int64_t i = 0; i < g_N; i++)
    for (int a = 0; a < 3; a++) v[3 * i + a] = grid.cells[i].phys_val.v[a];
  check(cudaMemcpy(d_vel, v.data(), sizeof(double) * 3 * g_N, cudaMemcpyHostToDevice), "SendVelocity");
}

// Compton scattering at the current frequency (cuda_interface_spectrum.cu:46-92): Illum [N][M]
int cuda::interface::separate_device::CalculateSpectrumIntScattering(const grid_directions_t &grid_dir, grid_t &grid,
                                                                     const IdType start_dir, const IdType end_dir,
                                                                     const e_cuda_stream_id_t stream) {
  (void)grid_dir;
  const int64_t M_loc = end_dir - start_dir;
  if (M_loc <= 0 || start_dir < 0 || end_dir > g_M) return e_completion_fail;
  const double frq = 0.5 * (grid.frq_grid[grid.cur_frq_id] + grid.frq_grid[grid.cur_frq_id + 1]);
  cudaStream_t s = cuda_streams[stream];
  check(cudaMemcpyAsync(d_I, grid.Illum, sizeof(double) * g_N * g_M, cudaMemcpyHostToDevice, s), "Illum");
  check(rrhd_compton_spectrum(g_dirs, d_I, d_vel, d_S, g_N, frq, (int32_t)start_dir, (int32_t)M_loc, (int32_t)M_loc, s),
        "rrhd_compton_spectrum");
  check(cudaMemcpyAsync(grid.scattering, d_S, sizeof(double) * g_N * M_loc, cudaMemcpyDeviceToHost, s), "scattering");
  check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  return e_completion_success;
}

// frequency-coupled Compton scattering over the whole spectrum (cuda_interface_spectrum.cu:94-140):
// Illum [N][M][100], scattering [N][end - start][100]
int cuda::interface::separate_device::CalculateFullSpectrumIntScattering(const grid_directions_t &grid_dir,
                                                                         grid_t &grid, const IdType start_dir,
                                                                         const IdType end_dir,
                                                                         const e_cuda_stream_id_t stream) {
  (void)grid_dir;
  const int64_t M_loc = end_dir - start_dir;
  if (M_loc <= 0 || start_dir < 0 || end_dir > g_M || grid.size_frq != 100) return e_completion_fail;
  cudaStream_t s = cuda_streams[stream];
  check(cudaMemcpyAsync(d_I, grid.Illum, sizeof(double) * g_N * g_M * 100, cudaMemcpyHostToDevice, s), "Illum");
  check(rrhd_compton_full_spectrum(g_dirs, d_I, d_vel, d_S, g_N, (int32_t)start_dir, (int32_t)M_loc, (int32_t)M_loc, s),
        "rrhd_compton_full_spectrum");
  check(cudaMemcpyAsync(grid.scattering, d_S, sizeof(double) * g_N * M_loc * 100, cudaMemcpyDeviceToHost, s),
        "scattering");
  check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  return e_completion_success;
}
#endif
#endif
