/* Test infrastructure, not product code.
 *
 * Host stand-in for <cuda_runtime.h>, used only to compile the reference's own
 * device source (the frequency-coupled Compton scattering kernel) with g++ so that
 * the oracle can run it on the CPU.  The CUDA qualifiers become no-ops and the
 * launch indices become per-thread host variables set by the caller before each
 * call of the kernel body. */
#ifndef RRHD_HOST_CUDA_RUNTIME_H
#define RRHD_HOST_CUDA_RUNTIME_H
#include <cmath>
#include <algorithm>
#define __host__
#define __device__
#define __global__
#define __forceinline__ inline
struct uint3 { unsigned int x, y, z; };
struct dim3 { unsigned int x, y, z; };
typedef struct CUstream_st *cudaStream_t;
typedef int cudaError_t;
extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
#endif
