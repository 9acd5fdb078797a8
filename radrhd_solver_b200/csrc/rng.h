// Counter-based RNG shared by host and device: every variate is a pure
// function of (seed, stream, index), so a field generated on the GPU equals the
// one generated on the CPU element for element.  splitmix64 finaliser.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define RRHD_HD __host__ __device__ __forceinline__
#else
#define RRHD_HD inline
#endif

RRHD_HD uint64_t rrhd_mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

RRHD_HD uint64_t rrhd_hash3(uint64_t seed, uint64_t stream, uint64_t index) {
  return rrhd_mix64(rrhd_mix64(seed ^ rrhd_mix64(stream * 0xD1B54A32D192ED03ull)) ^ index);
}

// uniform in [0, 1) with 53 random bits
RRHD_HD double rrhd_u01(uint64_t seed, uint64_t stream, uint64_t index) {
  return (double)(rrhd_hash3(seed, stream, index) >> 11) * 0x1.0p-53;
}
