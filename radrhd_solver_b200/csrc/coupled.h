// Internal entry points shared between the con2prim and coupled-step translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "rrhd.h"

namespace rrhd {

// Learned-guess con2prim of n states at U + stride i, W + stride i (stride 5 for
// separate arrays, 10 for a solver state [n][10]).  With G4 != NULL the
// radiation source tau G4 is added to U first.  Statistics are read back (and the
// stream synchronised) only when stats or n_guess_fallback is not NULL.
rrhd_status mlp_c2p(const rrhd_mlp *m, int eos, double gamma, double *U, double *W, int64_t stride,
                    const double *G4, double tau_src, uint8_t *status, int64_t n, int fallback, int k_stall,
                    rrhd_c2p_stats *stats, int64_t *n_guess_fallback, double *guess, cudaStream_t st);

}  // namespace rrhd
