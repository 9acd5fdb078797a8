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

// Scattering integral / moments with I and S in the cell-direction-group layout
// [cells][M][G] (rows cell * G + g of the row-layout entry points); G divides 64
// (FP64) or is 1, 2 or 4 (tensor cores).
rrhd_status scatter_fp64_cdg(const rrhd_dirs *d, const double *I, double *S, int64_t cells, int G, bool exact,
                             cudaStream_t st);
rrhd_status moments_fp64_cdg(const rrhd_dirs *d, const double *I, double *E, double *F, double *T, int64_t cells,
                             int G, cudaStream_t st);
rrhd_status scatter_tc_cdg(const rrhd_scatter_tc *t, const float *I, float *S, float *mom, int64_t cells, int G,
                           cudaStream_t st);
// Low-rank (Thomson) scattering and moments, cell-direction-group layout, G = 1, 2, 4:
// FP64 with the moments as E [rows], F [rows][3], T [rows][3][3] (any may be NULL
// together), FP32 with the moments as [rows][16] (mom may be NULL).
rrhd_status scatter_lowrank_fp64(const rrhd_dirs *d, const double *I, double *S, double *mE, double *mF, double *mT,
                                 int64_t cells, int G, cudaStream_t st);
rrhd_status scatter_lowrank_fp32(const rrhd_dirs *d, const float *I, float *S, float *mom, int64_t cells, int G,
                                 cudaStream_t st);

}  // namespace rrhd
