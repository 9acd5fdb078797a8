// The context behind rrhd_ctx: device-resident mesh and state of one solver.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "rrhd.h"

namespace rrhd {

// Scalars one hydro step produces; two slots used alternately so a step can
// read the previous step's max speed for its device-side time step.
struct StepScalars {
  double max_speed;
  double tau;
  unsigned long long n_fallback;
  unsigned long long n_failed;
};

struct BcTable {
  int32_t kind[8];
  double W[8][5];
  double U[8][5];
};

}  // namespace rrhd

struct rrhd_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int eos = 1;
  double gamma = 5.0 / 3.0;
  int64_t N = 0, F = 0;
  int cpb = 256;      // cells per CTA
  int nblocks = 0;
  int max_entries = 0;  // largest per-CTA face list
  int max_halo = 0;     // largest per-CTA list of neighbour cells owned by other CTAs
  int64_t n_entries = 0;
  size_t step_smem = 0; // dynamic shared memory of the step kernel

  // numbering: perm[new] = caller id, iperm[caller id] = new
  int32_t *d_perm = nullptr, *d_iperm = nullptr;
  std::vector<int32_t> h_perm;

  // per-CTA face lists
  int32_t *d_bface_off = nullptr;  // [nblocks+1]
  int2 *d_bface_lr = nullptr;      // [E] (l, r) as CTA-local state slots; r < 0: boundary code
  int32_t *d_halo_off = nullptr;   // [nblocks+1]
  int32_t *d_halo_ids = nullptr;   // neighbour cells (new numbering) staged after the CTA's own
  double4 *d_bface_nS = nullptr;   // [E] (n0, n1, n2, area)
  int32_t *d_bface_gid = nullptr;  // [E] caller face id on the owner CTA, else -1

  // per cell (new numbering)
  ushort4 *d_cell_slot = nullptr;  // local face slots
  uint8_t *d_cell_sign = nullptr;
  double *d_cell_V = nullptr;

  // state [N][10] = U(5), W(5); two buffers, `cur` holds the current one
  double *d_state[2] = {nullptr, nullptr};
  int cur = 0;
  uint8_t *d_status = nullptr;  // [N] status of the last step (new numbering)

  rrhd::StepScalars *d_scal = nullptr;  // [2]
  int scal_cur = 0;
  double cfl = 0.3, h_min = 0.0;

  bool keep_face_flux = false;
  double *d_face_flux = nullptr;  // [F][5] caller numbering

  rrhd::BcTable bc{};

  double *d_scratch_io = nullptr;  // [N][5] staging for strided host/device transfers
  double *h_pinned = nullptr;      // pinned staging for host transfers, N*10 doubles
};
