// The context behind rrhd_ctx: device-resident mesh and state of one solver.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <climits>

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

// One entry of a CTA's face list (40 bytes): the face's unit normal and area and
// its two sides as CTA-local state slots (r < 0: boundary code).
struct FaceRec {
  double n0, n1, n2, area;
  int32_t l, r;
};
// Marks the padding entry that rounds a CTA's face list up to an even count.
constexpr int32_t kFacePad = INT32_MIN;

// Per-cell record of the step (16 bytes): the CTA-local slots of the cell's four
// faces in id_faces order, each with the cell's sign_n bit of that face in bit
// 15, and the cell volume.
struct CellRec {
  uint16_t s[4];
  double V;
};
static_assert(sizeof(FaceRec) == 40 && sizeof(CellRec) == 16, "step record layout");

}  // namespace rrhd

struct rrhd_dirs;
struct rrhd_scatter_tc;

namespace rrhd {
// Pointers a sweep reads and writes, kept in device memory so that one captured
// graph of level launches serves every call.
struct SweepIO {
  const void *S;          // scattering integral
  void *I;                // intensity
  const int32_t *row_of;  // layout 0: context cell -> caller cell
  int32_t layout;         // 0: rows (cell * G + g) x M in caller numbering; 1: [N][M][G], context numbering
};

// Radiation part of a context: the transport sweep and the coupled step.
struct RadState {
  bool ready = false;
  const rrhd_dirs *dirs = nullptr;  // not owned
  int M = 0, G = 1, DB = 64, shift = 6, nbatch = 0;
  int prec = 0;  // RRHD_RAD_FP64 or RRHD_RAD_FP32: storage and arithmetic of the sweep
  int RW = 0;    // stride (values) of the per-cell record
  int GS = 0;    // stride (values) of one face-value slot: G rounded up to a 32-byte sector
  double bc = 0.0;
  int64_t last_cell = 0;  // context index of the caller's last cell (plain-mean quirk)
  void *d_w = nullptr;    // [M][3] directions in the sweep precision
  // per-cell record (context numbering, RW values): outward normals n_j (12), heights
  // H_j = 3 V / A_j (4), face-value slots of the faces (4 x int32) and neighbours (4 x int32,
  // context numbering or -1), then the step's source record {k, betta/k, alpha Q_g/k}
  void *d_rec = nullptr;
  void *d_area = nullptr;  // [N][4] face areas
  uint32_t *d_plan = nullptr;               // all batches: items (d << shift | cell) in level order
  bool item_geometry = false;
  uint4 *d_geo = nullptr;                   // item_geometry: per plan item {code, in-face distances}
  std::vector<std::vector<int64_t>> lvl;    // per batch: level offsets into d_plan
  int64_t levels = 0, max_level = 0;
  cudaGraphExec_t graph = nullptr;          // every level launch of one sweep
  SweepIO *d_io = nullptr;
  SweepIO h_io{};       // last pointers uploaded to d_io
  bool io_valid = false;
  // phase marks of the last coupled step: 0 start, 1 hydro done, 2 sweep done, 3 source
  // start and 4 source done (side stream), 5 join, 6 scattering done
  cudaEvent_t ev[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  cudaStream_t side = nullptr;  // the coupled step's source term runs here, beside the sweep
  void *d_fv = nullptr;  // [DB][F][GS] face values, direction-major
  // coupled step (context numbering, [N][M][G])
  void *d_I = nullptr, *d_S = nullptr;
  double *d_G4 = nullptr;                                    // [N][4] radiation 4-force of the last step
  double *d_mE = nullptr, *d_mF = nullptr, *d_mT = nullptr;  // FP64 moments per row [N*G], [N*G][3], [N*G][9]
  float *d_mom = nullptr;                                    // FP32 moments per row [N*G][16]
  unsigned long long *d_cnt = nullptr;                       // [8] counters of the source con2prim
  rrhd_scatter_tc *tc = nullptr;
  int tc_form = -1;
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
  rrhd::FaceRec *d_bface_rec = nullptr;  // [E] face records, every CTA's list padded to an even count
  int32_t *d_halo_off = nullptr;   // [nblocks+1]
  int32_t *d_halo_ids = nullptr;   // neighbour cells (new numbering) staged after the CTA's own
  int32_t *d_bface_gid = nullptr;  // [E] caller face id on the owner CTA, else -1

  // per cell (new numbering)
  rrhd::CellRec *d_cell_rec = nullptr;

  // state [N][10] = U(5), W(5); two buffers, `cur` holds the current one
  double *d_state[2] = {nullptr, nullptr};
  int cur = 0;
  uint8_t *d_status = nullptr;  // [N] status of the last step (new numbering)

  rrhd::StepScalars *d_scal = nullptr;  // [2]
  int scal_cur = 0;

  // split of the hydro step over ranks (rrhd_hydro_set_part): this context updates the
  // CTA blocks [part_b0, part_b1); the cells it sends / receives, grouped by peer rank
  int part_world = 1, part_rank = 0;
  int part_b0 = 0, part_b1 = 0;
  int64_t part_c0 = 0, part_c1 = 0;
  int64_t n_send = 0, n_recv = 0;
  std::vector<int64_t> send_counts, recv_counts;
  int32_t *d_send_ids = nullptr, *d_recv_ids = nullptr;
  double cfl = 0.3, h_min = 0.0;

  bool keep_face_flux = false;
  double *d_face_flux = nullptr;  // [F][5] caller numbering

  rrhd::BcTable bc{};

  double *d_scratch_io = nullptr;  // [N][5] staging for strided host/device transfers
  double *h_pinned = nullptr;      // pinned staging for host transfers, N*10 doubles

  // mesh arrays kept for the radiation set-up (caller numbering)
  std::vector<int32_t> h_cell_faces, h_face_l, h_face_r;
  std::vector<uint8_t> h_cell_sign;
  std::vector<double> h_face_n, h_face_area, h_cell_V;

  rrhd::RadState rad;
};

void rrhd_rad_release(rrhd_ctx *c);
