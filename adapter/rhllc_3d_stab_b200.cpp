// Drop-in replacement for solvers/rhllc/src/rhllc_3d_stab.cpp: the reference's
// void rhllc::Hllc3dStab(const Type tau, grid_t &grid) (solvers/rhllc/include/rhllc_calc.h:32)
// implemented on the B200 library's C ABI (include/rrhd.h).  Link this file into the
// reference's build in place of rhllc_3d_stab.cpp, plus radrhd_solver_b200/librrhd.so; the
// callers (RunRhllcModule, RunRadRHDModule) stay unchanged.
//
// What a call does, as the reference's body does on the host grid:
//   * on the first call for a grid (or when its size changes) the mesh -- grid.faces[].geo and
//     grid.cells[].geo -- is copied to the device once (rrhd_create);
//   * every call uploads cells[].conv_val / phys_val, runs the fused RHLLC flux + update +
//     con2prim step on the GPU, and downloads them back (rrhd_hydro_step_host: the state
//     records are read and written in place, with elem_t's size as the stride);
//   * in resident mode (SetResident(true)) the state stays on the device between calls:
//     the first call after SetResident or SyncToDevice uploads it, later calls only step,
//     and SyncToHost(grid) writes it back into grid.cells -- RunRhllcModule reads
//     grid.cells only in WriteSolution (rhllc::GetTimeStep reads max_signal_speed alone,
//     solvers/rhllc/src/rhllc_utils.cpp:15-23), so one SyncToHost before each
//     WriteSolution keeps its output identical while the per-step copies disappear;
//   * rhllc::max_signal_speed is set from the step; the face fluxes are written back into
//     grid.faces[].f only after KeepFaceFlux(true) (no reference caller reads faces[].f
//     outside Hllc3dStab, rhllc_main.cpp:42-57, so the 40 bytes per face of that download
//     are skipped by default);
//   * a cell where con2prim and PhysPressureFix both fail stops the program, as the
//     reference's DIE_IF does.
// The results are the reference's bit for bit (the library's FP64 step is compiled without
// contraction and follows the reference's operation order).
//
// Boundaries: codes the mesh uses default to transmissive (e_bound_free).  The reference
// chooses the other codes' states at compile time per GEOMETRY_TYPE (rhllc_utils.cpp:45-133);
// a build mirrors its choice with rhllc_b200::SetBoundary before the first step.
#if defined RHLLC && defined SOLVERS
#include "rhllc_calc.h"
#include "rhllc_utils.h"

#include "rhllc_3d_stab_b200.h"
#include "rrhd.h"

#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <vector>

namespace rhllc_b200 {

struct Bc {
  int32_t code, kind;
  double W[5];
};

static rrhd_ctx *g_ctx = nullptr;
static const elem_t *g_cells = nullptr;
static size_t g_n = 0, g_f = 0;
static bool g_face_flux = false;
static bool g_resident = false;
static bool g_dev_valid = false;  // resident mode: the device holds the latest state
static std::vector<Bc> g_bc;
static std::vector<double> g_flux;

static void fail(const char *what) {
  std::fprintf(stderr, "rhllc::Hllc3dStab (B200): %s: %s\n", what, rrhd_last_error());
  std::abort();
}

/// State of a boundary code for the following steps (kind RRHD_BC_TRANSMISSIVE,
/// RRHD_BC_FIXED with the primitive state W, or RRHD_BC_REFLECT).
void SetBoundary(int code, int kind, const double *W) {
  Bc b{code, kind, {0, 0, 0, 0, 0}};
  if (W)
    for (int i = 0; i < 5; i++) b.W[i] = W[i];
  g_bc.push_back(b);
  if (g_ctx && rrhd_set_boundary(g_ctx, code, kind, W) != RRHD_OK) fail("rrhd_set_boundary");
}

/// Whether grid.faces[].f is refreshed after each step (off by default; the reference's
/// step writes them, but none of its callers reads them).
void KeepFaceFlux(bool on) {
  g_face_flux = on;
  if (g_ctx && rrhd_keep_face_flux(g_ctx, on ? 1 : 0) != RRHD_OK) fail("rrhd_keep_face_flux");
}

/// Frees the device copy (the next call rebuilds it).  In resident mode, call
/// SyncToHost first: the device state is lost.
void Release() {
  if (g_ctx) rrhd_destroy(g_ctx);
  g_ctx = nullptr;
  g_cells = nullptr;
  g_n = g_f = 0;
  g_dev_valid = false;
}

static void state_ptrs(grid_t &grid, double **W, double **U, int64_t *stride) {
  static_assert(sizeof(flux_t) == 5 * sizeof(double), "flux_t must be 5 contiguous doubles");
  static_assert(sizeof(elem_t) % sizeof(double) == 0, "elem_t must be a whole number of doubles");
  elem_t &c0 = grid.cells[0];
  *W = reinterpret_cast<double *>(&c0.phys_val);
  *U = reinterpret_cast<double *>(&c0.conv_val);
  *stride = sizeof(elem_t) / sizeof(double);
}

/// Resident mode on or off.  On: the state is uploaded by the next call and then stays
/// on the device; grid.cells is refreshed only by SyncToHost.  Off (the default): every
/// call copies the state both ways.
void SetResident(bool on) {
  g_resident = on;
  g_dev_valid = false;
}

/// Resident mode: writes the device state into grid.cells (before WriteSolution or any
/// other read of the cells on the host).  No effect outside resident mode.
void SyncToHost(grid_t &grid) {
  if (!g_resident || !g_ctx || !g_dev_valid || g_cells != grid.cells.data()) return;
  double *W, *U;
  int64_t stride;
  state_ptrs(grid, &W, &U, &stride);
  if (rrhd_get_state(g_ctx, W, U, stride, RRHD_HOST) != RRHD_OK) fail("rrhd_get_state");
}

/// Resident mode: the host has changed grid.cells (e.g. a source term applied on the
/// host); the next call uploads them again.
void SyncToDevice(grid_t &) { g_dev_valid = false; }

static void init(const grid_t &grid) {
  Release();
  const size_t N = grid.cells.size(), F = grid.faces.size();
  std::vector<int32_t> fl(F), fr(F), cf(4 * N);
  std::vector<double> fn(3 * F), fs(F), cv(N), cc(3 * N);
  std::vector<uint8_t> sg(N);
  for (size_t f = 0; f < F; f++) {
    const geo_face_t &g = grid.faces[f].geo;
    fl[f] = (int32_t)g.id_l;
    fr[f] = (int32_t)g.id_r;
    fs[f] = g.S;
    for (int a = 0; a < 3; a++) fn[3 * f + a] = g.n[a];
  }
  for (size_t c = 0; c < N; c++) {
    const geo_cell_t &g = grid.cells[c].geo;
    for (int j = 0; j < 4; j++) cf[4 * c + j] = (int32_t)g.id_faces[j];
    sg[c] = (uint8_t)g.sign_n.bits;
    cv[c] = g.V;
    for (int a = 0; a < 3; a++) cc[3 * c + a] = g.center[a];
  }
  const rrhd_mesh_desc m = {(int64_t)N, (int64_t)F, fl.data(), fr.data(), fn.data(), fs.data(),
                            cf.data(),  sg.data(),  cv.data(), cc.data()};
  rrhd_opts o = {};
  o.eos = EOS == TAUB ? RRHD_EOS_TAUB : RRHD_EOS_IDEAL;  // include/hd_config.h
  o.gamma = kGamma1;                                      // lib/global_consts.h
  if (rrhd_create(&m, &o, &g_ctx) != RRHD_OK) fail("rrhd_create");
  for (const Bc &b : g_bc)
    if (rrhd_set_boundary(g_ctx, b.code, b.kind, b.W) != RRHD_OK) fail("rrhd_set_boundary");
  if (rrhd_keep_face_flux(g_ctx, g_face_flux ? 1 : 0) != RRHD_OK) fail("rrhd_keep_face_flux");
  g_cells = grid.cells.data();
  g_n = N;
  g_f = F;
  g_dev_valid = false;
}

}  // namespace rhllc_b200

void rhllc::Hllc3dStab(const Type tau, grid_t &grid) {
  using namespace rhllc_b200;
  if (!g_ctx || g_cells != grid.cells.data() || g_n != grid.cells.size() || g_f != grid.faces.size()) init(grid);
  double *W, *U;
  int64_t stride;
  state_ptrs(grid, &W, &U, &stride);
  rrhd_step_stats st;
  rrhd_status s;
  if (g_resident) {
    if (!g_dev_valid) {
      if (rrhd_set_state(g_ctx, W, U, stride, RRHD_HOST) != RRHD_OK) fail("rrhd_set_state");
      g_dev_valid = true;
    }
    s = rrhd_hydro_step(g_ctx, tau, &st);
  } else {
    s = rrhd_hydro_step_host(g_ctx, tau, W, U, stride, &st);
  }
  if (s == RRHD_ERR_C2P) fail("con2prim and PhysPressureFix failed in some cell");
  if (s != RRHD_OK) fail("rrhd_hydro_step_host");
  rhllc::max_signal_speed = st.max_speed;
  if (g_face_flux) {
    g_flux.resize(5 * g_f);
    if (rrhd_get_face_flux(g_ctx, g_flux.data()) != RRHD_OK) fail("rrhd_get_face_flux");
    for (size_t f = 0; f < g_f; f++) {
      flux_t &F = grid.faces[f].f;
      const double *p = g_flux.data() + 5 * f;
      F.d = p[0];
      F.v = Vector3(p[1], p[2], p[3]);
      F.p = p[4];
    }
  }
}
#endif
