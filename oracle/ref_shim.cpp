// Test infrastructure, not product code.
//
// C entry points around the reference implementation (Lartsev-Artem/RadRHD_solver)
// compiled from its own sources by oracle/Makefile into oracle/_ref/.  Only the
// tests, the smoke check and the CPU-baseline leg of bench.py load these
// libraries; nothing in the product path does.
//
// The shim owns no arithmetic of its own on the checked path: every number it
// returns comes out of a reference function.  What it does own is the glue the
// reference normally gets from its VTK/MPI drivers: building grid_t from plain
// arrays (the same face assembly as lib/geometry/src/convert_bin_to_geo.cpp:3-48)
// and a fixed-state inflow boundary that the reference only has as compile-time
// per-geometry code (solvers/rhllc/src/rhllc_utils.cpp:45-133).
//
// Build variants (selected by -D flags in oracle/Makefile):
//   RRHD_SHIM_HYDRO : -DSOLVERS -DRHLLC             (hydro: flux, update, con2prim)
//   RRHD_SHIM_ILLUM : -DSOLVERS -DILLUM             (CPU scattering + moments)
//   RRHD_SHIM_RAD   : -DSOLVERS -DILLUM -DRHLLC -DRAD_RHD -DUSE_CUDA (radiation 4-force)
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

#include "global_consts.h"
#include "solvers_struct.h"

#if defined RRHD_SHIM_HYDRO
#include "rhllc_calc.h"
#include "reader_bin.h"
#include "reader_txt.h"
#include "writer_bin.h"
#include "rhllc_flux_stab.h"
#include "rhllc_flux.h"
#include "rhllc_utils.h"
#if defined RRHD_ADAPTER_HYDRO
#include "rhllc_3d_stab_b200.h"
#endif
#endif
#if defined RRHD_SHIM_ILLUM
#include "illum_integrate.h"
#include "illum_utils.h"
#include "scattering.h"
#endif
#if defined RRHD_SHIM_RAD
#include "radRHD_utils.h"
#include "plunk.h"
#include "gas_state.h"
#include "illum_utils.h"
#endif

namespace {

inline void load_flux(flux_t &f, const double *p) {
  f.d = p[0];
  f.v = Vector3(p[1], p[2], p[3]);
  f.p = p[4];
}
inline void store_flux(const flux_t &f, double *p) {
  p[0] = f.d;
  p[1] = f.v[0];
  p[2] = f.v[1];
  p[3] = f.v[2];
  p[4] = f.p;
}

}  // namespace

extern "C" {

// Adiabatic index this variant was compiled with (kGamma1, lib/global_consts.h:20)
// and the equation of state (1 = IDEAL, 2 = TAUB, include/hd_config.h:16-20).
double ref_kgamma1(void) { return kGamma1; }
#if defined RRHD_SHIM_HYDRO
int ref_eos(void) { return EOS; }
#endif

#if defined RRHD_SHIM_HYDRO

// ---------------------------------------------------------------- per state
// rhllc::GetPhysValueStab (solvers/rhllc/src/rhllc_flux_stab.cpp:123-220)
void ref_c2p(const double *U, double *W, int32_t *codes, int64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    flux_t u, w;
    load_flux(u, U + 5 * i);
    load_flux(w, W + 5 * i);
    codes[i] = rhllc::GetPhysValueStab(u, w);
    store_flux(w, W + 5 * i);
  }
}

// rhllc::PhysPressureFix (rhllc_flux_stab.cpp:40-121); rewrites U.E.
void ref_pressure_fix(double *U, double *W, int32_t *codes, int64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    flux_t u, w;
    load_flux(u, U + 5 * i);
    load_flux(w, W + 5 * i);
    codes[i] = rhllc::PhysPressureFix(u, w);
    store_flux(u, U + 5 * i);
    store_flux(w, W + 5 * i);
  }
}

// rhllc::GetConvValueStab (rhllc_flux_stab.cpp:10-38); may rescale W.v.
void ref_p2c(double *W, double *U, int64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    flux_t u, w;
    load_flux(w, W + 5 * i);
    rhllc::GetConvValueStab(w, u);
    store_flux(w, W + 5 * i);
    store_flux(u, U + 5 * i);
  }
}

// rhllc::GetConvValue (solvers/rhllc/src/rhllc_flux.cpp:7-16), used by the
// reference for its fixed inflow states.
void ref_p2c_plain(const double *W, double *U, int64_t n) {
  for (int64_t i = 0; i < n; i++) {
    flux_t u, w;
    load_flux(w, W + 5 * i);
    rhllc::GetConvValue(w, u);
    store_flux(u, U + 5 * i);
  }
}

// rhllc::GetFluxStab (rhllc_flux_stab.cpp:240-431) for a batch of faces.
// normal [n][3], area [n]; F [n][5] gets the area-weighted flux.
void ref_flux(const double *UL, const double *UR, const double *WL, const double *WR,
              const double *normal, const double *area, double *F, double *speed,
              int64_t n) {
  for (int64_t i = 0; i < n; i++) {
    flux_t ul, ur, wl, wr;
    load_flux(ul, UL + 5 * i);
    load_flux(ur, UR + 5 * i);
    load_flux(wl, WL + 5 * i);
    load_flux(wr, WR + 5 * i);
    face_t f;
    f.geo.n = Vector3(normal[3 * i], normal[3 * i + 1], normal[3 * i + 2]);
    f.geo.S = area[i];
    speed[i] = rhllc::GetFluxStab(ul, ur, wl, wr, f);
    store_flux(f.f, F + 5 * i);
  }
}

// ---------------------------------------------------------------- whole mesh
struct ref_hydro {
  grid_t grid;
  // fixed-state boundary table for codes -1..-8 (index = -code-1):
  // kind 0 = reference BoundConditions, kind 1 = fixed (W,U) state.
  int bc_kind[8];
  double bc_W[8][5];
  double bc_U[8][5];
};

// Builds grid_t from plain arrays.  Face records mirror geo_face_t
// (lib/grids/include/solvers_struct.h:87-105), cell records geo_cell_t (:124-162).
void *ref_hydro_create(int64_t n_cells, int64_t n_faces, const int32_t *face_id_l,
                       const int32_t *face_id_r, const double *face_n,
                       const double *face_area, const int32_t *cell_faces,
                       const uint8_t *cell_sign, const double *cell_volume,
                       const double *cell_center) {
  ref_hydro *h = new ref_hydro();
  grid_t &g = h->grid;
  g.size = n_cells;
  g.cells.resize(n_cells);
  g.faces.resize(n_faces);
  for (int64_t f = 0; f < n_faces; f++) {
    geo_face_t &geo = g.faces[f].geo;
    geo.id_l = (uint32_t)face_id_l[f];
    geo.id_r = face_id_r[f];
    geo.n = Vector3(face_n[3 * f], face_n[3 * f + 1], face_n[3 * f + 2]);
    geo.S = face_area[f];
  }
  for (int64_t c = 0; c < n_cells; c++) {
    geo_cell_t &geo = g.cells[c].geo;
    for (int j = 0; j < 4; j++) geo.id_faces[j] = cell_faces[4 * c + j];
    geo.sign_n.bits = cell_sign[c];
    geo.V = cell_volume[c];
    geo.center = Vector3(cell_center[3 * c], cell_center[3 * c + 1], cell_center[3 * c + 2]);
  }
  for (int k = 0; k < 8; k++) h->bc_kind[k] = 0;
  return h;
}

void ref_hydro_destroy(void *p) { delete (ref_hydro *)p; }

void ref_hydro_set_bc(void *p, int32_t code, int32_t kind, const double *W, const double *U) {
  ref_hydro *h = (ref_hydro *)p;
  const int k = -code - 1;
  if (k < 0 || k >= 8) return;
  h->bc_kind[k] = kind;
  for (int i = 0; i < 5; i++) {
    h->bc_W[k][i] = W ? W[i] : 0.0;
    h->bc_U[k][i] = U ? U[i] : 0.0;
  }
}

void ref_hydro_set_state(void *p, const double *W, const double *U) {
  grid_t &g = ((ref_hydro *)p)->grid;
  for (int64_t c = 0; c < (int64_t)g.cells.size(); c++) {
    load_flux(g.cells[c].phys_val, W + 5 * c);
    load_flux(g.cells[c].conv_val, U + 5 * c);
  }
}

void ref_hydro_get_state(void *p, double *W, double *U) {
  grid_t &g = ((ref_hydro *)p)->grid;
  for (int64_t c = 0; c < (int64_t)g.cells.size(); c++) {
    store_flux(g.cells[c].phys_val, W + 5 * c);
    store_flux(g.cells[c].conv_val, U + 5 * c);
  }
}

// Face fluxes left in grid.faces[].f by the last step ([F][5]).
void ref_hydro_get_face_flux(void *p, double *F) {
  grid_t &g = ((ref_hydro *)p)->grid;
  for (int64_t f = 0; f < (int64_t)g.faces.size(); f++) store_flux(g.faces[f].f, F + 5 * f);
}

// One call of the reference step rhllc::Hllc3dStab (solvers/rhllc/src/rhllc_3d_stab.cpp:10-63)
// on the stored grid.  Returns rhllc::max_signal_speed (rhllc_utils.cpp:13).
double ref_hydro_step(void *p, double tau, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  rhllc::Hllc3dStab(tau, ((ref_hydro *)p)->grid);
  return rhllc::max_signal_speed;
}

// The same face/cell loops as rhllc::Hllc3dStab, but with the boundary table
// above for codes whose kind is 1 (fixed inflow state); every other face goes
// through the reference rhllc::BoundConditions.  Per-cell con2prim status is
// returned in codes[] (see below) instead of aborting the process as the
// reference does (DIE_IF).
double ref_hydro_step_bc(void *p, double tau, int nthreads, int32_t *codes) {
  ref_hydro *h = (ref_hydro *)p;
  grid_t &grid = h->grid;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  Type global_max = 0;
#pragma omp parallel default(shared)
  {
    Type max_speed = 0;
    flux_all_t bound_val;
    const int size_face = grid.faces.size();
#pragma omp for
    for (int i = 0; i < size_face; i++) {
      face_t &f = grid.faces[i];
      const int id_r = f.geo.id_r;
      const int k = -id_r - 1;
      if (id_r < 0 && k < 8 && h->bc_kind[k] == 1) {
        load_flux(bound_val.phys_val, h->bc_W[k]);
        load_flux(bound_val.conv_val, h->bc_U[k]);
      } else {
        rhllc::BoundConditions(f, grid.cells, bound_val);
      }
      max_speed = std::max(max_speed,
                           rhllc::GetFluxStab(grid.cells[f.geo.id_l].conv_val, bound_val.conv_val,
                                              grid.cells[f.geo.id_l].phys_val, bound_val.phys_val, f));
    }
    const int size_grid = grid.size;
#pragma omp for
    for (int i = 0; i < size_grid; i++) {
      elem_t &el = grid.cells[i];
      flux_t sumF;
      for (int j = 0; j < CELL_SIZE; j++) {
        if (el.geo.sign_n[j])
          sumF += grid.faces[el.geo.id_faces[j]].f;
        else
          sumF -= grid.faces[el.geo.id_faces[j]].f;
      }
      sumF *= (tau / el.geo.V);
      el.conv_val -= sumF;
      // status byte: bits 0-2 con2prim code, bit 4 fallback ran, bit 5 fallback failed
      int code = rhllc::GetPhysValueStab(el.conv_val, el.phys_val);
      if (code) {
        const int fix = rhllc::PhysPressureFix(el.conv_val, el.phys_val);
        code = code | 0x10 | (fix ? 0x20 : 0);
      }
      if (codes) codes[i] = code;
    }
#pragma omp critical
    { global_max = std::max(global_max, max_speed); }
  }
  rhllc::max_signal_speed = global_max;
  return global_max;
}

// rhllc::GetTimeStep (rhllc_utils.cpp:15-23) with an explicit max speed.
double ref_time_step(double cfl, double h_min, double max_speed) {
  hllc_value_t cfg;
  cfg.CFL = cfl;
  cfg.h_min = h_min;
  rhllc::max_signal_speed = max_speed;
  std::vector<elem_t> none;
  return rhllc::GetTimeStep(cfg, none);
}

// The reference's own binary formats (lib/files_sys): the solution files of
// files_sys::bin::WriteSolution (writer_bin.cpp:56-114), the geometry records of
// WriteGridGeo / ReadGridGeo (writer_bin.h:95-117, reader_bin.h:113-135) and the hydro
// initial state of ReadHllcInit (reader_bin.h:232-251).
int ref_write_solution(void *p, const char *dir) {
  return files_sys::bin::WriteSolution(std::string(dir), ((ref_hydro *)p)->grid);
}
int ref_write_geo(void *p, const char *faces_file, const char *cells_file) {
  grid_t &g = ((ref_hydro *)p)->grid;
  return files_sys::bin::WriteGridGeo(std::string(faces_file), g.faces) |
         files_sys::bin::WriteGridGeo(std::string(cells_file), g.cells);
}
// reads both files into a fresh grid; returns the sizes (0 on failure) and copies the fields
int64_t ref_read_geo(const char *faces_file, const char *cells_file, int64_t *n_faces, int32_t *face_id_l,
                     int32_t *face_id_r, double *face_n, double *face_area, int32_t *cell_faces, uint8_t *cell_sign,
                     double *cell_volume, double *cell_center) {
  std::vector<face_t> faces;
  std::vector<elem_t> cells;
  if (files_sys::bin::ReadGridGeo(std::string(faces_file), faces) ||
      files_sys::bin::ReadGridGeo(std::string(cells_file), cells))
    return 0;
  *n_faces = (int64_t)faces.size();
  if (face_id_l) {
    for (size_t f = 0; f < faces.size(); f++) {
      face_id_l[f] = (int32_t)faces[f].geo.id_l;
      face_id_r[f] = faces[f].geo.id_r;
      for (int a = 0; a < 3; a++) face_n[3 * f + a] = faces[f].geo.n[a];
      face_area[f] = faces[f].geo.S;
    }
    for (size_t c = 0; c < cells.size(); c++) {
      for (int j = 0; j < 4; j++) cell_faces[4 * c + j] = cells[c].geo.id_faces[j];
      cell_sign[c] = cells[c].geo.sign_n.bits;
      cell_volume[c] = cells[c].geo.V;
      for (int a = 0; a < 3; a++) cell_center[3 * c + a] = cells[c].geo.center[a];
    }
  }
  return (int64_t)cells.size();
}
int64_t ref_read_hllc_init(const char *file, double *W) {
  std::vector<elem_t> cells;
  if (files_sys::bin::ReadHllcInit(std::string(file), cells)) return 0;
  if (W)
    for (size_t c = 0; c < cells.size(); c++) {
      const flux_t &v = cells[c].phys_val;
      W[5 * c] = v.d;
      for (int a = 0; a < 3; a++) W[5 * c + 1 + a] = v.v[a];
      W[5 * c + 4] = v.p;
    }
  return (int64_t)cells.size();
}
// files_sys::txt::ReadSphereDirectionCartesian (lib/files_sys/src/reader_txt.cpp:6-37):
// returns the direction count (-1 on failure); dirs [M][3], areas [M], full_area.
int64_t ref_read_sphere_directions(const char *file, double *dirs, double *areas, double *full_area) {
  grid_directions_t gd;
  if (files_sys::txt::ReadSphereDirectionCartesian(std::string(file), gd) != e_completion_success) return -1;
  if (dirs)
    for (int64_t i = 0; i < (int64_t)gd.size; i++) {
      for (int a = 0; a < 3; a++) dirs[3 * i + a] = gd.directions[i].dir[a];
      areas[i] = gd.directions[i].area;
    }
  if (full_area) *full_area = gd.full_area;
  return (int64_t)gd.size;
}
int ref_record_sizes(int32_t *out) {
  out[0] = (int32_t)sizeof(geo_face_t);
  out[1] = (int32_t)sizeof(geo_cell_t);
  out[2] = (int32_t)sizeof(flux_t);
  return 0;
}

#if defined RRHD_ADAPTER_HYDRO
// The drop-in adapter's own controls (adapter/rhllc_3d_stab_b200.h), for the build that
// links the adapter in place of rhllc_3d_stab.cpp.
void ref_adapter_keep_face_flux(int on) { rhllc_b200::KeepFaceFlux(on != 0); }
void ref_adapter_set_resident(int on) { rhllc_b200::SetResident(on != 0); }
void ref_adapter_sync_to_host(void *p) { rhllc_b200::SyncToHost(((ref_hydro *)p)->grid); }
#endif

#endif  // RRHD_SHIM_HYDRO

#if defined RRHD_SHIM_ILLUM
namespace {
void make_dirs(grid_directions_t &gd, int M, const double *dirs, const double *areas,
               double full_area) {
  gd.size = M;
  gd.loc_size = M;
  gd.loc_shift = 0;
  gd.directions.resize(M);
  for (int k = 0; k < M; k++) {
    gd.directions[k].dir = Vector3(dirs[3 * k], dirs[3 * k + 1], dirs[3 * k + 2]);
    gd.directions[k].area = areas[k];
  }
  gd.full_area = full_area;
}
}  // namespace

// Scattering integral through illum::scattering::GetIntScatteringByDirection
// (solvers/illum/src/scattering.cpp:6-18) in the loop structure of
// CalculateIntCPU (:20-35; that function itself takes grid_t by value and is not
// callable safely).  I is cell-major [N][M]; it is replicated onto the 4 faces of
// each cell, the face layout the CPU function reads (avg of 4 equal values is exact).
void ref_scatter(int64_t N, int32_t M, const double *I, const double *dirs, const double *areas,
                 double full_area, double *S, int nthreads) {
  grid_directions_t gd;
  make_dirs(gd, M, dirs, areas, full_area);
  std::vector<double> face_layout((size_t)M * N * CELL_SIZE);
  for (int64_t c = 0; c < N; c++)
    for (int k = 0; k < M; k++)
      for (int f = 0; f < CELL_SIZE; f++)
        face_layout[((size_t)k * N + c) * CELL_SIZE + f] = I[(size_t)c * M + k];
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < M; k++) {
    const Vector3 direction = gd.directions[k].dir;
    for (int64_t c = 0; c < N; c++)
      S[(size_t)c * M + k] = illum::scattering::GetIntScatteringByDirection(
          CELL_SIZE * c, direction, N * CELL_SIZE, face_layout.data(), gd);
  }
}

// Energy / stream / impulse moments through illum::direction_integrator
// IntegrateByCell / IntegrateByFace3 / IntegrateByFace9
// (solvers/illum/src/illum_integrate.cpp:7-57) and GetAverageByCell, as
// illum::GetEnergy/GetStream/GetImpuls do (solvers/illum/src/illum_params.cpp:7-71).
// E [N], F [N][3], T [N][3][3] row-major T(i,k).
void ref_moments(int64_t N, int32_t M, const double *I, const double *dirs, const double *areas,
                 double full_area, double *E, double *F, double *T, int nthreads) {
  grid_directions_t gd;
  make_dirs(gd, M, dirs, areas, full_area);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
  {
    std::vector<Type> illum((size_t)M * CELL_SIZE);
#pragma omp for schedule(static)
    for (int64_t c = 0; c < N; c++) {
      for (int k = 0; k < M; k++)
        for (int f = 0; f < CELL_SIZE; f++) illum[(size_t)k * CELL_SIZE + f] = I[(size_t)c * M + k];
      E[c] = illum::direction_integrator::IntegrateByCell(illum, gd);
      Vector3 stream[CELL_SIZE];
      illum::direction_integrator::IntegrateByFace3(illum, gd, stream);
      Vector3 s = illum::GetAverageByCell(stream);
      Matrix3 imp[CELL_SIZE];
      illum::direction_integrator::IntegrateByFace9(illum, gd, imp);
      Matrix3 t = illum::GetAverageByCell(imp);
      for (int i = 0; i < 3; i++) {
        F[3 * c + i] = s[i];
        for (int k = 0; k < 3; k++) T[9 * c + 3 * i + k] = t(i, k);
      }
    }
  }
}
#endif  // RRHD_SHIM_ILLUM

#if defined RRHD_SHIM_RAD
}  // extern "C"
// Definitions that lib/grids/src/solvers_struct.cpp normally provides; that file
// does not compile with ILLUM, and none of the entry points below reach these.
solve_mode_t _solve_mode;
Type TableFunc::operator()(Type, Type) { return 0.0; }
extern "C" {

// rad_rhd::GetRadSource (solvers/RadRHD/src/radRHD_utils.cpp:44-101) for each
// cell.  W [N][5] primitive state, alpha/sigma [N] opacities, E [N], F [N][3],
// T [N][3][3] row-major radiation moments.  G [N][4].
void ref_rad_source(int64_t N, const double *W, const double *alpha, const double *sigma,
                    const double *E, const double *F, const double *T, double *G) {
  // grid_t's destructor lives in lib/grids/src/solvers_struct.cpp, which is not part
  // of this variant; one grid object is kept for the life of the process instead.
  static grid_t *g = new grid_t();
  g->size = N;
  g->cells.clear();
  g->cells.resize(N);
  std::vector<Type> energy(N);
  std::vector<Vector3> stream(N);
  std::vector<Matrix3> impuls(N);
  for (int64_t c = 0; c < N; c++) {
    load_flux(g->cells[c].phys_val, W + 5 * c);
    g->cells[c].illum_val.absorp_coef = alpha[c];
    g->cells[c].illum_val.scat_coef = sigma[c];
    energy[c] = E[c];
    stream[c] = Vector3(F[3 * c], F[3 * c + 1], F[3 * c + 2]);
    Matrix3 m;
    for (int i = 0; i < 3; i++)
      for (int k = 0; k < 3; k++) m(i, k) = T[9 * c + 3 * i + k];
    impuls[c] = m;
  }
  g->energy = energy.data();
  g->stream = stream.data();
  g->impuls = impuls.data();
  for (int64_t c = 0; c < N; c++) {
    Vector4 G4;
    rad_rhd::GetRadSource((int)c, *g, G4);
    for (int i = 0; i < 4; i++) G[4 * c + i] = G4[i];
  }
  g->energy = nullptr;
  g->stream = nullptr;
  g->impuls = nullptr;
  g->cells.clear();
}

// Out-face intensity of one short characteristic: illum::GetIllum(I0, s, k, rhs)
// (solvers/illum/src/illum_utils.cpp:454-490); I0 and s hold 3 values each.
double ref_get_illum(const double *I0, const double *s, double k, double rhs) {
  alignas(32) double i0[4] = {I0[0], I0[1], I0[2], 0.0};
  alignas(32) double ss[4] = {s[0], s[1], s[2], 0.0};
  return illum::GetIllum(i0, ss, k, rhs);
}

// Source function of the transfer equation: illum::GetRhsOpt
// (illum_utils.cpp:631-646) for a cell with opacities alpha, betta and
// temperature T; returns rhs, k_out = alpha + betta.
double ref_get_rhs(double alpha, double betta, double T, double S, double *k_out) {
  elem_t cell;
  full_phys_data_t data;
  data.alpha = alpha;
  data.betta = betta;
  data.T = T;
  cell.cell_data = &data;
  Type k = 0;
  const double r = illum::GetRhsOpt(Vector3(0, 0, 0), S, cell, k);
  cell.cell_data = nullptr;
  *k_out = k;
  return r;
}

// Cell intensities from face values for one direction:
// illum::separate_gpu::ReCalcIllumOpt (illum_utils.cpp:377-433).  Illum [N][M]
// in/out (column `dir` is rewritten); returns the norm it computes.
double ref_recalc_illum(int64_t N, int64_t F, const int32_t *cell_faces, const double *face_area,
                        const double *face_values, int32_t M, int32_t dir, double *Illum) {
  static grid_t *g = new grid_t();  // see ref_rad_source for why it is kept
  g->cells.clear();
  g->faces.clear();
  g->size = N;
  g->size_dir = M;
  g->cells.resize(N);
  g->faces.resize(F);
  for (int64_t c = 0; c < N; c++)
    for (int j = 0; j < 4; j++) g->cells[c].geo.id_faces[j] = cell_faces[4 * c + j];
  for (int64_t f = 0; f < F; f++) g->faces[f].geo.S = face_area[f];
  std::vector<Type> coef(face_values, face_values + F);
  g->Illum = Illum;
  const double norm = illum::separate_gpu::ReCalcIllumOpt(dir, coef, *g, 0);
  g->Illum = nullptr;
  g->cells.clear();
  g->faces.clear();
  return norm;
}

// The emission constants the reference compiles in: GetTemperature's
// g_idealGasConst (lib/physics/include/gas_state.h:22-27), kStefanBoltzmann, PI
// and kRadiation (lib/global_consts.h).
void ref_rad_constants(double *out4) {
  out4[0] = (kM_hydrogen / k_boltzmann) * kPressure / kDensity;
  out4[1] = kStefanBoltzmann;
  out4[2] = PI;
  out4[3] = kRadiation;
}
#endif  // RRHD_SHIM_RAD

}  // extern "C"
