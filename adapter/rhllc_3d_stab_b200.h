// Controls of the hydro drop-in (adapter/rhllc_3d_stab_b200.cpp), which defines the
// reference's rhllc::Hllc3dStab (solvers/rhllc/include/rhllc_calc.h:32) on the B200
// library.  A driver that wants more than the reference's behaviour includes this
// header; the reference's own drivers need none of it.
#pragma once
#include "solvers_struct.h"

namespace rhllc_b200 {
/// State of boundary code `code` (< 0) for the following steps: RRHD_BC_TRANSMISSIVE,
/// RRHD_BC_FIXED with the primitive state W = {rho, v, p}, or RRHD_BC_REFLECT.
void SetBoundary(int code, int kind, const double *W);
/// Refresh grid.faces[].f after each step (off by default).
void KeepFaceFlux(bool on);
/// Keep the state on the device between calls; grid.cells is refreshed by SyncToHost only.
void SetResident(bool on);
/// Resident mode: copy the device state into grid.cells (before WriteSolution).
void SyncToHost(grid_t &grid);
/// Resident mode: the host changed grid.cells; the next call uploads them.
void SyncToDevice(grid_t &grid);
/// Free the device copy of the mesh and state.
void Release();
}  // namespace rhllc_b200
