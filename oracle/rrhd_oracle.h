/* Test infrastructure, not product code.
 *
 * Plain-C restatement of the RadRHD_solver hot path (the checker for the CUDA
 * library).  Every function follows one reference function operation by
 * operation, in the same order, so that on x86-64 with IEEE double arithmetic
 * and no FMA contraction (gcc -O2 -ffp-contract=off) it reproduces the
 * reference bit for bit.  Each definition in rrhd_oracle.c cites the reference
 * file:line it restates.  Parity of this file with the reference is pinned by
 * tests/test_oracle_vs_ref.py against the reference compiled from its own
 * sources (oracle/Makefile "ref").
 *
 * States are 5 doubles: primitive W = {rho, vx, vy, vz, p}, conservative
 * U = {D, Sx, Sy, Sz, E} (E includes the rest mass), the flux_t layout of
 * lib/grids/include/solvers_struct.h:51-70.
 */
#ifndef RRHD_ORACLE_H
#define RRHD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_EOS_IDEAL = 1, ORC_EOS_TAUB = 2 };

typedef struct {
  int eos;       /* ORC_EOS_IDEAL or ORC_EOS_TAUB */
  double gamma1; /* adiabatic index (kGamma1); ideal gas only */
} orc_eos;

/* Mesh in the reference's face/cell form (geo_face_t / geo_cell_t). */
typedef struct {
  int64_t n_cells, n_faces;
  const int32_t *face_id_l;  /* [F] */
  const int32_t *face_id_r;  /* [F] neighbour or negative boundary code */
  const double *face_n;      /* [F][3] unit normal, outward from id_l */
  const double *face_area;   /* [F] */
  const int32_t *cell_faces; /* [N][4] */
  const uint8_t *cell_sign;  /* [N] bit j set: face j's normal is outward */
  const double *cell_volume; /* [N] */
  const double *cell_center; /* [N][3] */
} orc_mesh;

/* Boundary table for codes -1..-8 (index -code-1).
 * kind 0: transmissive copy of the inner cell (e_bound_free)
 * kind 1: fixed state (W, U)
 * kind 2: reflecting wall (e_bound_lock for non-Cone geometries) */
typedef struct {
  int32_t kind[8];
  double W[8][5];
  double U[8][5];
} orc_bc;

void orc_p2c(const orc_eos *eos, double *W, double *U);
void orc_p2c_plain(const orc_eos *eos, const double *W, double *U);
int orc_c2p(const orc_eos *eos, const double *U, double *W);
int orc_pressure_fix(const orc_eos *eos, double *U, double *W);
void orc_rotation(const double *n, double *T /* 3x3 row-major */);
double orc_flux(const orc_eos *eos, const double *UL, const double *UR, const double *WL,
                const double *WR, const double *n, double area, double *F);

/* One reference hydro step (flux loop, update loop, con2prim with fallback).
 * U, W [N][5] in/out; face_flux [F][5] scratch/out; status [N] (may be NULL):
 * bits 0-2 con2prim code, bit 4 fallback ran, bit 5 fallback failed.
 * Returns the max signal speed. */
double orc_hydro_step(const orc_eos *eos, const orc_mesh *mesh, const orc_bc *bc, double tau,
                      double *U, double *W, double *face_flux, int32_t *status, int nthreads);
double orc_time_step(double cfl, double h_min, double max_speed);

/* Scattering integral, cell-major I [N][M] -> S [N][M]. */
void orc_scatter(int64_t N, int32_t M, const double *I, const double *dirs, const double *areas,
                 double full_area, double *S, int nthreads);
/* Energy / stream / impulse moments: E [N], F [N][3], T [N][3][3] row-major. */
void orc_moments(int64_t N, int32_t M, const double *I, const double *dirs, const double *areas,
                 double full_area, double *E, double *F, double *T, int nthreads);

/* Emission constants of rad_rhd::GetRadSource: T = temp_coef*p/rho,
 * B = T^4 * sigma_sb / pi, q = -alpha*rho*B/rad_unit. */
typedef struct {
  double temp_coef, sigma_sb, pi, rad_unit;
} orc_emission;

void orc_rad_source(int64_t N, const orc_emission *em, const double *W, const double *alpha,
                    const double *sigma, const double *E, const double *F, const double *T,
                    double *G);

#ifdef __cplusplus
}
#endif
#endif
