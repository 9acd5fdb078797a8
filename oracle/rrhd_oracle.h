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

/* ---------------------------------------------------------------- transport sweep
 * Short-characteristics sweep of solvers/illum/src/mpi/multi_gpu/illum_multi_gpu_face_calc.cpp:91-190
 * on a tetrahedral mesh.  Local face j of a cell is the face opposite its vertex j
 * (cell_faces[c][j], the ConvertBinToGeo order); cell_nbr[c][j] is the cell across
 * it or -1 on the boundary (intensity bc there).  The outward normal of a cell's
 * face is the mesh face normal signed by cell_sign, so two neighbours always
 * classify their shared face consistently (in for one, out for the other). */
typedef struct {
  int64_t n_cells, n_faces;
  const double *cell_volume;    /* [N] */
  const int32_t *cell_faces;    /* [N][4] */
  const int32_t *cell_nbr;      /* [N][4] */
  const uint8_t *cell_sign;     /* [N] bit j: face j's normal is outward for this cell */
  const double *face_n;         /* [F][3] */
  const double *face_area;      /* [F] */
} orc_sweep_mesh;

/* illum::GetIllum (solvers/illum/src/illum_utils.cpp:454-490) */
double orc_get_illum(const double *I0, const double *s, double k, double rhs);
/* illum::GetRhsOpt (illum_utils.cpp:631-646) with the emission Q given */
double orc_get_rhs(double alpha, double betta, double Q, double S, double *k);
/* illum::separate_gpu::ReCalcIllumOpt (illum_utils.cpp:377-433): writes column dir
 * of Illum [N][M] from face values [F]; returns the relative-change norm. */
double orc_recalc_illum(int64_t N, const int32_t *cell_faces, const double *face_area,
                        const double *face_values, int32_t M, int32_t dir, double *Illum);
/* One sweep of all M directions and G groups: S [N*G][M] (rows cell*G+g) in,
 * I [N*G][M] out.  alpha, betta [N]; Q [N][G] emission per group.  Returns the
 * number of (cell, direction) pairs a dependency cycle left unswept (0 normally). */
void orc_trace_nodes(const orc_sweep_mesh *m, int32_t M, const double *dirs, int32_t *in_face, double *s);
int64_t orc_sweep(const orc_sweep_mesh *m, int32_t M, const double *dirs, int32_t G, const double *alpha,
               const double *betta, const double *Q, const double *S, double bc, double *I);

/* Frequency-coupled Compton scattering over the 100-bin spectrum
 * (cuda/src/short_characteristics/separate_gpu/spectrum/cuda_scat_full_spectrum.cu:8-118,
 * one call per (cell, direction, frequency) of Get_full_spectrum_multi_device).
 * I [cells][M][100], vel [cells][3] (units of c), dirs [M][3], areas [M];
 * S [cells][out_stride][100], directions dir_disp .. dir_disp + dir_count - 1. */
#define ORC_N_FRQ 100
void orc_compton_full_spectrum(int32_t M, const double *dirs, const double *areas, double full_area,
                               int64_t cells, const double *I, const double *vel, int32_t dir_disp,
                               int32_t dir_count, int32_t out_stride, double *S, int nthreads);
/* get_frq (cuda_scat_full_spectrum.cu:54-59) and get_frq_idx (:50-53), the latter with
 * the device's saturating float-to-int conversion (NaN -> 0). */
double orc_compton_frq(int32_t idx);
int32_t orc_compton_frq_idx(double frq);
/* Compton-shifted scattering integral at one frequency
 * (cuda/src/short_characteristics/separate_gpu/spectrum/cuda_scat_spectrum.cu:41-83,
 * Get_spectrum_multi_device; its GammaC :22-39 has no forward special case, cfl = 0.25).
 * I [cells][M] at frequency frq; S [cells][out_stride]. */
void orc_compton_spectrum(int32_t M, const double *dirs, const double *areas, double full_area, int64_t cells,
                          const double *I, const double *vel, double frq, int32_t dir_disp, int32_t dir_count,
                          int32_t out_stride, double *S, int nthreads);
/* Ray tracing of the image plane (cuda/src/ray_tracing/cuda_ray_calc.cu,
 * cuda_ray_geo_intersect.cu).  ray [6] = {orig, dir}; abc [9] = {A, B, C}.
 * Codes: -1 none, -2 disk, -3 sphere, -4 Roche lobe, else the triangle's id. */
#define ORC_RAY_NONE (-1)
#define ORC_RAY_DISK (-2)
#define ORC_RAY_SPHERE (-3)
#define ORC_RAY_ROCHE (-4)
double orc_ray_triangle(const double *ray, const double *abc);
int32_t orc_ray_roche(const double *ray, double *dist);
int32_t orc_ray_sphere_disk(const double *ray);
/* mode 0 RayTracing, 1 RayTracing_Phl1445, 2 InnerRayTracing, 3 RayTracingGrid; rays [M][6],
 * ids [N], abc [N][9]; out [M]. */
void orc_ray_trace(int32_t mode, const double *rays, int64_t M, const int32_t *ids, const double *abc, int64_t N,
                   int32_t *out, int nthreads);
/* ray_tracing::MakeRays(frame) (solvers/ray_tracing/src/ray_tracing_build_plane.cpp):
 * rays [600 * 300][6], ray i * 300 + j for pixel (i, j). */
void orc_ray_make_rays(int32_t frame, double *rays);

#ifdef __cplusplus
}
#endif
#endif
