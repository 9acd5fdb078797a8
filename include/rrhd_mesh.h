/* rrhd_mesh.h - synthetic inputs for the RadRHD_solver hot path.
 *
 * The reference reads its tetrahedral meshes from VTK files and converts them
 * with ConvertBinToGeo (lib/geometry/src/convert_bin_to_geo.cpp:3-48); VTK is
 * not available here, so meshes are generated: an axis-aligned hex grid, each
 * hex split into the 6 Kuhn tetrahedra that share its main diagonal, interior
 * vertices jittered by a seeded counter-based RNG.  Faces are assembled in the
 * same order and orientation as ConvertBinToGeo: cells are scanned in order,
 * local faces 0..3; a face is created at its first incidence, takes that cell as
 * id_l and that cell's outward normal; the second incidence becomes id_r.
 *
 * Direction sets mirror the "N, area x y z ..., full_area" sphere files read by
 * files_sys::txt::ReadSphereDirectionCartesian (lib/files_sys/src/reader_txt.cpp:6-37).
 * No entry point here has a counterpart among the reference's hot-path calls.
 */
#ifndef RRHD_MESH_H
#define RRHD_MESH_H

#include <stdint.h>

#include "rrhd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int32_t nx, ny, nz; /* hexes per axis                                        */
  double lo[3], hi[3];/* box                                                    */
  double jitter;      /* vertex jitter, fraction of the hex edge (e.g. 0.15)    */
  uint64_t seed;
  int32_t bc_code[6]; /* boundary code of the x-, x+, y-, y+, z-, z+ planes      */
                      /* (0 means -1, e_bound_free)                            */
  double inflow_radius; /* > 0: z- faces whose centroid lies within this radius */
  int32_t inflow_code;  /*      of the box axis get this code                   */
} rrhd_kuhn_params;

rrhd_status rrhd_mesh_kuhn_sizes(const rrhd_kuhn_params *p, int64_t *n_cells, int64_t *n_faces,
                                 int64_t *n_vertices);

/* All outputs are caller-allocated host arrays sized by rrhd_mesh_kuhn_sizes.
 * vertices [V][3] and cell_vertices [N][4] may be NULL.  h_min receives
 * min over cells of 3V / (largest face area). */
rrhd_status rrhd_mesh_kuhn_build(const rrhd_kuhn_params *p, int32_t *face_id_l,
                                 int32_t *face_id_r, double *face_n, double *face_area,
                                 int32_t *cell_faces, uint8_t *cell_sign, double *cell_volume,
                                 double *cell_center, double *h_min, double *vertices,
                                 int32_t *cell_vertices);

/* Fibonacci sphere with equal weights 4 pi / M and full_area = 4 pi. */
rrhd_status rrhd_directions_fibonacci(int32_t M, double *dirs, double *areas, double *full_area);

/* Synthetic intensity I [rows][M] on the device (rows = cells x groups, cell-major):
 *   kind 0: exp(sigma z) * exp(-|x_c|^2 / 0.2), x_c from centers [cells][3] (device; NULL: no envelope)
 *   kind 1: 10^(-6 + 6 g / (groups - 1)) * exp(sigma z), g = row % groups
 * z standard normal (Box-Muller on the counter-based RNG), a pure function of (seed, row, k). */
rrhd_status rrhd_fill_intensity_f32(float *I, int64_t rows, int32_t M, int32_t groups, int32_t kind,
                                    double sigma, const double *centers, uint64_t seed, void *stream);
rrhd_status rrhd_fill_intensity_f64(double *I, int64_t rows, int32_t M, int32_t groups, int32_t kind,
                                    double sigma, const double *centers, uint64_t seed, void *stream);

/* Primitive states W [n][5] on the device for the con2prim benchmark: rho
 * log-uniform [1e-4, 1e2], p/rho log-uniform [1e-6, 1e2], Lorentz factor
 * log-uniform [1, 50], isotropic velocity direction (counter-based RNG). */
rrhd_status rrhd_fill_c2p_states(double *W, int64_t n, uint64_t seed, void *stream);

/* Counter-based uniform [0,1) variate: the same value on host and device. */
double rrhd_rng_u01(uint64_t seed, uint64_t stream, uint64_t index);

#ifdef __cplusplus
}
#endif
#endif
