/* rrhd.h - C ABI of the B200 implementation of the RadRHD_solver coupled step.
 *
 * Drop-in boundary for the reference's hot path (Lartsev-Artem/RadRHD_solver):
 * the relativistic HLLC hydro step with con2prim, the radiation scattering
 * integral and its energy/stream/impulse moments, and the radiation 4-force
 * source.  Every entry point below names the reference interface it stands
 * behind (paths are inside the reference project).
 *
 * Conventions
 *  - Plain pointers and sizes only.  States are 5 doubles per cell, the flux_t
 *    layout of lib/grids/include/solvers_struct.h:51-70: primitive
 *    W = {rho, vx, vy, vz, p}; conservative U = {D, Sx, Sy, Sz, E}.
 *  - Every function returns rrhd_status (0 = success) and never aborts the
 *    process; rrhd_last_error() gives a message for the calling thread.
 *  - Pointers marked "device" must be device memory of the context's GPU;
 *    "host" pointers may be pageable or pinned.  Functions taking a `where`
 *    argument accept either (RRHD_HOST / RRHD_DEVICE).
 *  - Work is ordered on the context's CUDA stream (or the stream argument);
 *    functions that return data to host pointers synchronise that stream.
 *  - One context per host thread at a time.
 */
#ifndef RRHD_H
#define RRHD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t rrhd_status;
#define RRHD_OK 0
#define RRHD_ERR_INVALID 1 /* bad argument */
#define RRHD_ERR_CUDA 2    /* a CUDA call failed */
#define RRHD_ERR_OOM 3     /* device allocation failed */
#define RRHD_ERR_C2P 4     /* con2prim failed in some cells even after the fallback */
#define RRHD_ERR_STATE 5   /* call made in the wrong order / missing data */
#define RRHD_ERR_LIMIT 6   /* size beyond a fixed limit of the entry point */

#define RRHD_HOST 0
#define RRHD_DEVICE 1

#define RRHD_EOS_IDEAL 1 /* h = 1 + Gamma/(Gamma-1) p/rho   (include/hd_config.h:17) */
#define RRHD_EOS_TAUB 2  /* Taub-Matthews h                  (include/hd_config.h:18) */

/* Boundary kinds for negative face neighbour codes (lib/global_types.h:25-31). */
#define RRHD_BC_TRANSMISSIVE 0 /* copy of the inner cell (e_bound_free)            */
#define RRHD_BC_FIXED 1        /* fixed primitive state, e.g. an inflow nozzle      */
#define RRHD_BC_REFLECT 2      /* wall: normal velocity reversed (e_bound_lock)     */

/* Per-cell status byte written by the hydro step and the batch con2prim:
 * bits 0-2: code of rhllc::GetPhysValueStab (0 ok, 1 no solution, 2 p<0,
 *           3 inaccurate, 4 NaN, 5 Lorentz factor < 1 where the reference aborts);
 * bit 4: the PhysPressureFix fallback ran; bit 5: the fallback failed too. */
#define RRHD_STATUS_FALLBACK 0x10
#define RRHD_STATUS_FAILED 0x20

typedef struct rrhd_ctx rrhd_ctx;

/* Mesh in the reference's face/cell form: geo_face_t / geo_cell_t,
 * lib/grids/include/solvers_struct.h:87-162, as assembled by ConvertBinToGeo
 * (lib/geometry/src/convert_bin_to_geo.cpp:3-48).  Host pointers. */
typedef struct {
  int64_t n_cells;
  int64_t n_faces;
  const int32_t *face_id_l;  /* [F] cell on the normal's tail side            */
  const int32_t *face_id_r;  /* [F] neighbour cell, or negative boundary code  */
  const double *face_n;      /* [F][3] unit normal, outward from id_l         */
  const double *face_area;   /* [F]                                            */
  const int32_t *cell_faces; /* [N][4] face ids (id_faces)                     */
  const uint8_t *cell_sign;  /* [N] bit j set: face j's normal points outward  */
  const double *cell_volume; /* [N]                                            */
  const double *cell_center; /* [N][3]                                         */
} rrhd_mesh_desc;

typedef struct {
  int32_t eos;             /* RRHD_EOS_IDEAL (default when 0) or RRHD_EOS_TAUB        */
  double gamma;            /* adiabatic index, ideal gas (default 5/3 when 0)        */
  int32_t device;          /* CUDA device ordinal                                    */
  int32_t cells_per_block; /* cells per CTA in the fused step; 0 = default (256)     */
  int32_t renumber;        /* 0 = default Morton renumbering, -1 = keep input order  */
} rrhd_opts;

typedef struct {
  double max_speed;     /* max signal speed of the step (rhllc::max_signal_speed) */
  int64_t n_fallback;   /* cells where PhysPressureFix ran                        */
  int64_t n_failed;     /* cells where the fallback failed too                    */
} rrhd_step_stats;

/* ------------------------------------------------------------------ context */

/* Device-resident copy of the mesh and state.  Stands behind
 * cuda::interface::separate_device::InitDevice
 * (cuda/include/short_characteristics/separate_gpu/cuda_multi_interface.h:44)
 * and grid_t::InitMemory (lib/grids/src/solvers_struct.cpp:146-180). */
rrhd_status rrhd_create(const rrhd_mesh_desc *mesh, const rrhd_opts *opts, rrhd_ctx **out);
/* The step kernel's layout (no counterpart in the reference): cells per CTA, the number of
 * CTA blocks, and face_entries, the length of all CTAs' face lists together (a face between
 * two CTAs' blocks is fluxed by both; each list is padded to an even length), against the
 * mesh's faces.  Any pointer may be NULL. */
rrhd_status rrhd_hydro_layout_info(const rrhd_ctx *ctx, int32_t *cells_per_block, int32_t *blocks,
                                   int64_t *face_entries, int64_t *faces);

/* Frees everything.  Stands behind separate_device::ClearDevice / ClearHost
 * (cuda_multi_interface.h:50, :57). */
rrhd_status rrhd_destroy(rrhd_ctx *ctx);

/* The context's CUDA stream (a cudaStream_t). */
void *rrhd_stream(rrhd_ctx *ctx);
rrhd_status rrhd_sync(rrhd_ctx *ctx);

/* Boundary state for a negative face code (-1..-8).  W is the primitive state
 * for RRHD_BC_FIXED (its conservative state is made by rhllc::GetConvValue,
 * solvers/rhllc/src/rhllc_flux.cpp:7-16); ignored otherwise.  Stands behind the
 * compile-time per-geometry states of rhllc::BoundConditions
 * (solvers/rhllc/src/rhllc_utils.cpp:45-133). */
rrhd_status rrhd_set_boundary(rrhd_ctx *ctx, int32_t code, int32_t kind, const double *W);

/* Cell state in the caller's numbering, [N] records of `stride` doubles whose
 * first 5 are the state (stride 5 for packed arrays).  Either pointer may be
 * NULL to skip it.  Mirrors grid.cells[i].phys_val / conv_val. */
rrhd_status rrhd_set_state(rrhd_ctx *ctx, const double *W, const double *U, int64_t stride,
                           int32_t where);
rrhd_status rrhd_get_state(rrhd_ctx *ctx, double *W, double *U, int64_t stride, int32_t where);

/* Sets W (rescaling |v| >= 1 as the reference does) and derives U on the
 * device: rhllc::HllcPhysToConv / GetConvValueStab
 * (solvers/rhllc/src/rhllc_utils.cpp:25-33, rhllc_flux_stab.cpp:10-38). */
rrhd_status rrhd_set_state_prim(rrhd_ctx *ctx, const double *W, int64_t stride, int32_t where);

/* One hydro step: RHLLC face fluxes, conservative update and con2prim with the
 * PhysPressureFix fallback, fused in one kernel.  Stands behind
 * void rhllc::Hllc3dStab(const Type tau, grid_t &grid)
 * (solvers/rhllc/include/rhllc_calc.h:32, solvers/rhllc/src/rhllc_3d_stab.cpp:10-63).
 * tau > 0: that time step.  tau <= 0: tau = CFL*h_min/max_speed of the previous
 * step, computed on the device (rhllc::GetTimeStep, rhllc_utils.cpp:15-23;
 * set CFL/h_min with rrhd_set_time_step).  stats may be NULL (no host sync);
 * otherwise the call synchronises and fills it.  Returns RRHD_ERR_C2P when some
 * cell failed even after the fallback (the reference aborts there). */
rrhd_status rrhd_hydro_step(rrhd_ctx *ctx, double tau, rrhd_step_stats *stats);
rrhd_status rrhd_set_time_step(rrhd_ctx *ctx, double cfl, double h_min, double initial_max_speed);
/* Last time step used and the max signal speed it produced (synchronises). */
rrhd_status rrhd_get_step_info(rrhd_ctx *ctx, double *tau_used, double *max_speed);

/* Drop-in with host buffers: uploads W and U, runs one step, downloads W and U
 * (the whole body of rhllc::Hllc3dStab on a host grid_t).  stride as above. */
rrhd_status rrhd_hydro_step_host(rrhd_ctx *ctx, double tau, double *W, double *U, int64_t stride,
                                 rrhd_step_stats *stats);

/* Keep the face fluxes of the following steps in a [F][5] device array
 * (off by default: it costs F*40 bytes of writes per step). */
rrhd_status rrhd_keep_face_flux(rrhd_ctx *ctx, int32_t on);
/* Face fluxes of the last step, [F][5] in the caller's face numbering (the
 * grid.faces[].f the reference leaves behind).  Host pointer. */
rrhd_status rrhd_get_face_flux(rrhd_ctx *ctx, double *F);
/* Per-cell status bytes of the last step (bits above), caller's numbering. */
rrhd_status rrhd_get_cell_status(rrhd_ctx *ctx, uint8_t *status);

/* ------------------------------------------------ hydro step split over ranks */

/* Cell order of a context built on `mesh` with rrhd_opts.renumber = `renumber`:
 * order[k] = caller id of the context's k-th cell (Morton order of the cell centres, or
 * the input order when renumber < 0).  Host only; needs no device. */
rrhd_status rrhd_cell_order(const rrhd_mesh_desc *mesh, int32_t renumber, int32_t *order);

/* Split of the hydro step over `world` ranks, each holding the whole mesh: rank q updates
 * the CTA blocks [nb q/world, nb (q+1)/world) of the context order (nb blocks of
 * `cells_per_block` cells; 0 = 256) and exchanges with the other ranks the states of the
 * face neighbours of its cells that they update.  Host only; needs no device.
 *   cell_range[2]   this rank's cells [begin, end) in context order;
 *   send_counts, recv_counts [world]: cells sent to / received from each rank;
 *   send_ids, recv_ids: context-order cell ids grouped by peer in rank order, ascending
 *                   within a peer (NULL for a counts-only call).
 * rank q's recv_ids from rank p equal rank p's send_ids to rank q.  Stands behind
 * rhllc_mpi::InitMpiConfig (solvers/rhllc/src/rhllc_3d_mpi.cpp:86-369), whose partition
 * is a caller-grouped METIS map; here it is Morton-ordered CTA blocks. */
rrhd_status rrhd_part_plan(const rrhd_mesh_desc *mesh, const int32_t *order, int32_t cells_per_block,
                           int32_t world, int32_t rank, int64_t *cell_range, int64_t *send_counts,
                           int64_t *recv_counts, int32_t *send_ids, int32_t *recv_ids);

/* Restricts the context's hydro step to rank `rank`'s blocks of rrhd_part_plan and keeps
 * its exchange lists on the device; world = 1 restores the whole-mesh step.  Cells outside
 * the rank's range are not written by the step.  A rank's step follows the reference's
 * rhllc_mpi::Hllc3dStab (rhllc_3d_mpi.cpp:371-486):
 *   rrhd_hydro_pack_halo -> exchange of the send / recv buffers between ranks ->
 *   rrhd_hydro_unpack_halo -> rrhd_hydro_step -> max-reduction over ranks of the double
 *   at rrhd_hydro_max_speed_ptr (the next step's tau <= 0 reads it).
 * Kept face fluxes (rrhd_keep_face_flux) are written for the faces whose id_l cell the rank
 * updates.  The coupled step and rrhd_hydro_step_host refuse a split context. */
rrhd_status rrhd_hydro_set_part(rrhd_ctx *ctx, int32_t world, int32_t rank);
/* cell_range[2], send_counts / recv_counts [world] of the split, and the caller ids of the
 * rank's cells [cell_range[1] - cell_range[0]].  Any pointer may be NULL. */
rrhd_status rrhd_hydro_part_info(rrhd_ctx *ctx, int64_t *cell_range, int64_t *send_counts,
                                 int64_t *recv_counts, int32_t *cells);
/* Gathers the current states (U(5), W(5): 10 doubles a cell) of the cells to send into
 * send_buf [sum send_counts][10] (device), in send_ids order, on the context's stream.
 * Stands behind the send side of StartExchangeBoundaryCells (rhllc_3d_mpi.cpp:69-80). */
rrhd_status rrhd_hydro_pack_halo(rrhd_ctx *ctx, double *send_buf);
/* Scatters recv_buf [sum recv_counts][10] (device) into the current states of the
 * received cells, on the context's stream (SyncExchangeBoundaryCells, :81-85). */
rrhd_status rrhd_hydro_unpack_halo(rrhd_ctx *ctx, const double *recv_buf);
/* Device address of the last step's max signal speed (one double; the address alternates
 * between steps, so query it after every step).  rhllc::max_signal_speed, which
 * rhllc_mpi::Hllc3dStab reduces with MPI_MAX over ranks (:461-485). */
rrhd_status rrhd_hydro_max_speed_ptr(rrhd_ctx *ctx, double **max_speed);

/* ------------------------------------------------------------ batch kernels */

/* con2prim for n states, device pointers, on `stream` (a cudaStream_t, may be
 * NULL).  rhllc::GetPhysValueStab (rhllc_flux_stab.cpp:123-220), and when
 * fallback != 0 rhllc::PhysPressureFix (:40-121) where it fails, which also
 * rewrites U.E as the reference does.  status [n] may be NULL. */
rrhd_status rrhd_con2prim_batch(int32_t eos, double gamma, double *U, double *W, uint8_t *status,
                                int64_t n, int32_t fallback, void *stream);
/* Totals over a con2prim batch. */
typedef struct {
  int64_t n_ok;         /* states solved by the Newton iteration                 */
  int64_t n_fallback;   /* states that went to PhysPressureFix                   */
  int64_t n_failed;     /* states where the fallback failed too (or no fallback) */
  int64_t newton_iters; /* Newton iterations summed over all states              */
  int32_t max_iters;    /* largest Newton iteration count of one state           */
} rrhd_c2p_stats;

/* rrhd_con2prim_batch plus the totals above, reduced per CTA into a device
 * scratch buffer and then summed in a fixed order.  The scratch is one buffer
 * per (device, stream), allocated on first use and grown (after synchronising
 * that stream) when a batch needs more: calls on one stream are ordered, calls
 * on different streams or host threads use separate buffers and may overlap.
 * Synchronises `stream` when stats is not NULL.  Same reference
 * functions as rrhd_con2prim_batch (rhllc::GetPhysValueStab / PhysPressureFix);
 * the iteration counts are those of the loop at rhllc_flux_stab.cpp:153-183. */
rrhd_status rrhd_con2prim_batch_stats(int32_t eos, double gamma, double *U, double *W,
                                      uint8_t *status, int64_t n, int32_t fallback,
                                      rrhd_c2p_stats *stats, void *stream);

/* The same computation as rrhd_con2prim_batch_stats without allocating any
 * device memory (no counterpart in the reference).  For callers that cannot
 * call cudaMalloc: hosts whose memory pool or arena already reserves the GPU,
 * and latency-critical loops that cannot take cudaMalloc's implicit device
 * synchronisation.  The per-CTA partial totals live in a fixed file-scope
 * device array of 320 KiB, held by every GPU that loads the library until the
 * process exits, so n is limited to 16,777,216 states (RRHD_ERR_LIMIT beyond).
 * The first call on a device (and the first after the device was reset) looks
 * up that array's device address (make it before any stream capture).  Every
 * call shares the array: calls that overlap on the GPU race and must be
 * serialised by the caller. */
rrhd_status rrhd_con2prim_batch_stats_noalloc(int32_t eos, double gamma, double *U, double *W,
                                              uint8_t *status, int64_t n, int32_t fallback,
                                              rrhd_c2p_stats *stats, void *stream);

/* ------------------------------------------------ learned con2prim guess
 * A 3-64-64-1 ReLU network predicting log(p/tau), tau = E - D, from
 * (log(Q/tau), log(|S|/tau), log(tau/D)), Q = E - sqrt(|S|^2 + D^2) (all built in
 * FP64 from D, |S|/tau, tau/D); trained on the device by this library's
 * own forward/backward/Adam kernels; its prediction seeds the Newton solve of
 * rhllc::GetPhysValueStab (rhllc_flux_stab.cpp:123-220), which has no learned
 * part of its own.  Parameters: 4481 floats = W1[64][3], b1[64], W2[64][64]
 * (row = output), b2[64], W3[64], b3; normalisation: 8 floats = mu[3],
 * sigma[3] of the features, mu, sigma of the target. */
typedef struct rrhd_mlp rrhd_mlp;
int32_t rrhd_mlp_num_params(void);
rrhd_status rrhd_mlp_create(int32_t device, uint64_t seed, rrhd_mlp **out);
rrhd_status rrhd_mlp_destroy(rrhd_mlp *m);
/* host copies of the parameters / normalisation (either pointer may be NULL) */
rrhd_status rrhd_mlp_set(rrhd_mlp *m, const float *theta, const float *norm);
rrhd_status rrhd_mlp_get(const rrhd_mlp *m, float *theta, float *norm);
/* Adam on labelled states U [n][5], p [n] (device): mini-batches of `batch`
 * (multiple of 128) in a seeded order; lr halved at 50 % and 75 % of the epochs;
 * set_norm != 0 derives the normalisation from the data; loss_hist (host
 * [epochs], may be NULL) gets each epoch's mean squared normalised error. */
rrhd_status rrhd_mlp_train(rrhd_mlp *m, const double *U, const double *p, int64_t n, int32_t epochs,
                           int32_t batch, float lr, uint64_t seed, int32_t set_norm, float *loss_hist,
                           void *stream);
/* Gradient (host [4481]) and loss of the mean squared normalised error over
 * all n labelled states at the current parameters. */
rrhd_status rrhd_mlp_gradient(rrhd_mlp *m, const double *U, const double *p, int64_t n, float *grad,
                              float *loss);
/* con2prim batch seeded by the network: Newton from the learned guess for at
 * most k_stall iterations, else the reference solve from its own guess, then
 * PhysPressureFix when fallback != 0.  stats / n_guess_fallback (host) and
 * guess (device [n], the learned initial pressures, 0 where the network gives
 * no usable guess) may be NULL.  The network object holds the call's scratch
 * (per-CTA statistics, the guesses when guess is NULL): calls with one object
 * must not overlap (one stream, or the caller serialises them). */
rrhd_status rrhd_con2prim_batch_mlp(const rrhd_mlp *m, int32_t eos, double gamma, double *U, double *W,
                                    uint8_t *status, int64_t n, int32_t fallback, int32_t k_stall,
                                    rrhd_c2p_stats *stats, int64_t *n_guess_fallback, double *guess,
                                    void *stream);

/* prim->cons for n states, device pointers: rhllc::GetConvValueStab. */
rrhd_status rrhd_prim2con_batch(int32_t eos, double gamma, double *W, double *U, int64_t n,
                                void *stream);

/* ------------------------------------------------------------ radiation */

typedef struct rrhd_dirs rrhd_dirs;

/* Direction set on the device: unit vectors [M][3], quadrature weights [M] and
 * their normaliser full_area (grid_directions_t, lib/geometry/include/geo_types.h:110-127,
 * read by files_sys::txt::ReadSphereDirectionCartesian, lib/files_sys/src/reader_txt.cpp:6-37). */
rrhd_status rrhd_dirs_create(int32_t M, const double *dirs, const double *areas, double full_area,
                             int32_t device, rrhd_dirs **out);
rrhd_status rrhd_dirs_destroy(rrhd_dirs *d);

/* Scattering integral S[r][k] = sum_d Gamma(w_d.w_k) I[r][d] a_d / full_area with
 * the Thomson Gamma = 3(1+mu^2)/4, FP64, same operation order as
 * cuda::kernel::GetS_MPI_multi_device (cuda/src/short_characteristics/cuda_scattering.cu:82-105).
 * I, S device [rows][M], rows = cells x groups.  Stands behind
 * separate_device::CalculateIntScatteringAsync (cuda_multi_interface.h:81). */
rrhd_status rrhd_scatter_fp64(const rrhd_dirs *d, const double *I, double *S, int64_t rows,
                              void *stream);

/* The same contraction with one FMA per term on the precomputed matrix
 * K[d][k] = Gamma(d,k) a_d / full_area (differs from the reference's three
 * roundings per term by a few ulp). */
rrhd_status rrhd_scatter_fp64_fma(const rrhd_dirs *d, const double *I, double *S, int64_t rows,
                                  void *stream);
int32_t rrhd_dirs_count(const rrhd_dirs *d);
/* Device pointer to K [M][M] (row d), for callers that build their own kernels. */
const double *rrhd_dirs_device_kernel(const rrhd_dirs *d);

/* Energy E[r], stream F[r][3], impulse T[r][3][3] (row-major) moments, FP64,
 * same order as cuda_sep::kernel::MakeIllumParam
 * (cuda/src/short_characteristics/separate_gpu/cuda_illum_sep_param.cu:9-83).
 * Stands behind separate_device::CalculateAllParamAsync (cuda_multi_interface.h:69).
 * Device pointers. */
rrhd_status rrhd_moments_fp64(const rrhd_dirs *d, const double *I, double *E, double *F,
                              double *T, int64_t rows, void *stream);

/* Scattering integral and moments on the tensor cores (tcgen05), FP32 in/out.
 * The same contraction as rrhd_scatter_fp64 plus the moments as 16 extra
 * output columns, with the kernel matrix split into 16-bit parts once at
 * creation.  Forms (maximum relative error against FP64 measured by the tests on the
 * 256- and 512-direction cases, intensities over 12 decades):
 *   RRHD_TC_BF16X3 : bf16 hi/lo split of I and K, three products        (about 1e-5)
 *   RRHD_TC_F16X3  : per-row power-of-two scaled fp16 hi/lo split, three
 *                    products                                           (below 1e-6)
 *   RRHD_TC_F16    : per-row scaled fp16, one product                   (about 5e-4)
 *   RRHD_TC_BF16   : bf16, one product
 * The scaled forms put only the anisotropic part 3 mu^2 / 4 of the Thomson kernel on the
 * tensor cores and add the isotropic 3/4 E (E = sum_d a_d I_d / A, summed in FP64) to every
 * output; their moments are summed in FP64 by the same row pass (stored as FP32), not on the
 * tensor cores.  M must be 64 or a multiple of 128
 * (<= 1024).  Stands behind
 * CalculateIntScatteringAsync + CalculateAllParamAsync (cuda_multi_interface.h:69, :81). */
#define RRHD_TC_BF16X3 0
#define RRHD_TC_F16X3 1
#define RRHD_TC_F16 2
#define RRHD_TC_BF16 3
typedef struct rrhd_scatter_tc rrhd_scatter_tc;
rrhd_status rrhd_scatter_tc_create(const rrhd_dirs *d, int32_t form, rrhd_scatter_tc **out);
rrhd_status rrhd_scatter_tc_destroy(rrhd_scatter_tc *t);
/* I [rows][M] FP32 -> S [rows][M] FP32 and, when moments is not NULL, moments
 * [rows][16] FP32 = {E, Fx, Fy, Fz, Txx, Txy, Txz, Tyy, Tyz, Tzz, 0...}.  All
 * device pointers, 16-byte aligned. */
rrhd_status rrhd_scatter_tc_run(const rrhd_scatter_tc *t, const float *I, float *S, float *moments,
                                int64_t rows, void *stream);
/* The same three contractions on the cell-direction-group layout the coupled
 * step keeps its intensity in: I, S [cells][M][groups] (row cell * groups + g of
 * the row-layout calls above; moments stay [rows][...]).  groups divides 64 for
 * the FP64 calls and is 1, 2 or 4 for the tensor cores. */
rrhd_status rrhd_scatter_fp64_cdg(const rrhd_dirs *d, const double *I, double *S, int64_t cells, int32_t groups,
                                  int32_t exact, void *stream);
rrhd_status rrhd_moments_fp64_cdg(const rrhd_dirs *d, const double *I, double *E, double *F, double *T,
                                  int64_t cells, int32_t groups, void *stream);
rrhd_status rrhd_scatter_tc_run_cdg(const rrhd_scatter_tc *t, const float *I, float *S, float *moments,
                                    int64_t cells, int32_t groups, void *stream);
/* Scattering integral and moments through the rank-7 structure of the Thomson
 * Gamma: 3/4 (1 + (w_d.w_k)^2) = 3/4 (1 + sum_ij w_d,i w_d,j w_k,i w_k,j), so
 *   S[r][k] = 3/4 (E[r] + w_k^T T[r] w_k),  E = sum_d a_d I / A,  T = sum_d a_d w_d w_d^T I / A,
 * the energy and impulse moments.  One pass over I, O(M) per row instead of O(M^2),
 * FP64 arithmetic throughout; agrees with rrhd_scatter_fp64 to about 1e-15 relative.
 * No counterpart in the reference, whose kernels sum the O(M^2) form
 * (cuda_scattering.cu:82-105); valid for its phase function (scattering.h:32-35) only.
 * I, S device [cells][M][groups] (groups 1 = the row layout [rows][M]), in FP64
 * (precision RRHD_RAD_FP64) or FP32 (RRHD_RAD_FP32); moments NULL or [rows][16] in the
 * same precision = {E, Fx, Fy, Fz, Txx, Txy, Txz, Tyy, Tyz, Tzz, 0...}. */
rrhd_status rrhd_scatter_lowrank(const rrhd_dirs *d, const void *I, void *S, void *moments, int64_t cells,
                                 int32_t groups, int32_t precision, void *stream);
/* Max and rms relative error of an FP32 scattering integral S_test (same layout as
 * rrhd_scatter_lowrank's FP32 case) against the FP64 low-rank values, over every
 * row and direction.  Synchronises `stream`. */
rrhd_status rrhd_scatter_lowrank_error(const rrhd_dirs *d, const float *I, const float *S_test, int64_t cells,
                                       int32_t groups, double *max_rel, double *rms_rel, void *stream);
/* Frequency-coupled Compton scattering integral over the 100-bin spectrum, replacing
 * cuda::kernel::Get_full_spectrum_multi_device
 * (cuda/src/short_characteristics/separate_gpu/spectrum/cuda_scat_full_spectrum.cu:61-118)
 * as CalculateFullSpectrumIntScattering launches it
 * (cuda/src/short_characteristics/separate_gpu/spectrum/cuda_interface_spectrum.cu:94-140):
 *   S[i][k][f] = sum_d GammaC(w_{dir_disp+k}, w_d, frq_f, v_i) I[i][d][bin(frq1)] a_d / A
 * with the Doppler and recoil frequency shift, the Klein-Nishina weight and the
 * low/high cut-offs of that kernel (CGS constants of lib/global_consts.h:34-44).
 * I device FP64 [cells][M][100] (I[i][d][99] is never read: the top bin is always cut);
 * velocity device FP64 [cells][3] in units of c (velocity[shift_gpu + i] of the
 * reference: pass the pointer to this chunk's first cell); S device FP64
 * [cells][out_stride][100] (local_scattering_size = out_stride), output directions
 * dir_disp .. dir_disp + dir_count - 1 (local_scattering_disp, end_dir).  I and S
 * 16-byte aligned.  Asynchronous on `stream`. */
rrhd_status rrhd_compton_full_spectrum(const rrhd_dirs *d, const double *I, const double *velocity, double *S,
                                       int64_t cells, int32_t dir_disp, int32_t dir_count, int32_t out_stride,
                                       void *stream);
/* Compton-shifted scattering integral at one frequency frq (Hz), replacing
 * cuda::kernel::Get_spectrum_multi_device
 * (cuda/src/short_characteristics/separate_gpu/spectrum/cuda_scat_spectrum.cu:41-83) as
 * CalculateSpectrumIntScattering launches it (cuda_interface_spectrum.cu:46-92):
 *   S[i][k] = 0.25 sum_d GammaC(w_{dir_disp+k}, w_d, frq, v_i) I[i][d] a_d / A
 * (that kernel's weight has no forward special case; 0.25 is its cfl factor).
 * I device FP64 [cells][M] at frq; velocity device FP64 [cells][3] in units of c;
 * S device FP64 [cells][out_stride].  Asynchronous on `stream`. */
rrhd_status rrhd_compton_spectrum(const rrhd_dirs *d, const double *I, const double *velocity, double *S,
                                  int64_t cells, double frq, int32_t dir_disp, int32_t dir_count, int32_t out_stride,
                                  void *stream);
/* ---- Image-plane ray tracing (solvers/ray_tracing, cuda/src/ray_tracing) ----------
 * A surface of triangles resident on the device, replacing cuda::ray_tracing::interface::
 * InitDevice / ClearDevice (cuda/src/ray_tracing/cuda_ray_interface.cu:83-99).  face_cells:
 * n FaceCell records as the reference stores them (lib/geometry/include/geo_types.h:77-83:
 * int32 face_id, 4 bytes padding, double A[3], B[3], C[3]; 80 bytes), host or device. */
typedef struct rrhd_ray_surface rrhd_ray_surface;
rrhd_status rrhd_ray_surface_create(const void *face_cells, int64_t n, int32_t device, rrhd_ray_surface **out);
rrhd_status rrhd_ray_surface_destroy(rrhd_ray_surface *s);
/* First intersection of each ray, replacing StartTracing / TracingGrid / FindInnerIntersection
 * (cuda_ray_interface.cu:17-80) and their kernels (cuda/src/ray_tracing/cuda_ray_calc.cu):
 *   mode RRHD_RAY_SURFACE (RayTracing), RRHD_RAY_ROCHE (RayTracing_Phl1445: the donor's Roche
 *   lobe, cuda_ray_geo_intersect.cu:22-86, then nearer triangles), RRHD_RAY_INNER
 *   (InnerRayTracing: accretor sphere / disk, :110-169, else the triangles), RRHD_RAY_GRID
 *   (RayTracingGrid).  rays device [M] Ray_t records {orig[3], direction[3]} (48 bytes);
 *   codes device [M]: the triangle's face_id, or RRHD_RAY_NONE / _DISK / _SPHERE / _LOBE
 *   (e_ray_intersect_code, ray_tracing_const.h).  Asynchronous on `stream`.  Rays sharing one
 *   direction (an image plane) are answered through image-plane bins kept with the surface, so
 *   calls on one surface must not overlap on the GPU; the first call, and a call with more rays
 *   than any before, allocates them. */
#define RRHD_RAY_SURFACE 0
#define RRHD_RAY_ROCHE 1
#define RRHD_RAY_INNER 2
#define RRHD_RAY_GRID 3
#define RRHD_RAY_NONE (-1)
#define RRHD_RAY_DISK (-2)
#define RRHD_RAY_SPHERE (-3)
#define RRHD_RAY_LOBE (-4)
rrhd_status rrhd_ray_trace(const rrhd_ray_surface *s, const double *rays, int64_t M, int32_t mode, int32_t *codes,
                           void *stream);
/* The image-plane rays of frame `frame` (ray_tracing::MakeRays, solvers/ray_tracing/src/
 * ray_tracing_build_plane.cpp, constants of ray_tracing_const.h): host [600 * 300][6],
 * ray i * 300 + j for pixel (i, j).  Host code. */
rrhd_status rrhd_ray_make_rays(int32_t frame, double *rays);
/* One frame of MakeIllumAndCurve / MakeEnergyAndCurve (ray_tracing_calc_illum.cpp): image[i]
 * = value by code (0 none, 1e-5 Roche lobe, 5 disk, 10 sphere, else value[code / cell_size]),
 * *curve = sum of image[i] * pixel_factor (pixel area for the illumination curve, 1 for the
 * energy curve), in a fixed order.  *bad is OR-ed with 1 for a negative code the reference
 * would stop on (DIE_IF).  All pointers device; asynchronous on `stream`. */
rrhd_status rrhd_ray_image(const int32_t *codes, int64_t M, const double *value, int32_t cell_size,
                           double pixel_factor, double *image, double *curve, int32_t *bad, void *stream);
/* Reads (and with clear != 0 resets) the error word of the tensor-core kernels:
 * RRHD_ERR_CUDA if a bounded pipeline wait timed out.  Synchronises `stream`. */
rrhd_status rrhd_scatter_tc_check(const rrhd_scatter_tc *t, void *stream, int32_t clear);

/* Emission constants of rad_rhd::GetRadSource: T = temp_coef*p/rho,
 * B = T^4*sigma_sb/pi, q = -alpha*rho*B/rad_unit (lib/physics/src/plunk.cpp:87-90,
 * lib/physics/include/gas_state.h:22-27).  rrhd_emission_reference() gives the
 * reference's compiled-in CGS values. */
typedef struct {
  double temp_coef, sigma_sb, pi, rad_unit;
} rrhd_emission;
rrhd_emission rrhd_emission_reference(void);

/* Radiation 4-force G [n][4] per cell, rad_rhd::GetRadSource
 * (solvers/RadRHD/src/radRHD_utils.cpp:44-101), device pointers: W [n][5],
 * alpha/sigma [n], E [n], F [n][3], T [n][9]. */
rrhd_status rrhd_rad_source(const rrhd_emission *em, const double *W, const double *alpha,
                            const double *sigma, const double *E, const double *F, const double *T,
                            double *G, int64_t n, void *stream);

/* ------------------------------------------------------------ transport sweep
 * Short-characteristics sweep of illum::separate_gpu::CalculateIllum
 * (solvers/illum/src/mpi/multi_gpu/illum_multi_gpu_face_calc.cpp:20-190, one
 * iteration of its direction loop): for every direction, cells in upwind order;
 * each out-face value is the mean over its three interpolation nodes of
 * illum::GetIllum (illum_utils.cpp:454-490) with the source illum::GetRhsOpt
 * (illum_utils.cpp:631-646); each cell value is illum::separate_gpu::ReCalcIllumOpt
 * (illum_utils.cpp:377-433), area-weighted face mean (plain mean for the last
 * cell).  The upwind order (the reference's sorted_graph, made offline by its
 * graph/ and make_trace/ tools) is built on the device at setup as levels of
 * cells whose upwind neighbours are all done; one level is one kernel launch,
 * all launches of a sweep are one CUDA graph. */
#define RRHD_RAD_FP64 0  /* sweep arithmetic and storage in double */
#define RRHD_RAD_FP32 1  /* in float (input of the tensor-core scattering) */
#define RRHD_RAD_MIXED 2 /* the sweep in double (geometry, records, face values, arithmetic)
                            with the scattering integral S read and the intensity I written
                            in float, the tensor-core scattering's input and output: the
                            intensity is the double sweep's rounded once.  Caller arrays
                            (rrhd_sweep) are float.  Storing the face values in float lets
                            the rounding accumulate along each characteristic; rounding the
                            geometry to float moves the attenuation of faces at grazing
                            incidence and the choice between nearly equally distant
                            in-faces, which over 100 coupled steps of a 5.3M-cell jet moved
                            the hydro state by 8e-7 against 2e-10 with double geometry */
typedef struct {
  int32_t groups;         /* frequency groups G >= 1 (grey copies, rows cell * G + g)           */
  int32_t precision;      /* RRHD_RAD_FP64, RRHD_RAD_FP32 or RRHD_RAD_MIXED                     */
  int32_t dirs_per_batch; /* directions swept together (face values [dirs_per_batch][F][groups] are
                             kept for them): power of two <= 256; 0 = min(64, M)                */
  double boundary_value;  /* intensity entering through boundary faces (illum::BoundaryConditions
                             returns 0 for free, lock and outer boundaries, illum_utils.cpp:52-65) */
  int32_t item_geometry;  /* 1: precompute at setup, per (cell, direction) item in sweep order, which
                             faces are in- and out-faces, the in-face each interpolation node is
                             traced to and the in-face distances H_f / -cos_f (16 bytes per item,
                             cells x directions x 16 bytes of device memory); the sweep then reads
                             that stream in order instead of each item's cell normals and heights.
                             RRHD_RAD_FP32 and RRHD_RAD_MIXED only: the distances are stored as
                             float (FP32: the same values; MIXED: the double distance rounded
                             once, every choice made in double).  0: off                         */
} rrhd_rad_opts;
/* Builds the sweep geometry and plan for ctx's mesh and the direction set (which
 * must outlive the context's radiation use).  RRHD_ERR_STATE if the mesh has a
 * dependency cycle for some direction. */
rrhd_status rrhd_rad_setup(rrhd_ctx *ctx, const rrhd_dirs *dirs, const rrhd_rad_opts *opts);
/* Levels summed over direction batches and the largest level (items). */
rrhd_status rrhd_rad_plan_info(const rrhd_ctx *ctx, int64_t *levels, int64_t *max_level_items);
/* The plan as the reference's sweep order would number it: levels [M][N] (caller cell
 * numbering) the level of direction d's batch in which cell c is swept for d -- the
 * depth of c in the upwind graph of d, which is the index of the front graph::
 * RunGraphModule puts c in (graph/src/graph_by_direction.cpp).  Synchronises. */
rrhd_status rrhd_rad_plan_levels(const rrhd_ctx *ctx, int32_t *levels);
/* One sweep of all directions and groups on ctx's stream.  Device pointers of the
 * setup's precision (double for RRHD_RAD_FP64, float otherwise), caller cell
 * numbering: alpha, betta [N] absorption and scattering
 * coefficients, Q [N][G] emission B / kRadiation per group, S [N*G][M] scattering
 * integral in, I [N*G][M] intensity out. */
rrhd_status rrhd_sweep(rrhd_ctx *ctx, const void *alpha, const void *betta, const void *Q, const void *S, void *I);

/* ------------------------------------------------------------ coupled step
 * One step of the RadRHD loop (solvers/RadRHD/src/radRHD_main.cpp:96-139):
 * rhllc::Hllc3dStab; opacities alpha = absorption rho, betta = scattering rho and
 * emission Q = B(T) / kRadiation / G from the new primitives; the sweep with the
 * scattering integral of the previous step; the 4-force rad_rhd::GetRadSource
 * from the moments of the previous step's intensity (the reference computes them
 * asynchronously at the start of each radiation iteration, before the sweep,
 * illum_multi_gpu_face_calc.cpp:59-66) added as U.E += tau G0, U.S += tau G,
 * then con2prim without fallback; finally the scattering integral and moments
 * of the new intensity for the next step.  The 4-force and the source con2prim
 * share no data with the sweep and run on a second stream beside it; the call
 * joins that stream before the scattering, so the context's stream orders
 * everything that follows. */
#define RRHD_SCATTER_FP64 (-1)    /* rrhd_scatter_fp64_fma + rrhd_moments_fp64 (RRHD_RAD_FP64) */
#define RRHD_SCATTER_LOWRANK (-2) /* rrhd_scatter_lowrank, either sweep precision */
typedef struct {
  int32_t scatter;        /* RRHD_SCATTER_FP64, RRHD_SCATTER_LOWRANK, or an RRHD_TC_* form (FP32)  */
  const rrhd_mlp *guess;  /* NULL: the reference's initial guess in the source con2prim; else the
                             learned guess (Newton for at most k_stall iterations from it)        */
  int32_t k_stall;        /* 0 = 12                                                             */
  double absorption;      /* alpha = absorption * rho                                           */
  double scattering;      /* betta = scattering * rho                                           */
  rrhd_emission emission;
} rrhd_coupled_opts;
/* tau > 0.  hydro / source (host, may be NULL): statistics of the hydro step and
 * of the source con2prim; either one synchronises the stream. */
rrhd_status rrhd_coupled_step(rrhd_ctx *ctx, double tau, const rrhd_coupled_opts *opts, rrhd_step_stats *hydro,
                              rrhd_c2p_stats *source);
/* Device time (ms) of the phases of the last coupled step: hydro step + opacities;
 * sweep; 4-force + source con2prim (on a second stream, concurrent with the sweep,
 * so it is not added to the step time); scattering + moments.  Synchronises. */
rrhd_status rrhd_coupled_phase_ms(rrhd_ctx *ctx, float *ms4);
/* Host copies (caller cell numbering, double) of the coupled step's radiation
 * arrays: RRHD_RAD_I / RRHD_RAD_S [N*G][M], RRHD_RAD_G4 [N][4] (4-force of the
 * last step), RRHD_RAD_MOM [N*G][10] (energy, stream and impulse moments of the
 * last scattering per row cell * G + g: E, F0..2, T00, T01, T02, T11, T12, T22,
 * as cuda_sep::MakeEnergy/MakeStream/MakeImpuls give them,
 * cuda/src/short_characteristics/separate_gpu/cuda_illum_sep_param.cu:9-69);
 * rrhd_rad_set writes I or S (e.g. the scattering integral of a previous run). */
#define RRHD_RAD_I 0
#define RRHD_RAD_S 1
#define RRHD_RAD_G4 2
#define RRHD_RAD_MOM 3
rrhd_status rrhd_rad_get(rrhd_ctx *ctx, int32_t what, double *out);
/* Pieces of the coupled step on caller arrays, for a step composed over ranks
 * (rad_rhd::RunRadRHDMpiModule, solvers/RadRHD/src/radRHD_mpi_main.cpp:107-122), where each
 * rank runs them on its share of cells or rows.  Device pointers; W, U [n][stride] with the
 * five primitives / conservatives first.
 *   rrhd_rad_opacities       alpha = absorption rho, betta = scattering rho, Q [n][groups]
 *                            = B(T) / rad_unit / groups (the coupled step's rule)
 *   rrhd_rad_source_rows     the 4-force G4 [n][4] of each cell from the FP64 moments of its
 *                            groups' rows (E [n groups], F [n groups][3], T [n groups][9], as
 *                            rrhd_moments_fp64 writes them), summed over the groups
 *   rrhd_rad_source_con2prim U.E += tau G0, U.S += tau G[1..3], then GetPhysValueStab from its
 *                            own guess without fallback (the coupled step's source update);
 *                            stats (may be NULL) synchronise the stream. */
rrhd_status rrhd_rad_opacities(const rrhd_emission *em, const double *W, int64_t stride, int64_t n,
                               double absorption, double scattering, int32_t groups, double *alpha,
                               double *betta, double *Q, void *stream);
rrhd_status rrhd_rad_source_rows(const rrhd_emission *em, const double *W, int64_t stride, int64_t n,
                                 double absorption, double scattering, int32_t groups, const double *E,
                                 const double *F, const double *T, double *G4, void *stream);
rrhd_status rrhd_rad_source_con2prim(int32_t eos, double gamma, double *U, double *W, int64_t stride,
                                     const double *G4, double tau, int64_t n, rrhd_c2p_stats *stats,
                                     void *stream);

/* Accuracy of the reduced-precision scattering of the last coupled step (FP32 or
 * mixed sweep precision; not FP64): on every (N / sample_cells)-th cell, the FP32
 * scattering integral against its FP64 value from the same FP32 intensity (per
 * (cell, group, direction), relative to itself: max and rms) and the moments against
 * theirs (max; F and T relative to E).  Synchronises the context's stream. */
rrhd_status rrhd_coupled_scatter_error(rrhd_ctx *ctx, int64_t sample_cells, double *max_rel, double *rms_rel,
                                       double *moments_max);

rrhd_status rrhd_rad_set(rrhd_ctx *ctx, int32_t what, const double *in);

/* ------------------------------------------------------------ misc */
const char *rrhd_last_error(void);
const char *rrhd_version(void);

#ifdef __cplusplus
}
#endif
#endif /* RRHD_H */
