/* Test infrastructure, not product code: the checker, never the thing measured.
 *
 * Plain-C restatement of the RadRHD_solver hot path.  Each function restates one
 * reference function in the same operation order (citations below are paths
 * inside the reference project).  Eigen's evaluation order, which the reference
 * inherits for its 3-vector arithmetic, is spelled out explicitly: with gcc -O2
 * on x86-64 a Vector3 dot product is (x0 + x1) + x2, a Matrix3 * Vector3 product
 * gives rows 0 and 1 as (x0 + x1) + x2 and row 2 as x0 + (x1 + x2), and
 * Matrix3.transpose() * Vector3 gives every row as (x0 + x1) + x2.
 */
#include "rrhd_oracle.h"

#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#define MAX_ITER 40 /* solvers/rhllc/src/rhllc_flux_stab.cpp:8 */
static const double kMinPressure = 1e-12; /* lib/global_consts.h:16 */

/* std::min / std::max semantics (NaN handling included). */
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double smax(double a, double b) { return (a < b) ? b : a; }

static inline double dot3(const double *a, const double *b) {
  return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}
/* Matrix3 * Vector3 (row-major T) */
static inline void matvec(const double *T, const double *v, double *r) {
  r[0] = (T[0] * v[0] + T[1] * v[1]) + T[2] * v[2];
  r[1] = (T[3] * v[0] + T[4] * v[1]) + T[5] * v[2];
  r[2] = T[6] * v[0] + (T[7] * v[1] + T[8] * v[2]);
}
/* Matrix3.transpose() * Vector3 (row-major T) */
static inline void matTvec(const double *T, const double *v, double *r) {
  r[0] = (T[0] * v[0] + T[3] * v[1]) + T[6] * v[2];
  r[1] = (T[1] * v[0] + T[4] * v[1]) + T[7] * v[2];
  r[2] = (T[2] * v[0] + T[5] * v[1]) + T[8] * v[2];
}

static inline double gamma_g(const orc_eos *e) { return e->gamma1 / (e->gamma1 - 1.0); }

/* rhllc::GetConvValueStab, solvers/rhllc/src/rhllc_flux_stab.cpp:10-38 */
void orc_p2c(const orc_eos *eos, double *W, double *U) {
  double h;
  if (eos->eos == ORC_EOS_IDEAL) {
    h = 1 + gamma_g(eos) * W[4] / W[0];
  } else {
    double theta = W[4] / W[0];
    h = 2.5 * theta + sqrt(2.25 * theta * theta + 1.0);
  }
  double g = dot3(W + 1, W + 1);
  if (g >= 1.0) {
    const double beta_fix = 0.9999;
    g = beta_fix / sqrt(g);
    W[1] *= g;
    W[2] *= g;
    W[3] *= g;
    g = beta_fix * beta_fix;
  }
  g = 1.0 / (1.0 - g);
  double scrh = W[0] * h * g;
  g = sqrt(g);
  U[0] = W[0] * g;
  U[1] = scrh * W[1];
  U[2] = scrh * W[2];
  U[3] = scrh * W[3];
  U[4] = scrh - W[4];
}

/* rhllc::GetConvValue, solvers/rhllc/src/rhllc_flux.cpp:7-16 (fixed inflow states) */
void orc_p2c_plain(const orc_eos *eos, const double *W, double *U) {
  const double d = W[0];
  const double Gamma = 1. / sqrt(1 - dot3(W + 1, W + 1));
  const double h = 1 + gamma_g(eos) * W[4] / d;
  const double dhGG = d * h * Gamma * Gamma;
  U[0] = Gamma * W[0];
  U[1] = dhGG * W[1];
  U[2] = dhGG * W[2];
  U[3] = dhGG * W[3];
  U[4] = dhGG - W[4];
}

static inline double enthalpy_fix(const orc_eos *eos, double D, double plor, double alpha) {
  if (eos->eos == ORC_EOS_IDEAL) return D + plor * alpha;
  return 2.5 * plor + sqrt(2.25 * plor * plor + D * D);
}

/* rhllc::PhysPressureFix, rhllc_flux_stab.cpp:40-121 */
int orc_pressure_fix(const orc_eos *eos, double *U, double *W) {
  double p = kMinPressure;
  double D = U[0];
  double m2 = dot3(U + 1, U + 1);
  double m = sqrt(m2);
  double umax = m / D;
  double u0 = umax;
  double lor = sqrt(1.0 + u0 * u0);
  double plor = p * lor;
  const double alpha = (eos->eos == ORC_EOS_IDEAL) ? eos->gamma1 / (eos->gamma1 - 1.0) : 2.5;
  double Dh = enthalpy_fix(eos, D, plor, alpha);
  double f0 = m / Dh - u0;
  double u1 = (-D + sqrt(D * D + 4.0 * m * alpha * p)) / (2.0 * alpha * p);
  int done = 0;
  double f1, du;
  for (int k = 1; k < MAX_ITER; k++) {
    lor = sqrt(1.0 + u1 * u1);
    plor = p * lor;
    Dh = enthalpy_fix(eos, D, plor, alpha);
    f1 = m / Dh - u1;
    if (done == 1) break;
    du = (u1 - u0) / (f1 - f0) * f1;
    u0 = u1;
    f0 = f1;
    u1 -= du;
    u1 = smin(u1, umax);
    u1 = smax(u1, 0.0);
    if (fabs(f1) < 1.e-9) done = 1;
  }
  if (done != 1) return 2;
  lor = sqrt(1.0 + u1 * u1);
  plor = p * lor;
  Dh = enthalpy_fix(eos, D, plor, alpha);
  W[0] = U[0] / lor;
  W[4] = p;
  U[4] = Dh * lor - p;
  f0 = 1.0 / (Dh * lor);
  W[1] = U[1] * f0;
  W[2] = U[2] * f0;
  W[3] = U[3] * f0;
  return 0;
}

/* rhllc::GetPhysValueStab, rhllc_flux_stab.cpp:123-220.  Returns 5 where the
 * reference would abort the process (DIE_IF(lor2 < 1.0), :149). */
int orc_c2p(const orc_eos *eos, const double *U, double *W) {
  const double tol = 1.e-11;
  const double eps2 = 1.e-12;
  const double kg = gamma_g(eos);
  double D = U[0];
  double E = U[4];
  double m2 = dot3(U + 1, U + 1);
  double Q = E - sqrt(m2 + D * D);
  if (Q < 0.0) return 1;
  double m = sqrt(m2);
  double p = smax(m - E, 0.0);
  double D_1 = 1.0 / D;
  double pmin = sqrt(m2 / (1.0 - eps2)) - E;
  double alpha, alpha2, lor2, lor, tau, theta;
  double h, dh_dp, dh_dtau, yp = 0, dp, dyp, scrh;
  p = smax(p, pmin);
  int iter;
  for (iter = 0; iter < MAX_ITER; iter++) {
    alpha = E + p;
    alpha2 = alpha * alpha;
    lor2 = 1.0 - m2 / alpha2;
    lor2 = 1.0 / lor2;
    if (lor2 < 1.0) return 5;
    lor = sqrt(lor2);
    tau = lor * D_1;
    theta = p * tau;
    if (eos->eos == ORC_EOS_IDEAL) {
      h = 1.0 + kg * theta;
      dh_dp = kg * tau;
      dh_dtau = kg * p;
    } else {
      h = 2.5 * theta + sqrt(2.25 * theta * theta + 1.0);
      scrh = (5.0 * h - 8.0 * theta) / (2.0 * h - 5.0 * theta);
      dh_dp = tau * scrh;
      dh_dtau = p * scrh;
    }
    yp = D * h * lor - E - p;
    dyp = D * lor * dh_dp - m2 * lor2 * lor / (alpha2 * alpha) * (lor * dh_dtau + D * h) - 1.0;
    dp = yp / dyp;
    p -= dp;
    if (p < pmin) p = pmin;
    if (fabs(dp) < tol * E) break;
  }
  if (p < 0.0) return 2;
  if (isnan(p)) return 4;
  if (iter >= MAX_ITER || fabs(yp / (E + p)) > 1.e-4 || p < (m - E)) return 3;
  alpha = E + p;
  alpha2 = alpha * alpha;
  lor2 = alpha2 / (alpha2 - m2);
  lor = sqrt(lor2);
  tau = lor * D_1;
  W[0] = 1.0 / tau;
  W[4] = p;
  const double den = U[4] + p;
  W[1] = U[1] / den;
  W[2] = U[2] / den;
  W[3] = U[3] / den;
  return 0;
}

/* GetRotationMatrix, lib/geometry/src/linear_alg.cpp:3-42 (row-major T) */
void orc_rotation(const double *n, double *T) {
  for (int i = 0; i < 9; i++) T[i] = 0.0;
  const double eps = 1e-12;
  if (fabs(n[2] * n[2] - 1) > eps) {
    T[0] = n[0];
    T[1] = n[1];
    T[2] = n[2];
    double sqr = sqrt(1 - n[2] * n[2]);
    double sqr_inv = 1. / sqr;
    T[3] = -n[1] * sqr_inv;
    T[4] = n[0] * sqr_inv;
    T[6] = -n[0] * n[2] * sqr_inv;
    T[7] = -n[1] * n[2] * sqr_inv;
    T[8] = sqr;
  } else if (n[2] > 0) {
    T[2] = 1;
    T[4] = 1;
    T[6] = -1;
  } else {
    T[2] = -1;
    T[4] = -1;
    T[6] = 1;
  }
}

/* GetSignalSpeed, rhllc_flux_stab.cpp:231-238 */
static void signal_speed(double cs2, double Vn, double V2_norm, double *cmin, double *cmax) {
  const double Vn2 = Vn * Vn;
  const double Vt2 = V2_norm - Vn2;
  const double sroot_L = sqrt(cs2 * (1 - Vn2 - Vt2 * cs2) * (1 - V2_norm));
  *cmax = (Vn * (1.0 - cs2) + sroot_L) / (1.0 - V2_norm * cs2);
  *cmin = (Vn * (1.0 - cs2) - sroot_L) / (1.0 - V2_norm * cs2);
}

static void sound_speed(const orc_eos *eos, double d, double p, double *cs2) {
  if (eos->eos == ORC_EOS_IDEAL) {
    const double h = 1 + gamma_g(eos) * p / d;
    *cs2 = ((eos->gamma1 * p) / (d * h));
  } else {
    double theta = p / d;
    const double h = 2.5 * theta + sqrt(2.25 * theta * theta + 1.0);
    *cs2 = theta / (3.0 * h) * (5.0 * h - 8.0 * theta) / (h - theta);
  }
}

/* rhllc::GetFluxStab, rhllc_flux_stab.cpp:240-431.  F gets the flux times area. */
double orc_flux(const orc_eos *eos, const double *UL0, const double *UR0, const double *WL0,
                const double *WR0, const double *n, double area, double *Fout) {
  double T[9];
  orc_rotation(n, T);
  double UL[5], UR[5], WL[5], WR[5];
  UL[0] = UL0[0];
  UL[4] = UL0[4];
  matvec(T, UL0 + 1, UL + 1);
  UR[0] = UR0[0];
  UR[4] = UR0[4];
  matvec(T, UR0 + 1, UR + 1);
  WL[0] = WL0[0];
  WL[4] = WL0[4];
  matvec(T, WL0 + 1, WL + 1);
  WR[0] = WR0[0];
  WR[4] = WR0[4];
  matvec(T, WR0 + 1, WR + 1);

  const double *Vel_L = WL + 1, *Vel_R = WR + 1;
  const double d_L = WL[0], d_R = WR[0];
  const double p_L = WL[4], p_R = WR[4];
  const double VV_L = dot3(Vel_L, Vel_L);
  const double VV_R = dot3(Vel_R, Vel_R);
  double cs_L2, cs_R2;
  sound_speed(eos, d_L, p_L, &cs_L2);
  sound_speed(eos, d_R, p_R, &cs_R2);

  double cmax_L, cmax_R, cmin_L, cmin_R;
  signal_speed(cs_L2, Vel_L[0], VV_L, &cmin_L, &cmax_L);
  signal_speed(cs_R2, Vel_R[0], VV_R, &cmin_R, &cmax_R);
  const double lambda_L = smin(cmin_L, cmin_R);
  const double lambda_R = smax(cmax_L, cmax_R);

  double F[5];
  if (lambda_L >= 0.0) {
    F[0] = UL[0] * Vel_L[0];
    F[1] = UL[1] * Vel_L[0];
    F[2] = UL[2] * Vel_L[0];
    F[3] = UL[3] * Vel_L[0];
    F[4] = UL[1];
    F[1] += p_L;
  } else if (lambda_R <= 0.0) {
    F[0] = UR[0] * Vel_R[0];
    F[1] = UR[1] * Vel_R[0];
    F[2] = UR[2] * Vel_R[0];
    F[3] = UR[3] * Vel_R[0];
    F[4] = UR[1];
    F[1] += p_R;
  } else {
    double F_L[5] = {UL[0] * Vel_L[0], UL[1] * Vel_L[0], UL[2] * Vel_L[0], UL[3] * Vel_L[0], UL[1]};
    double F_R[5] = {UR[0] * Vel_R[0], UR[1] * Vel_R[0], UR[2] * Vel_R[0], UR[3] * Vel_R[0], UR[1]};
    double AL = lambda_L * UL[4] - F_L[4];
    double AR = lambda_R * UR[4] - F_R[4];
    double BL = lambda_L * UL[1] - F_L[1] - p_L;
    double BR = lambda_R * UR[1] - F_R[1] - p_R;
    double a = AR * lambda_L - AL * lambda_R;
    double b = AL + BL * lambda_R - AR - BR * lambda_L;
    double c = BR - BL;
    double scrh = -0.5 * (b + (b < 0.0 ? -1.0 : 1.0) * sqrt(b * b - 4.0 * a * c));
    double us = c / scrh;
    double ps = (AL * us - BL) / (1.0 - us * lambda_L);
    if (us >= 0.0) {
      double usl[5];
      double dif = 1.0 / (lambda_L - us);
      usl[0] = UL[0] * (lambda_L - Vel_L[0]) * dif;
      usl[1] = (lambda_L * (UL[4] + ps) - UL[1]) * us * dif;
      usl[2] = UL[2] * (lambda_L - Vel_L[0]) * dif;
      usl[3] = UL[3] * (lambda_L - Vel_L[0]) * dif;
      usl[4] = UL[4] + (usl[1] - UL[1]) / lambda_L;
      for (int i = 0; i < 5; i++) usl[i] -= UL[i];
      for (int i = 0; i < 5; i++) usl[i] *= lambda_L;
      for (int i = 0; i < 5; i++) F[i] = F_L[i] + usl[i];
      F[1] += p_L;
    } else {
      double usr[5];
      double dif = 1.0 / (lambda_R - us);
      usr[0] = UR[0] * (lambda_R - Vel_R[0]) * dif;
      usr[1] = (lambda_R * (UR[4] + ps) - UR[1]) * us * dif;
      usr[2] = UR[2] * (lambda_R - Vel_R[0]) * dif;
      usr[3] = UR[3] * (lambda_R - Vel_R[0]) * dif;
      usr[4] = UR[4] + (usr[1] - UR[1]) / lambda_R;
      for (int i = 0; i < 5; i++) usr[i] -= UR[i];
      for (int i = 0; i < 5; i++) usr[i] *= lambda_R;
      for (int i = 0; i < 5; i++) F[i] = F_R[i] + usr[i];
      F[1] += p_R;
    }
  }
  Fout[0] = F[0];
  Fout[4] = F[4];
  matTvec(T, F + 1, Fout + 1);
  for (int i = 0; i < 5; i++) Fout[i] *= area;
  return smax(lambda_L, lambda_R);
}

/* rhllc::BoundConditions, solvers/rhllc/src/rhllc_utils.cpp:45-133, with the
 * boundary states taken from a runtime table instead of compile-time geometry. */
static void boundary_state(const orc_mesh *m, const orc_bc *bc, int64_t f, const double *U,
                           const double *W, double *Ub, double *Wb) {
  const int32_t id_l = m->face_id_l[f];
  const int32_t id_r = m->face_id_r[f];
  if (id_r >= 0) {
    memcpy(Ub, U + 5 * (int64_t)id_r, 5 * sizeof(double));
    memcpy(Wb, W + 5 * (int64_t)id_r, 5 * sizeof(double));
    return;
  }
  const int k = -id_r - 1;
  const int kind = (k < 8 && bc) ? bc->kind[k] : 0;
  if (kind == 1) {
    memcpy(Ub, bc->U[k], 5 * sizeof(double));
    memcpy(Wb, bc->W[k], 5 * sizeof(double));
    return;
  }
  memcpy(Ub, U + 5 * (int64_t)id_l, 5 * sizeof(double));
  memcpy(Wb, W + 5 * (int64_t)id_l, 5 * sizeof(double));
  if (kind == 2) {
    /* reflecting wall: rotate into the face frame, negate the normal
     * component, rotate back with the transposed matrix (rhllc_utils.cpp:96-114) */
    double T[9], Tt[9], r[3];
    orc_rotation(m->face_n + 3 * f, T);
    matvec(T, Ub + 1, r);
    memcpy(Ub + 1, r, sizeof r);
    matvec(T, Wb + 1, r);
    memcpy(Wb + 1, r, sizeof r);
    Ub[1] = -Ub[1];
    Wb[1] = -Wb[1];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) Tt[3 * i + j] = T[3 * j + i];
    matvec(Tt, Ub + 1, r);
    memcpy(Ub + 1, r, sizeof r);
    matvec(Tt, Wb + 1, r);
    memcpy(Wb + 1, r, sizeof r);
  }
}

/* rhllc::Hllc3dStab, solvers/rhllc/src/rhllc_3d_stab.cpp:10-63 */
double orc_hydro_step(const orc_eos *eos, const orc_mesh *m, const orc_bc *bc, double tau,
                      double *U, double *W, double *face_flux, int32_t *status, int nthreads) {
  double max_speed_all = 0;
  const int64_t F = m->n_faces, N = m->n_cells;
  (void)nthreads;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
  {
    double max_speed = 0;
#pragma omp for schedule(static)
    for (int64_t f = 0; f < F; f++) {
      double Ub[5], Wb[5];
      boundary_state(m, bc, f, U, W, Ub, Wb);
      const int64_t l = m->face_id_l[f];
      const double s = orc_flux(eos, U + 5 * l, Ub, W + 5 * l, Wb, m->face_n + 3 * f,
                                m->face_area[f], face_flux + 5 * f);
      max_speed = smax(max_speed, s);
    }
#pragma omp for schedule(static)
    for (int64_t c = 0; c < N; c++) {
      double sumF[5] = {0, 0, 0, 0, 0};
      for (int j = 0; j < 4; j++) {
        const double *fl = face_flux + 5 * (int64_t)m->cell_faces[4 * c + j];
        if ((m->cell_sign[c] >> j) & 1)
          for (int i = 0; i < 5; i++) sumF[i] += fl[i];
        else
          for (int i = 0; i < 5; i++) sumF[i] -= fl[i];
      }
      const double s = (tau / m->cell_volume[c]);
      for (int i = 0; i < 5; i++) sumF[i] *= s;
      for (int i = 0; i < 5; i++) U[5 * c + i] -= sumF[i];
      int code = orc_c2p(eos, U + 5 * c, W + 5 * c);
      if (code) {
        const int fix = orc_pressure_fix(eos, U + 5 * c, W + 5 * c);
        code = code | 0x10 | (fix ? 0x20 : 0);
      }
      if (status) status[c] = code;
    }
#pragma omp critical
    { max_speed_all = smax(max_speed_all, max_speed); }
  }
  return max_speed_all;
}

/* rhllc::GetTimeStep, solvers/rhllc/src/rhllc_utils.cpp:15-23 */
double orc_time_step(double cfl, double h_min, double max_speed) {
  return cfl * h_min / max_speed;
}

/* Thomson phase function Gamma, cuda/src/short_characteristics/cuda_integrator.cu:10-13
 * (same arithmetic as solvers/illum/include/scattering.h:32-35). */
static inline double thomson(const double *a, const double *b) {
  const double sum = dot3(a, b);
  return (3. * (1. + sum * sum)) / 4.;
}

/* Scattering integral, cell-major: cuda::kernel::GetS_MPI_multi_device,
 * cuda/src/short_characteristics/cuda_scattering.cu:82-105 (the CPU
 * GetIntScatteringByDirection, solvers/illum/src/scattering.cpp:6-18, has the
 * same sum in the same direction order). */
void orc_scatter(int64_t N, int32_t M, const double *I, const double *dirs, const double *areas,
                 double full_area, double *S, int nthreads) {
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
  for (int64_t c = 0; c < N; c++) {
    const double *Ic = I + (size_t)c * M;
    for (int32_t k = 0; k < M; k++) {
      double scatter = 0;
      for (int32_t d = 0; d < M; d++)
        scatter += thomson(dirs + 3 * d, dirs + 3 * k) * Ic[d] * areas[d];
      S[(size_t)c * M + k] = scatter / full_area;
    }
  }
}

/* Moments, cuda_sep::device::MakeEnergy / MakeStream / MakeImpuls,
 * cuda/src/short_characteristics/separate_gpu/cuda_illum_sep_param.cu:9-69. */
void orc_moments(int64_t N, int32_t M, const double *I, const double *dirs, const double *areas,
                 double full_area, double *E, double *F, double *T, int nthreads) {
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
  for (int64_t c = 0; c < N; c++) {
    const double *Ic = I + (size_t)c * M;
    double e = 0, s[3] = {0, 0, 0}, t[9] = {0};
    for (int32_t k = 0; k < M; k++) e += Ic[k] * areas[k];
    for (int32_t k = 0; k < M; k++) {
      const double Ia = Ic[k] * areas[k];
      for (int i = 0; i < 3; i++) s[i] += dirs[3 * k + i] * Ia;
    }
    for (int32_t d = 0; d < M; d++) {
      const double Ia = Ic[d] * areas[d];
      for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) t[3 * i + k] += dirs[3 * d + i] * dirs[3 * d + k] * Ia;
    }
    E[c] = e / full_area;
    for (int i = 0; i < 3; i++) F[3 * c + i] = s[i] / full_area;
    for (int i = 0; i < 9; i++) T[9 * c + i] = t[i] / full_area;
  }
}

/* rad_rhd::GetRadSource, solvers/RadRHD/src/radRHD_utils.cpp:44-101
 * (ISOTROPIC_INTENSITY 0: the impulse moment is used directly), with the
 * emission B_Plank(GetTemperature(rho, p)) / kRadiation of
 * lib/physics/src/plunk.cpp:87-90 and lib/physics/include/gas_state.h:22-27. */
void orc_rad_source(int64_t N, const orc_emission *em, const double *W, const double *alpha,
                    const double *sigma, const double *E, const double *F, const double *T,
                    double *G) {
  for (int64_t c = 0; c < N; c++) {
    const double abs_op = alpha[c];
    const double scat_op = sigma[c];
    const double tot_op = abs_op + scat_op;
    const double rho = W[5 * c + 0];
    const double prs = W[5 * c + 4];
    const double *v = W + 5 * c + 1;
    const double Ur = E[c];
    const double *Fr = F + 3 * c;
    const double *Tr = T + 9 * c; /* Tr(j,i) = Tr[3*j+i] */

    double gamma = dot3(v, v);
    double u2 = gamma;
    double gamma2 = 1.0 / (1.0 - gamma);
    u2 *= gamma2;
    gamma = sqrt(gamma2);
    double u[3] = {gamma * v[0], gamma * v[1], gamma * v[2]};

    double uuD = 0.;
    double uF = dot3(u, Fr);
    double uD[3];
    double D;
    for (int i = 0; i < 3; i++) {
      uD[i] = 0.;
      for (int j = 0; j < 3; j++) {
        D = Tr[3 * j + i];
        uD[i] += u[j] * D;
        uuD += u[i] * u[j] * D;
      }
    }
    double rhogamma = rho * gamma;
    const double Tgas = em->temp_coef * prs / rho;
    const double T2 = Tgas * Tgas;
    const double B = (T2 * T2) * em->sigma_sb / em->pi;
    double q = -abs_op * rho * B / em->rad_unit;

    G[4 * c + 0] = q * gamma + rhogamma * (abs_op - scat_op * (u2 + uuD)) * Ur -
                   rho * (abs_op - scat_op * (u2 + gamma2)) * uF;
    for (int i = 0; i < 3; i++)
      G[4 * c + i + 1] = q * u[i] - rho * (tot_op * uD[i] + scat_op * u[i] * (gamma2 + uuD)) * Ur +
                         rhogamma * (tot_op * Fr[i] + scat_op * 2.0 * uF * u[i]);
  }
}

/* ------------------------------------------------------------------ sweep */

/* illum::GetIllum, solvers/illum/src/illum_utils.cpp:454-490 (TRANSFER_CELL_TO_FACE) */
double orc_get_illum(const double *I0, const double *s, double k, double rhs) {
  double Icur = exp(-k * s[0]) * (I0[0] - rhs) + rhs;
  Icur += (exp(-k * s[1]) * (I0[1] - rhs) + rhs);
  Icur += (exp(-k * s[2]) * (I0[2] - rhs) + rhs);
  return (Icur * 0.3333333333333333);
}

/* illum::GetRhsOpt, illum_utils.cpp:631-646 (Q = B_Plank(T) / kRadiation given) */
double orc_get_rhs(double alpha, double betta, double Q, double S, double *k) {
  *k = alpha + betta;
  return (alpha * Q + betta * S) / *k;
}

/* illum::separate_gpu::ReCalcIllumOpt, illum_utils.cpp:377-433: area-weighted face
 * mean for every cell but the last, plain mean for the last one. */
double orc_recalc_illum(int64_t N, const int32_t *cell_faces, const double *face_area,
                        const double *fv, int32_t M, int32_t dir, double *Illum) {
  double norm = -1;
  for (int64_t c = 0; c < N - 1; c++) {
    const size_t id = (size_t)c * M + dir;
    double curI = 0, S = 0;
    for (int j = 0; j < 4; j++) {
      const int32_t f = cell_faces[4 * c + j];
      curI += fv[f] * face_area[f];
      S += face_area[f];
    }
    curI /= S;
    norm = smax(norm, fabs((Illum[id] - curI) / curI));
    Illum[id] = curI;
  }
  {
    const int64_t c = N - 1;
    const size_t id = (size_t)c * M + dir;
    double curI = 0;
    for (int j = 0; j < 4; j++) curI += fv[cell_faces[4 * c + j]];
    curI /= 4;
    norm = smax(norm, fabs((Illum[id] - curI) / curI));
    Illum[id] = curI;
  }
  return norm;
}

/* Short characteristics of the out-face j of a cell for direction w.  The three
 * interpolation nodes of the face (barycentric weight 2/3 at one face vertex and
 * 1/6 at the other two: the nodes of BaseTetra_t, lib/geometry/include/geo_types.h:163-212)
 * are traced back along -w to the in-face the ray leaves the cell through: the
 * in-face h (cos_h = n_h.w < 0) with the smallest ray parameter
 *     t_h = lam_h * (H_h / -cos_h),
 * lam_h the node's barycentric weight of vertex h (the vertex opposite face h) and
 * H_h = 3 V / A_h that vertex's height over face h, since the signed distance of a
 * point to the plane of face h is -lam_h H_h.  First in face order on ties.
 * Output: in-face index h[3] and distance s[3]. */
static void trace_face(const double *H, const double *cosf, int j, int *h, double *s) {
  double r[4];
  for (int f = 0; f < 4; f++) r[f] = cosf[f] < 0 ? H[f] / -cosf[f] : 0.0;
  for (int q = 0; q < 3; q++) {
    const int vq = (j + 1 + q) & 3;
    double tmin = 0;
    int hmin = -1;
    for (int f = 0; f < 4; f++) {
      if (!(cosf[f] < 0)) continue;
      const double lam = f == vq ? 2.0 / 3.0 : 1.0 / 6.0;
      const double t = lam * r[f];
      if (hmin < 0 || t < tmin) {
        tmin = t;
        hmin = f;
      }
    }
    h[q] = hmin;
    s[q] = tmin;
  }
}

/* Outward normal of local face j of cell c: the mesh face normal signed by the
 * cell's orientation bit, so two neighbours classify a shared face consistently. */
static void cell_normal(const orc_sweep_mesh *m, int64_t c, int j, double *n) {
  const double *fn = m->face_n + 3 * (int64_t)m->cell_faces[4 * c + j];
  if ((m->cell_sign[c] >> j) & 1) {
    n[0] = fn[0];
    n[1] = fn[1];
    n[2] = fn[2];
  } else {
    n[0] = -fn[0];
    n[1] = -fn[1];
    n[2] = -fn[2];
  }
}

/* The short-characteristic geometry orc_sweep uses, for every (direction d, cell c,
 * local face j, node q): the in-face h and the distance s of trace_face where face j is
 * an out-face (cos_j > 0), -1 and 0 elsewhere; in_face and s are [M][N][4][3]. */
void orc_trace_nodes(const orc_sweep_mesh *m, int32_t M, const double *dirs, int32_t *in_face, double *s) {
  const int64_t N = m->n_cells;
  for (int32_t dd = 0; dd < M; dd++) {
    const double *w = dirs + 3 * dd;
    for (int64_t c = 0; c < N; c++) {
      double n[4][3], H[4], cosf[4];
      for (int j = 0; j < 4; j++) {
        cell_normal(m, c, j, n[j]);
        H[j] = 3.0 * m->cell_volume[c] / m->face_area[m->cell_faces[4 * c + j]];
        cosf[j] = dot3(n[j], w);
      }
      for (int j = 0; j < 4; j++) {
        int32_t *hf = in_face + (((int64_t)dd * N + c) * 4 + j) * 3;
        double *sd = s + (((int64_t)dd * N + c) * 4 + j) * 3;
        int h[3] = {-1, -1, -1};
        double sdist[3] = {0, 0, 0};
        if (cosf[j] > 0) trace_face(H, cosf, j, h, sdist);
        for (int q = 0; q < 3; q++) {
          hf[q] = h[q];
          sd[q] = sdist[q];
        }
      }
    }
  }
}

int64_t orc_sweep(const orc_sweep_mesh *m, int32_t M, const double *dirs, int32_t G, const double *alpha,
                  const double *betta, const double *Q, const double *S, double bc, double *I) {
  const int64_t N = m->n_cells, F = m->n_faces;
  double *geo = (double *)malloc(sizeof(double) * 16 * N); /* n_j[3], then H_j */
  for (int64_t c = 0; c < N; c++) {
    for (int j = 0; j < 4; j++) {
      cell_normal(m, c, j, geo + 16 * c + 3 * j);
      geo[16 * c + 12 + j] = 3.0 * m->cell_volume[c] / m->face_area[m->cell_faces[4 * c + j]];
    }
  }
  double *fv = (double *)malloc(sizeof(double) * F * G);
  double *col = (double *)malloc(sizeof(double) * N * M);
  double *fvg = (double *)malloc(sizeof(double) * F);
  int32_t *indeg = (int32_t *)malloc(sizeof(int32_t) * N);
  int64_t *queue = (int64_t *)malloc(sizeof(int64_t) * N);
  int64_t missing = 0;
  for (int32_t dd = 0; dd < M; dd++) {
    const double *w = dirs + 3 * dd;
    /* faces nobody writes in this direction (boundary in-faces, faces parallel to w)
     * hold the boundary value */
    for (int64_t i = 0; i < F * G; i++) fv[i] = bc;
    int64_t qh = 0, qt = 0;
    for (int64_t c = 0; c < N; c++) {
      int cnt = 0;
      for (int j = 0; j < 4; j++)
        if (dot3(geo + 16 * c + 3 * j, w) < 0 && m->cell_nbr[4 * c + j] >= 0) cnt++;
      indeg[c] = cnt;
      if (cnt == 0) queue[qt++] = c;
    }
    while (qh < qt) {
      const int64_t c = queue[qh++];
      double cosf[4];
      for (int j = 0; j < 4; j++) cosf[j] = dot3(geo + 16 * c + 3 * j, w);
      for (int j = 0; j < 4; j++) {
        if (!(cosf[j] > 0)) continue;
        int h[3];
        double sdist[3];
        trace_face(geo + 16 * c + 12, cosf, j, h, sdist);
        for (int g = 0; g < G; g++) {
          double I0[3], k, rhs;
          for (int q = 0; q < 3; q++) {
            const int hf = h[q];
            I0[q] = (hf >= 0 && m->cell_nbr[4 * c + hf] >= 0) ? fv[(int64_t)m->cell_faces[4 * c + hf] * G + g] : bc;
          }
          rhs = orc_get_rhs(alpha[c], betta[c], Q[c * G + g], S[((size_t)c * G + g) * M + dd], &k);
          fv[(int64_t)m->cell_faces[4 * c + j] * G + g] = orc_get_illum(I0, sdist, k, rhs);
        }
        const int32_t nb = m->cell_nbr[4 * c + j];
        if (nb >= 0 && --indeg[nb] == 0) queue[qt++] = nb;
      }
    }
    missing += N - qt;
    for (int g = 0; g < G; g++) {
      for (int64_t f = 0; f < F; f++) fvg[f] = fv[f * G + g];
      for (int64_t c = 0; c < N; c++) col[(size_t)c * M + dd] = I[((size_t)c * G + g) * M + dd];
      orc_recalc_illum(N, m->cell_faces, m->face_area, fvg, M, dd, col);
      for (int64_t c = 0; c < N; c++) I[((size_t)c * G + g) * M + dd] = col[(size_t)c * M + dd];
    }
  }
  free(geo);
  free(fv);
  free(col);
  free(fvg);
  free(indeg);
  free(queue);
  return missing;
}

/* ------------------------------------------------------------------ Compton
 * Frequency-coupled Compton scattering over the full spectrum, restating
 * cuda/src/short_characteristics/separate_gpu/spectrum/cuda_scat_full_spectrum.cu in the
 * same operation order (the reference has it as device code only; its CGS constants are
 * lib/global_consts.h:34-44, written here as the same products). */
#define CMP_C_LIGHT (3 * 1e10)                                   /* kC_Light */
#define CMP_C_LIGHT_INV (1.0 / (CMP_C_LIGHT))                    /* kC_LightInv */
#define CMP_VELOCITY CMP_C_LIGHT                                 /* kVelocity, global_consts.h:74 */
#define CMP_HMC ((6.62 * 1e-27) / (((9.109383701528 * 1e-28) * CMP_C_LIGHT) * CMP_C_LIGHT))
#define CMP_COEF (((2 * 3.1415926535897932384626433832795) * (2.8179403 * 1e-13)) * (2.8179403 * 1e-13))
static const double cmp_frq0 = 1e24; /* cuda_scat_full_spectrum.cu:48 */
static const double cmp_betta = 350; /* :49 */

/* :54-59 */
double orc_compton_frq(int32_t idx) {
  if (idx <= 0) return 0;
  const double x = ORC_N_FRQ - idx;
  return cmp_frq0 * exp((-x * x) / cmp_betta);
}

/* :50-53; (int)floor(...) converts like the device's cvt.rzi (NaN -> 0, saturating) */
int32_t orc_compton_frq_idx(double frq) {
  const double t = floor(sqrt(-cmp_betta * log(frq / cmp_frq0)) + 1);
  int m;
  if (t != t) m = 0;
  else if (t >= 2147483647.0) m = 2147483647;
  else if (t <= -2147483648.0) m = -2147483647 - 1;
  else m = (int)t;
  m = m < ORC_N_FRQ ? m : ORC_N_FRQ;
  m = m > 0 ? m : 0;
  return ORC_N_FRQ - m;
}

/* get_compton_frq, :8-14 and :16-20 */
static inline double cmp_frq_doppler(double frq, double v, double cosf, double cosf1, double cosTh, double lorenz) {
  const double eps = CMP_HMC * frq;
  return frq * (1. - v * cosf) / (1. + eps / lorenz * (1 - cosTh) - v * cosf1);
}
static inline double cmp_frq_recoil(double frq, double cosTh) {
  const double eps = CMP_HMC * frq;
  return frq / (1. + eps * (1.0 - cosTh));
}

/* GammaC, :22-44 */
static inline double cmp_gamma(double cosf, double v, const double *vel, double frq, double lorenz,
                               const double *main_dir, const double *scat_dir, double *frq1) {
  const double cosTh = dot3(main_dir, scat_dir);
  if (v > (1. / CMP_VELOCITY)) {
    const double cosf1 = dot3(vel, scat_dir) / v;
    *frq1 = cmp_frq_doppler(frq, v, cosf, cosf1, cosTh, lorenz);
  } else {
    if (cosTh > 0.99999999) {
      *frq1 = frq;
      return 2.0 * CMP_COEF;
    }
    *frq1 = cmp_frq_recoil(frq, cosTh);
  }
  const double frq_frac = *frq1 / frq;
  const double frq1_inv = 1. / frq_frac;
  const double ds = CMP_COEF * frq_frac * frq_frac * (frq_frac + frq1_inv + cosTh * cosTh - 1.0);
  return frq1_inv * ds;
}

/* Get_full_spectrum_multi_device, :61-118, for every (cell, direction, frequency).  The
 * reference reads the intensity before the two cut-offs replace it by zero; reading it
 * only when it is kept gives the same sum and stays inside the array. */
void orc_compton_full_spectrum(int32_t M, const double *dirs, const double *areas, double full_area,
                               int64_t cells, const double *I, const double *vel, int32_t dir_disp,
                               int32_t dir_count, int32_t out_stride, double *S, int nthreads) {
  const double low = 0.5 * (orc_compton_frq(0 + 1) + orc_compton_frq(0));
  const double high = orc_compton_frq(ORC_N_FRQ - 1);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
  for (int64_t i = 0; i < cells; i++) {
    const double *v3 = vel + 3 * i;
    for (int32_t k = 0; k < dir_count; k++) {
      const double *cur_dir = dirs + 3 * (int64_t)(dir_disp + k);
      for (int f = 0; f < ORC_N_FRQ; f++) {
        const double frq = 0.5 * (orc_compton_frq(f + 1) + orc_compton_frq(f));
        const double v2 = dot3(v3, v3);
        double lorenz = 1.0, v = 0.0, cosf = 0.0;
        if (v2 > CMP_C_LIGHT_INV) {
          lorenz = 1. / sqrt(1. - (v2));
          v = sqrt(v2);
          cosf = dot3(v3, cur_dir) / v;
        }
        double scatter = 0;
        for (int32_t d = 0; d < M; d++) {
          double frq1;
          const double G = cmp_gamma(cosf, v, v3, frq, lorenz, cur_dir, dirs + 3 * (int64_t)d, &frq1);
          double Iv = 0;
          if (!(frq1 < low) && !(frq1 > high))
            Iv = I[((int64_t)i * M + d) * ORC_N_FRQ + orc_compton_frq_idx(frq1)];
          scatter += G * Iv * areas[d];
        }
        const double cfl = 1.0;
        S[((int64_t)i * out_stride + k) * ORC_N_FRQ + f] = cfl * scatter / full_area;
      }
    }
  }
}

/* GammaC of cuda_scat_spectrum.cu:22-39: the same weight as the full-spectrum kernel's
 * without its forward-scattering special case. */
static inline double cmp_gamma_one(double cosf, double v, const double *vel, double frq, double lorenz,
                                   const double *main_dir, const double *scat_dir) {
  const double cosTh = dot3(main_dir, scat_dir);
  double frq1;
  if (v > (1. / CMP_VELOCITY)) {
    const double cosf1 = dot3(vel, scat_dir) / v;
    frq1 = cmp_frq_doppler(frq, v, cosf, cosf1, cosTh, lorenz);
  } else {
    frq1 = cmp_frq_recoil(frq, cosTh);
  }
  const double frq_frac = frq1 / frq;
  const double frq1_inv = 1. / frq_frac;
  const double ds = CMP_COEF * frq_frac * frq_frac * (frq_frac + frq1_inv + cosTh * cosTh - 1.0);
  return frq1_inv * ds;
}

/* Get_spectrum_multi_device, cuda_scat_spectrum.cu:41-83, for every (cell, direction). */
void orc_compton_spectrum(int32_t M, const double *dirs, const double *areas, double full_area, int64_t cells,
                          const double *I, const double *vel, double frq, int32_t dir_disp, int32_t dir_count,
                          int32_t out_stride, double *S, int nthreads) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
  for (int64_t i = 0; i < cells; i++) {
    const double *v3 = vel + 3 * i;
    for (int32_t k = 0; k < dir_count; k++) {
      const double *cur_dir = dirs + 3 * (int64_t)(dir_disp + k);
      const double v2 = dot3(v3, v3);
      double lorenz = 1.0, v = 0.0, cosf = 0.0;
      if (v2 > CMP_C_LIGHT_INV) {
        lorenz = 1. / sqrt(1. - (v2));
        v = sqrt(v2);
        cosf = dot3(v3, cur_dir) / v;
      }
      double scatter = 0;
      for (int32_t d = 0; d < M; d++) {
        const double Iv = I[(int64_t)i * M + d];
        scatter += cmp_gamma_one(cosf, v, v3, frq, lorenz, cur_dir, dirs + 3 * (int64_t)d) * Iv * areas[d];
      }
      const double cfl = 0.25;
      S[(int64_t)i * out_stride + k] = cfl * scatter / full_area;
    }
  }
}

/* ------------------------------------------------------------------ ray tracing
 * Restates cuda/src/ray_tracing/cuda_ray_calc.cu and cuda_ray_geo_intersect.cu, and the
 * image-plane construction of solvers/ray_tracing/src/ray_tracing_build_plane.cpp,
 * in the reference's operation order (Eigen's cross product component by component
 * as (a1 b2 - a2 b1, a2 b0 - a0 b2, a0 b1 - a1 b0)). */
static inline void cross3(const double *a, const double *b, double *r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}

/* RayIntersectsTriangle, cuda_ray_calc.cu:10-44 */
double orc_ray_triangle(const double *ray, const double *abc) {
  const double eps = 1e-10;
  const double *o = ray, *dir = ray + 3, *A = abc, *B = abc + 3, *C = abc + 6;
  double e1[3], e2[3], h[3], s[3], q[3];
  for (int k = 0; k < 3; k++) {
    e1[k] = B[k] - A[k];
    e2[k] = C[k] - A[k];
  }
  cross3(dir, e2, h);
  const double det = dot3(e1, h);
  if (det > -eps && det < eps) return -1;
  const double inv_det = 1.0 / det;
  for (int k = 0; k < 3; k++) s[k] = o[k] - A[k];
  const double u = inv_det * dot3(s, h);
  if (u < 0.0 || u > 1.0) return -1;
  cross3(s, e1, q);
  const double v = inv_det * dot3(dir, q);
  if (v < 0.0 || u + v > 1.0) return -1;
  const double dist = inv_det * dot3(e2, q);
  if (dist > 0.0) return dist;
  return -1;
}

/* Rosh, cuda_ray_geo_intersect.cu:22-42 */
static double ray_rosh(const double *ray, double t) {
  const double max_potential = -1.82547, m = 0.8795180722891566;
  const double *S = ray, *a = ray + 3;
  const double x1 = S[0] + a[0] * t;
  const double x2 = (S[1] + a[1] * t) * (S[1] + a[1] * t);
  const double x3 = (S[2] + a[2] * t) * (S[2] + a[2] * t);
  return -max_potential - ((x1 - m) * (x1 - m) + x2 + x3) * 0.5 - m / sqrt((x1 - 1) * (x1 - 1) + x2 + x3) -
         (1 - m) / sqrt(x1 * x1 + x2 + x3);
}

/* FindRoshRoots (:44-64) and GetIntersectionWithRosh (:66-86).  The reference stores the
 * roots in an array of 6 without a bound; more than 6 sign changes would overrun it.  Here
 * the count goes on, only the first 6 are stored (the result needs roots[1] and a count of
 * 4 or 6), and the bubble sort of the already ascending roots is the identity. */
int32_t orc_ray_roche(const double *ray, double *dist) {
  const int n = 1001;
  const double a = -3, b = 3;
  const double step = (b - a) / (n - 1);
  double roots[6];
  int size = 0;
  double fi_1 = ray_rosh(ray, a + 0 * step);
  for (int i = 1; i < n; ++i) {
    const double fi_2 = ray_rosh(ray, a + (i)*step);
    if (fi_1 * fi_2 < 0) {
      if (size < 6) roots[size] = ((2 * a + (2. * i - 1) * step) / 2.);
      size++;
    }
    fi_1 = fi_2;
  }
  if (size == 6 || size == 4) {
    const double x0 = ray[0] + ray[3] * roots[1];
    if (x0 < 0.3) {
      *dist = roots[1];
      return ORC_RAY_ROCHE;
    }
  }
  *dist = -1;
  return ORC_RAY_NONE;
}

/* IntersectionWithPlane (:88-101) and GetIntersectionWithSphereOfDisk (:110-169); the
 * reference returns "sphere" as soon as the ray meets the accretor sphere (the code after
 * that return never runs). */
int32_t orc_ray_sphere_disk(const double *ray) {
  const double A[3] = {1, 0, 0}, B[3] = {0, 0.9928768384869221, 0.11914522061843064}, C[3] = {2, 0, 0};
  const double *o = ray, *n = ray + 3;
  const double pa = A[1] * (B[2] - C[2]) + B[1] * (C[2] - A[2]) + C[1] * (A[2] - B[2]);
  const double pb = A[0] * (C[2] - B[2]) + B[0] * (A[2] - C[2]) + C[0] * (B[2] - A[2]);
  const double pc = A[0] * (B[1] - C[1]) + B[0] * (C[1] - A[1]) + C[0] * (A[1] - B[1]);
  const double pd = A[0] * (C[1] * B[2] - B[1] * C[2]) + B[0] * (A[1] * C[2] - C[1] * A[2]) +
                    C[0] * (B[1] * A[2] - A[1] * B[2]);
  const double t = -(pa * o[0] + pb * o[1] + pc * o[2] + pd) / (pa * n[0] + pb * n[1] + pc * n[2]);
  double res[3];
  for (int k = 0; k < 3; k++) res[k] = n[k] * t + o[k];
  const double vec_1[3] = {1, 0, 0}, vec_2[3] = {0, -0.992877, -0.119145};
  double loc0 = 0, loc1 = 0;
  for (int k = 0; k < 3; k++) {
    loc0 += (res[k]) * vec_1[k];
    loc1 += (res[k]) * vec_2[k];
  }
  const double loc_x = loc0 - 1, loc_y = loc1 - 0;
  const double loc_sq = loc_x * loc_x + loc_y * loc_y;
  const double An = dot3(n, n);
  const double oc[3] = {o[0] - 1, o[1] - 0, o[2] - 0};
  const double proj = dot3(oc, n);
  const double r_s = 0.01, r_in = 0.01, r_ex = 0.06;
  const double radical = 4. * (proj * proj - An * (1 - 2 * o[0] + dot3(o, o) - r_s * r_s));
  if (radical >= 0) return ORC_RAY_SPHERE;
  if (loc_sq < r_ex * r_ex && (loc_sq > r_in * r_in)) return ORC_RAY_DISK;
  return ORC_RAY_NONE;
}

/* RayTracing (:46-73), RayTracing_Phl1445 (:75-114), InnerRayTracing (:116-152),
 * RayTracingGrid (:154-177): the nearest triangle hit (strictly closer than the best so
 * far, so the first in index order among equal distances), after the Roche lobe (mode 1)
 * or instead of the triangles when the accretor sphere or disk is met (mode 2). */
void orc_ray_trace(int32_t mode, const double *rays, int64_t M, const int32_t *ids, const double *abc, int64_t N,
                   int32_t *out, int nthreads) {
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads > 0 ? nthreads : 1)
  for (int64_t r = 0; r < M; r++) {
    const double *ray = rays + 6 * r;
    int32_t loc_id = ORC_RAY_NONE;
    double loc_dist = 1e10;
    if (mode == 1) {
      double rd;
      if (orc_ray_roche(ray, &rd) != ORC_RAY_NONE) {
        loc_dist = rd;
        loc_id = ORC_RAY_ROCHE;
      }
    } else if (mode == 2) {
      const int32_t code = orc_ray_sphere_disk(ray);
      if (code != ORC_RAY_NONE) {
        out[r] = code;
        continue;
      }
    }
    for (int64_t i = 0; i < N; i++) {
      const double d = orc_ray_triangle(ray, abc + 9 * i);
      if (d > 0 && d < loc_dist) {
        loc_id = ids[i];
        loc_dist = d;
      }
    }
    out[r] = loc_id;
  }
}

/* Eigen normalize: v / sqrt((x^2 + y^2) + z^2) component by component */
static void normalize3(double *v) {
  const double z = dot3(v, v);
  if (z > 0) {
    const double s = sqrt(z);
    for (int k = 0; k < 3; k++) v[k] = v[k] / s;
  }
}

/* intersection::SetBasis (lib/geometry/src/intersections.cpp:3-40), row-major basis */
static void ray_set_basis(const double *nrm, double *basis) {
  double v1[3], v2[3];
  if (fabs(nrm[1]) < 1e-20) {
    v1[0] = 0;
    v1[1] = 1;
    v1[2] = 0;
  } else {
    v1[0] = 1;
    v1[2] = 0;
    v1[1] = -(nrm[0] * v1[0] + nrm[2] * v1[2]) / nrm[1];
  }
  if (nrm[1] < 0)
    for (int k = 0; k < 3; k++) v1[k] = -v1[k];
  cross3(nrm, v1, v2);
  normalize3(v1);
  normalize3(v2);
  for (int k = 0; k < 3; k++) {
    basis[k] = v2[k];
    basis[3 + k] = v1[k];
    basis[6 + k] = nrm[k];
  }
}

/* MakeRays(num_frame, rays) and MakeRays(center_ray, rays), ray_tracing_build_plane.cpp;
 * constants of solvers/ray_tracing/include/ray_tracing_const.h (GRB_TASK plane 1.2 x 0.6,
 * 600 x 300 pixels, 120 frames, height 0.1 above the centre of mass (0.879518, 0, 0)). */
void orc_ray_make_rays(int32_t frame, double *rays) {
  const double PIv = 3.1415926535897932384626433832795, com[3] = {0.879518, 0, 0};
  const int nw = 600, nh = 300, nframes = 120;
  const double width = 1.2, height = 0.6, above = 0.1;
  const double start_angle = 2 * PIv / nframes * frame;
  const double start[3] = {cos(start_angle) + com[0], sin(start_angle) + com[1], above + com[2]};
  double dir[3] = {com[0] - start[0], com[1] - start[1], com[2] - start[2]};
  normalize3(dir);
  double basis[9];
  ray_set_basis(dir, basis);
  const double ap[3] = {-(width / 2), -(height / 2), 0};
  const double step_x = width / nw, step_y = height / nh;
  for (int i = 0; i < nw; ++i)
    for (int j = 0; j < nh; ++j) {
      const double o2[3] = {ap[0] + i * step_x, ap[1] + j * step_y, 0};
      double o3[3];
      matTvec(basis, o2, o3);
      double *r = rays + 6 * ((int64_t)i * nh + j);
      for (int k = 0; k < 3; k++) {
        r[k] = o3[k] + start[k];
        r[3 + k] = dir[k];
      }
    }
}
