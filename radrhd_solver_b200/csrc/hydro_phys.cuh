// FP64 device physics of the relativistic HLLC step.
//
// Each function performs the reference's arithmetic in the reference's order
// (solvers/rhllc/src/rhllc_flux_stab.cpp, lib/geometry/src/linear_alg.cpp),
// including Eigen's association order for 3-vectors as compiled by gcc -O2 on
// x86-64: dot = (x0 + x1) + x2; Matrix3 * Vector3 rows 0,1 = (x0 + x1) + x2 and
// row 2 = x0 + (x1 + x2); Matrix3.transpose() * Vector3 = (x0 + x1) + x2.
// Translation units including this header are compiled with --fmad=false, so
// every + - * / sqrt is one IEEE-rounded operation as on the CPU, and results
// equal the reference bit for bit.
#pragma once
#include <stdint.h>

namespace rrhd {

struct Eos {
  int eos;    // 1 ideal, 2 Taub
  double g1;  // kGamma1
  double gg;  // kGamma_g = g1 / (g1 - 1)
};

#define RRHD_MAX_ITER 40

__device__ __forceinline__ double smin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double smax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dot3(double a0, double a1, double a2, double b0, double b1,
                                       double b2) {
  return (a0 * b0 + a1 * b1) + a2 * b2;
}

// Orthonormal frame with row 0 = n: GetRotationMatrix, linear_alg.cpp:3-42.
struct Rot {
  double t[9];
};
__device__ __forceinline__ void rotation(double n0, double n1, double n2, Rot &R) {
  double *T = R.t;
#pragma unroll
  for (int i = 0; i < 9; i++) T[i] = 0.0;
  if (fabs(n2 * n2 - 1) > 1e-12) {
    T[0] = n0;
    T[1] = n1;
    T[2] = n2;
    const double sqr = sqrt(1 - n2 * n2);
    const double sqr_inv = 1. / sqr;
    T[3] = -n1 * sqr_inv;
    T[4] = n0 * sqr_inv;
    T[6] = -n0 * n2 * sqr_inv;
    T[7] = -n1 * n2 * sqr_inv;
    T[8] = sqr;
  } else if (n2 > 0) {
    T[2] = 1;
    T[4] = 1;
    T[6] = -1;
  } else {
    T[2] = -1;
    T[4] = -1;
    T[6] = 1;
  }
}
__device__ __forceinline__ void matvec(const Rot &R, const double *v, double *r) {
  const double *T = R.t;
  r[0] = (T[0] * v[0] + T[1] * v[1]) + T[2] * v[2];
  r[1] = (T[3] * v[0] + T[4] * v[1]) + T[5] * v[2];
  r[2] = T[6] * v[0] + (T[7] * v[1] + T[8] * v[2]);
}
// T.transpose() materialised as a Matrix3 and then times v (the Matrix3 * Vector3 order above).
__device__ __forceinline__ void matvec_transposed(const Rot &R, const double *v, double *r) {
  const double *T = R.t;
  r[0] = (T[0] * v[0] + T[3] * v[1]) + T[6] * v[2];
  r[1] = (T[1] * v[0] + T[4] * v[1]) + T[7] * v[2];
  r[2] = T[2] * v[0] + (T[5] * v[1] + T[8] * v[2]);
}
__device__ __forceinline__ void matTvec(const Rot &R, const double *v, double *r) {
  const double *T = R.t;
  r[0] = (T[0] * v[0] + T[3] * v[1]) + T[6] * v[2];
  r[1] = (T[1] * v[0] + T[4] * v[1]) + T[7] * v[2];
  r[2] = (T[2] * v[0] + T[5] * v[1]) + T[8] * v[2];
}

// GetConvValueStab, rhllc_flux_stab.cpp:10-38 (W may be rescaled).
__device__ __forceinline__ void p2c(const Eos &e, double *W, double *U) {
  double h;
  if (e.eos == 1) {
    h = 1 + e.gg * W[4] / W[0];
  } else {
    const double theta = W[4] / W[0];
    h = 2.5 * theta + sqrt(2.25 * theta * theta + 1.0);
  }
  double g = dot3(W[1], W[2], W[3], W[1], W[2], W[3]);
  if (g >= 1.0) {
    const double beta_fix = 0.9999;
    g = beta_fix / sqrt(g);
    W[1] *= g;
    W[2] *= g;
    W[3] *= g;
    g = beta_fix * beta_fix;
  }
  g = 1.0 / (1.0 - g);
  const double scrh = W[0] * h * g;
  g = sqrt(g);
  U[0] = W[0] * g;
  U[1] = scrh * W[1];
  U[2] = scrh * W[2];
  U[3] = scrh * W[3];
  U[4] = scrh - W[4];
}

// GetConvValue, solvers/rhllc/src/rhllc_flux.cpp:7-16 (fixed inflow states).
__host__ __device__ inline void p2c_plain(double gg, const double *W, double *U) {
  const double d = W[0];
  const double Gamma = 1. / sqrt(1 - ((W[1] * W[1] + W[2] * W[2]) + W[3] * W[3]));
  const double h = 1 + gg * W[4] / d;
  const double dhGG = d * h * Gamma * Gamma;
  U[0] = Gamma * W[0];
  U[1] = dhGG * W[1];
  U[2] = dhGG * W[2];
  U[3] = dhGG * W[3];
  U[4] = dhGG - W[4];
}

__device__ __forceinline__ double dh_fix(const Eos &e, double D, double plor, double alpha) {
  if (e.eos == 1) return D + plor * alpha;
  return 2.5 * plor + sqrt(2.25 * plor * plor + D * D);
}

// PhysPressureFix, rhllc_flux_stab.cpp:40-121 (rewrites U[4]).
__device__ __forceinline__ int pressure_fix(const Eos &e, double *U, double *W) {
  const double p = 1e-12;  // kMinPressure
  const double D = U[0];
  const double m2 = dot3(U[1], U[2], U[3], U[1], U[2], U[3]);
  const double m = sqrt(m2);
  const double umax = m / D;
  double u0 = umax;
  double lor = sqrt(1.0 + u0 * u0);
  double plor = p * lor;
  const double alpha = (e.eos == 1) ? e.gg : 2.5;
  double Dh = dh_fix(e, D, plor, alpha);
  double f0 = m / Dh - u0;
  double u1 = (-D + sqrt(D * D + 4.0 * m * alpha * p)) / (2.0 * alpha * p);
  int done = 0;
  double f1, du;
  for (int k = 1; k < RRHD_MAX_ITER; k++) {
    lor = sqrt(1.0 + u1 * u1);
    plor = p * lor;
    Dh = dh_fix(e, D, plor, alpha);
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
  Dh = dh_fix(e, D, plor, alpha);
  W[0] = U[0] / lor;
  W[4] = p;
  U[4] = Dh * lor - p;
  f0 = 1.0 / (Dh * lor);
  W[1] = U[1] * f0;
  W[2] = U[2] * f0;
  W[3] = U[3] * f0;
  return 0;
}

// GetPhysValueStab, rhllc_flux_stab.cpp:123-220.  Newton on the pressure from
// the initial guess p0; returns the reference's code (5 where it would abort).
// W is written only on success.  iters (if non-null) gets the Newton count.
__device__ __forceinline__ int c2p_from(const Eos &e, const double *U, double *W, double p0,
                                        bool use_guess, int *iters, int max_iter = RRHD_MAX_ITER) {
  const double tol = 1.e-11;
  const double eps2 = 1.e-12;
  const double D = U[0];
  const double E = U[4];
  const double m2 = dot3(U[1], U[2], U[3], U[1], U[2], U[3]);
  const double Q = E - sqrt(m2 + D * D);
  if (Q < 0.0) return 1;
  const double m = sqrt(m2);
  double p = smax(m - E, 0.0);
  const double D_1 = 1.0 / D;
  const double pmin = sqrt(m2 / (1.0 - eps2)) - E;
  if (use_guess) p = p0;
  p = smax(p, pmin);
  double alpha, alpha2, lor2, lor, tau, theta, h, dh_dp, dh_dtau, yp = 0, dp, dyp;
  int iter;
  for (iter = 0; iter < max_iter; iter++) {
    alpha = E + p;
    alpha2 = alpha * alpha;
    lor2 = 1.0 - m2 / alpha2;
    lor2 = 1.0 / lor2;
    if (lor2 < 1.0) {
      if (iters) *iters = iter;
      return 5;
    }
    lor = sqrt(lor2);
    tau = lor * D_1;
    theta = p * tau;
    if (e.eos == 1) {
      h = 1.0 + e.gg * theta;
      dh_dp = e.gg * tau;
      dh_dtau = e.gg * p;
    } else {
      h = 2.5 * theta + sqrt(2.25 * theta * theta + 1.0);
      const double scrh = (5.0 * h - 8.0 * theta) / (2.0 * h - 5.0 * theta);
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
  if (iters) *iters = iter;
  if (p < 0.0) return 2;
  if (isnan(p)) return 4;
  if (iter >= max_iter || fabs(yp / (E + p)) > 1.e-4 || p < (m - E)) return 3;
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

__device__ __forceinline__ int c2p(const Eos &e, const double *U, double *W) {
  return c2p_from(e, U, W, 0.0, false, nullptr);
}

// con2prim with the reference's fallback; returns the status byte
// (code | 0x10 when PhysPressureFix ran | 0x20 when it failed as well).
__device__ __forceinline__ uint8_t c2p_with_fix(const Eos &e, double *U, double *W) {
  int code = c2p(e, U, W);
  if (code) {
    const int fix = pressure_fix(e, U, W);
    code = code | 0x10 | (fix ? 0x20 : 0);
  }
  return (uint8_t)code;
}

__device__ __forceinline__ void signal_speed(double cs2, double Vn, double V2, double &cmin,
                                             double &cmax) {
  const double Vn2 = Vn * Vn;
  const double Vt2 = V2 - Vn2;
  const double sroot = sqrt(cs2 * (1 - Vn2 - Vt2 * cs2) * (1 - V2));
  cmax = (Vn * (1.0 - cs2) + sroot) / (1.0 - V2 * cs2);
  cmin = (Vn * (1.0 - cs2) - sroot) / (1.0 - V2 * cs2);
}

__device__ __forceinline__ double sound_speed2(const Eos &e, double d, double p) {
  if (e.eos == 1) {
    const double h = 1 + e.gg * p / d;
    return ((e.g1 * p) / (d * h));
  }
  const double theta = p / d;
  const double h = 2.5 * theta + sqrt(2.25 * theta * theta + 1.0);
  return theta / (3.0 * h) * (5.0 * h - 8.0 * theta) / (h - theta);
}

// GetFluxStab, rhllc_flux_stab.cpp:240-431, split in three parts so that a thread
// holds few values at a time (the step kernel is latency-bound and runs more warps
// when each needs fewer registers).  Every value is formed by the reference's
// operations in the reference's order, so the flux is the reference's bit for bit:
//   face_side    one side's rotated normal velocity and momentum, energy, pressure,
//                sound speed and signal speeds (:257-318);
//   face_star    the wave speeds lambda_L/R, the branch, and in the HLLC branch the
//                contact speed us and pressure ps (:319-394);
//   face_flux    the flux of the side the branch selects, from that side's state
//                reloaded in the global frame, rotated back and times the area
//                (:331-346, :395-431).
struct FaceSide {
  double cmin, cmax;  // signal speeds (GetSignalSpeed, :231-238)
  double m1;          // momentum along the normal: row 0 of T * U.v
  double E;           // U.p (total energy)
  double vn;          // velocity along the normal: row 0 of T * W.v
  double p;           // W.p
};

// cs2 = sound_speed2(e, W[0], W[4]): a function of the cell's state alone, so the step
// computes it once per staged cell rather than once per face and side.
__device__ __forceinline__ FaceSide face_side(const Rot &R, const double *U, const double *W, double cs2) {
  double vel[3];
  matvec(R, W + 1, vel);
  FaceSide s;
  s.m1 = (R.t[0] * U[1] + R.t[1] * U[2]) + R.t[2] * U[3];
  s.E = U[4];
  s.vn = vel[0];
  s.p = W[4];
  const double VV = dot3(vel[0], vel[1], vel[2], vel[0], vel[1], vel[2]);
  signal_speed(cs2, vel[0], VV, s.cmin, s.cmax);
  return s;
}

// Which side's flux the face takes and the star-state parameters.
struct FaceStar {
  double vmax;  // max(lambda_L, lambda_R), the value GetFluxStab returns
  double lam;   // the selected side's wave speed (HLLC branch)
  double us, ps;
  bool right;   // the flux is built from the right state
  bool star;    // HLLC branch (star state), else the upwind flux of one side
};

__device__ __forceinline__ FaceStar face_star(const FaceSide &L, const FaceSide &R) {
  const double lambda_L = smin(L.cmin, R.cmin);
  const double lambda_R = smax(L.cmax, R.cmax);
  FaceStar f;
  f.vmax = smax(lambda_L, lambda_R);
  f.lam = 0.0;
  f.us = 0.0;
  f.ps = 0.0;
  f.star = false;
  if (lambda_L >= 0.0) {
    f.right = false;
  } else if (lambda_R <= 0.0) {
    f.right = true;
  } else {
    // F_L = {D vn, m vn, m1}: F_L.p = m1, F_L.v[0] = m1 vn
    const double AL = lambda_L * L.E - L.m1;
    const double AR = lambda_R * R.E - R.m1;
    const double BL = lambda_L * L.m1 - L.m1 * L.vn - L.p;
    const double BR = lambda_R * R.m1 - R.m1 * R.vn - R.p;
    const double a = AR * lambda_L - AL * lambda_R;
    const double b = AL + BL * lambda_R - AR - BR * lambda_L;
    const double c = BR - BL;
    const double scrh = -0.5 * (b + (b < 0.0 ? -1.0 : 1.0) * sqrt(b * b - 4.0 * a * c));
    f.us = c / scrh;
    f.ps = (AL * f.us - BL) / (1.0 - f.us * lambda_L);
    f.star = true;
    f.right = !(f.us >= 0.0);
    f.lam = f.right ? lambda_R : lambda_L;
  }
  return f;
}

// Fout = area * flux in the global frame, from the selected side's conservative
// state U (global frame) and its FaceSide values.
__device__ __forceinline__ void face_flux(const Rot &R, const double *U, const FaceSide &s, const FaceStar &f,
                                          double area, double *Fout) {
  double Ur[5];
  Ur[0] = U[0];
  Ur[4] = U[4];
  matvec(R, U + 1, Ur + 1);
  const double vn = s.vn;
  double F[5] = {Ur[0] * vn, Ur[1] * vn, Ur[2] * vn, Ur[3] * vn, Ur[1]};
  if (f.star) {
    const double lam = f.lam, us = f.us;
    double st[5];
    const double dif = 1.0 / (lam - us);
    st[0] = Ur[0] * (lam - vn) * dif;
    st[1] = (lam * (Ur[4] + f.ps) - Ur[1]) * us * dif;
    st[2] = Ur[2] * (lam - vn) * dif;
    st[3] = Ur[3] * (lam - vn) * dif;
    st[4] = Ur[4] + (st[1] - Ur[1]) / lam;
#pragma unroll
    for (int i = 0; i < 5; i++) st[i] -= Ur[i];
#pragma unroll
    for (int i = 0; i < 5; i++) st[i] *= lam;
#pragma unroll
    for (int i = 0; i < 5; i++) F[i] = F[i] + st[i];
  }
  F[1] += s.p;
  Fout[0] = F[0] * area;
  Fout[4] = F[4] * area;
  double Fv[3];
  matTvec(R, F + 1, Fv);
  Fout[1] = Fv[0] * area;
  Fout[2] = Fv[1] * area;
  Fout[3] = Fv[2] * area;
}

}  // namespace rrhd
