// Per-cell radiation 4-force of rad_rhd::GetRadSource
// (solvers/RadRHD/src/radRHD_utils.cpp:44-101), shared by the batch entry point
// and the coupled step.  Compile with --fmad=false: the operation order is the
// reference's, so the result matches it bit for bit.
#pragma once
#include <cuda_runtime.h>

namespace rrhd {

struct Emission {
  double temp_coef, sigma_sb, pi, rad_unit;
};

// T = temp_coef p / rho, B = T^4 sigma_sb / pi (B_Plank, lib/physics/src/plunk.cpp:87-90)
__device__ __forceinline__ double planck_B(const Emission &em, double rho, double prs) {
  const double Tg = em.temp_coef * prs / rho;
  const double T2 = Tg * Tg;
  return (T2 * T2) * em.sigma_sb / em.pi;
}

// W = {rho, v[3], p}; Tr [9] read as Tr[3 j + i] = T(i, j) (Eigen column-major).
__device__ __forceinline__ void rad_source_cell(const Emission &em, const double *W, double abs_op, double scat_op,
                                                double Ur, const double *Fr, const double *Tr, double *G) {
  const double tot_op = abs_op + scat_op;
  const double rho = W[0];
  const double prs = W[4];
  const double v[3] = {W[1], W[2], W[3]};
  double gamma = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
  double u2 = gamma;
  const double gamma2 = 1.0 / (1.0 - gamma);
  u2 *= gamma2;
  gamma = sqrt(gamma2);
  const double u[3] = {gamma * v[0], gamma * v[1], gamma * v[2]};
  double uuD = 0.;
  const double uF = (u[0] * Fr[0] + u[1] * Fr[1]) + u[2] * Fr[2];
  double uD[3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    uD[i] = 0.;
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const double D = Tr[3 * j + i];
      uD[i] += u[j] * D;
      uuD += u[i] * u[j] * D;
    }
  }
  const double rhogamma = rho * gamma;
  const double B = planck_B(em, rho, prs);
  const double q = -abs_op * rho * B / em.rad_unit;
  G[0] = q * gamma + rhogamma * (abs_op - scat_op * (u2 + uuD)) * Ur - rho * (abs_op - scat_op * (u2 + gamma2)) * uF;
#pragma unroll
  for (int i = 0; i < 3; i++)
    G[i + 1] = q * u[i] - rho * (tot_op * uD[i] + scat_op * u[i] * (gamma2 + uuD)) * Ur +
               rhogamma * (tot_op * Fr[i] + scat_op * 2.0 * uF * u[i]);
}

}  // namespace rrhd
