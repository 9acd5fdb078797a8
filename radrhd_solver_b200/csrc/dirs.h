// Device-resident direction set shared by the FP64 and tensor-core radiation kernels.
#pragma once
#include <vector>

struct rrhd_dirs {
  int device = 0;
  int M = 0;
  double full_area = 0;
  double *d_w = nullptr;  // [M][3]
  double *d_a = nullptr;  // [M]
  double *d_G = nullptr;  // [M][M] Gamma(w_d . w_k), row d
  double *d_K = nullptr;  // [M][M] Gamma * a_d / full_area, row d
  std::vector<double> h_w, h_a;
};
