// cn_hsc.h -- host construction of the HSC preconditioner (cn_hsc.cpp).
// Not part of the public ABI.
#pragma once

#include <vector>

#include "cn_internal.h"

namespace cn {

struct HscParams {
  double theta = 0.01;  // fill kept when |S_ij| >= theta sqrt(S_ii S_jj)
  int keep_k = 3;       // ... or when among the keep_k strongest of its row / column
  int n_coarse = 512;   // dense coarse solve at or below this size
  int max_levels = 64;
};

// HSC hierarchy in "HSC positions": the eliminated sets F_0, F_1, ... and the
// coarse set are consecutive ranges; order[p] = row of A at position p.
struct HscHost {
  int n = 0, coarse_off = 0, nc = 0;
  std::vector<int> order;
  struct Level {
    int off = 0, nf = 0;                 // F = positions [off, off + nf)
    std::vector<int> R_rows, R_ptr, R_col;  // rows: C positions; cols: F positions
    std::vector<double> R_val, dinv;     // R = M_CF D_F^{-1}; dinv over F
    std::vector<int> P_ptr, P_col;       // rows: F (local); cols: C positions
    std::vector<double> P_val;           // P = M_FC
  };
  std::vector<Level> levels;
  std::vector<double> Sinv;              // nc x nc, row-major
};

cn_status hsc_build(int n, const int* ptr, const int* col, const double* val, const HscParams& prm,
                    HscHost& out);

}  // namespace cn
