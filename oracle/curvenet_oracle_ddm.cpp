// curvenet_oracle_ddm.cpp -- CPU FP64 restatement of the Direct Delta Mush
// runtime kernel and bind-time post-processing (TEST INFRASTRUCTURE ONLY: the
// checker of the product's cn_lbs_matvec_device and cn_ddm_bind).
//
//   DirectDeltaMush.lean:70-74    applyTransform4x4
//   DirectDeltaMush.lean:84-102   lbsMatvec
//   DirectDeltaMushBind.lean:72-94   smoothWeights (damped neighbour mean)
//   DirectDeltaMushBind.lean:104-133 sparsifyTopK (selection sort by |w|
//                                    with swaps, then renormalisation)
// Compiled with -ffp-contract=off: every a*b+c rounds twice, as Lean's Float.
#include <cmath>
#include <vector>

extern "C" {

// T row-major 4x4; the point is (x, y, z, 1).
void orc_apply_transform4x4(const double* T, double x, double y, double z, double* out) {
  out[0] = T[0] * x + T[1] * y + T[2] * z + T[3];
  out[1] = T[4] * x + T[5] * y + T[6] * z + T[7];
  out[2] = T[8] * x + T[9] * y + T[10] * z + T[11];
}

// One vertex: sum over its influences (in order) of w * (T_i (r, 1)).
void orc_lbs_matvec(const double* transforms, int n_infl, const int* idx, const double* w, double rx, double ry,
                    double rz, double* out) {
  double x = 0.0, y = 0.0, z = 0.0;
  for (int k = 0; k < n_infl; ++k) {
    double t[3];
    orc_apply_transform4x4(transforms + 16 * (size_t)idx[k], rx, ry, rz, t);
    x = x + w[k] * t[0];
    y = y + w[k] * t[1];
    z = z + w[k] * t[2];
  }
  out[0] = x;
  out[1] = y;
  out[2] = z;
}

// All vertices, influences in CSR (start[v] .. start[v + 1]).
void orc_lbs_matvec_csr(int nv, const double* rest, const double* transforms, const int* start, const int* idx,
                        const double* w, double* out) {
  for (int v = 0; v < nv; ++v)
    orc_lbs_matvec(transforms, start[v + 1] - start[v], idx + start[v], w + start[v], rest[3 * v],
                   rest[3 * v + 1], rest[3 * v + 2], out + 3 * (size_t)v);
}

// W: n x nh row-major; adjacency adj_ptr / adj_idx (neighbour order as
// given); nu passes of w' = (1 - omega) w + omega * (sum of neighbours / count).
void orc_smooth_weights(int n, int nh, const double* W, const int* adj_ptr, const int* adj_idx, int nu,
                        double omega, double* out) {
  std::vector<double> cur(W, W + (size_t)n * nh), next((size_t)n * nh);
  for (int pass = 0; pass < nu; ++pass) {
    for (int v = 0; v < n; ++v) {
      const int count = adj_ptr[v + 1] - adj_ptr[v];
      for (int i = 0; i < nh; ++i) {
        double nb = 0.0;
        if (count > 0) {
          for (int e = adj_ptr[v]; e < adj_ptr[v + 1]; ++e) nb = nb + cur[(size_t)adj_idx[e] * nh + i];
          nb = nb / (double)count;
        }
        next[(size_t)v * nh + i] = (1.0 - omega) * cur[(size_t)v * nh + i] + omega * nb;
      }
    }
    cur.swap(next);
  }
  for (size_t q = 0; q < cur.size(); ++q) out[q] = cur[q];
}

// Per row: the selection sort of the spec (position k takes the first
// entry of largest |w| among positions >= k, then swaps), keep
// take = min(K, nh) entries, divide them by their sum when it is not 0.
// out_idx / out_w: n x take.
void orc_sparsify_topk(int n, int nh, const double* W, int K, int* out_idx, double* out_w) {
  const int take = K < nh ? K : nh;
  std::vector<int> pi(nh);
  std::vector<double> pw(nh);
  for (int v = 0; v < n; ++v) {
    for (int i = 0; i < nh; ++i) {
      pi[i] = i;
      pw[i] = W[(size_t)v * nh + i];
    }
    for (int k = 0; k < take; ++k) {
      int best = k;
      for (int j = k + 1; j < nh; ++j)
        if (std::fabs(pw[j]) > std::fabs(pw[best])) best = j;
      std::swap(pi[k], pi[best]);
      std::swap(pw[k], pw[best]);
    }
    double sum = 0.0;
    for (int k = 0; k < take; ++k) sum = sum + pw[k];
    for (int k = 0; k < take; ++k) {
      out_idx[(size_t)v * take + k] = pi[k];
      out_w[(size_t)v * take + k] = sum != 0.0 ? pw[k] / sum : pw[k];
    }
  }
}

}  // extern "C"
