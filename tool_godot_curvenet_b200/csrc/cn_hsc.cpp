// cn_hsc.cpp -- host construction of the HSC (hierarchical sparsify and
// compensate) preconditioner of a reduced system A.
//
// The reference specifies the elimination primitive
// (HierarchicalSparsifyCompensate.lean:97-125): eliminating vertex v adds
// w(v,i) w(v,j) / deg(v) to the edge (i, j) of every pair of v's neighbours
// and drops v's edges.  The hierarchy completes it:
//   * the M-matrix part of A: a positive off-diagonal a_ij is moved onto the
//     diagonals (A + a_ij (e_i - e_j)(e_i - e_j)^T, still SPD);
//   * per level, F = the greedy maximal independent set in index order and C
//     the rest; eliminating the independent set is the spec's rule applied to
//     every v in F (deg(v) = M_vv with the Dirichlet excess), i.e. the Schur
//     complement S = M_CC - M_CF D_F^{-1} M_FC;
//   * sparsify: a fill entry of S absent from M_CC is kept if
//     |S_ij| >= theta sqrt(S_ii S_jj) or if it is among the keep_k largest
//     off-diagonals of row i or row j; a dropped entry is added to the
//     diagonal of its row (row sums, hence the action on constants and the
//     Dirichlet excess, are unchanged);
//   * recurse down to at most n_coarse unknowns, whose matrix is inverted
//     densely (Cholesky).
// The V-cycle application runs in the persistent solve (cn_pcg_body.cuh).
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "cn_hsc.h"

namespace cn {
namespace {

struct Csr {
  int n = 0;
  std::vector<int> ptr, col;
  std::vector<double> val;
};

double find(const Csr& M, int r, int c) {
  auto b = M.col.begin() + M.ptr[r], e = M.col.begin() + M.ptr[r + 1];
  auto it = std::lower_bound(b, e, c);
  return (it != e && *it == c) ? M.val[it - M.col.begin()] : 0.0;
}

}  // namespace

cn_status hsc_build(int n, const int* ptr, const int* col, const double* val, const HscParams& prm,
                    HscHost& out) {
  // ---- M-matrix part
  Csr M;
  M.n = n;
  M.ptr.assign(n + 1, 0);
  {
    std::vector<double> extra(n, 0.0);
    for (int i = 0; i < n; ++i)
      for (int e = ptr[i]; e < ptr[i + 1]; ++e)
        if (col[e] != i && val[e] > 0.0) extra[i] += val[e];
    for (int i = 0; i < n; ++i) {
      for (int e = ptr[i]; e < ptr[i + 1]; ++e) {
        const int j = col[e];
        double v = val[e];
        if (j != i && v > 0.0) continue;
        if (j == i) v += extra[i];
        M.col.push_back(j);
        M.val.push_back(v);
      }
      M.ptr[i + 1] = (int)M.col.size();
    }
  }
  std::vector<int> gid(n);
  std::iota(gid.begin(), gid.end(), 0);
  out = HscHost{};
  out.n = n;
  std::vector<std::vector<int>> level_C_gid;  // to map C rows to HSC positions at the end
  int off = 0;
  while (M.n > prm.n_coarse && (int)out.levels.size() < prm.max_levels) {
    const int m = M.n;
    // greedy maximal independent set in index order
    std::vector<char> sel(m, 0), blocked(m, 0);
    for (int v = 0; v < m; ++v)
      if (!blocked[v]) {
        sel[v] = 1;
        for (int e = M.ptr[v]; e < M.ptr[v + 1]; ++e) blocked[M.col[e]] = 1;
      }
    std::vector<int> F, C, fidx(m, -1), cidx(m, -1);
    for (int v = 0; v < m; ++v) {
      if (sel[v]) { fidx[v] = (int)F.size(); F.push_back(v); }
      else { cidx[v] = (int)C.size(); C.push_back(v); }
    }
    if ((double)F.size() < 0.02 * m) break;
    HscHost::Level L;
    L.off = off;
    L.nf = (int)F.size();
    L.dinv.resize(F.size());
    for (size_t k = 0; k < F.size(); ++k) L.dinv[k] = 1.0 / find(M, F[k], F[k]);
    // R: rows C (local C order), cols F (local F index) : M_iv * (1 / M_vv)
    L.R_ptr.assign(C.size() + 1, 0);
    for (size_t k = 0; k < C.size(); ++k) {
      const int i = C[k];
      for (int e = M.ptr[i]; e < M.ptr[i + 1]; ++e) {
        const int v = M.col[e];
        if (fidx[v] >= 0) {
          L.R_col.push_back(fidx[v]);
          L.R_val.push_back(M.val[e] * L.dinv[fidx[v]]);
        }
      }
      L.R_ptr[k + 1] = (int)L.R_col.size();
    }
    // P: rows F, cols C (local C index) : M_vj
    L.P_ptr.assign(F.size() + 1, 0);
    for (size_t k = 0; k < F.size(); ++k) {
      const int v = F[k];
      for (int e = M.ptr[v]; e < M.ptr[v + 1]; ++e)
        if (cidx[M.col[e]] >= 0) {
          L.P_col.push_back(cidx[M.col[e]]);
          L.P_val.push_back(M.val[e]);
        }
      L.P_ptr[k + 1] = (int)L.P_col.size();
    }
    // Schur complement on C
    const int nc = (int)C.size();
    Csr S;
    S.n = nc;
    S.ptr.assign(nc + 1, 0);
    std::vector<char> base_flag;
    {
      std::vector<double> acc(nc, 0.0);
      std::vector<int> mark(nc, -1), touched;
      std::vector<char> isbase(nc, 0);
      for (int k = 0; k < nc; ++k) {
        const int i = C[k];
        touched.clear();
        for (int e = M.ptr[i]; e < M.ptr[i + 1]; ++e) {
          const int j = cidx[M.col[e]];
          if (j < 0) continue;
          if (mark[j] != k) { mark[j] = k; acc[j] = 0.0; touched.push_back(j); }
          acc[j] += M.val[e];
          isbase[j] = 1;
        }
        for (int e = L.R_ptr[k]; e < L.R_ptr[k + 1]; ++e) {
          const int v = F[L.R_col[e]];
          const double coef = L.R_val[e];
          for (int q = M.ptr[v]; q < M.ptr[v + 1]; ++q) {
            const int j = cidx[M.col[q]];
            if (j < 0) continue;
            if (mark[j] != k) { mark[j] = k; acc[j] = 0.0; touched.push_back(j); isbase[j] = 0; }
            acc[j] -= coef * M.val[q];
          }
        }
        std::sort(touched.begin(), touched.end());
        for (int j : touched) {
          S.col.push_back(j);
          S.val.push_back(acc[j]);
          base_flag.push_back(isbase[j]);
          isbase[j] = 0;
        }
        S.ptr[k + 1] = (int)S.col.size();
      }
    }
    // sparsify with row-sum compensation
    std::vector<double> diag(nc, 0.0);
    for (int i = 0; i < nc; ++i) diag[i] = find(S, i, i);
    std::vector<char> top(S.col.size(), 0);
    {
      std::vector<int> idx;
      for (int i = 0; i < nc; ++i) {
        idx.clear();
        for (int e = S.ptr[i]; e < S.ptr[i + 1]; ++e)
          if (S.col[e] != i) idx.push_back(e);
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
          const double ma = std::fabs(S.val[a]), mb = std::fabs(S.val[b]);
          if (ma != mb) return ma > mb;
          return S.col[a] < S.col[b];
        });
        for (int q = 0; q < (int)idx.size() && q < prm.keep_k; ++q) top[idx[q]] = 1;
      }
    }
    auto entry = [&](int r, int c) {
      auto b = S.col.begin() + S.ptr[r], e = S.col.begin() + S.ptr[r + 1];
      auto it = std::lower_bound(b, e, c);
      return (it != e && *it == c) ? (int)(it - S.col.begin()) : -1;
    };
    Csr S2;
    S2.n = nc;
    S2.ptr.assign(nc + 1, 0);
    for (int i = 0; i < nc; ++i) {
      double comp = 0.0;
      int dpos = -1;
      for (int e = S.ptr[i]; e < S.ptr[i + 1]; ++e) {
        const int j = S.col[e];
        bool keep = true;
        if (j != i && !base_flag[e]) {
          const bool weak = std::fabs(S.val[e]) < prm.theta * std::sqrt(diag[i] * diag[j]);
          const int t = entry(j, i);
          const bool strong = top[e] || (t >= 0 && top[t]);
          keep = !weak || strong;
        }
        if (!keep) { comp += S.val[e]; continue; }
        if (j == i) dpos = (int)S2.col.size();
        S2.col.push_back(j);
        S2.val.push_back(S.val[e]);
      }
      if (dpos >= 0) S2.val[dpos] += comp;
      S2.ptr[i + 1] = (int)S2.col.size();
    }
    for (int v : F) out.order.push_back(gid[v]);
    std::vector<int> cg(nc);
    for (int k = 0; k < nc; ++k) cg[k] = gid[C[k]];
    level_C_gid.push_back(cg);
    out.levels.push_back(std::move(L));
    off += (int)F.size();
    M = std::move(S2);
    gid = std::move(cg);
  }
  for (int v = 0; v < M.n; ++v) out.order.push_back(gid[v]);
  out.coarse_off = off;
  out.nc = M.n;
  // map level-local indices to HSC positions
  std::vector<int> pos_of(n);
  for (int p = 0; p < n; ++p) pos_of[out.order[p]] = p;
  for (size_t l = 0; l < out.levels.size(); ++l) {
    HscHost::Level& L = out.levels[l];
    L.R_rows.resize(level_C_gid[l].size());
    for (size_t k = 0; k < level_C_gid[l].size(); ++k) L.R_rows[k] = pos_of[level_C_gid[l][k]];
    for (int& c : L.R_col) c += L.off;  // F positions of this level are contiguous
    for (int& c : L.P_col) c = pos_of[level_C_gid[l][c]];
  }
  // coarse: dense Cholesky, then the inverse
  const int nc = M.n;
  std::vector<double> D((size_t)nc * nc, 0.0), Lc((size_t)nc * nc, 0.0);
  for (int i = 0; i < nc; ++i)
    for (int e = M.ptr[i]; e < M.ptr[i + 1]; ++e) D[(size_t)i * nc + M.col[e]] = M.val[e];
  for (int j = 0; j < nc; ++j) {
    double s = D[(size_t)j * nc + j];
    for (int k = 0; k < j; ++k) s -= Lc[(size_t)j * nc + k] * Lc[(size_t)j * nc + k];
    if (!(s > 0.0)) return CN_NONPOS_PIVOT;
    const double d = std::sqrt(s);
    Lc[(size_t)j * nc + j] = d;
    for (int i = j + 1; i < nc; ++i) {
      double t = D[(size_t)i * nc + j];
      for (int k = 0; k < j; ++k) t -= Lc[(size_t)i * nc + k] * Lc[(size_t)j * nc + k];
      Lc[(size_t)i * nc + j] = t / d;
    }
  }
  out.Sinv.assign((size_t)nc * nc, 0.0);
  std::vector<double> y(nc), x(nc);
  for (int c = 0; c < nc; ++c) {  // column c of the inverse: solve L L^T x = e_c
    for (int i = 0; i < nc; ++i) {
      double s = i == c ? 1.0 : 0.0;
      for (int k = 0; k < i; ++k) s -= Lc[(size_t)i * nc + k] * y[k];
      y[i] = s / Lc[(size_t)i * nc + i];
    }
    for (int i = nc - 1; i >= 0; --i) {
      double s = y[i];
      for (int k = i + 1; k < nc; ++k) s -= Lc[(size_t)k * nc + i] * x[k];
      x[i] = s / Lc[(size_t)i * nc + i];
    }
    for (int i = 0; i < nc; ++i) out.Sinv[(size_t)i * nc + c] = x[i];
  }
  return CN_OK;
}

}  // namespace cn
