// curvenet_oracle_sparse.cpp -- sparse FP64 restatement (CSR assembly,
// Dirichlet reduction, greedy colouring, IC(0), PCG, HSC elimination) of the
// reference's Lean specification.
//
// TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline); the
// product never links it.  Built with -ffp-contract=off.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

extern "C" void orc_triangle_cot_laplacian(const double*, const double*, const double*, double*);
extern "C" void orc_robust_triangle_cot_laplacian(double, const double*, const double*,
                                                  const double*, double*);

namespace {

struct Csr {
  int n = 0;
  std::vector<int> ptr, col;
  std::vector<double> val;
};

// CSR pattern of the vertex adjacency of a triangle list, diagonal included,
// columns sorted.
Csr pattern_from_tris(int nv, int nt, const int* tris) {
  std::vector<uint64_t> keys;
  keys.reserve((size_t)nt * 6 + nv);
  for (int v = 0; v < nv; ++v) keys.push_back(((uint64_t)v << 32) | (uint32_t)v);
  for (int f = 0; f < nt; ++f)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        if (a != b)
          keys.push_back(((uint64_t)(uint32_t)tris[3 * f + a] << 32) | (uint32_t)tris[3 * f + b]);
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  Csr K;
  K.n = nv;
  K.ptr.assign(nv + 1, 0);
  K.col.resize(keys.size());
  for (size_t e = 0; e < keys.size(); ++e) {
    K.ptr[(keys[e] >> 32) + 1]++;
    K.col[e] = (int)(keys[e] & 0xffffffffu);
  }
  for (int v = 0; v < nv; ++v) K.ptr[v + 1] += K.ptr[v];
  K.val.assign(keys.size(), 0.0);
  return K;
}

int find_entry(const Csr& A, int r, int c) {
  auto b = A.col.begin() + A.ptr[r], e = A.col.begin() + A.ptr[r + 1];
  auto it = std::lower_bound(b, e, c);
  return (it != e && *it == c) ? (int)(it - A.col.begin()) : -1;
}

// K = V^T L_h V as a sparse sum over faces in ascending order
// (CutMeshLaplacian.lean:56-93).  Each triangle is laid out as the spec's
// faceLoop walks it, starting at halfedge 3f whose target is t1
// (HalfedgeBuilder.lean:43-45): polygon (t1, t2, t0).
Csr assemble_K(int nv, int nt, const int* tris, const double* pos, int kind, double delta) {
  Csr K = pattern_from_tris(nv, nt, tris);
  for (int f = 0; f < nt; ++f) {
    int g[3] = {tris[3 * f + 1], tris[3 * f + 2], tris[3 * f + 0]};
    double m[9];
    if (kind == 1)
      orc_robust_triangle_cot_laplacian(delta, pos + 3 * g[0], pos + 3 * g[1], pos + 3 * g[2], m);
    else
      orc_triangle_cot_laplacian(pos + 3 * g[0], pos + 3 * g[1], pos + 3 * g[2], m);
    for (int li = 0; li < 3; ++li)
      for (int lj = 0; lj < 3; ++lj) {
        int e = find_entry(K, g[li], g[lj]);
        K.val[e] = K.val[e] + m[li * 3 + lj];
      }
  }
  return K;
}

// GraphColoring.lean:41-56 greedyColor: vertices in index order, smallest
// colour not used by an earlier-indexed neighbour.
std::vector<int> greedy_color(const Csr& G) {
  std::vector<int> color(G.n, 0);
  std::vector<int> mark;
  for (int i = 0; i < G.n; ++i) {
    mark.assign(G.ptr[i + 1] - G.ptr[i] + 2, 0);
    for (int p = G.ptr[i]; p < G.ptr[i + 1]; ++p) {
      int j = G.col[p];
      if (j < i && color[j] < (int)mark.size()) mark[color[j]] = 1;
    }
    int c = 0;
    while (c < (int)mark.size() && mark[c]) ++c;
    color[i] = c;
  }
  return color;
}

// Symmetric permutation B = A[perm, perm] (perm: new -> old), columns sorted.
Csr permute(const Csr& A, const std::vector<int>& perm) {
  int n = A.n;
  std::vector<int> inv(n);
  for (int i = 0; i < n; ++i) inv[perm[i]] = i;
  Csr B;
  B.n = n;
  B.ptr.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) B.ptr[i + 1] = B.ptr[i] + (A.ptr[perm[i] + 1] - A.ptr[perm[i]]);
  B.col.resize(A.col.size());
  B.val.resize(A.val.size());
  std::vector<std::pair<int, double>> row;
  for (int i = 0; i < n; ++i) {
    int o = perm[i];
    row.clear();
    for (int p = A.ptr[o]; p < A.ptr[o + 1]; ++p) row.push_back({inv[A.col[p]], A.val[p]});
    std::sort(row.begin(), row.end(),
              [](const std::pair<int, double>& a, const std::pair<int, double>& b) { return a.first < b.first; });
    for (size_t k = 0; k < row.size(); ++k) {
      B.col[B.ptr[i] + k] = row[k].first;
      B.val[B.ptr[i] + k] = row[k].second;
    }
  }
  return B;
}

// Elimination order of the free unknowns: natural (0) or greedy colour (1);
// then stable-sorted by the level of the lower-triangular dependency DAG so
// every level is a contiguous row range.  Level sorting keeps the relative
// order of every adjacent pair, so the IC(0) factor is the one of the chosen
// order, relabelled.
std::vector<int> solve_order(const Csr& A, int ordering, int* nlev_out) {
  int n = A.n;
  std::vector<int> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  if (ordering == 1) {
    std::vector<int> color = greedy_color(A);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return color[a] < color[b]; });
  }
  std::vector<int> pos(n);
  for (int i = 0; i < n; ++i) pos[ord[i]] = i;
  std::vector<int> level(n, 0);
  int nlev = n ? 1 : 0;
  for (int i = 0; i < n; ++i) {
    int v = ord[i], l = 0;
    for (int p = A.ptr[v]; p < A.ptr[v + 1]; ++p) {
      int u = A.col[p];
      if (pos[u] < i) l = std::max(l, level[u] + 1);
    }
    level[v] = l;
    nlev = std::max(nlev, l + 1);
  }
  std::vector<int> out = ord;
  std::stable_sort(out.begin(), out.end(), [&](int a, int b) { return level[a] < level[b]; });
  if (nlev_out) *nlev_out = nlev;
  return out;
}

// IC(0) of a CSR matrix (IncompleteCholesky.lean:30-33, :49-69): rows of L
// hold the strictly-lower pattern of A in ascending column order followed by
// the diagonal.  L_ij = (A_ij - sum_{k<j} L_ik L_jk) / L_jj and
// L_ii = sqrt(A_ii (1 + shift) - sum_k L_ik^2), each sum subtracted term by
// term in ascending k as factor3 does (shift = 0 is the spec's factor).
// Returns -1 - row on a non-positive pivot.
int ic0(const Csr& A, Csr& L, double shift = 0.0) {
  int n = A.n;
  L.n = n;
  L.ptr.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    int c = 0;
    for (int p = A.ptr[i]; p < A.ptr[i + 1]; ++p) c += A.col[p] < i;
    L.ptr[i + 1] = L.ptr[i] + c + 1;
  }
  L.col.assign(L.ptr[n], 0);
  L.val.assign(L.ptr[n], 0.0);
  for (int i = 0; i < n; ++i) {
    int q = L.ptr[i];
    double aii = 0.0;
    for (int p = A.ptr[i]; p < A.ptr[i + 1]; ++p) {
      if (A.col[p] < i) { L.col[q] = A.col[p]; L.val[q] = A.val[p]; ++q; }
      if (A.col[p] == i) aii = A.val[p];
    }
    if (shift != 0.0) aii = aii * (1.0 + shift);
    L.col[q] = i;
    int ilo = L.ptr[i], ihi = L.ptr[i + 1] - 1;  // strictly lower entries of row i
    for (int e = ilo; e < ihi; ++e) {
      int j = L.col[e];
      double s = L.val[e];
      int a = ilo, b = L.ptr[j], bhi = L.ptr[j + 1] - 1;
      while (a < e && b < bhi) {
        if (L.col[a] == L.col[b]) { s = s - L.val[a] * L.val[b]; ++a; ++b; }
        else if (L.col[a] < L.col[b]) ++a;
        else ++b;
      }
      L.val[e] = s / L.val[L.ptr[j + 1] - 1];
    }
    double d = aii;
    for (int e = ilo; e < ihi; ++e) d = d - L.val[e] * L.val[e];
    if (!(d > 0.0)) return -1 - i;
    L.val[ihi] = std::sqrt(d);
  }
  return 0;
}

void spmv(const Csr& A, const double* x, double* y) {
  for (int i = 0; i < A.n; ++i) {
    double s = 0.0;
    for (int p = A.ptr[i]; p < A.ptr[i + 1]; ++p) s = s + A.val[p] * x[A.col[p]];
    y[i] = s;
  }
}

double dot(const double* a, const double* b, int n) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s = s + a[i] * b[i];
  return s;
}

// z = L^{-T} L^{-1} r (IncompleteCholesky.lean:83-101 forwardSub3/backwardSub3
// in CSR form); the backward sweep reads L column-wise through Lt.
struct Ic0Apply {
  const Csr* L;
  Csr Lt;  // transpose of the strictly-lower part: row j holds (i, L_ij), i > j
  std::vector<double> y;
  explicit Ic0Apply(const Csr& Lf) : L(&Lf) {
    int n = Lf.n;
    Lt.n = n;
    Lt.ptr.assign(n + 1, 0);
    for (int i = 0; i < n; ++i)
      for (int e = Lf.ptr[i]; e < Lf.ptr[i + 1] - 1; ++e) Lt.ptr[Lf.col[e] + 1]++;
    for (int i = 0; i < n; ++i) Lt.ptr[i + 1] += Lt.ptr[i];
    Lt.col.resize(Lt.ptr[n]);
    Lt.val.resize(Lt.ptr[n]);
    std::vector<int> fill(Lt.ptr.begin(), Lt.ptr.end() - 1);
    for (int i = 0; i < n; ++i)
      for (int e = Lf.ptr[i]; e < Lf.ptr[i + 1] - 1; ++e) {
        int j = Lf.col[e];
        Lt.col[fill[j]] = i;
        Lt.val[fill[j]] = Lf.val[e];
        fill[j]++;
      }
    y.resize(n);
  }
  void apply(const double* r, double* z) {
    const Csr& Lf = *L;
    int n = Lf.n;
    for (int i = 0; i < n; ++i) {
      double s = r[i];
      for (int e = Lf.ptr[i]; e < Lf.ptr[i + 1] - 1; ++e) s = s - Lf.val[e] * y[Lf.col[e]];
      y[i] = s / Lf.val[Lf.ptr[i + 1] - 1];
    }
    for (int ii = 0; ii < n; ++ii) {
      int i = n - 1 - ii;
      double s = y[i];
      for (int e = Lt.ptr[i]; e < Lt.ptr[i + 1]; ++e) s = s - Lt.val[e] * z[Lt.col[e]];
      z[i] = s / Lf.val[Lf.ptr[i + 1] - 1];
    }
  }
};

// PCG of SparseLinAlg.lean:137-163 (cgWithGuess) with a pluggable
// preconditioner and the relative stopping test ||r|| < tol ||b||.
// Returns the iteration count.
template <class Prec>
int pcg(const Csr& A, const double* b, double* x, int max_iter, double tol, Prec&& prec) {
  int n = A.n;
  std::vector<double> r(n), z(n), p(n), Ap(n);
  spmv(A, x, Ap.data());
  for (int i = 0; i < n; ++i) r[i] = b[i] - Ap[i];
  prec(r.data(), z.data());
  p = z;
  double rz = dot(r.data(), z.data(), n);
  double tolsq = tol * tol * dot(b, b, n);
  int it = 0;
  for (; it < max_iter; ++it) {
    spmv(A, p.data(), Ap.data());
    double pAp = dot(p.data(), Ap.data(), n);
    if (pAp == 0.0) break;
    double alpha = rz / pAp;
    for (int i = 0; i < n; ++i) x[i] = x[i] + alpha * p[i];
    for (int i = 0; i < n; ++i) r[i] = r[i] + (-alpha) * Ap[i];
    double rr = dot(r.data(), r.data(), n);
    if (rr < tolsq) { ++it; break; }
    prec(r.data(), z.data());
    double rzn = dot(r.data(), z.data(), n);
    double beta = rz == 0.0 ? 0.0 : rzn / rz;
    for (int i = 0; i < n; ++i) p[i] = 1.0 * z[i] + beta * p[i];
    rz = rzn;
  }
  return it;
}

// The assembled, reduced, ordered and factored system of one mesh.
struct System {
  int nv = 0, nt = 0, n = 0, nh = 0, nlev = 0;
  std::vector<double> pos;
  Csr K;                       // all vertices, original numbering
  std::vector<int> free_of;    // solve row -> vertex
  std::vector<int> row_of;     // vertex -> solve row or -1
  std::vector<int> hidx;       // vertex -> handle index or -1
  Csr A;                       // K[free, free] in solve order
  Csr L;                       // IC(0) factor of A (precond 1)
  int precond = 1;
  int status = 0;
  double shift = 0.0;          // diagonal shift the IC(0) factor needed
};

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// CSR assembly of K over all vertices (two-call: pass rowptr=NULL for nnz).
long long orc_assemble_csr(int nv, int nt, const int* tris, const double* pos, int kind,
                           double delta, int* rowptr, int* colidx, double* vals) {
  Csr K = assemble_K(nv, nt, tris, pos, kind, delta);
  if (rowptr) {
    std::memcpy(rowptr, K.ptr.data(), sizeof(int) * (nv + 1));
    std::memcpy(colidx, K.col.data(), sizeof(int) * K.col.size());
    std::memcpy(vals, K.val.data(), sizeof(double) * K.val.size());
  }
  return (long long)K.col.size();
}

// GraphColoring.lean:41-56 on a CSR adjacency (self loops ignored).
void orc_greedy_color(int n, const int* adj_ptr, const int* adj, int* color_out) {
  Csr G;
  G.n = n;
  G.ptr.assign(adj_ptr, adj_ptr + n + 1);
  G.col.assign(adj, adj + adj_ptr[n]);
  std::vector<int> c = greedy_color(G);
  std::memcpy(color_out, c.data(), sizeof(int) * n);
}

// IC(0) of a square CSR matrix with sorted columns (no reordering).
// Two-call: L_ptr filled always (n+1), L_col/L_val when non-NULL.
int orc_ic0_factor(int n, const int* ptr, const int* col, const double* val, int* L_ptr,
                   int* L_col, double* L_val) {
  Csr A;
  A.n = n;
  A.ptr.assign(ptr, ptr + n + 1);
  A.col.assign(col, col + ptr[n]);
  A.val.assign(val, val + ptr[n]);
  Csr L;
  int st = ic0(A, L);
  std::memcpy(L_ptr, L.ptr.data(), sizeof(int) * (n + 1));
  if (L_col) {
    std::memcpy(L_col, L.col.data(), sizeof(int) * L.col.size());
    std::memcpy(L_val, L.val.data(), sizeof(double) * L.val.size());
  }
  return st;
}

// SparseLinAlg.lean:104-130 cg / :137-163 cgWithGuess exactly as specified:
// Jacobi preconditioner (zero diagonal -> 0, :89-97), absolute test rr < tol^2.
// x0 may be NULL (zero guess).  Returns iterations performed.
int orc_cg_ref(int n, const int* ptr, const int* col, const double* val, const double* b,
               const double* x0, int max_iter, double tol, double* x) {
  Csr A;
  A.n = n;
  A.ptr.assign(ptr, ptr + n + 1);
  A.col.assign(col, col + ptr[n]);
  A.val.assign(val, val + ptr[n]);
  std::vector<double> d(n, 0.0);  // diagonal (:78-87)
  for (int i = 0; i < n; ++i)
    for (int p = A.ptr[i]; p < A.ptr[i + 1]; ++p)
      if (A.col[p] == i) { d[i] = A.val[p]; break; }
  auto jac = [&](const double* r, double* z) {
    for (int i = 0; i < n; ++i) z[i] = d[i] == 0.0 ? 0.0 : r[i] / d[i];
  };
  for (int i = 0; i < n; ++i) x[i] = x0 ? x0[i] : 0.0;
  std::vector<double> r(n), z(n), p(n), Ap(n);
  if (x0) {
    spmv(A, x, Ap.data());
    for (int i = 0; i < n; ++i) r[i] = 1.0 * b[i] + (-1.0) * Ap[i];
  } else {
    for (int i = 0; i < n; ++i) r[i] = b[i];
  }
  jac(r.data(), z.data());
  p = z;
  double rz = dot(r.data(), z.data(), n), tolsq = tol * tol;
  int it = 0;
  for (; it < max_iter; ++it) {
    spmv(A, p.data(), Ap.data());
    double pAp = dot(p.data(), Ap.data(), n);
    if (pAp == 0.0) break;
    double alpha = rz / pAp;
    for (int i = 0; i < n; ++i) x[i] = x[i] + alpha * p[i];
    for (int i = 0; i < n; ++i) r[i] = r[i] + (-alpha) * Ap[i];
    double rr = dot(r.data(), r.data(), n);
    if (rr < tolsq) { ++it; break; }
    jac(r.data(), z.data());
    double rzn = dot(r.data(), z.data(), n);
    double beta = rz == 0.0 ? 0.0 : rzn / rz;
    for (int i = 0; i < n; ++i) p[i] = 1.0 * z[i] + beta * p[i];
    rz = rzn;
  }
  return it;
}

// ---------------------------------------------------------------------------
// HierarchicalSparsifyCompensate.lean:97-125 eliminateVertex on the spec's
// edge-list graph (edges (u, v, w), u < v).  Output capacity: ne + deg^2/2.
// Returns the output edge count.
int orc_hsc_eliminate(int ne, const int* eu, const int* ev, const double* ew, int v,
                      int* ou, int* ov, double* ow) {
  std::vector<std::pair<int, double>> nbrs;  // neighborsOf (:71-79)
  double dv = 0.0;                            // degreeWeight (:62-68)
  for (int e = 0; e < ne; ++e) {
    if (eu[e] == v || ev[e] == v) dv = dv + ew[e];
    if (eu[e] == v) nbrs.push_back({ev[e], ew[e]});
    else if (ev[e] == v) nbrs.push_back({eu[e], ew[e]});
  }
  int m = 0;
  for (int e = 0; e < ne; ++e)
    if (eu[e] != v && ev[e] != v) { ou[m] = eu[e]; ov[m] = ev[e]; ow[m] = ew[e]; ++m; }
  if (dv > 0.0) {
    for (size_t i = 0; i < nbrs.size(); ++i)
      for (size_t j = i + 1; j < nbrs.size(); ++j) {
        int ni = nbrs[i].first, nj = nbrs[j].first;
        int lo = std::min(ni, nj), hi = std::max(ni, nj);
        double comp = nbrs[i].second * nbrs[j].second / dv;
        bool found = false;
        for (int k = 0; k < m; ++k)
          if (ou[k] == lo && ov[k] == hi) { ow[k] = ow[k] + comp; found = true; break; }
        if (!found) { ou[m] = lo; ov[m] = hi; ow[m] = comp; ++m; }
      }
  }
  return m;
}

// ---------------------------------------------------------------------------
// Mesh-level system: assemble K, reduce to the free unknowns, order, factor.
// ordering: 0 natural, 1 greedy colour.  precond: 0 Jacobi, 1 IC(0).
// Status codes (same meaning as the product's): 0 ok, 2 singular component,
// 3 non-positive pivot, 7 bad input.
void* orc_system_create(int nv, int nt, const int* tris, const double* pos, int nh,
                        const int* handles, int lap_kind, double delta, int ordering,
                        int precond) {
  System* S = new System;
  S->nv = nv; S->nt = nt; S->nh = nh; S->precond = precond;
  S->pos.assign(pos, pos + 3 * (size_t)nv);
  S->K = assemble_K(nv, nt, tris, pos, lap_kind, delta);
  S->hidx.assign(nv, -1);
  for (int h = 0; h < nh; ++h) {
    if (handles[h] < 0 || handles[h] >= nv || S->hidx[handles[h]] >= 0) { S->status = 7; return S; }
    S->hidx[handles[h]] = h;
  }
  // every connected component needs a handle (union-find over triangles)
  std::vector<int> par(nv);
  std::iota(par.begin(), par.end(), 0);
  auto find = [&](int a) { while (par[a] != a) { par[a] = par[par[a]]; a = par[a]; } return a; };
  for (int f = 0; f < nt; ++f) {
    int a = find(tris[3 * f]), b = find(tris[3 * f + 1]), c = find(tris[3 * f + 2]);
    par[b] = a; par[find(c)] = a;
  }
  std::vector<char> has(nv, 0);
  for (int h = 0; h < nh; ++h) has[find(handles[h])] = 1;
  for (int v = 0; v < nv; ++v)
    if (!has[find(v)]) { S->status = 2; return S; }
  // free unknowns in vertex order, then K[free, free]
  std::vector<int> fidx(nv, -1), fverts;
  for (int v = 0; v < nv; ++v)
    if (S->hidx[v] < 0) { fidx[v] = (int)fverts.size(); fverts.push_back(v); }
  int n = (int)fverts.size();
  Csr Af;
  Af.n = n;
  Af.ptr.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    int v = fverts[i];
    for (int p = S->K.ptr[v]; p < S->K.ptr[v + 1]; ++p)
      if (fidx[S->K.col[p]] >= 0) { Af.col.push_back(fidx[S->K.col[p]]); Af.val.push_back(S->K.val[p]); }
    Af.ptr[i + 1] = (int)Af.col.size();
  }
  std::vector<int> ord = solve_order(Af, ordering, &S->nlev);
  S->A = permute(Af, ord);
  S->n = n;
  S->free_of.resize(n);
  S->row_of.assign(nv, -1);
  for (int i = 0; i < n; ++i) { S->free_of[i] = fverts[ord[i]]; S->row_of[S->free_of[i]] = i; }
  // A non-positive pivot (the jittered cot Laplacian is not an M-matrix) is
  // retried on A + shift diag(A) (Manteuffel), shift in {1e-3, 1e-2, 1e-1};
  // the shifted factor preconditions the unshifted A.
  if (precond == 1) {
    const double shifts[] = {0.0, 1e-3, 1e-2, 1e-1};
    S->status = 3;
    for (double sh : shifts) {
      if (ic0(S->A, S->L, sh) == 0) { S->status = 0; S->shift = sh; break; }
    }
  }
  return S;
}

void orc_system_free(void* s) { delete (System*)s; }

// sizes: {status, n, nnz_A, nnz_L, nlev, nnz_K, shift * 1e6}
void orc_system_sizes(void* s, long long* out) {
  System* S = (System*)s;
  out[0] = S->status; out[1] = S->n; out[2] = (long long)S->A.col.size();
  out[3] = (long long)S->L.col.size(); out[4] = S->nlev; out[5] = (long long)S->K.col.size();
  out[6] = (long long)(S->shift * 1e6 + 0.5);
}

// Solve order (row -> vertex), A in that order, and the IC(0) factor.
void orc_system_export(void* s, int* free_of, int* A_ptr, int* A_col, double* A_val,
                       int* L_ptr, int* L_col, double* L_val) {
  System* S = (System*)s;
  std::memcpy(free_of, S->free_of.data(), sizeof(int) * S->n);
  std::memcpy(A_ptr, S->A.ptr.data(), sizeof(int) * (S->n + 1));
  std::memcpy(A_col, S->A.col.data(), sizeof(int) * S->A.col.size());
  std::memcpy(A_val, S->A.val.data(), sizeof(double) * S->A.val.size());
  if (L_ptr && !S->L.ptr.empty()) {
    std::memcpy(L_ptr, S->L.ptr.data(), sizeof(int) * (S->n + 1));
    std::memcpy(L_col, S->L.col.data(), sizeof(int) * S->L.col.size());
    std::memcpy(L_val, S->L.val.data(), sizeof(double) * S->L.val.size());
  }
}

// Right-hand side of the reduced system (HarmonicSolve.lean:51-66 for mode 0,
// DeformSolve.lean:123-135 Stage 2 with F_f = I for mode 1):
//   b_f = -(K diff)_f,  diff_v = X_c(v) - [mode 1] rest_v  (handle v)
//                               = -[mode 1] rest_v          (free v)
// For mode 1, RHS column c uses coordinate c % 3.
static void rhs(const System* S, int k, const double* targets, int mode, double* b) {
  for (int i = 0; i < S->n; ++i) {
    int v = S->free_of[i];
    for (int c = 0; c < k; ++c) {
      double s = 0.0;
      for (int p = S->K.ptr[v]; p < S->K.ptr[v + 1]; ++p) {
        int u = S->K.col[p];
        double rest = mode == 1 ? S->pos[3 * u + c % 3] : 0.0;
        double d = S->hidx[u] >= 0 ? targets[(size_t)S->hidx[u] * k + c] - rest : -rest;
        s = s + S->K.val[p] * d;
      }
      b[(size_t)i * k + c] = -s;
    }
  }
}

// Solve k right-hand sides (handle targets nh x k) to relative residual tol.
// Columns run on up to nthreads threads.  x0 (nv x k) may be NULL.  Outputs
// x_out (nv x k, handles overlaid), per-column iterations and the true final
// relative residual ||b - A x|| / ||b||.
int orc_system_solve(void* s, int k, const double* targets, int mode, double tol,
                     int max_iter, int nthreads, const double* x0, double* x_out,
                     int* iters_out, double* relres_out) {
  System* S = (System*)s;
  if (S->status) return S->status;
  int n = S->n;
  std::vector<double> b((size_t)n * k);
  rhs(S, k, targets, mode, b.data());
  std::atomic<int> next(0);
  auto worker = [&]() {
    std::vector<double> bc(n), xc(n), tmp(n);
    Ic0Apply* ica = S->precond == 1 ? new Ic0Apply(S->L) : nullptr;
    std::vector<double> dinv(n);
    for (int i = 0; i < n; ++i)
      for (int p = S->A.ptr[i]; p < S->A.ptr[i + 1]; ++p)
        if (S->A.col[p] == i) dinv[i] = S->A.val[p] == 0.0 ? 0.0 : 1.0 / S->A.val[p];
    for (int c; (c = next.fetch_add(1)) < k;) {
      for (int i = 0; i < n; ++i) {
        bc[i] = b[(size_t)i * k + c];
        xc[i] = x0 ? x0[(size_t)S->free_of[i] * k + c] : 0.0;
      }
      int it;
      if (ica)
        it = pcg(S->A, bc.data(), xc.data(), max_iter, tol,
                 [&](const double* r, double* z) { ica->apply(r, z); });
      else
        it = pcg(S->A, bc.data(), xc.data(), max_iter, tol, [&](const double* r, double* z) {
          for (int i = 0; i < n; ++i) z[i] = r[i] * dinv[i];
        });
      spmv(S->A, xc.data(), tmp.data());
      double rr = 0.0, bb = dot(bc.data(), bc.data(), n);
      for (int i = 0; i < n; ++i) { double d = bc[i] - tmp[i]; rr = rr + d * d; }
      if (iters_out) iters_out[c] = it;
      if (relres_out) relres_out[c] = bb > 0.0 ? std::sqrt(rr / bb) : std::sqrt(rr);
      for (int i = 0; i < n; ++i) x_out[(size_t)S->free_of[i] * k + c] = xc[i];
      for (int v = 0; v < S->nv; ++v)
        if (S->hidx[v] >= 0) x_out[(size_t)v * k + c] = targets[(size_t)S->hidx[v] * k + c];
    }
    delete ica;
  };
  int nt = std::max(1, std::min(nthreads, k));
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(worker);
  worker();
  for (auto& t : th) t.join();
  return 0;
}

// Right-hand side only (free rows in solve order, n x k).
void orc_system_rhs(void* s, int k, const double* targets, int mode, double* b) {
  rhs((System*)s, k, targets, mode, b);
}

}  // extern "C"
