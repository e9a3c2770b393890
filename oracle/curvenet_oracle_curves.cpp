// curvenet_oracle_curves.cpp -- FP64 restatement of the curve side of the
// reference (Bezier evaluation, isolated-segment deformation gradient) and the
// CPU FP64 adjoint of the handle-constrained solve.
//
// TEST INFRASTRUCTURE ONLY (the checker for the product's deform/adjoint
// entry points); the product never links it.  Built with -ffp-contract=off.
//
// The curve -> handle-target map has no counterpart in the reference beyond
// the Bezier sample and the isolated-segment gradient; its definition here is
// the one the product documents:
//   handle h bound to (curve c_h, parameter tau_h) with per-curve weight w_c:
//   X_c(h) = rest(h) + w_c (B_posed,c(tau_h) - B_rest,c(tau_h)),
//   handles with c_h < 0 stay at rest.
// A curve is a composite cubic Bezier of S segments (3S+1 control points);
// tau in [0, S] selects segment s = min(floor(tau), S-1) and t = tau - s.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

extern "C" int orc_system_solve(void*, int, const double*, int, double, int, int,
                                const double*, double*, int*, double*);
extern "C" void orc_system_sizes(void*, long long*);

namespace {

// EndToEndExample.lean:52-60 bezier3
void bezier3(const double* P0, const double* P1, const double* P2, const double* P3, double t,
             double* out) {
  double u = 1.0 - t;
  double c0 = u * u * u;
  double c1 = 3.0 * u * u * t;
  double c2 = 3.0 * u * t * t;
  double c3 = t * t * t;
  for (int d = 0; d < 3; ++d) out[d] = c0 * P0[d] + c1 * P1[d] + c2 * P2[d] + c3 * P3[d];
}

void bern(double t, double* c) {
  double u = 1.0 - t;
  c[0] = u * u * u; c[1] = 3.0 * u * u * t; c[2] = 3.0 * u * t * t; c[3] = t * t * t;
}

void seg_of(double tau, int S, int* s, double* t) {
  int k = (int)std::floor(tau);
  if (k > S - 1) k = S - 1;
  if (k < 0) k = 0;
  *s = k;
  *t = tau - (double)k;
}

void eval_curve(const double* P, int S, double tau, double* out) {
  int s; double t;
  seg_of(tau, S, &s, &t);
  bezier3(P + 9 * s, P + 9 * s + 3, P + 9 * s + 6, P + 9 * s + 9, t, out);
}

}  // namespace

extern "C" {

void orc_bezier3(const double* P4, double t, double* out) {
  bezier3(P4, P4 + 3, P4 + 6, P4 + 9, t, out);
}

// ScaledFrames.lean tangentLength / smallestRotation / isolatedSegmentGradient
void orc_isolated_segment_gradient(const double* rp, const double* rq, const double* pp,
                                   const double* pq, double* F) {
  auto tl = [](const double* p, const double* q, double* t) {
    double d[3] = {q[0] - p[0], q[1] - p[1], q[2] - p[2]};
    double l = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double inv = l == 0.0 ? 0.0 : 1.0 / l;
    t[0] = d[0] * inv; t[1] = d[1] * inv; t[2] = d[2] * inv;
    return l;
  };
  double tr[3], tp[3];
  double lr = tl(rp, rq, tr), lp = tl(pp, pq, tp);
  double r = lr == 0.0 ? 0.0 : lp / lr;
  double cx = tr[1] * tp[2] - tr[2] * tp[1];
  double cy = tr[2] * tp[0] - tr[0] * tp[2];
  double cz = tr[0] * tp[1] - tr[1] * tp[0];
  double cosT = tr[0] * tp[0] + tr[1] * tp[1] + tr[2] * tp[2];
  double K[9] = {0.0, -cz, cy, cz, 0.0, -cx, -cy, cx, 0.0};
  double K2[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      K2[i * 3 + j] = K[i * 3 + 0] * K[0 * 3 + j] + K[i * 3 + 1] * K[1 * 3 + j] + K[i * 3 + 2] * K[2 * 3 + j];
  double denom = 1.0 + cosT;
  double invd = denom == 0.0 ? 0.0 : 1.0 / denom;
  double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int k = 0; k < 9; ++k) F[k] = r * ((I[k] + K[k]) + invd * K2[k]);
}

// Handle targets from curves.  rest_cp / posed_cp: ncurves x (3S+1) x 3,
// weights: ncurves, curve_of/tau: per handle, rest: nv x 3, handles: nh.
// out: nh x 3.
void orc_curve_targets(int ncurves, int S, const double* rest_cp, const double* posed_cp,
                       const double* weights, int nh, const int* handles, const int* curve_of,
                       const double* tau, const double* rest, double* out) {
  int np = 3 * S + 1;
  for (int h = 0; h < nh; ++h) {
    const double* x = rest + 3 * (size_t)handles[h];
    int c = curve_of[h];
    if (c < 0 || c >= ncurves) { for (int d = 0; d < 3; ++d) out[3 * h + d] = x[d]; continue; }
    double bp[3], br[3];
    eval_curve(posed_cp + (size_t)c * np * 3, S, tau[h], bp);
    eval_curve(rest_cp + (size_t)c * np * 3, S, tau[h], br);
    for (int d = 0; d < 3; ++d) out[3 * h + d] = x[d] + weights[c] * (bp[d] - br[d]);
  }
}

// Forward deform solve from curve parameters (mode 1, k = 3) followed by the
// FP64 adjoint of L = 1/2 ||x - x_target||^2 (all vertices):
//   lambda = A^{-1} (x_f - xt_f)
//   G_h    = -(K_{h,f} lambda) + (X_c(h) - xt_h)
//   dL/dP[c][j] = sum_{h on c} w_c bern_j(tau_h) G_h,
//   dL/dw_c     = sum_{h on c} (B_posed - B_rest)(tau_h) . G_h.
// Needs the System of a mesh (orc_system_create) plus its K/A (exported by
// the caller as CSR to keep this file independent of System's layout).
// K: nv-row CSR of all vertices; free_of: solve row -> vertex (n rows).
// Returns the loss; fills x (nv x 3), dP (like posed_cp), dw (ncurves).
double orc_deform_adjoint(void* sys, int nv, const int* K_ptr, const int* K_col,
                          const double* K_val, int n, const int* free_of, int ncurves, int S,
                          const double* rest_cp, const double* posed_cp, const double* weights,
                          int nh, const int* handles, const int* curve_of, const double* tau,
                          const double* rest, const double* x_target, double tol, int max_iter,
                          double* x, double* dP, double* dw) {
  std::vector<double> Xc(3 * (size_t)nh);
  orc_curve_targets(ncurves, S, rest_cp, posed_cp, weights, nh, handles, curve_of, tau, rest,
                    Xc.data());
  orc_system_solve(sys, 3, Xc.data(), 1, tol, max_iter, 3, nullptr, x, nullptr, nullptr);
  double loss = 0.0;
  for (size_t i = 0; i < 3 * (size_t)nv; ++i) { double d = x[i] - x_target[i]; loss = loss + 0.5 * d * d; }
  // Adjoint solve A lambda = g_f with a plain Jacobi-PCG on A = K[free, free]
  // (A is symmetric, so the transpose solve is the same system).
  std::vector<int> row_of(nv, -1);
  for (int i = 0; i < n; ++i) row_of[free_of[i]] = i;
  // A in solve order from K
  std::vector<int> Ap(n + 1, 0), Ac;
  std::vector<double> Av;
  for (int i = 0; i < n; ++i) {
    int v = free_of[i];
    std::vector<std::pair<int, double>> row;
    for (int p = K_ptr[v]; p < K_ptr[v + 1]; ++p)
      if (row_of[K_col[p]] >= 0) row.push_back({row_of[K_col[p]], K_val[p]});
    std::sort(row.begin(), row.end(),
              [](const std::pair<int, double>& a, const std::pair<int, double>& b) { return a.first < b.first; });
    for (auto& e : row) { Ac.push_back(e.first); Av.push_back(e.second); }
    Ap[i + 1] = (int)Ac.size();
  }
  std::vector<double> lam((size_t)n * 3, 0.0);
  for (int c = 0; c < 3; ++c) {
    std::vector<double> g(n), l(n, 0.0), r(n), z(n), p(n), q(n), dinv(n);
    for (int i = 0; i < n; ++i) g[i] = x[3 * (size_t)free_of[i] + c] - x_target[3 * (size_t)free_of[i] + c];
    for (int i = 0; i < n; ++i)
      for (int e = Ap[i]; e < Ap[i + 1]; ++e)
        if (Ac[e] == i) dinv[i] = 1.0 / Av[e];
    double bb = 0.0;
    for (int i = 0; i < n; ++i) bb = bb + g[i] * g[i];
    r = g;
    for (int i = 0; i < n; ++i) z[i] = r[i] * dinv[i];
    p = z;
    double rz = 0.0;
    for (int i = 0; i < n; ++i) rz = rz + r[i] * z[i];
    for (int it = 0; it < max_iter && bb > 0.0; ++it) {
      for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int e = Ap[i]; e < Ap[i + 1]; ++e) s = s + Av[e] * p[Ac[e]];
        q[i] = s;
      }
      double pq = 0.0;
      for (int i = 0; i < n; ++i) pq = pq + p[i] * q[i];
      if (pq == 0.0) break;
      double a = rz / pq, rr = 0.0;
      for (int i = 0; i < n; ++i) { l[i] = l[i] + a * p[i]; r[i] = r[i] - a * q[i]; rr = rr + r[i] * r[i]; }
      if (rr < tol * tol * bb) break;
      double rzn = 0.0;
      for (int i = 0; i < n; ++i) { z[i] = r[i] * dinv[i]; rzn = rzn + r[i] * z[i]; }
      double beta = rzn / rz;
      for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
      rz = rzn;
    }
    for (int i = 0; i < n; ++i) lam[(size_t)i * 3 + c] = l[i];
  }
  int np = 3 * S + 1;
  std::memset(dP, 0, sizeof(double) * (size_t)ncurves * np * 3);
  std::memset(dw, 0, sizeof(double) * ncurves);
  for (int h = 0; h < nh; ++h) {
    int v = handles[h];
    double G[3];
    for (int d = 0; d < 3; ++d) {
      double s = 0.0;
      for (int p = K_ptr[v]; p < K_ptr[v + 1]; ++p) {
        int r = row_of[K_col[p]];
        if (r >= 0) s = s + K_val[p] * lam[(size_t)r * 3 + d];
      }
      G[d] = -s + (Xc[3 * h + d] - x_target[3 * (size_t)v + d]);
    }
    int c = curve_of[h];
    if (c < 0 || c >= ncurves) continue;
    int s; double t, b[4];
    seg_of(tau[h], S, &s, &t);
    bern(t, b);
    for (int j = 0; j < 4; ++j)
      for (int d = 0; d < 3; ++d) dP[((size_t)c * np + 3 * s + j) * 3 + d] += weights[c] * b[j] * G[d];
    double bp[3], br[3];
    eval_curve(posed_cp + (size_t)c * np * 3, S, tau[h], bp);
    eval_curve(rest_cp + (size_t)c * np * 3, S, tau[h], br);
    for (int d = 0; d < 3; ++d) dw[c] += (bp[d] - br[d]) * G[d];
  }
  return loss;
}

}  // extern "C"
