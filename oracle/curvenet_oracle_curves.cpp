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

// ---------------------------------------------------------------------------
// The curvenet (DeGoes22 section 3): the primitives of ScaledFrames.lean,
// IntersectionFrames.lean and CurveInterp.lean, and their assembly into
// per-handle F_c / X_c as the product documents it (curvenet_b200.h,
// cn_curvenet_desc).

// ScaledFrames.lean:40-45 tangentLength
double orc_tangent_length(const double* p, const double* q, double* t) {
  double d[3] = {q[0] - p[0], q[1] - p[1], q[2] - p[2]};
  double l = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  double inv = l == 0.0 ? 0.0 : 1.0 / l;
  t[0] = d[0] * inv; t[1] = d[1] * inv; t[2] = d[2] * inv;
  return l;
}

// ScaledFrames.lean:71-84 smallestRotation: R = (I + K) + K^2 / (1 + cos)
void orc_smallest_rotation(const double* f, const double* to, double* R) {
  double cx = f[1] * to[2] - f[2] * to[1];
  double cy = f[2] * to[0] - f[0] * to[2];
  double cz = f[0] * to[1] - f[1] * to[0];
  double cosT = f[0] * to[0] + f[1] * to[1] + f[2] * to[2];
  double K[9] = {0.0, -cz, cy, cz, 0.0, -cx, -cy, cx, 0.0};
  double denom = 1.0 + cosT;
  double invd = denom == 0.0 ? 0.0 : 1.0 / denom;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double k2 = K[i * 3 + 0] * K[0 * 3 + j] + K[i * 3 + 1] * K[1 * 3 + j] + K[i * 3 + 2] * K[2 * 3 + j];
      double id = i == j ? 1.0 : 0.0;
      R[i * 3 + j] = (id + K[i * 3 + j]) + invd * k2;
    }
}

// ScaledFrames.lean:59-65 mat3Mul
void orc_mat3_mul(const double* a, const double* b, double* o) {
  double t[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      t[i * 3 + j] = a[i * 3 + 0] * b[0 * 3 + j] + a[i * 3 + 1] * b[1 * 3 + j] + a[i * 3 + 2] * b[2 * 3 + j];
  std::memcpy(o, t, sizeof t);
}

// ScaledFrames.lean:120-131 mat3Det
double orc_mat3_det(const double* m) {
  double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
  return a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
}

// ScaledFrames.lean:135-160 mat3Inv (adjugate / det; det = 0 gives 0)
void orc_mat3_inv(const double* m, double* o) {
  double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
  double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
  double inv = det == 0.0 ? 0.0 : 1.0 / det;
  double t[9] = {inv * (e * i - f * h), inv * (c * h - b * i), inv * (b * f - c * e),
                 inv * (f * g - d * i), inv * (a * i - c * g), inv * (c * d - a * f),
                 inv * (d * h - e * g), inv * (b * g - a * h), inv * (a * e - b * d)};
  std::memcpy(o, t, sizeof t);
}

// ScaledFrames.lean:164-166 deformationGradient = posed * rest^-1
void orc_deformation_gradient(const double* rest, const double* posed, double* F) {
  double inv[9];
  orc_mat3_inv(rest, inv);
  orc_mat3_mul(posed, inv, F);
}

// IntersectionFrames.lean:65-110 cornerVectors / cornerNormals (with the
// T-junction fallback, eps 1e-12); t: n x 3 unit tangents in CCW order.
void orc_corner_normals(int n, const double* t, double* cv, double* m) {
  for (int i = 0; i < n; ++i) {
    const double* a = t + 3 * i;
    const double* b = t + 3 * ((i + 1) % n);
    cv[3 * i + 0] = a[1] * b[2] - a[2] * b[1];
    cv[3 * i + 1] = a[2] * b[0] - a[0] * b[2];
    cv[3 * i + 2] = a[0] * b[1] - a[1] * b[0];
  }
  const double eps = 1.0e-12;
  for (int i = 0; i < n; ++i) {
    const double* c = cv + 3 * i;
    double nrm = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    if (nrm > eps) {
      double s = 1.0 / nrm;
      m[3 * i + 0] = s * c[0]; m[3 * i + 1] = s * c[1]; m[3 * i + 2] = s * c[2];
    } else {
      const double* cP = cv + 3 * ((i + 1) % n);
      const double* cM = cv + 3 * ((i + n - 1) % n);
      double sum[3] = {cP[0] + cM[0], cP[1] + cM[1], cP[2] + cM[2]};
      double sn = std::sqrt(sum[0] * sum[0] + sum[1] * sum[1] + sum[2] * sum[2]);
      if (sn > eps) {
        double s = 1.0 / sn;
        m[3 * i + 0] = s * sum[0]; m[3 * i + 1] = s * sum[1]; m[3 * i + 2] = s * sum[2];
      } else {
        m[3 * i + 0] = 0.0; m[3 * i + 1] = 0.0; m[3 * i + 2] = 0.0;
      }
    }
  }
}

// IntersectionFrames.lean:128-143 perSideWidths
void orc_per_side_widths(int n, const double* t, const double* l, double* wp, double* wm) {
  std::vector<double> cv(3 * (size_t)n), m(3 * (size_t)n);
  orc_corner_normals(n, t, cv.data(), m.data());
  for (int i = 0; i < n; ++i) {
    double li = l[i], liP = l[(i + 1) % n], liM = l[(i + n - 1) % n];
    const double* c = &cv[3 * i];
    const double* cm = &cv[3 * ((i + n - 1) % n)];
    double cMag = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    double cMagM = std::sqrt(cm[0] * cm[0] + cm[1] * cm[1] + cm[2] * cm[2]);
    wp[i] = li + cMag * (liP - li);
    wm[i] = li + cMagM * (liM - li);
  }
}

// IntersectionFrames.lean:160-170 scaledFrame
void orc_scaled_frame(const double* t, const double* n, double l, double w, double* M) {
  double bx = n[1] * t[2] - n[2] * t[1];
  double by = n[2] * t[0] - n[0] * t[2];
  double bz = n[0] * t[1] - n[1] * t[0];
  double h = std::sqrt(l * w);
  M[0] = t[0] * l; M[1] = bx * w; M[2] = n[0] * h;
  M[3] = t[1] * l; M[4] = by * w; M[5] = n[1] * h;
  M[6] = t[2] * l; M[7] = bz * w; M[8] = n[2] * h;
}

// CurveInterp.lean:45-60 interpAlongCurve; a side record is (n[3], w) and a
// segment record (plus side, minus side) = 8 doubles.  out: n x 8.
void orc_interp_along_curve(const double* first, const double* last, int n, double* out) {
  if (n <= 0) return;
  if (n == 1) { for (int k = 0; k < 8; ++k) out[k] = first[k]; return; }
  double denom = (double)(n - 1);
  for (int i = 0; i < n; ++i) {
    double t = (double)i / denom;
    for (int k = 0; k < 8; ++k) out[8 * i + k] = (1.0 - t) * first[k] + t * last[k];
  }
}

// The assembly into F_c / X_c per pose (see cn_curvenet_desc).  Inputs as the
// product takes them; rest: vertex positions (n_verts x 3), handles: nh ids.
// Fc: n_poses x nh x 9, Xc: n_poses x nh x 3.  Returns 0, or -1 on a
// malformed curvenet.
int orc_curvenet_constraints(int C, int S, int M, const double* rest_cp, const double* tau, const int* closed,
                             int n_nodes, const int* node_ptr, const int* node_ends, int nh,
                             const int* h_curve, const int* h_sample, const int* h_side, const int* handles,
                             const double* rest, int n_poses, const double* posed_cp, double* Fc, double* Xc) {
  const int np = 3 * S + 1;
  std::vector<int> seg_off(C + 1, 0), kind(C, 0);
  for (int c = 0; c < C; ++c) seg_off[c + 1] = seg_off[c] + ((closed && closed[c]) ? M : M - 1);
  for (int j = 0; j < n_nodes; ++j)
    for (int q = node_ptr[j]; q < node_ptr[j + 1]; ++q) kind[node_ends[q] >> 1] |= (node_ends[q] & 1) ? 2 : 1;
  for (int pose = 0; pose < n_poses; ++pose) {
    const double* PP = posed_cp + (size_t)pose * C * np * 3;
    // segment records: [cfg][t(3), l]
    std::vector<double> seg(8 * (size_t)seg_off[C]);
    for (int c = 0; c < C; ++c)
      for (int i = 0; i < seg_off[c + 1] - seg_off[c]; ++i) {
        int j = i + 1 < M ? i + 1 : 0;
        double* o = &seg[8 * (size_t)(seg_off[c] + i)];
        for (int cfg = 0; cfg < 2; ++cfg) {
          const double* P = (cfg == 0 ? rest_cp : PP) + (size_t)c * np * 3;
          double a[3], b[3];
          eval_curve(P, S, tau[(size_t)c * M + i], a);
          eval_curve(P, S, tau[(size_t)c * M + j], b);
          o[4 * cfg + 3] = orc_tangent_length(a, b, o + 4 * cfg);
        }
      }
    // curve-end side records: [end][cfg][plus n, plus w, minus n, minus w]
    std::vector<double> ends(32 * (size_t)C, 0.0);
    for (int jn = 0; jn < n_nodes; ++jn) {
      int b = node_ptr[jn], n = node_ptr[jn + 1] - b;
      if (n < 2) return -1;
      for (int cfg = 0; cfg < 2; ++cfg) {
        std::vector<double> t(3 * (size_t)n), l(n), cv(3 * (size_t)n), m(3 * (size_t)n), wp(n), wm(n);
        for (int q = 0; q < n; ++q) {
          int e = node_ends[b + q], c = e >> 1;
          int sg = (e & 1) ? seg_off[c + 1] - 1 : seg_off[c];
          const double* s = &seg[8 * (size_t)sg + 4 * cfg];
          for (int d = 0; d < 3; ++d) t[3 * q + d] = (e & 1) ? -s[d] : s[d];
          l[q] = s[3];
        }
        orc_corner_normals(n, t.data(), cv.data(), m.data());
        orc_per_side_widths(n, t.data(), l.data(), wp.data(), wm.data());
        for (int q = 0; q < n; ++q) {
          int e = node_ends[b + q];
          bool swap = (e & 1) != 0;
          const double* nP = &m[3 * q];
          const double* nM = &m[3 * ((q + n - 1) % n)];
          double* o = &ends[(((size_t)(e >> 1)) * 2 + (e & 1)) * 16 + 8 * cfg];
          const double* a = swap ? nM : nP;
          const double* bb = swap ? nP : nM;
          o[0] = a[0]; o[1] = a[1]; o[2] = a[2]; o[3] = swap ? wm[q] : wp[q];
          o[4] = bb[0]; o[5] = bb[1]; o[6] = bb[2]; o[7] = swap ? wp[q] : wm[q];
        }
      }
    }
    for (int h = 0; h < nh; ++h) {
      double* F = Fc + ((size_t)pose * nh + h) * 9;
      double* X = Xc + ((size_t)pose * nh + h) * 3;
      int c = h_curve[h];
      if (c < 0) {
        for (int k = 0; k < 9; ++k) F[k] = (k % 4 == 0) ? 1.0 : 0.0;
        for (int d = 0; d < 3; ++d) X[d] = rest[3 * (size_t)handles[h] + d];
        continue;
      }
      int i = h_sample[h], side = h_side[h];
      int nseg = seg_off[c + 1] - seg_off[c];
      int si = i < nseg ? i : nseg - 1;
      const double* s = &seg[8 * (size_t)(seg_off[c] + si)];
      if (kind[c] == 0) {
        double R[9];
        orc_smallest_rotation(s, s + 4, R);
        double r = s[3] == 0.0 ? 0.0 : s[7] / s[3];
        for (int k = 0; k < 9; ++k) F[k] = r * R[k];
      } else {
        const double* E = &ends[(size_t)c * 32];
        const double* first = (kind[c] & 1) ? E : E + 16;
        const double* last = (kind[c] & 2) ? E + 16 : E;
        double fr[2][9];
        for (int cfg = 0; cfg < 2; ++cfg) {
          double f8[8], g8[8];
          for (int k = 0; k < 8; ++k) { f8[k] = first[8 * cfg + k]; g8[k] = last[8 * cfg + k]; }
          std::vector<double> arr(8 * (size_t)nseg);
          orc_interp_along_curve(f8, g8, nseg, arr.data());
          const double* sd = &arr[8 * (size_t)si + 4 * side];
          orc_scaled_frame(s + 4 * cfg, sd, s[4 * cfg + 3], sd[3], fr[cfg]);
        }
        orc_deformation_gradient(fr[0], fr[1], F);
      }
      eval_curve(PP + (size_t)c * np * 3, S, tau[(size_t)c * M + i], X);
    }
  }
  return 0;
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
