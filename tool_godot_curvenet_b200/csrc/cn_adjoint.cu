// cn_adjoint.cu -- profile-curve handle targets and the adjoint of the
// deform solve (sm_100a).
//
// Curve -> handle map (the reference has the Bezier sample,
// EndToEndExample.lean:52-60, and nearest-vertex projection,
// SurfaceProjection.lean:46-64, but no per-curve weights; this definition is
// the library's): handle h is bound at rest to curve c_h at parameter tau_h;
// with per-curve weight w_c,
//     X_c(h) = rest(h) + w_c (B_posed,c(tau_h) - B_rest,c(tau_h)),
// handles with c_h < 0 stay at rest.  A curve is a composite cubic Bezier of
// S segments (3S+1 control points); tau in [0, S] selects segment
// s = min(floor(tau), S-1) and t = tau - s.
//
// Adjoint of x = overlay(X_c) on handles, x_f = A^{-1} b(X_c) with
// b = -(K diff)_f: for an upstream gradient g = dL/dx,
//     lambda = A^{-1} g_f                      (A symmetric: the same factor)
//     G_h    = dL/dX_c(h) = -(K_{h,free} lambda) + g_h
//     dL/dP_posed[c][3s+j] += w_c bern_j(t) G_h,   dL/dw_c += (B_posed - B_rest)(tau_h) . G_h
// The lambda solve is the persistent solve in right-hand-side mode; these
// kernels build its right-hand side and fold lambda into the gradients.
#include "cn_internal.h"

namespace cn {
namespace {

__device__ void seg_of(double tau, int S, int* s, double* t) {
  int k = (int)floor(tau);
  k = k > S - 1 ? S - 1 : (k < 0 ? 0 : k);
  *s = k;
  *t = tau - (double)k;
}

// EndToEndExample.lean:52-60 bezier3 weights
__device__ void bern(double t, double* c) {
  const double u = 1.0 - t;
  c[0] = u * u * u;
  c[1] = 3.0 * u * u * t;
  c[2] = 3.0 * u * t * t;
  c[3] = t * t * t;
}

__device__ void eval_curve(const double* P, int S, double tau, double* out) {
  int s;
  double t, c[4];
  seg_of(tau, S, &s, &t);
  bern(t, c);
  const double* Q = P + 9 * s;
  for (int d = 0; d < 3; ++d) out[d] = c[0] * Q[d] + c[1] * Q[3 + d] + c[2] * Q[6 + d] + c[3] * Q[9 + d];
}

__global__ void k_curve_targets(CurveArgs c, double* targets) {
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= c.nh) return;
  const int v = c.handles[h];
  const int cv = c.curve_of[h];
  double x[3] = {c.pos[3 * v], c.pos[3 * v + 1], c.pos[3 * v + 2]};
  if (cv >= 0 && cv < c.ncurves) {
    const int np = 3 * c.nseg + 1;
    double bp[3], br[3];
    eval_curve(c.posed_cp + (size_t)cv * np * 3, c.nseg, c.tau[h], bp);
    eval_curve(c.rest_cp + (size_t)cv * np * 3, c.nseg, c.tau[h], br);
    for (int d = 0; d < 3; ++d) x[d] += c.weights[cv] * (bp[d] - br[d]);
  }
  for (int d = 0; d < 3; ++d) targets[3 * h + d] = x[d];
}

__global__ void k_adjoint_rhs(int n, const int* free_of, const double* dLdx, double* b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int v = free_of[i];
  for (int d = 0; d < 3; ++d) b[3 * i + d] = dLdx[3 * v + d];
}

__global__ void k_adjoint_grad(CurveArgs c, const int* K_ptr, const int* K_col, const double* K_val,
                               const int* row_of, const double* lambda, const double* dLdx, double* dP,
                               double* dw) {
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= c.nh) return;
  const int v = c.handles[h];
  double G[3] = {dLdx[3 * v], dLdx[3 * v + 1], dLdx[3 * v + 2]};
  for (int e = K_ptr[v]; e < K_ptr[v + 1]; ++e) {
    const int r = row_of[K_col[e]];
    if (r < 0) continue;
    for (int d = 0; d < 3; ++d) G[d] -= K_val[e] * lambda[3 * (size_t)r + d];
  }
  const int cv = c.curve_of[h];
  if (cv < 0 || cv >= c.ncurves) return;
  const int np = 3 * c.nseg + 1;
  int s;
  double t, b[4];
  seg_of(c.tau[h], c.nseg, &s, &t);
  bern(t, b);
  const double w = c.weights[cv];
  for (int j = 0; j < 4; ++j)
    for (int d = 0; d < 3; ++d) atomicAdd(&dP[((size_t)cv * np + 3 * s + j) * 3 + d], w * b[j] * G[d]);
  double bp[3], br[3];
  eval_curve(c.posed_cp + (size_t)cv * np * 3, c.nseg, c.tau[h], bp);
  eval_curve(c.rest_cp + (size_t)cv * np * 3, c.nseg, c.tau[h], br);
  atomicAdd(&dw[cv], (bp[0] - br[0]) * G[0] + (bp[1] - br[1]) * G[1] + (bp[2] - br[2]) * G[2]);
}

inline int blocks_for(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_curve_targets(const CurveArgs& c, double* targets, cudaStream_t s) {
  if (c.nh > 0) k_curve_targets<<<blocks_for(c.nh, 128), 128, 0, s>>>(c, targets);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_rhs(int n, const int* free_of, const double* dLdx, double* b, cudaStream_t s) {
  if (n > 0) k_adjoint_rhs<<<blocks_for(n, 256), 256, 0, s>>>(n, free_of, dLdx, b);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_grad(const CurveArgs& c, const int* K_ptr, const int* K_col, const double* K_val,
                                const int* row_of, const double* lambda, const double* dLdx, double* dP,
                                double* dw, cudaStream_t s) {
  const size_t np = 3 * (size_t)c.nseg + 1;
  cudaError_t e = cudaMemsetAsync(dP, 0, sizeof(double) * c.ncurves * np * 3, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(dw, 0, sizeof(double) * c.ncurves, s);
  if (e != cudaSuccess) return e;
  if (c.nh > 0)
    k_adjoint_grad<<<blocks_for(c.nh, 128), 128, 0, s>>>(c, K_ptr, K_col, K_val, row_of, lambda, dLdx, dP, dw);
  return cudaGetLastError();
}

}  // namespace cn
