// cn_ddm.cu -- Direct Delta Mush on the GPU (sm_100a): the bind-time
// influence bake (DirectDeltaMushBind.lean:6-40) and the runtime kernel
// (DirectDeltaMush.lean:84-102, SlangCodegen/DirectDeltaMush.lean:11-22).
//
// Bind, per chunk of up to 9 handles (the harmonic solve of the handle with
// k = 9 unit right-hand sides, HarmonicSolve.lean:51-66, fills W[:, chunk]):
//   k_ddm_smooth  nu passes of w' = (1 - omega) w + omega * mean of the
//                 neighbours (DirectDeltaMushBind.lean:72-94), FP64 without
//                 contraction, neighbours in ascending vertex order (the
//                 off-diagonal entries of K's row);
//   k_ddm_topk    merges the chunk into each vertex's running top-K list,
//                 ordered by |w| descending, ties by lower handle index
//                 (DirectDeltaMushBind.lean:104-133 picks by |w| with a
//                 selection sort);
// then k_ddm_finish divides each row by the sum of its kept weights.
// Runtime: one thread per vertex, pos = sum_k w_k (T_{i_k} (rest, 1)).
#include "cn_internal.h"

namespace cn {
namespace {

__global__ void k_unit_targets(int nh, int c0, int kc, double* t) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nh * 9) return;
  const int h = q / 9, j = q - h * 9;
  t[q] = (j < kc && h == c0 + j) ? 1.0 : 0.0;
}

__global__ void k_ddm_smooth(int nv, const int* __restrict__ ptr, const int* __restrict__ col, const double* in,
                             double* out, double omega) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nv * 9) return;
  const int v = q / 9, j = q - v * 9;
  double nb = 0.0;
  int count = 0;
  for (int e = ptr[v]; e < ptr[v + 1]; ++e) {
    const int u = col[e];
    if (u == v) continue;
    nb = __dadd_rn(nb, in[(size_t)u * 9 + j]);
    ++count;
  }
  if (count > 0) nb = __ddiv_rn(nb, (double)count);
  out[q] = __dadd_rn(__dmul_rn(__dsub_rn(1.0, omega), in[q]), __dmul_rn(omega, nb));
}

__global__ void k_ddm_topk(int nv, int c0, int kc, int K, const double* __restrict__ W, int* bidx, double* bw,
                           int* cnt) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  int* li = bidx + (size_t)v * K;
  double* lw = bw + (size_t)v * K;
  int c = cnt[v];
  for (int j = 0; j < kc; ++j) {
    const double w = W[(size_t)v * 9 + j];
    const double a = fabs(w);
    // first position whose entry this candidate beats (strictly larger |w|;
    // candidates arrive in increasing handle index, so ties keep the earlier)
    int p = c;
    while (p > 0 && a > fabs(lw[p - 1])) --p;
    if (p >= K) continue;
    const int last = c < K ? c : K - 1;
    for (int q = last; q > p; --q) {
      li[q] = li[q - 1];
      lw[q] = lw[q - 1];
    }
    li[p] = c0 + j;
    lw[p] = w;
    if (c < K) ++c;
  }
  cnt[v] = c;
}

__global__ void k_ddm_finish(int nv, int take, double* bw) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  double* lw = bw + (size_t)v * take;
  double sum = 0.0;
  for (int k = 0; k < take; ++k) sum = __dadd_rn(sum, lw[k]);
  if (sum != 0.0)
    for (int k = 0; k < take; ++k) lw[k] = __ddiv_rn(lw[k], sum);
}

template <typename T>
__global__ void __launch_bounds__(256) k_lbs_matvec(int nv, const T* __restrict__ rest, const T* __restrict__ tr,
                                                    const int* __restrict__ start, const int* __restrict__ idx,
                                                    const T* __restrict__ w, T* __restrict__ out) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const T rx = rest[3 * (size_t)v], ry = rest[3 * (size_t)v + 1], rz = rest[3 * (size_t)v + 2];
  T x = 0, y = 0, z = 0;
  const int s = start[v], e = start[v + 1];
  for (int k = s; k < e; ++k) {
    const T* M = tr + 16 * (size_t)__ldg(idx + k);
    const T wk = __ldg(w + k);
    const T tx = __ldg(M + 0) * rx + __ldg(M + 1) * ry + __ldg(M + 2) * rz + __ldg(M + 3);
    const T ty = __ldg(M + 4) * rx + __ldg(M + 5) * ry + __ldg(M + 6) * rz + __ldg(M + 7);
    const T tz = __ldg(M + 8) * rx + __ldg(M + 9) * ry + __ldg(M + 10) * rz + __ldg(M + 11);
    x += wk * tx;
    y += wk * ty;
    z += wk * tz;
  }
  out[3 * (size_t)v] = x;
  out[3 * (size_t)v + 1] = y;
  out[3 * (size_t)v + 2] = z;
}

__global__ void k_copy_columns(const double* src, int rows, int ks, int s0, double* dst, int kd, int d0,
                               int ncols) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)rows * ncols) return;
  const int r = (int)(q / ncols), c = (int)(q - (long long)r * ncols);
  dst[(size_t)r * kd + d0 + c] = src[(size_t)r * ks + s0 + c];
}

inline unsigned blocks_for(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_copy_columns(const double* src, int rows, int ks, int s0, double* dst, int kd, int d0, int ncols,
                                cudaStream_t s) {
  if (rows > 0 && ncols > 0)
    k_copy_columns<<<blocks_for((long long)rows * ncols, 256), 256, 0, s>>>(src, rows, ks, s0, dst, kd, d0, ncols);
  return cudaGetLastError();
}

cudaError_t launch_ddm_unit_targets(int nh, int c0, int kc, double* t, cudaStream_t s) {
  if (nh > 0) k_unit_targets<<<blocks_for((long long)nh * 9, 256), 256, 0, s>>>(nh, c0, kc, t);
  return cudaGetLastError();
}

cudaError_t launch_ddm_smooth(int nv, const int* ptr, const int* col, const double* in, double* out, double omega,
                              cudaStream_t s) {
  if (nv > 0) k_ddm_smooth<<<blocks_for((long long)nv * 9, 256), 256, 0, s>>>(nv, ptr, col, in, out, omega);
  return cudaGetLastError();
}

cudaError_t launch_ddm_topk(int nv, int c0, int kc, int K, const double* W, int* bidx, double* bw, int* cnt,
                            cudaStream_t s) {
  if (nv > 0) k_ddm_topk<<<blocks_for(nv, 128), 128, 0, s>>>(nv, c0, kc, K, W, bidx, bw, cnt);
  return cudaGetLastError();
}

cudaError_t launch_ddm_finish(int nv, int take, double* bw, cudaStream_t s) {
  if (nv > 0) k_ddm_finish<<<blocks_for(nv, 256), 256, 0, s>>>(nv, take, bw);
  return cudaGetLastError();
}

cudaError_t launch_lbs_matvec(int nv, int precision, const void* rest, const void* tr, const int* start,
                              const int* idx, const void* w, void* out, cudaStream_t s) {
  if (nv <= 0) return cudaSuccess;
  if (precision == CN_PREC_MIXED)
    k_lbs_matvec<float><<<blocks_for(nv, 256), 256, 0, s>>>(nv, (const float*)rest, (const float*)tr, start, idx,
                                                            (const float*)w, (float*)out);
  else
    k_lbs_matvec<double><<<blocks_for(nv, 256), 256, 0, s>>>(nv, (const double*)rest, (const double*)tr, start,
                                                             idx, (const double*)w, (double*)out);
  return cudaGetLastError();
}

}  // namespace cn
