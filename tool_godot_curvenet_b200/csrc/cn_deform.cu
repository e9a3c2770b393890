// cn_deform.cu -- the bridge between the two stages of the DeGoes22 solve
// (DeformSolve.lean:110-135) on the GPU (sm_100a).
//
// Stage 1 solves (V^T L_h V) F_v = -V^T L_h (C F_c) for the 9 entries of the
// deformation gradient (a k = 9 harmonic solve, handles overlaid with F_c).
// The bridge, per face (each triangle's halfedges are its 3 corners, in the
// spec's faceLoop order t1, t2, t0):
//   F_h  = F_v at the corner's vertex (F_c at a handle)      computeFh   :40-53
//   F_f  = (1/3) sum of the 3 corner values                   averageOverFaces :57-70
//   y_h  = F_f rest(corner)                                   computeYh   :75-97
//   diff = C X_c - y_h  (C X_c is X_c at a handle corner, else 0)
//   c_f[a] = sum_b L_f[a][b] diff[b]   (L_f the face's 3x3 cot Laplacian)
// and per free row v the Stage-2 right-hand side b_v = -sum over the faces of
// v (ascending) of c_f[corner of v]  (= -(V^T L_h (C X_c - y_h))_v, :123-132).
#include "cn_internal.h"

namespace cn {
namespace {

// face_m layout: {m00, m11, m22, m01, m02, m12} of the face's faceLoop order.
__device__ __forceinline__ double fm(const double* m, int a, int b) {
  if (a == b) return m[a];
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  return m[lo == 0 ? (hi == 1 ? 3 : 4) : 5];
}

__global__ void k_face_bridge(DeformArgs d) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= d.nt) return;
  const int g[3] = {d.tris[3 * f + 1], d.tris[3 * f + 2], d.tris[3 * f + 0]};
  double Ff[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    double s = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) s += d.Fv[(size_t)g[a] * 9 + q];
    Ff[q] = s * (1.0 / 3.0);
  }
  double diff[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double* p = d.pos + 3 * (size_t)g[a];
    const int h = d.hidx[g[a]];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double y = p[0] * Ff[3 * i] + p[1] * Ff[3 * i + 1] + p[2] * Ff[3 * i + 2];
      const double cx = h >= 0 ? d.Xc[(size_t)h * 3 + i] : 0.0;
      diff[a][i] = cx - y;
    }
  }
  const double* m = d.face_m + 6 * (size_t)f;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double s = 0.0;
#pragma unroll
      for (int b = 0; b < 3; ++b) s += fm(m, a, b) * diff[b][i];
      d.contrib[(size_t)(3 * f + a) * 3 + i] = s;  // slot a is faceLoop corner a
    }
}

__global__ void k_stage2_rhs(DeformArgs d) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= d.n) return;
  const int v = d.free_of[row];
  double s[3] = {0.0, 0.0, 0.0};
  for (int q = d.vf_ptr[v]; q < d.vf_ptr[v + 1]; ++q) {
    const int f = d.vf_face[q];
    const int a = (d.vf_corner[q] + 2) % 3;  // corner t0,t1,t2 -> faceLoop slot 2,0,1
#pragma unroll
    for (int i = 0; i < 3; ++i) s[i] += d.contrib[(size_t)(3 * f + a) * 3 + i];
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) d.b[(size_t)row * 3 + i] = -s[i];
}

inline int blocks_for(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_deform_bridge(const DeformArgs& d, cudaStream_t s) {
  if (d.nt > 0) k_face_bridge<<<blocks_for(d.nt, 128), 128, 0, s>>>(d);
  if (d.n > 0) k_stage2_rhs<<<blocks_for(d.n, 256), 256, 0, s>>>(d);
  return cudaGetLastError();
}

}  // namespace cn
