// cn_assemble.cu -- GPU assembly of K = V^T L_h V into CSR and the IC(0)
// factorisation (sm_100a).
//
// Assembly is gather-based (no atomics): one thread per face computes the
// face's 3x3 cotangent Laplacian (PolygonLaplacian.lean:32-71, or the
// mollified one of RobustLaplacian.lean:83-140), then one thread per CSR
// entry adds its face contributions in ascending face order, the order in
// which CutMeshLaplacian.lean:56-71 accumulates them.  All arithmetic uses the
// explicitly rounded intrinsics (__dadd_rn, __dmul_rn, ...), so no FMA is
// contracted and the FP64 values equal the spec's evaluation bit for bit.
//
// The IC(0) factor runs one launch per level set (rows of one level are
// independent); each row computes its strictly-lower entries in ascending
// column order and then its pivot, in FP64 (IncompleteCholesky.lean:49-69).
#include "cn_internal.h"

namespace cn {
namespace {

struct P3 {
  double x, y, z;
};

__device__ __forceinline__ P3 ld3(const double* p, int v) {
  return {p[3 * v], p[3 * v + 1], p[3 * v + 2]};
}

// PolygonLaplacian.lean:32-40
__device__ double cot_at(P3 apex, P3 o1, P3 o2) {
  const double ax = __dsub_rn(o1.x, apex.x), ay = __dsub_rn(o1.y, apex.y), az = __dsub_rn(o1.z, apex.z);
  const double bx = __dsub_rn(o2.x, apex.x), by = __dsub_rn(o2.y, apex.y), bz = __dsub_rn(o2.z, apex.z);
  const double dot = __dadd_rn(__dadd_rn(__dmul_rn(ax, bx), __dmul_rn(ay, by)), __dmul_rn(az, bz));
  const double cx = __dsub_rn(__dmul_rn(ay, bz), __dmul_rn(az, by));
  const double cy = __dsub_rn(__dmul_rn(az, bx), __dmul_rn(ax, bz));
  const double cz = __dsub_rn(__dmul_rn(ax, by), __dmul_rn(ay, bx));
  const double len = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(cx, cx), __dmul_rn(cy, cy)), __dmul_rn(cz, cz)));
  return __ddiv_rn(dot, len);
}

__device__ double dist(P3 u, P3 v) {
  const double dx = __dsub_rn(u.x, v.x), dy = __dsub_rn(u.y, v.y), dz = __dsub_rn(u.z, v.z);
  return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
}

// RobustLaplacian.lean:106-109
__device__ double cot_len(double eo, double e1, double e2) {
  const double s = __dmul_rn(__dadd_rn(__dadd_rn(eo, e1), e2), 0.5);
  const double area = __dsqrt_rn(__dmul_rn(__dmul_rn(__dmul_rn(s, __dsub_rn(s, eo)), __dsub_rn(s, e1)),
                                           __dsub_rn(s, e2)));
  const double num = __dsub_rn(__dadd_rn(__dmul_rn(e1, e1), __dmul_rn(e2, e2)), __dmul_rn(eo, eo));
  return __ddiv_rn(num, __dmul_rn(4.0, area));
}

// Face f's 3x3 in the spec's faceLoop layout (t1, t2, t0): face_m = {m00, m11,
// m22, m01, m02, m12}.
__global__ void k_face_weights(BuildArgs b) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= b.nt) return;
  const P3 A = ld3(b.pos, b.tris[3 * f + 1]);
  const P3 B = ld3(b.pos, b.tris[3 * f + 2]);
  const P3 C = ld3(b.pos, b.tris[3 * f + 0]);
  double cotA, cotB, cotC;
  if (b.lap_kind == CN_LAPLACIAN_ROBUST) {
    double eA = dist(B, C), eB = dist(A, C), eC = dist(A, B);  // RobustLaplacian.lean:66-72
    const double ra = __dsub_rn(__dsub_rn(__dadd_rn(b.delta, eA), eB), eC);
    const double rb = __dsub_rn(__dsub_rn(__dadd_rn(b.delta, eB), eA), eC);
    const double rc = __dsub_rn(__dsub_rn(__dadd_rn(b.delta, eC), eA), eB);
    const double m = fmax(ra, fmax(rb, rc));
    const double eps = fmax(0.0, m);  // :83-89
    eA = __dadd_rn(eA, eps); eB = __dadd_rn(eB, eps); eC = __dadd_rn(eC, eps);
    cotA = cot_len(eA, eB, eC);
    cotB = cot_len(eB, eA, eC);
    cotC = cot_len(eC, eA, eB);
  } else {
    cotA = cot_at(A, B, C);
    cotB = cot_at(B, A, C);
    cotC = cot_at(C, A, B);
  }
  const double w_bc = __dmul_rn(cotA, 0.5), w_ac = __dmul_rn(cotB, 0.5), w_ab = __dmul_rn(cotC, 0.5);
  double* m = b.face_m + 6 * (size_t)f;
  m[0] = __dadd_rn(w_ab, w_ac);
  m[1] = __dadd_rn(w_ab, w_bc);
  m[2] = __dadd_rn(w_ac, w_bc);
  m[3] = -w_ab;
  m[4] = -w_ac;
  m[5] = -w_bc;
}

// CSR values of K: contributions in ascending face order (CutMeshLaplacian.lean:56-71).
__global__ void k_assemble_k(BuildArgs b) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= b.nnzK) return;
  double s = 0.0;
  for (int c = b.K_cptr[e]; c < b.K_cptr[e + 1]; ++c) s = __dadd_rn(s, b.face_m[b.K_contrib[c]]);
  b.K_val[e] = s;
}

// A = K[free, free] in solve order, FP64 and FP32 copies.
__global__ void k_gather_a(BuildArgs b) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= b.nnzA) return;
  const double v = b.K_val[b.A_src[e]];
  b.A_val64[e] = v;
  b.A_val32[e] = __double2float_rn(v);
}

// One level of IC(0): L_ij = (A_ij - sum_k L_ik L_jk) / L_jj, then
// L_ii = sqrt(A_ii (1 + shift) - sum_k L_ik^2).  Jacobi keeps L strictly
// empty and only takes the pivots.
__global__ void k_factor_level(BuildArgs b, int lo, int hi) {
  const int i = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= hi) return;
  double d = b.A_val64[b.A_diag[i]];
  if (b.shift != 0.0) d = __dmul_rn(d, __dadd_rn(1.0, b.shift));
  for (int e = b.L_ptr[i]; e < b.L_ptr[i + 1]; ++e) {
    const int j = b.L_col[e];
    double s = b.A_val64[b.L_src[e]];
    for (int t = b.T_ptr[e]; t < b.T_ptr[e + 1]; ++t)
      s = __dsub_rn(s, __dmul_rn(b.L_val64[b.T_a[t]], b.L_val64[b.T_b[t]]));
    const double l = __ddiv_rn(s, b.Ld64[j]);
    b.L_val64[e] = l;
    d = __dsub_rn(d, __dmul_rn(l, l));
  }
  if (!(d > 0.0)) {
    atomicMin(b.status, i);
    d = 1.0;
  }
  b.Ld64[i] = __dsqrt_rn(d);
}

__global__ void k_factor_finish(BuildArgs b) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < b.nnzL) {
    b.L_val32[e] = __double2float_rn(b.L_val64[e]);
    const double u = b.L_val64[b.U_src[e]];
    b.U_val64[e] = u;
    b.U_val32[e] = __double2float_rn(u);
  }
  if (e < b.n) {
    const double di = __ddiv_rn(1.0, b.Ld64[e]);
    b.dinv64[e] = di;
    b.dinv32[e] = __double2float_rn(di);
  }
}

inline int blocks_for(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_assemble(const BuildArgs& b, cudaStream_t s) {
  if (b.nt > 0) k_face_weights<<<blocks_for(b.nt, 256), 256, 0, s>>>(b);
  if (b.nnzK > 0) k_assemble_k<<<blocks_for(b.nnzK, 256), 256, 0, s>>>(b);
  if (b.nnzA > 0) k_gather_a<<<blocks_for(b.nnzA, 256), 256, 0, s>>>(b);
  return cudaGetLastError();
}

// The level bounds are launch arguments, read from the host copy h_lev_ptr.
cudaError_t launch_factor(const BuildArgs& b, cudaStream_t s) {
  const int* lp = b.h_lev_ptr;
  for (int l = 0; l < b.nlev; ++l) {
    const int lo = lp[l], hi = lp[l + 1];
    if (hi > lo) k_factor_level<<<blocks_for(hi - lo, 128), 128, 0, s>>>(b, lo, hi);
  }
  const long long m = b.nnzL > b.n ? b.nnzL : b.n;
  if (m > 0) k_factor_finish<<<blocks_for(m, 256), 256, 0, s>>>(b);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Plain FP64 Jacobi-PCG primitives (one kernel each; SlangCodegen/SpmvMulti,
// DotReduceMulti, AxpyMulti, SaxpbyMulti, JacobiMulti shapes).
namespace {

__global__ void kp_spmv(PlainArgs a, const double* x, double* y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  for (int c = 0; c < a.K; ++c) {
    double s = 0.0;
    for (int e = a.A_ptr[i]; e < a.A_ptr[i + 1]; ++e) s += a.A_val[e] * x[(size_t)a.A_col[e] * a.K + c];
    y[(size_t)i * a.K + c] = s;
  }
}

__global__ void kp_dot(PlainArgs a, const double* u, const double* v) {
  __shared__ double red[256];
  for (int c = 0; c < a.K; ++c) {
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x)
      s += u[(size_t)i * a.K + c] * v[(size_t)i * a.K + c];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) a.partials[(size_t)blockIdx.x * a.K + c] = red[0];
    __syncthreads();
  }
}

__global__ void kp_axpy2(PlainArgs a, const double* alpha) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  for (int c = 0; c < a.K; ++c) {
    const size_t ix = (size_t)i * a.K + c;
    a.x[ix] += alpha[c] * a.p[ix];
    a.r[ix] -= alpha[c] * a.Ap[ix];
  }
}

__global__ void kp_jacobi(PlainArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const double d = a.A_val[a.A_diag[i]];
  for (int c = 0; c < a.K; ++c) {
    const size_t ix = (size_t)i * a.K + c;
    a.z[ix] = d == 0.0 ? 0.0 : a.r[ix] / d;  // SparseLinAlg.lean:92-97
  }
}

__global__ void kp_saxpby(PlainArgs a, const double* beta) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  for (int c = 0; c < a.K; ++c) {
    const size_t ix = (size_t)i * a.K + c;
    a.p[ix] = a.z[ix] + beta[c] * a.p[ix];
  }
}

__global__ void kp_rhs_init(SolveArgs sa, PlainArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int v = sa.free_of[i];
  for (int c = 0; c < a.K; ++c) {
    double s = 0.0;
    if (sa.mode != CN_MODE_RHS) {
      for (int e = sa.K_ptr[v]; e < sa.K_ptr[v + 1]; ++e) {
        const int u = sa.K_col[e];
        const int h = sa.hidx[u];
        const double rest = sa.mode == CN_MODE_DEFORM ? sa.pos[3 * u + c % 3] : 0.0;
        s += sa.K_val[e] * (h >= 0 ? sa.targets[(size_t)h * a.K + c] - rest : -rest);
      }
    }
    const size_t ix = (size_t)i * a.K + c;
    a.b[ix] = sa.mode == CN_MODE_RHS ? sa.targets[ix] : -s;
    a.x[ix] = sa.x0 ? sa.x0[(size_t)v * a.K + c] : 0.0;
  }
}

__global__ void kp_residual(PlainArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  for (int c = 0; c < a.K; ++c) {
    double s = 0.0;
    for (int e = a.A_ptr[i]; e < a.A_ptr[i + 1]; ++e) s += a.A_val[e] * a.x[(size_t)a.A_col[e] * a.K + c];
    a.r[(size_t)i * a.K + c] = a.b[(size_t)i * a.K + c] - s;
  }
}

__global__ void kp_output(SolveArgs sa, PlainArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.n) {
    const int v = sa.free_of[i];
    for (int c = 0; c < a.K; ++c) sa.x_out[(size_t)v * a.K + c] = a.x[(size_t)i * a.K + c];
  }
  if (i < sa.nh) {
    const int v = sa.handles[i];
    for (int c = 0; c < a.K; ++c)
      sa.x_out[(size_t)v * a.K + c] = sa.mode == CN_MODE_RHS ? 0.0 : sa.targets[(size_t)i * a.K + c];
  }
}

}  // namespace

cudaError_t plain_spmv(const PlainArgs& a, const double* x, double* y, cudaStream_t s) {
  kp_spmv<<<blocks_for(a.n, 256), 256, 0, s>>>(a, x, y);
  return cudaGetLastError();
}
cudaError_t plain_dot(const PlainArgs& a, const double* u, const double* v, cudaStream_t s) {
  kp_dot<<<a.blocks, 256, 0, s>>>(a, u, v);
  return cudaGetLastError();
}
cudaError_t plain_axpy2(const PlainArgs& a, const double* alpha, cudaStream_t s) {
  kp_axpy2<<<blocks_for(a.n, 256), 256, 0, s>>>(a, alpha);
  return cudaGetLastError();
}
cudaError_t plain_jacobi(const PlainArgs& a, cudaStream_t s) {
  kp_jacobi<<<blocks_for(a.n, 256), 256, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t plain_saxpby(const PlainArgs& a, const double* beta, cudaStream_t s) {
  kp_saxpby<<<blocks_for(a.n, 256), 256, 0, s>>>(a, beta);
  return cudaGetLastError();
}
cudaError_t plain_rhs_and_init(const SolveArgs& sa, const PlainArgs& a, cudaStream_t s) {
  if (a.n > 0) kp_rhs_init<<<blocks_for(a.n, 256), 256, 0, s>>>(sa, a);
  return cudaGetLastError();
}
cudaError_t plain_residual(const PlainArgs& a, cudaStream_t s) {
  if (a.n > 0) kp_residual<<<blocks_for(a.n, 256), 256, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t plain_output(const SolveArgs& sa, const PlainArgs& a, cudaStream_t s) {
  const int m = a.n > sa.nh ? a.n : sa.nh;
  if (m > 0) kp_output<<<blocks_for(m, 256), 256, 0, s>>>(sa, a);
  return cudaGetLastError();
}
cudaError_t plain_set_scalars(double* d_dst, const double* h_src, int K, cudaStream_t s) {
  return cudaMemcpyAsync(d_dst, h_src, sizeof(double) * K, cudaMemcpyHostToDevice, s);
}

}  // namespace cn
