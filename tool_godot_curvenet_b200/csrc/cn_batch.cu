// cn_batch.cu -- batched solves of many uneven meshes in one persistent launch
// (sm_100a).
//
// The grid is made of thread-block clusters; each cluster takes the next mesh
// from an atomic work queue (meshes ordered longest first) and solves all of
// its right-hand sides (poses x 3 coordinates) with the same algorithm as the
// single-mesh persistent solve (cn_pcg.cu): right-hand-side assembly, FP64
// residual refinement around an inner PCG in T with the IC(0) level-scheduled
// sweeps, and the output scatter.  The team barrier is the hardware cluster
// barrier (barrier.cluster.arrive.release / wait.acquire) and the partial
// sums of the dot products live in each block's shared memory, read by the
// other blocks of the cluster through distributed shared memory, in rank
// order, so every block takes the same branch.  A mesh's working vectors
// stay in a per-cluster scratch that is reused mesh after mesh, so they tend
// to stay in L2 while the cluster iterates.
//
// Thread mapping for many right-hand sides: C lanes per row, each lane owns
// K / C consecutive columns and walks the row's entries; the C lanes of a row
// read one neighbour row's K values as one contiguous, coalesced segment.
// With K = 24 a mesh takes C = 8 (4 rows per warp) or C = 4 (8 rows per
// warp), chosen per size class by the autotuner: the meshes of each C are one
// work queue of one persistent kernel, and both kernels are nodes of the same
// CUDA graph, running side by side on disjoint clusters.
#include <cooperative_groups.h>

#include "cn_batch.h"
#include "cn_pcg_body.cuh"

namespace cg = cooperative_groups;

namespace cn {
namespace {

using pcg::gather_row;
using pcg::kBB;
using pcg::kPAP;
using pcg::kRR;
using pcg::kRR64;
using pcg::kRZ;

struct ClusterTeam {
  int r, s;
  __device__ __forceinline__ int rank() const { return r; }
  __device__ __forceinline__ int size() const { return s; }
  __device__ __forceinline__ bool sync() const {
    cg::this_cluster().sync();
    return true;
  }
};

template <int K>
struct SmemW {
  double red[32 * K];
  double part[5][K];  // this block's partial of each reduction (read over DSMEM)
  double sum[K];
  double alpha[K], beta[K], rz[K], rr0[K], bb[K], stop[K];
  int active[K];
  int flag;
};

// Block sums of K columns where a thread holds CPL = K / C columns starting at
// (lane % C) * CPL.  Result in out[0..K), fixed order.
template <int K, int C>
__device__ void block_reduce_wide(double (&v)[K / C], double* red, double* out) {
  constexpr int CPL = K / C;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int c = 0; c < CPL; ++c) {
    double t = v[c];
#pragma unroll
    for (int o = C; o < 32; o <<= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane < C) red[warp * K + lane * CPL + c] = t;
  }
  __syncthreads();
  if (warp == 0) {
    for (int c = lane; c < K; c += 32) {
      double t = 0.0;
      for (int w = 0; w < nw; ++w) t += red[w * K + c];
      out[c] = t;
    }
  }
  __syncthreads();
}

// After a cluster barrier: sum slot `slot` over the cluster's blocks in rank
// order (distributed shared memory); result in s->sum.
template <int K>
__device__ void cluster_sum(SmemW<K>* s, int slot, int csize) {
  if (threadIdx.x < 32) {
    cg::cluster_group cl = cg::this_cluster();
    for (int c = threadIdx.x; c < K; c += 32) {
      double t = 0.0;
      for (int r = 0; r < csize; ++r) {
        const SmemW<K>* rs = cl.map_shared_rank(s, r);
        t += rs->part[slot][c];
      }
      s->sum[c] = t;
    }
  }
  __syncthreads();
}

template <typename T, int K, int C>
__device__ void solve_body_wide(const SolveArgs& a, const ClusterTeam& team, SmemW<K>* s) {
  constexpr int CPL = K / C;
  const T* Aval = (const T*)a.A_val;
  const T* Lval = (const T*)a.L_val;
  const T* Uval = (const T*)a.U_val;
  const T* dinv = (const T*)a.dinv;
  T* r = (T*)a.r;
  T* y = (T*)a.y;
  T* z = (T*)a.z;
  T* pa = (T*)a.p0;
  T* pb = (T*)a.p1;
  T* Ap = (T*)a.Ap;
  T* xin = (T*)a.xin;
  const int n = a.n, nlev = a.nlev;
  const int gpb = blockDim.x / C;
  const int grp = threadIdx.x / C, sub = threadIdx.x % C;
  const int c0 = sub * CPL;
  const int row0 = team.rank() * gpb + grp, rstride = team.size() * gpb;
  const int csize = team.size();
  int status = CN_OK, total_iters = 0, refinements = 0;
  // entries of a row gathered together: FP32 runs three 512-thread CTAs per
  // SM (40 registers; more clusters in flight hide more of the HBM latency
  // than wider gathers), FP64 two (64 registers)
  constexpr int UW = sizeof(T) == 4 ? 2 : 4;

  // ---- right-hand side (HarmonicSolve.lean:51-66 / DeformSolve.lean:123-135)
  {
    double bb[CPL];
#pragma unroll
    for (int c = 0; c < CPL; ++c) bb[c] = 0.0;
    for (int row = row0; row < n; row += rstride) {
      double acc[CPL];
#pragma unroll
      for (int c = 0; c < CPL; ++c) acc[c] = 0.0;
      const int v = a.free_of[row];
      if (a.mode != CN_MODE_RHS) {
        const bool deform = a.mode == CN_MODE_DEFORM;
        gather_row<CPL, 1, UW>(a.K_ptr[v], a.K_ptr[v + 1], 0, a.K_col, a.K_val,
                               [&](int u, double* d) {
                                 const int h = a.hidx[u];
#pragma unroll
                                 for (int c = 0; c < CPL; ++c) {
                                   const int cc = c0 + c;
                                   const double rest = deform ? a.pos[3 * u + cc % 3] : 0.0;
                                   d[c] = h >= 0 ? a.targets[(size_t)h * K + cc] - rest : -rest;
                                 }
                               },
                               acc);
      }
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        const size_t ix = (size_t)row * K + c0 + c;
        const double b = a.mode == CN_MODE_RHS ? a.targets[ix] : -acc[c];
        a.b64[ix] = b;
        bb[c] += b * b;
        a.x64[ix] = 0.0;
      }
    }
    block_reduce_wide<K, C>(bb, s->red, s->part[kBB]);
    team.sync();
    cluster_sum<K>(s, kBB, csize);
    if (threadIdx.x < K) s->bb[threadIdx.x] = s->sum[threadIdx.x];
    __syncthreads();
  }

  for (int refine = 0;; ++refine) {
    // ---- FP64 residual r = b - A x
    {
      double rr[CPL];
#pragma unroll
      for (int c = 0; c < CPL; ++c) rr[c] = 0.0;
      for (int row = row0; row < n; row += rstride) {
        double acc[CPL];
#pragma unroll
        for (int c = 0; c < CPL; ++c) acc[c] = 0.0;
        gather_row<CPL, 1, UW>(a.A_ptr[row], a.A_ptr[row + 1], 0, a.A_col, a.A_val64,
                               [&](int j, double* x) {
                                 const double* xj = a.x64 + (size_t)j * K + c0;
#pragma unroll
                                 for (int c = 0; c < CPL; ++c) x[c] = xj[c];
                               },
                               acc);
#pragma unroll
        for (int c = 0; c < CPL; ++c) {
          const size_t ix = (size_t)row * K + c0 + c;
          const double rv = a.b64[ix] - acc[c];
          r[ix] = (T)rv;
          xin[ix] = (T)0;
          rr[c] += rv * rv;
        }
      }
      block_reduce_wide<K, C>(rr, s->red, s->part[kRR64]);
      team.sync();
      cluster_sum<K>(s, kRR64, csize);
      if (threadIdx.x == 0) {
        int any = 0, bad = 0;
        for (int c = 0; c < K; ++c) {
          const double rr64 = s->sum[c], bb = s->bb[c];
          const double rel = bb > 0.0 ? sqrt(rr64 / bb) : sqrt(rr64);
          if (team.rank() == 0 && c < 32) a.stats->rel_residual[c] = rel;
          if (!(rel == rel)) bad = 1;
          const int act = rel > a.tol;
          s->active[c] = act;
          any |= act;
          s->rr0[c] = rr64;
          const double want = bb > 0.0 ? 0.5 * a.tol * sqrt(bb / (rr64 > 0.0 ? rr64 : 1.0)) : 0.0;
          const double tau = fmax(a.inner_tol, want);
          s->stop[c] = tau * tau * rr64;
          s->beta[c] = 0.0;
        }
        s->flag = bad ? 2 : (any ? 1 : 0);
      }
      __syncthreads();
      if (s->flag == 2) { status = CN_NAN; break; }
      if (s->flag == 0) { status = CN_OK; break; }
      if (refine >= a.max_refine) { status = CN_MAX_ITER; break; }
      refinements = refine + 1;
    }

    int it = 0;
    bool first = true;
    // x += alpha p of an iteration is applied where that p is read next: in
    // the following iteration's SpMV pass, or after the loop for the last one
    const T* plast = nullptr;
    T alast[CPL];
    for (;;) {
      if (!first) {
        double pap[CPL];
#pragma unroll
        for (int c = 0; c < CPL; ++c) pap[c] = 0.0;
        T beta[CPL];
#pragma unroll
        for (int c = 0; c < CPL; ++c) beta[c] = (T)s->beta[c0 + c];
        // On the first iteration every beta is 0 and p_old is not read: the
        // reused scratch may hold anything (another mesh, another precision).
        const bool b0 = it == 0;
        const T* pold = (it & 1) ? pb : pa;
        T* pnew = (it & 1) ? pa : pb;
        T aprev[CPL];
#pragma unroll
        for (int c = 0; c < CPL; ++c) aprev[c] = (T)s->alpha[c0 + c];
        for (int row = row0; row < n; row += rstride) {
          T acc[CPL];
#pragma unroll
          for (int c = 0; c < CPL; ++c) acc[c] = (T)0;
          if (b0) {
            gather_row<CPL, 1, UW>(a.A_ptr[row], a.A_ptr[row + 1], 0, a.A_col, Aval,
                                   [&](int j, T* x) {
                                     const size_t jb = (size_t)j * K + c0;
#pragma unroll
                                     for (int c = 0; c < CPL; ++c) x[c] = z[jb + c];
                                   },
                                   acc);
          } else {
            // A p = A z + beta A p_old: only z is gathered, A p_old is this
            // row's own entry of Ap
            gather_row<CPL, 1, UW>(a.A_ptr[row], a.A_ptr[row + 1], 0, a.A_col, Aval,
                                   [&](int j, T* x) {
                                     const size_t jb = (size_t)j * K + c0;
#pragma unroll
                                     for (int c = 0; c < CPL; ++c) x[c] = z[jb + c];
                                   },
                                   acc);
          }
#pragma unroll
          for (int c = 0; c < CPL; ++c) {
            const size_t ix = (size_t)row * K + c0 + c;
            T pi = z[ix];
            if (!b0) {
              const T po = pold[ix];
              xin[ix] += aprev[c] * po;  // the previous iteration's x update
              pi += beta[c] * po;
            }
            const T api = b0 ? acc[c] : acc[c] + beta[c] * Ap[ix];
            pnew[ix] = pi;
            Ap[ix] = api;
            pap[c] += (double)pi * (double)api;
          }
        }
        block_reduce_wide<K, C>(pap, s->red, s->part[kPAP]);
        team.sync();
        cluster_sum<K>(s, kPAP, csize);
        if (threadIdx.x < K) {
          const int c = threadIdx.x;
          const double v = s->sum[c];
          if (s->active[c] && !(v > 0.0)) s->active[c] = 0;
          s->alpha[c] = s->active[c] ? s->rz[c] / v : 0.0;
        }
        __syncthreads();
      }

      const T* pcur = (it & 1) ? pa : pb;
      double rrp[CPL], rzp[CPL];
#pragma unroll
      for (int c = 0; c < CPL; ++c) { rrp[c] = 0.0; rzp[c] = 0.0; }
      T alpha[CPL];
#pragma unroll
      for (int c = 0; c < CPL; ++c) alpha[c] = (T)s->alpha[c0 + c];
      for (int l = 0; l < nlev; ++l) {
        const int lo = a.lev_ptr[l], hi = a.lev_ptr[l + 1];
        const bool last = l == nlev - 1;
        for (int row = lo + row0; row < hi; row += rstride) {
          T acc[CPL];
#pragma unroll
          for (int c = 0; c < CPL; ++c) acc[c] = (T)0;
          gather_row<CPL, 1, UW>(a.L_ptr[row], a.L_ptr[row + 1], 0, a.L_col, Lval,
                                 [&](int j, T* x) {
                                   const size_t jb = (size_t)j * K + c0;
#pragma unroll
                                   for (int c = 0; c < CPL; ++c) x[c] = y[jb + c];
                                 },
                                 acc);
          const T di = dinv[row];
#pragma unroll
          for (int c = 0; c < CPL; ++c) {
            const size_t ix = (size_t)row * K + c0 + c;
            T rv = r[ix];
            if (!first) {
              rv -= alpha[c] * Ap[ix];
              r[ix] = rv;
            }
            const T yv = (rv - acc[c]) * di;
            y[ix] = yv;
            rrp[c] += (double)rv * (double)rv;
            // (r, M^-1 r) = (L y, L^-T y) = ||y||^2 with M = L L^T, y = L^-1 r:
            // the backward sweep need not read r again
            rzp[c] += (double)yv * (double)yv;
            if (last) z[ix] = yv * di;
          }
        }
        if (!last) team.sync();
      }
      for (int l = nlev - 2; l >= 0; --l) {
        team.sync();
        const int lo = a.lev_ptr[l], hi = a.lev_ptr[l + 1];
        for (int row = lo + row0; row < hi; row += rstride) {
          T acc[CPL];
#pragma unroll
          for (int c = 0; c < CPL; ++c) acc[c] = (T)0;
          gather_row<CPL, 1, UW>(a.U_ptr[row], a.U_ptr[row + 1], 0, a.U_col, Uval,
                                 [&](int j, T* x) {
                                   const size_t jb = (size_t)j * K + c0;
#pragma unroll
                                   for (int c = 0; c < CPL; ++c) x[c] = z[jb + c];
                                 },
                                 acc);
          const T di = dinv[row];
#pragma unroll
          for (int c = 0; c < CPL; ++c) {
            const size_t ix = (size_t)row * K + c0 + c;
            z[ix] = (y[ix] - acc[c]) * di;
          }
        }
      }
      block_reduce_wide<K, C>(rrp, s->red, s->part[kRR]);
      block_reduce_wide<K, C>(rzp, s->red, s->part[kRZ]);
      team.sync();
      cluster_sum<K>(s, kRR, csize);
      double rrv = threadIdx.x < K ? s->sum[threadIdx.x] : 0.0;
      __syncthreads();
      cluster_sum<K>(s, kRZ, csize);
      if (threadIdx.x < K) {
        const int c = threadIdx.x;
        const double rzn = s->sum[c];
        if (!first && s->active[c] && rrv < s->stop[c]) s->active[c] = 0;
        s->beta[c] = first ? 0.0 : (s->rz[c] == 0.0 ? 0.0 : rzn / s->rz[c]);
        s->rz[c] = rzn;
        s->red[c] = (!(rrv == rrv) || !(rzn == rzn)) ? 1.0 : 0.0;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int any = 0, bad = 0;
        for (int c = 0; c < K; ++c) {
          any |= s->active[c];
          bad |= s->red[c] != 0.0;
        }
        s->flag = bad ? 2 : (any ? 1 : 0);
      }
      __syncthreads();
      if (!first) {
        plast = pcur;
#pragma unroll
        for (int c = 0; c < CPL; ++c) alast[c] = alpha[c];
        ++it;
        ++total_iters;
      }
      if (s->flag == 2) { status = CN_NAN; goto done; }
      first = false;
      if (s->flag == 0 || it >= a.max_iter) break;
    }
    for (int row = row0; row < n; row += rstride) {
#pragma unroll
      for (int c = 0; c < CPL; ++c) {
        const size_t ix = (size_t)row * K + c0 + c;
        T xv = xin[ix];
        if (plast) xv += alast[c] * plast[ix];  // the last iteration's x update
        a.x64[ix] += (double)xv;
      }
    }
    team.sync();
  }

  if (a.x_out) {
    for (int row = row0; row < n; row += rstride) {
      const int v = a.free_of[row];
#pragma unroll
      for (int c = 0; c < CPL; ++c) a.x_out[(size_t)v * K + c0 + c] = a.x64[(size_t)row * K + c0 + c];
    }
    for (int h = row0; h < a.nh; h += rstride) {
      const int v = a.handles[h];
#pragma unroll
      for (int c = 0; c < CPL; ++c)
        a.x_out[(size_t)v * K + c0 + c] = a.mode == CN_MODE_RHS ? 0.0 : a.targets[(size_t)h * K + c0 + c];
    }
  }

done:
  if (team.rank() == 0 && threadIdx.x == 0) {
    a.stats->status = status;
    a.stats->iterations = total_iters;
    a.stats->refinements = refinements;
  }
  // all blocks leave the mesh together (the next mesh reuses the scratch)
  team.sync();
}

template <typename T, int K, int C>
__global__ void __launch_bounds__(512, sizeof(T) == 4 ? 3 : 2) k_batch(BatchArgs ba) {
  __shared__ SmemW<K> s;
  __shared__ int s_mesh;
  cg::cluster_group cl = cg::this_cluster();
  const int csize = (int)cl.num_blocks();
  ClusterTeam team{(int)cl.block_rank(), csize};
  const int cid = ba.cluster_base + blockIdx.x / csize;
  T* vt = (T*)ba.vec_T + (size_t)cid * 7 * ba.stride;
  double* v64 = ba.vec_64 + (size_t)cid * 2 * ba.stride;
  for (;;) {
    if (team.rank() == 0 && threadIdx.x == 0) s_mesh = atomicAdd(ba.queue, 1);
    cl.sync();
    const int q = *cl.map_shared_rank(&s_mesh, 0);
    cl.sync();
    if (q >= ba.n_meshes) break;
    const int m = ba.order[q];
    SolveArgs a = ba.meshes[m];
    a.targets = ba.targets + ba.tgt_off[m];
    a.x_out = ba.x_out ? ba.x_out + ba.out_off[m] : nullptr;
    a.r = vt; a.y = vt + ba.stride; a.z = vt + 2 * ba.stride; a.p0 = vt + 3 * ba.stride;
    a.p1 = vt + 4 * ba.stride; a.Ap = vt + 5 * ba.stride; a.xin = vt + 6 * ba.stride;
    a.b64 = v64;
    a.x64 = v64 + ba.stride;
    a.stats = ba.stats + m;
    solve_body_wide<T, K, C>(a, team, &s);
  }
}

template <typename T, int K, int C>
cudaError_t launch_kc(const BatchArgs& ba, int csize, int nclusters, int block, cudaStream_t st) {
  auto kern = k_batch<T, K, C>;
  if (csize > 8) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nclusters * csize);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, ba);
}

template <typename T, int K, int C>
int max_clusters_kc(int csize, int block) {
  auto kern = k_batch<T, K, C>;
  if (csize > 8) cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(csize);
  cfg.blockDim = dim3(block);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess) return 0;
  return n;
}

}  // namespace

cudaError_t launch_batch(const BatchArgs& ba, int precision, int K, int lanes, int csize, int nclusters, int block,
                         cudaStream_t st) {
  if (K == 24 && lanes == 4) {
    if (precision == CN_PREC_MIXED) return launch_kc<float, 24, 4>(ba, csize, nclusters, block, st);
    return launch_kc<double, 24, 4>(ba, csize, nclusters, block, st);
  }
  if (K == 24) {
    if (precision == CN_PREC_MIXED) return launch_kc<float, 24, 8>(ba, csize, nclusters, block, st);
    return launch_kc<double, 24, 8>(ba, csize, nclusters, block, st);
  }
  if (K == 3) {
    if (precision == CN_PREC_MIXED) return launch_kc<float, 3, 1>(ba, csize, nclusters, block, st);
    return launch_kc<double, 3, 1>(ba, csize, nclusters, block, st);
  }
  return cudaErrorInvalidValue;
}

int batch_max_clusters(int precision, int K, int lanes, int csize, int block) {
  if (K == 24 && lanes == 4) {
    if (precision == CN_PREC_MIXED) return max_clusters_kc<float, 24, 4>(csize, block);
    return max_clusters_kc<double, 24, 4>(csize, block);
  }
  if (K == 24) {
    if (precision == CN_PREC_MIXED) return max_clusters_kc<float, 24, 8>(csize, block);
    return max_clusters_kc<double, 24, 8>(csize, block);
  }
  if (K == 3) {
    if (precision == CN_PREC_MIXED) return max_clusters_kc<float, 3, 1>(csize, block);
    return max_clusters_kc<double, 3, 1>(csize, block);
  }
  return 0;
}

}  // namespace cn
