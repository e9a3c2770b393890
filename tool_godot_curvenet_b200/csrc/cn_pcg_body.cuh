// cn_pcg_body.cuh -- the device code of the persistent preconditioned-CG
// solve (team barriers, deterministic reductions, the solve body), shared by
// the kernels of cn_pcg.cu and cn_noalloc.cu.  See cn_pcg.cu for the
// algorithm.
#pragma once

#include "cn_internal.h"

namespace cn {
namespace pcg {


__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// All blocks of a cooperative grid.  A monotonic arrival counter: barrier
// number e completes when the counter reaches e * gridDim.x (the host zeroes
// it before the launch).  Each block's thread 0 adds 1 with a fire-and-forget
// reduction after a fence, then polls with acquire loads; the wait is bounded
// by timeout_ns (checked at the first poll and every 64th) and by the shared
// abort flag (set by the first block whose wait runs out; the others leave
// at their next wait).
struct GridTeam {
  Control* ctl;
  long long timeout_ns;
  mutable unsigned epoch;
  __device__ __forceinline__ int rank() const { return blockIdx.x; }
  __device__ __forceinline__ int size() const { return gridDim.x; }
  __device__ bool sync() const {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
      int ok = 1;
      ++epoch;
      const unsigned target = epoch * gridDim.x;
      __threadfence();
      asm volatile("red.relaxed.gpu.global.add.u32 [%0], 1;" ::"l"(&ctl->bar_count) : "memory");
      if (ld_acquire_u32(&ctl->bar_count) < target) {
        const unsigned long long t0 = global_ns();
        unsigned spins = 0;
        while (ld_acquire_u32(&ctl->bar_count) < target) {
          // the clock at the first poll (a limit shorter than one barrier
          // ends the solve at its first barrier) and then with the abort
          // flag every 64th: reading the global timer at every poll spaced
          // the polls out and lengthened every barrier
          const unsigned sp = spins++;
          if (sp == 0 || (sp & 63u) == 63u) {
            if ((long long)(global_ns() - t0) > timeout_ns) {
              atomicExch(&ctl->abort, 1);
              ok = 0;
              break;
            }
            if (sp != 0 && *(volatile int*)&ctl->abort) { ok = 0; break; }
          }
        }
      }
      s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
  }
};

// One block solving alone: the barrier is __syncthreads.
struct CtaTeam {
  __device__ __forceinline__ int rank() const { return 0; }
  __device__ __forceinline__ int size() const { return 1; }
  __device__ __forceinline__ bool sync() const {
    __syncthreads();
    return true;
  }
};

constexpr int kMaxWarps = 32;

enum Slot { kBB = 0, kRR64 = 1, kPAP = 2, kRR = 3, kRZ = 4 };

template <int K>
struct Smem {
  double red[kMaxWarps * K];
  double sum[K];
  double alpha[K], beta[K], rz[K], rr0[K], bb[K], stop[K];
  int active[K];
  int flag;
};

// Sum v[0..K) over the block (warp shuffles, then one warp over the warp
// partials) and store it to out[0..K) from thread 0.  Fixed order.
template <int K>
__device__ void block_reduce_store(double (&v)[K], double* red, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int c = 0; c < K; ++c) {
    double t = v[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) red[warp * K + c] = t;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int c = 0; c < K; ++c) {
      double t = lane < nw ? red[lane * K + c] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (lane == 0) out[c] = t;
    }
  }
  __syncthreads();
}

// After a barrier: every block adds the team's partials of one slot; every
// thread loads at most a few partials (independent loads, one L2 latency),
// then a fixed-order block reduction lands the K sums in s->sum.
template <int K>
__device__ void team_sum(const double* part, int size, Smem<K>* s) {
  double v[K];
#pragma unroll
  for (int c = 0; c < K; ++c) v[c] = 0.0;
  const int tot = size * K;
  for (int i = threadIdx.x; i < tot; i += blockDim.x) {
    const double x = __ldcg(part + i);
    const int ci = i % K;
#pragma unroll
    for (int c = 0; c < K; ++c)
      if (c == ci) v[c] += x;
  }
  block_reduce_store<K>(v, s->red, s->sum);
}

template <int G>
__device__ __forceinline__ unsigned group_mask() {
  if (G == 32) return 0xffffffffu;
  const unsigned lane = threadIdx.x & 31;
  return ((1u << G) - 1u) << (lane & ~(unsigned)(G - 1));
}

template <int G, typename V>
__device__ __forceinline__ V group_sum(V v, unsigned mask) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
  return v;
}

// acc[c] += sum of val[e] * X(col[e], c) over this lane's entries of a row
// (e = e0 + sub, e0 + sub + G, ... < e1).  Up to U entries at a time: their
// column indices and values are loaded first, then all U gathers are issued
// before any of them is used, so one row costs about two dependent memory
// latencies instead of two per entry.  Entries past e1 contribute zero and
// read nothing.
template <int K, int G, int U, typename V, typename A, typename F>
__device__ __forceinline__ void gather_row(int e0, int e1, int sub, const int* __restrict__ col,
                                           const V* __restrict__ val, F&& load, A (&acc)[K]) {
  for (int e = e0 + sub; e < e1; e += G * U) {
    int j[U];
    A w[U];
    bool ok[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int ee = e + u * G;
      ok[u] = ee < e1;
      j[u] = ok[u] ? col[ee] : 0;
      w[u] = ok[u] ? (A)val[ee] : (A)0;
    }
    A x[U][K];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (ok[u]) {
        load(j[u], x[u]);
      } else {
#pragma unroll
        for (int c = 0; c < K; ++c) x[u][c] = (A)0;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int c = 0; c < K; ++c) acc[c] += w[u] * x[u][c];
  }
}

template <typename T, int K, int G, class Team>
__device__ void solve_body(const SolveArgs& a, const Team& team, Smem<K>* s) {
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
  const int gpb = blockDim.x / G;
  const int grp = threadIdx.x / G, sub = threadIdx.x % G;
  const int row0 = team.rank() * gpb + grp, rstride = team.size() * gpb;
  const unsigned gmask = group_mask<G>();
  const int tsize = team.size();
  double* part = a.partials;
  auto slot_ptr = [&](int slot) { return part + ((size_t)slot * tsize) * K; };
  auto write_partial = [&](int slot, double (&v)[K]) {
    block_reduce_store<K>(v, s->red, slot_ptr(slot) + (size_t)team.rank() * K);
  };
  int status = CN_OK, total_iters = 0, refinements = 0;
  // entries gathered together per lane: a row of ~7 entries in one or two passes
  constexpr int UR = K <= 3 ? (G >= 8 ? 1 : 8 / G) : 2;

  // ---- phase A: right-hand side (HarmonicSolve.lean:51-66 / DeformSolve.lean:123-135)
  {
    double bb[K];
#pragma unroll
    for (int c = 0; c < K; ++c) bb[c] = 0.0;
    for (int row = row0; row < n; row += rstride) {
      double acc[K];
#pragma unroll
      for (int c = 0; c < K; ++c) acc[c] = 0.0;
      const int v = a.free_of[row];
      if (a.mode != CN_MODE_RHS) {
        const bool deform = a.mode == CN_MODE_DEFORM;
        gather_row<K, G, UR>(a.K_ptr[v], a.K_ptr[v + 1], sub, a.K_col, a.K_val,
                             [&](int u, double* d) {
                               const int h = a.hidx[u];
#pragma unroll
                               for (int c = 0; c < K; ++c) {
                                 const double rest = deform ? a.pos[3 * u + c % 3] : 0.0;
                                 d[c] = h >= 0 ? a.targets[(size_t)h * K + c] - rest : -rest;
                               }
                             },
                             acc);
      }
#pragma unroll
      for (int c = 0; c < K; ++c) acc[c] = group_sum<G>(acc[c], gmask);
      if (sub == 0) {
#pragma unroll
        for (int c = 0; c < K; ++c) {
          const double b = a.mode == CN_MODE_RHS ? a.targets[(size_t)row * K + c] : -acc[c];
          a.b64[(size_t)row * K + c] = b;
          bb[c] += b * b;
          if (!a.warm) a.x64[(size_t)row * K + c] = a.x0 ? a.x0[(size_t)v * K + c] : 0.0;
        }
      }
    }
    write_partial(kBB, bb);
    if (!team.sync()) { status = CN_TIMEOUT; goto done; }
    team_sum<K>(slot_ptr(kBB), tsize, s);
    if (threadIdx.x < K) s->bb[threadIdx.x] = s->sum[threadIdx.x];
    __syncthreads();
  }

  for (int refine = 0;; ++refine) {
    // ---- phase R: FP64 residual r = b - A x (stays FP64 in every precision)
    {
      double rr[K];
#pragma unroll
      for (int c = 0; c < K; ++c) rr[c] = 0.0;
      for (int row = row0; row < n; row += rstride) {
        double acc[K];
#pragma unroll
        for (int c = 0; c < K; ++c) acc[c] = 0.0;
        gather_row<K, G, UR>(a.A_ptr[row], a.A_ptr[row + 1], sub, a.A_col, a.A_val64,
                             [&](int j, double* x) {
#pragma unroll
                               for (int c = 0; c < K; ++c) x[c] = a.x64[(size_t)j * K + c];
                             },
                             acc);
#pragma unroll
        for (int c = 0; c < K; ++c) acc[c] = group_sum<G>(acc[c], gmask);
        if (sub == 0) {
#pragma unroll
          for (int c = 0; c < K; ++c) {
            const double rv = a.b64[(size_t)row * K + c] - acc[c];
            r[(size_t)row * K + c] = (T)rv;
            xin[(size_t)row * K + c] = (T)0;
            rr[c] += rv * rv;
          }
        }
      }
      write_partial(kRR64, rr);
      if (!team.sync()) { status = CN_TIMEOUT; goto done; }
      team_sum<K>(slot_ptr(kRR64), tsize, s);
      if (threadIdx.x == 0) {
        int any = 0, bad = 0;
        for (int c = 0; c < K; ++c) {
          const double rr64 = s->sum[c], bb = s->bb[c];
          const double rel = bb > 0.0 ? sqrt(rr64 / bb) : sqrt(rr64);
          if (c < 32) a.stats->rel_residual[c] = rel;
          if (!(rel == rel)) bad = 1;
          const int act = rel > a.tol;
          s->active[c] = act;
          any |= act;
          s->rr0[c] = rr64;
          // inner stopping threshold on ||r||^2 of this refinement step
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
      // max_refine bounds the number of inner solves
      if (refine >= a.max_refine) { status = CN_MAX_ITER; break; }
      refinements = refine + 1;
    }

    // ---- initial preconditioning z = M^{-1} r (sweeps without the update)
    // then the inner PCG iterations.
    int it = 0;
    bool first = true;
    for (;;) {
      // SPMV (skipped before the first preconditioning)
      if (!first) {
        double pap[K];
#pragma unroll
        for (int c = 0; c < K; ++c) pap[c] = 0.0;
        T beta[K];
        bool b0 = true;
#pragma unroll
        for (int c = 0; c < K; ++c) { beta[c] = (T)s->beta[c]; b0 = b0 && s->beta[c] == 0.0; }
        const T* pold = (it & 1) ? pb : pa;
        T* pnew = (it & 1) ? pa : pb;
        for (int row = row0; row < n; row += rstride) {
          T acc[K];
#pragma unroll
          for (int c = 0; c < K; ++c) acc[c] = (T)0;
          // A p = A z + beta A p_old: only z is gathered, A p_old is the
          // row's own entry of Ap
          gather_row<K, G, UR>(a.A_ptr[row], a.A_ptr[row + 1], sub, a.A_col, Aval,
                               [&](int j, T* x) {
#pragma unroll
                                 for (int c = 0; c < K; ++c) x[c] = z[(size_t)j * K + c];
                               },
                               acc);
#pragma unroll
          for (int c = 0; c < K; ++c) acc[c] = group_sum<G>(acc[c], gmask);
          if (sub == 0) {
#pragma unroll
            for (int c = 0; c < K; ++c) {
              const size_t ix = (size_t)row * K + c;
              T pi = z[ix];
              if (!b0) pi += beta[c] * pold[ix];
              const T api = b0 ? acc[c] : acc[c] + beta[c] * Ap[ix];
              pnew[ix] = pi;
              Ap[ix] = api;
              pap[c] += (double)pi * (double)api;
            }
          }
        }
        write_partial(kPAP, pap);
        if (!team.sync()) { status = CN_TIMEOUT; goto done; }
        team_sum<K>(slot_ptr(kPAP), tsize, s);
        if (threadIdx.x == 0) {
          for (int c = 0; c < K; ++c) {
            const double v = s->sum[c];
            // SparseLinAlg.lean:118 stops on pAp == 0; a non-positive value
            // ends this column's inner solve (the next FP64 residual decides
            // whether it restarts).
            if (s->active[c] && !(v > 0.0)) s->active[c] = 0;
            s->alpha[c] = s->active[c] ? s->rz[c] / v : 0.0;
          }
        }
        __syncthreads();
      }

      // FWD sweeps by level; the last level also finishes z.
      const T* pcur = (it & 1) ? pa : pb;
      double rrp[K], rzp[K];
#pragma unroll
      for (int c = 0; c < K; ++c) { rrp[c] = 0.0; rzp[c] = 0.0; }
      T alpha[K];
#pragma unroll
      for (int c = 0; c < K; ++c) alpha[c] = (T)s->alpha[c];
      if (a.hsc) {
        // HSC V-cycle (the block-LDL^T solve of the hierarchy): w = r (with
        // the CG update), down the levels w_C -= R w_F, the coarse
        // z_c = S^{-1} w_c, up the levels z_F = D_F^{-1} (w_F - P z_C).
        T* w = y;
        const T* Rv = (const T*)a.hsc_rval;
        const T* Pv = (const T*)a.hsc_pval;
        const T* hd = (const T*)a.hsc_dinv;
        const T* Si = (const T*)a.hsc_sinv;
        for (int row = row0; row < n; row += rstride) {
          if (sub == 0) {
#pragma unroll
            for (int c = 0; c < K; ++c) {
              const size_t ix = (size_t)row * K + c;
              T rv = r[ix];
              if (!first) {
                xin[ix] += alpha[c] * pcur[ix];
                rv -= alpha[c] * Ap[ix];
                r[ix] = rv;
              }
              w[ix] = rv;
              rrp[c] += (double)rv * (double)rv;
            }
          }
        }
        if (!team.sync()) { status = CN_TIMEOUT; goto done; }
        const int HL = a.hsc_L, tail = a.hsc_tail;
        auto down = [&](int l, int q0, int qs) {
          for (int q = a.hsc_rlev[l] + q0; q < a.hsc_rlev[l + 1]; q += qs) {
            T acc[K];
#pragma unroll
            for (int c = 0; c < K; ++c) acc[c] = (T)0;
            gather_row<K, G, UR>(a.hsc_rptr[q], a.hsc_rptr[q + 1], sub, a.hsc_rcol, Rv,
                                 [&](int j, T* x) {
#pragma unroll
                                   for (int c = 0; c < K; ++c) x[c] = w[(size_t)j * K + c];
                                 },
                                 acc);
#pragma unroll
            for (int c = 0; c < K; ++c) acc[c] = group_sum<G>(acc[c], gmask);
            if (sub == 0) {
              const int i = a.hsc_rrow[q];
#pragma unroll
              for (int c = 0; c < K; ++c) w[(size_t)i * K + c] -= acc[c];
            }
          }
        };
        auto up = [&](int l, int v0, int vs) {
          for (int v = a.hsc_off[l] + v0; v < a.hsc_off[l + 1]; v += vs) {
            T acc[K];
#pragma unroll
            for (int c = 0; c < K; ++c) acc[c] = (T)0;
            gather_row<K, G, UR>(a.hsc_pptr[v], a.hsc_pptr[v + 1], sub, a.hsc_pcol, Pv,
                                 [&](int j, T* x) {
#pragma unroll
                                   for (int c = 0; c < K; ++c) x[c] = z[(size_t)j * K + c];
                                 },
                                 acc);
#pragma unroll
            for (int c = 0; c < K; ++c) acc[c] = group_sum<G>(acc[c], gmask);
            if (sub == 0) {
              const T di = hd[v];
#pragma unroll
              for (int c = 0; c < K; ++c) {
                const size_t ix = (size_t)v * K + c;
                const T zv = (w[ix] - acc[c]) * di;
                z[ix] = zv;
                rzp[c] += (double)r[ix] * (double)zv;
              }
            }
          }
        };
        for (int l = 0; l < tail; ++l) {
          down(l, row0, rstride);
          if (!team.sync()) { status = CN_TIMEOUT; goto done; }
        }
        if (team.rank() == 0) {
          // the small levels and the dense coarse solve: one block,
          // __syncthreads between the steps
          for (int l = tail; l < HL; ++l) {
            down(l, grp, gpb);
            __syncthreads();
          }
          const int co = a.hsc_off[HL], nc = a.hsc_nc;
          const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
          for (int i = co + warp; i < n; i += nw) {
            T acc[K];
#pragma unroll
            for (int c = 0; c < K; ++c) acc[c] = (T)0;
            const T* srow = Si + (size_t)(i - co) * nc;
            for (int j = lane; j < nc; j += 32) {
              const T sv = srow[j];
#pragma unroll
              for (int c = 0; c < K; ++c) acc[c] += sv * w[(size_t)(co + j) * K + c];
            }
#pragma unroll
            for (int c = 0; c < K; ++c)
#pragma unroll
              for (int o = 16; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
            if (lane == 0) {
#pragma unroll
              for (int c = 0; c < K; ++c) {
                const size_t ix = (size_t)i * K + c;
                z[ix] = acc[c];
                rzp[c] += (double)r[ix] * (double)acc[c];
              }
            }
          }
          __syncthreads();
          for (int l = HL - 1; l >= tail; --l) {
            up(l, grp, gpb);
            __syncthreads();
          }
        }
        for (int l = tail - 1; l >= 0; --l) {
          if (!team.sync()) { status = CN_TIMEOUT; goto done; }
          up(l, row0, rstride);
        }
      } else {
      for (int l = 0; l < nlev; ++l) {
        const int lo = a.lev_ptr[l], hi = a.lev_ptr[l + 1];
        const bool last = l == nlev - 1;
        for (int row = lo + row0; row < hi; row += rstride) {
          T acc[K];
#pragma unroll
          for (int c = 0; c < K; ++c) acc[c] = (T)0;
          gather_row<K, G, UR>(a.L_ptr[row], a.L_ptr[row + 1], sub, a.L_col, Lval,
                               [&](int j, T* x) {
#pragma unroll
                                 for (int c = 0; c < K; ++c) x[c] = y[(size_t)j * K + c];
                               },
                               acc);
#pragma unroll
          for (int c = 0; c < K; ++c) acc[c] = group_sum<G>(acc[c], gmask);
          if (sub == 0) {
            const T di = dinv[row];
#pragma unroll
            for (int c = 0; c < K; ++c) {
              const size_t ix = (size_t)row * K + c;
              T rv = r[ix];
              if (!first) {
                xin[ix] += alpha[c] * pcur[ix];
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
        }
        if (!last) {
          if (!team.sync()) { status = CN_TIMEOUT; goto done; }
        }
      }
      // BWD sweeps, levels nlev-2 .. 0 (each needs the later levels' z).
      for (int l = nlev - 2; l >= 0; --l) {
        if (!team.sync()) { status = CN_TIMEOUT; goto done; }
        const int lo = a.lev_ptr[l], hi = a.lev_ptr[l + 1];
        for (int row = lo + row0; row < hi; row += rstride) {
          T acc[K];
#pragma unroll
          for (int c = 0; c < K; ++c) acc[c] = (T)0;
          gather_row<K, G, UR>(a.U_ptr[row], a.U_ptr[row + 1], sub, a.U_col, Uval,
                               [&](int j, T* x) {
#pragma unroll
                                 for (int c = 0; c < K; ++c) x[c] = z[(size_t)j * K + c];
                               },
                               acc);
#pragma unroll
          for (int c = 0; c < K; ++c) acc[c] = group_sum<G>(acc[c], gmask);
          if (sub == 0) {
            const T di = dinv[row];
#pragma unroll
            for (int c = 0; c < K; ++c) {
              const size_t ix = (size_t)row * K + c;
              z[ix] = (y[ix] - acc[c]) * di;
            }
          }
        }
      }
      }  // IC(0) / Jacobi sweeps
      write_partial(kRR, rrp);
      write_partial(kRZ, rzp);
      if (!team.sync()) { status = CN_TIMEOUT; goto done; }
      team_sum<K>(slot_ptr(kRR), tsize, s);
      double rrv[K];
#pragma unroll
      for (int c = 0; c < K; ++c) rrv[c] = s->sum[c];
      __syncthreads();
      team_sum<K>(slot_ptr(kRZ), tsize, s);
      if (threadIdx.x == 0) {
        int any = 0, bad = 0;
        for (int c = 0; c < K; ++c) {
          const double rzn = s->sum[c];
          if (!(rrv[c] == rrv[c]) || !(rzn == rzn)) bad = 1;
          if (!first && s->active[c] && rrv[c] < s->stop[c]) s->active[c] = 0;
          s->beta[c] = first ? 0.0 : (s->rz[c] == 0.0 ? 0.0 : rzn / s->rz[c]);
          s->rz[c] = rzn;
          any |= s->active[c];
        }
        s->flag = bad ? 2 : (any ? 1 : 0);
      }
      __syncthreads();
      if (!first) {
        ++it;
        ++total_iters;
      }
      if (s->flag == 2) { status = CN_NAN; goto done; }
      first = false;
      if (s->flag == 0 || it >= a.max_iter) break;
    }
    // ---- x64 += xin (FP64 accumulation of the correction)
    for (int row = row0; row < n; row += rstride) {
      if (sub == 0) {
#pragma unroll
        for (int c = 0; c < K; ++c) {
          const size_t ix = (size_t)row * K + c;
          a.x64[ix] += (double)xin[ix];
        }
      }
    }
    if (!team.sync()) { status = CN_TIMEOUT; goto done; }
  }

  // ---- output: free rows, then the handle overlay (DeformSolve.lean:108-109)
  if (a.x_out) {
    for (int row = row0; row < n; row += rstride)
      if (sub == 0) {
        const int v = a.free_of[row];
#pragma unroll
        for (int c = 0; c < K; ++c) a.x_out[(size_t)v * K + c] = a.x64[(size_t)row * K + c];
      }
    for (int h = row0; h < a.nh; h += rstride)
      if (sub == 0) {
        const int v = a.handles[h];
#pragma unroll
        for (int c = 0; c < K; ++c)
          a.x_out[(size_t)v * K + c] = a.mode == CN_MODE_RHS ? 0.0 : a.targets[(size_t)h * K + c];
      }
  }

done:
  if (team.rank() == 0 && threadIdx.x == 0) {
    a.stats->status = status;
    a.stats->iterations = total_iters;
    a.stats->refinements = refinements;
  }
}

}  // namespace pcg
}  // namespace cn
