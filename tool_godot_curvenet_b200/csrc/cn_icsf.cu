// cn_icsf.cu -- IC(0)-preconditioned CG with synchronisation-free triangular
// sweeps (sm_100a): the solve of an IC(0) handle in mixed precision (FP32
// inner solve) and, for large systems, in FP64.
//
// Same problem, right-hand sides, FP64 residual refinement and output as the
// level-scheduled persistent solve (cn_pcg.cu), and the same preconditioner:
// M = L~ L~^T with the handle's IC(0) factor (IncompleteCholesky.lean:30-101),
// applied as a forward sweep y = L~^-1 r and a backward sweep u = L~^-T y
// over the levels of the factor's lower-triangular graph.
//
// The level-scheduled kernel separates the levels by grid barriers (2 x
// levels per iteration).  Here no grid barrier separates them: every value a
// sweep publishes is stored together with the number of the preconditioner
// application it belongs to, one 64-bit word per column (the FP32 bits in
// the low half, the application number in the high half; FP64: two words,
// one per half of the double), and a row's
// thread reads its neighbours' words until every one carries the current
// number.  A naturally aligned 64-bit access is single-copy atomic, so a word
// with the current number holds the current value; no fence or flag orders
// the value and its number.  Each thread walks its own rows level by level
// (ascending in the forward sweep, descending in the backward one), and a
// row only waits for rows of lower (higher) levels, so by induction over the
// levels every wait ends (the launch is cooperative: all blocks co-resident).
// A block barrier closes each level: correctness needs only the numbers, but
// without it the polls of rows levels away from ready slowed the whole solve
// (each thread walking its rows on the numbers alone measured 1.7x slower).
//
// The CG is the single-reduction form of Chronopoulos & Gear ("s-step
// iterative methods for symmetric linear systems", J. Comput. Appl. Math.
// 25, 1989):
//
//   u = M^-1 r ; w = A u                       (sweeps and product, no barrier)
//   gamma = (r, u), delta = (w, u), ||r||^2    one reduction -> ONE grid barrier
//   beta = gamma / gamma' ; alpha = gamma / (delta - beta gamma / alpha')
//   p = u + beta p ; s = w + beta s ; x += alpha p ; r -= alpha s
//
// and the update of a row is done by its thread in the forward sweep, just
// before the row's y, so an iteration is: the forward sweep (with the
// update), the backward sweep, the product w = A u, the partial sums, one grid
// barrier.  A word of application a is overwritten only in application a + 1,
// which starts after a grid barrier that every reader of application a has
// passed, so no reader sees a value replaced too early.
//
// Ownership: the rows of level l are cut into one chunk of ceil(size / grid)
// consecutive rows per block (every block gets an equal share of every
// level); inside block b's chunk, position q goes to thread (q + o_l) mod
// blockDim, o_l the sum of the lower levels' chunk sizes.  A row's neighbours
// mostly belong to other blocks (about three quarters of the entries of L on
// the torus 512x256 workload); blocks owning mesh patches instead measured
// slower (the levels no longer split evenly).
//
// Every wait is bounded: it reads the global timer at its first poll and every
// 64th and the shared abort flag every 64th; a wait that runs out raises the
// abort flag, the others leave at their next check, and the solve ends with
// CN_TIMEOUT at the next block-uniform check.
#include "cn_pcg_body.cuh"

namespace cn {
namespace {

using namespace pcg;

constexpr int kIcsfMaxLev = 256;

__device__ __forceinline__ void ld_pair(const unsigned long long* p, unsigned long long& a, unsigned long long& b) {
  asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p));
}

__device__ __forceinline__ void st_pair(unsigned long long* p, unsigned long long a, unsigned long long b) {
  asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(a), "l"(b) : "memory");
}

__device__ __forceinline__ unsigned long long tag_bits(unsigned bits, unsigned app) {
  return ((unsigned long long)app << 32) | (unsigned long long)bits;
}

// The words of a row.  FP32: one word per column (value bits, number),
// K padded to an even count so a row is whole 16-byte pairs.  FP64: two
// words per column, the high and the low half of the value each with the
// number; a reader takes a column when both carry the current number (each
// half is written once per application, so both then come from it).
template <typename T, int K>
struct Words;

template <int K>
struct Words<float, K> {
  static constexpr int W = (K + 1) & ~1;  // words of a row
  static constexpr int N = W;             // words read
  static constexpr int R = K;             // words whose numbers are checked
  __device__ __forceinline__ static void load(const unsigned long long* p, unsigned long long (&x)[N]) {
#pragma unroll
    for (int i = 0; i < W; i += 2) ld_pair(p + i, x[i], x[i + 1]);
  }
  __device__ __forceinline__ static float value(const unsigned long long (&x)[N], int c) { return __uint_as_float((unsigned)x[c]); }
  __device__ __forceinline__ static void publish(unsigned long long* p, const float (&v)[K], unsigned app) {
#pragma unroll
    for (int i = 0; i < W / 2; ++i)
      st_pair(p + 2 * i, tag_bits(__float_as_uint(2 * i < K ? v[2 * i] : 0.f), app),
              tag_bits(__float_as_uint(2 * i + 1 < K ? v[2 * i + 1] : 0.f), app));
  }
};

template <int K>
struct Words<double, K> {
  static constexpr int W = 2 * K;
  static constexpr int N = 2 * K;
  static constexpr int R = 2 * K;
  __device__ __forceinline__ static void load(const unsigned long long* p, unsigned long long (&x)[N]) {
#pragma unroll
    for (int c = 0; c < K; ++c) ld_pair(p + 2 * c, x[2 * c], x[2 * c + 1]);
  }
  __device__ __forceinline__ static double value(const unsigned long long (&x)[N], int c) {
    return __hiloint2double((int)(unsigned)x[2 * c], (int)(unsigned)x[2 * c + 1]);
  }
  __device__ __forceinline__ static void publish(unsigned long long* p, const double (&v)[K], unsigned app) {
#pragma unroll
    for (int c = 0; c < K; ++c)
      st_pair(p + 2 * c, tag_bits((unsigned)__double2hiint(v[c]), app), tag_bits((unsigned)__double2loint(v[c]), app));
  }
};

template <typename T, int K>
__device__ __forceinline__ void publish(unsigned long long* words, int row, const T (&v)[K], unsigned app) {
  Words<T, K>::publish(words + (size_t)row * Words<T, K>::W, v, app);
}

// the first R words of x carry `app`
template <int R, int N>
__device__ __forceinline__ bool words_ready(const unsigned long long (&x)[N], unsigned app) {
  bool ok = true;
#pragma unroll
  for (int i = 0; i < R; ++i) ok = ok && (unsigned)(x[i] >> 32) == app;
  return ok;
}

// The bounded wait of one thread in one phase.
struct Spin {
  Control* ctl;
  long long limit_ns;
  unsigned long long t0;
  unsigned n;
  bool dead;
  // false: stop waiting (limit reached, or another wait raised the abort flag)
  __device__ __forceinline__ bool poll() {
    if (dead) return false;
    const unsigned k = n++;
    if (k == 0) {
      t0 = global_ns();
    } else if ((k & 63u) == 63u) {
      if (*(volatile int*)&ctl->abort) {
        dead = true;
        return false;
      }
      if ((long long)(global_ns() - t0) > limit_ns) {
        atomicExch(&ctl->abort, 1);
        dead = true;
        return false;
      }
    }
    return true;
  }
};

// acc[c] = sum over the row's entries e0..e1 of val[e] * word(col[e], c),
// every word read until it carries `app`.  U entries at a time: their indices
// and values, then all their words, then the waits and the multiply-adds in
// entry order.
template <typename T, int K, int U>
__device__ __forceinline__ void gather_tagged(int e0, int e1, const int* __restrict__ col, const T* __restrict__ val,
                                              const unsigned long long* words, unsigned app, Spin& sp,
                                              T (&acc)[K]) {
  using Wd = Words<T, K>;
  constexpr int W = Wd::W, N = Wd::N;
#pragma unroll
  for (int c = 0; c < K; ++c) acc[c] = (T)0;
  for (int e = e0; e < e1; e += U) {
    int j[U];
    T v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const bool ok = e + u < e1;
      j[u] = ok ? __ldg(col + e + u) : -1;
      v[u] = ok ? __ldg(val + e + u) : (T)0;
    }
    unsigned long long x[U][N];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (j[u] >= 0) {
        Wd::load(words + (size_t)j[u] * W, x[u]);
      } else {
#pragma unroll
        for (int i = 0; i < N; ++i) x[u][i] = (unsigned long long)app << 32;  // no entry: ready, value 0
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      for (;;) {
        if (words_ready<Wd::R>(x[u], app) || !sp.poll()) break;
        Wd::load(words + (size_t)j[u] * W, x[u]);
      }
#pragma unroll
      for (int c = 0; c < K; ++c) acc[c] += v[u] * Wd::value(x[u], c);
    }
  }
}

// Rows of level l owned by this thread: block b's chunk of the level,
// positions q = (t - o) mod B, q + B, ... below the chunk's row count.
struct LevelRows {
  int base, cnt, q0;
};

__device__ __forceinline__ LevelRows level_rows(const int* lev, const int* loff, int l) {
  const int lo = lev[l], hi = lev[l + 1];
  const int G = gridDim.x, B = blockDim.x;
  const int cs = (hi - lo + G - 1) / G;
  LevelRows r;
  r.base = lo + blockIdx.x * cs;
  r.cnt = min(cs, hi - r.base);
  int q0 = ((int)threadIdx.x - loff[l] % B) % B;
  if (q0 < 0) q0 += B;
  r.q0 = q0;
  return r;
}

template <int K>
struct IcsfSmem {
  double red[kMaxWarps * 3 * K];
  double sum[3 * K];
  double bb[K], stop[K], gprev[K], aprev[K], alpha[K], beta[K];
  int active[K];
  int flag;
  int abort;
  int lev[kIcsfMaxLev + 1];
  int loff[kIcsfMaxLev];  // ownership offset of each level: chunk sizes of the lower levels
};

// Sum the V values of every block's partials (V-wide records) in block order;
// result in sum[0..V).
template <int V>
__device__ void team_sum_wide(const double* part, int size, double* red, double* sum) {
  double v[V];
#pragma unroll
  for (int c = 0; c < V; ++c) v[c] = 0.0;
  for (int i = threadIdx.x; i < size * V; i += blockDim.x) {
    const double x = __ldcg(part + i);
    const int ci = i % V;
#pragma unroll
    for (int c = 0; c < V; ++c)
      if (c == ci) v[c] += x;
  }
  block_reduce_store<V>(v, red, sum);
}

template <typename T, int K>
__global__ void __launch_bounds__(512) k_icsf(SolveArgs a) {
  __shared__ IcsfSmem<K> s;
  GridTeam team{a.ctl, a.timeout_ns, 0u};
  const T* Aval = (const T*)a.A_val;
  const T* Lval = (const T*)a.L_val;
  const T* Uval = (const T*)a.U_val;
  const T* dinv = (const T*)a.dinv;
  T* r = (T*)a.r;
  T* u = (T*)a.z;   // M^-1 r of the own rows
  T* w = (T*)a.y;   // A u of the own rows
  T* p = (T*)a.p0;
  T* sv = (T*)a.Ap; // s = A p
  T* xin = (T*)a.xin;
  unsigned long long* yw = (unsigned long long*)a.m0;  // forward-sweep words
  unsigned long long* uw = (unsigned long long*)a.m1;  // backward-sweep words
  using Wd = Words<T, K>;
  constexpr int W = Wd::W;
  // entries whose words are in flight together: rows of L and U hold ~3
  // entries, rows of A ~7 (FP64: twice the words an entry)
  constexpr int kUL = K <= 3 && sizeof(T) == 4 ? 4 : 2;
  constexpr int kUA = K <= 3 ? (sizeof(T) == 4 ? 8 : 4) : 2;
  const int n = a.n, nlev = a.nlev;
  const int row0 = blockIdx.x * blockDim.x + threadIdx.x, rstride = gridDim.x * blockDim.x;
  const int tsize = gridDim.x;
  double* part = a.partials;
  int status = CN_OK, total_iters = 0, refinements = 0;
  unsigned app = 0;
  Spin sp{a.ctl, a.timeout_ns, 0ull, 0u, false};

  for (int i = threadIdx.x; i <= nlev; i += blockDim.x) s.lev[i] = a.lev_ptr[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    int o = 0;
    for (int l = 0; l < nlev; ++l) {
      s.loff[l] = o;
      o += (s.lev[l + 1] - s.lev[l] + (int)gridDim.x - 1) / (int)gridDim.x;
    }
  }
  __syncthreads();
  // every word starts with application number 0 (applications count from 1)
  for (size_t i = row0; i < (size_t)n * W; i += rstride) {
    yw[i] = 0ull;
    uw[i] = 0ull;
  }

  // ---- right-hand side (HarmonicSolve.lean:51-66 / DeformSolve.lean:123-135)
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
        gather_row<K, 1, 4>(a.K_ptr[v], a.K_ptr[v + 1], 0, a.K_col, a.K_val,
                            [&](int uu, double* d) {
                              const int h = a.hidx[uu];
#pragma unroll
                              for (int c = 0; c < K; ++c) {
                                const double rest = deform ? a.pos[3 * uu + c % 3] : 0.0;
                                d[c] = h >= 0 ? a.targets[(size_t)h * K + c] - rest : -rest;
                              }
                            },
                            acc);
      }
#pragma unroll
      for (int c = 0; c < K; ++c) {
        const double b = a.mode == CN_MODE_RHS ? a.targets[(size_t)row * K + c] : -acc[c];
        a.b64[(size_t)row * K + c] = b;
        bb[c] += b * b;
        if (!a.warm) a.x64[(size_t)row * K + c] = a.x0 ? a.x0[(size_t)v * K + c] : 0.0;
      }
    }
    block_reduce_store<K>(bb, s.red, part + (size_t)blockIdx.x * K);
    if (!team.sync()) { status = CN_TIMEOUT; goto done; }
    team_sum_wide<K>(part, tsize, s.red, s.sum);
    if (threadIdx.x < K) s.bb[threadIdx.x] = s.sum[threadIdx.x];
    __syncthreads();
  }

  for (int refine = 0;; ++refine) {
    // ---- FP64 residual r = b - A x (stays FP64)
    {
      double rr[K];
#pragma unroll
      for (int c = 0; c < K; ++c) rr[c] = 0.0;
      for (int row = row0; row < n; row += rstride) {
        double acc[K];
#pragma unroll
        for (int c = 0; c < K; ++c) acc[c] = 0.0;
        gather_row<K, 1, 4>(a.A_ptr[row], a.A_ptr[row + 1], 0, a.A_col, a.A_val64,
                            [&](int j, double* x) {
#pragma unroll
                              for (int c = 0; c < K; ++c) x[c] = a.x64[(size_t)j * K + c];
                            },
                            acc);
#pragma unroll
        for (int c = 0; c < K; ++c) {
          const double rv = a.b64[(size_t)row * K + c] - acc[c];
          r[(size_t)row * K + c] = (T)rv;
          xin[(size_t)row * K + c] = (T)0;
          rr[c] += rv * rv;
        }
      }
      double* pslot = part + (size_t)tsize * K;
      block_reduce_store<K>(rr, s.red, pslot + (size_t)blockIdx.x * K);
      if (!team.sync()) { status = CN_TIMEOUT; goto done; }
      team_sum_wide<K>(pslot, tsize, s.red, s.sum);
      if (threadIdx.x == 0) {
        int any = 0, bad = 0;
        for (int c = 0; c < K; ++c) {
          const double rr64 = s.sum[c], bb = s.bb[c];
          const double rel = bb > 0.0 ? sqrt(rr64 / bb) : sqrt(rr64);
          if (c < 32) a.stats->rel_residual[c] = rel;
          if (!(rel == rel)) bad = 1;
          const int act = rel > a.tol;
          s.active[c] = act;
          any |= act;
          const double want = bb > 0.0 ? 0.5 * a.tol * sqrt(bb / (rr64 > 0.0 ? rr64 : 1.0)) : 0.0;
          const double tau = fmax(a.inner_tol, want);
          s.stop[c] = tau * tau * rr64;
          s.alpha[c] = 0.0;
          s.beta[c] = 0.0;
        }
        s.flag = bad ? 2 : (any ? 1 : 0);
      }
      __syncthreads();
      if (s.flag == 2) { status = CN_NAN; break; }
      if (s.flag == 0) { status = CN_OK; break; }
      if (refine >= a.max_refine) { status = CN_MAX_ITER; break; }
      refinements = refine + 1;
    }

    // ---- inner single-reduction PCG in FP32
    int it = 0;
    bool first = true;
    for (;;) {
      T al[K], be[K];
#pragma unroll
      for (int c = 0; c < K; ++c) {
        al[c] = (T)s.alpha[c];
        be[c] = (T)s.beta[c];
      }
      ++app;
      sp.n = 0;

      // forward sweep y = L~^-1 r, the update of each row first; the top
      // level's u = y / L_ii is final and goes straight to the u words
      for (int l = 0; l < nlev; ++l) {
        const LevelRows lr = level_rows(s.lev, s.loff, l);
        const bool top = l == nlev - 1;
        for (int q = lr.q0; q < lr.cnt; q += blockDim.x) {
          const int row = lr.base + q;
          T rv[K];
          if (!first) {
#pragma unroll
            for (int c = 0; c < K; ++c) {
              const size_t ix = (size_t)row * K + c;
              // beta = 0 (an inner solve's first update, or an inactive
              // column): p = u, s = w, whatever the previous p, s hold
              const T pv = be[c] == (T)0 ? u[ix] : u[ix] + be[c] * p[ix];
              const T svv = be[c] == (T)0 ? w[ix] : w[ix] + be[c] * sv[ix];
              p[ix] = pv;
              sv[ix] = svv;
              xin[ix] += al[c] * pv;
              rv[c] = r[ix] - al[c] * svv;
              r[ix] = rv[c];
            }
          } else {
#pragma unroll
            for (int c = 0; c < K; ++c) rv[c] = r[(size_t)row * K + c];
          }
          T acc[K];
          gather_tagged<T, K, kUL>(a.L_ptr[row], a.L_ptr[row + 1], a.L_col, Lval, yw, app, sp, acc);
          const T di = dinv[row];
          T yv[K];
#pragma unroll
          for (int c = 0; c < K; ++c) yv[c] = (rv[c] - acc[c]) * di;
          if (top) {
            T uv[K];
#pragma unroll
            for (int c = 0; c < K; ++c) {
              uv[c] = yv[c] * di;
              u[(size_t)row * K + c] = uv[c];
            }
            publish<T, K>(uw, row, uv, app);
          } else {
            publish<T, K>(yw, row, yv, app);
          }
        }
        // the block's rows of this level are published before any of its
        // rows of the next level reads them; rows of other blocks carry
        // their application number
        __syncthreads();
      }
      // backward sweep u = L~^-T y, levels nlev-2 .. 0 (own y from the words)
      for (int l = nlev - 2; l >= 0; --l) {
        const LevelRows lr = level_rows(s.lev, s.loff, l);
        for (int q = lr.q0; q < lr.cnt; q += blockDim.x) {
          const int row = lr.base + q;
          // the row's own y (this thread's words) before the waits
          unsigned long long yx[Wd::N];
          Wd::load(yw + (size_t)row * W, yx);
          const T di = dinv[row];
          T acc[K];
          gather_tagged<T, K, kUL>(a.U_ptr[row], a.U_ptr[row + 1], a.U_col, Uval, uw, app, sp, acc);
          T uv[K];
#pragma unroll
          for (int c = 0; c < K; ++c) {
            uv[c] = (Wd::value(yx, c) - acc[c]) * di;
            u[(size_t)row * K + c] = uv[c];
          }
          publish<T, K>(uw, row, uv, app);
        }
        __syncthreads();
      }
      // w = A u and the partial sums (r, u), (w, u), ||r||^2
      double ga[K], de[K], rr[K];
#pragma unroll
      for (int c = 0; c < K; ++c) { ga[c] = 0.0; de[c] = 0.0; rr[c] = 0.0; }
      for (int l = 0; l < nlev; ++l) {
        const LevelRows lr = level_rows(s.lev, s.loff, l);
        for (int q = lr.q0; q < lr.cnt; q += blockDim.x) {
          const int row = lr.base + q;
          T acc[K];
          gather_tagged<T, K, kUA>(a.A_ptr[row], a.A_ptr[row + 1], a.A_col, Aval, uw, app, sp, acc);
#pragma unroll
          for (int c = 0; c < K; ++c) {
            const size_t ix = (size_t)row * K + c;
            w[ix] = acc[c];
            const double uu = (double)u[ix], rv = (double)r[ix];
            ga[c] += rv * uu;
            de[c] += (double)acc[c] * uu;
            rr[c] += rv * rv;
          }
        }
      }
      {
        double v[3 * K];
#pragma unroll
        for (int c = 0; c < K; ++c) { v[c] = ga[c]; v[K + c] = de[c]; v[2 * K + c] = rr[c]; }
        // partials alternate between two 3K-wide tables by iteration parity
        double* pslot = part + (size_t)tsize * K * (2 + 3 * (app & 1u));
        block_reduce_store<3 * K>(v, s.red, pslot + (size_t)blockIdx.x * 3 * K);
        // a wait of this iteration that gave up (here or in another block)
        // ends the solve; the decision is the block's, read once
        if (threadIdx.x == 0) s.abort = *(volatile int*)&a.ctl->abort;
        __syncthreads();
        if (s.abort) { status = CN_TIMEOUT; goto done; }
        if (!team.sync()) { status = CN_TIMEOUT; goto done; }
        team_sum_wide<3 * K>(pslot, tsize, s.red, s.sum);
      }
      if (threadIdx.x == 0) {
        int any = 0, bad = 0;
        for (int c = 0; c < K; ++c) {
          const double g = s.sum[c], d = s.sum[K + c], rrv = s.sum[2 * K + c];
          if (!(g == g) || !(d == d) || !(rrv == rrv)) bad = 1;
          if (!first && s.active[c] && rrv < s.stop[c]) s.active[c] = 0;
          double be2 = 0.0, al2 = 0.0;
          if (s.active[c]) {
            be2 = first || s.gprev[c] == 0.0 ? 0.0 : g / s.gprev[c];
            const double den = first ? d : d - be2 * g / s.aprev[c];
            // SparseLinAlg.lean:118 stops on pAp == 0; a non-positive
            // curvature ends this column's inner solve (the next FP64
            // residual decides whether it restarts)
            if (den > 0.0) al2 = g / den;
            else s.active[c] = 0;
          }
          if (!s.active[c]) { be2 = 0.0; al2 = 0.0; }
          s.beta[c] = be2;
          s.alpha[c] = al2;
          s.gprev[c] = g;
          if (al2 != 0.0) s.aprev[c] = al2;
          any |= s.active[c];
        }
        s.flag = bad ? 2 : (any ? 1 : 0);
      }
      __syncthreads();
      if (s.flag == 2) { status = CN_NAN; goto done; }
      if (s.flag == 0 || it >= a.max_iter) break;
      // the update of the next forward sweep is this iteration
      ++it;
      ++total_iters;
      first = false;
    }
    // ---- x64 += xin (FP64 accumulation of the correction), own rows
    {
      for (int l = 0; l < nlev; ++l) {
        const LevelRows lr = level_rows(s.lev, s.loff, l);
        for (int q = lr.q0; q < lr.cnt; q += blockDim.x) {
          const int row = lr.base + q;
#pragma unroll
          for (int c = 0; c < K; ++c) {
            const size_t ix = (size_t)row * K + c;
            a.x64[ix] += (double)xin[ix];
          }
        }
      }
    }
    if (!team.sync()) { status = CN_TIMEOUT; goto done; }
  }

  // ---- output: free rows, then the handle overlay (DeformSolve.lean:108-109)
  if (a.x_out) {
    for (int row = row0; row < n; row += rstride) {
      const int v = a.free_of[row];
#pragma unroll
      for (int c = 0; c < K; ++c) a.x_out[(size_t)v * K + c] = a.x64[(size_t)row * K + c];
    }
    for (int h = row0; h < a.nh; h += rstride) {
      const int v = a.handles[h];
#pragma unroll
      for (int c = 0; c < K; ++c)
        a.x_out[(size_t)v * K + c] = a.mode == CN_MODE_RHS ? 0.0 : a.targets[(size_t)h * K + c];
    }
  }

done:
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.stats->status = status;
    a.stats->iterations = total_iters;
    a.stats->refinements = refinements;
  }
}

template <typename T, int K>
cudaError_t launch_k(const SolveArgs& a, int block, int grid, cudaStream_t st) {
  SolveArgs copy = a;
  void* args[] = {&copy};
  return cudaLaunchCooperativeKernel((const void*)k_icsf<T, K>, dim3(grid), dim3(block), args, 0, st);
}

template <typename T, int K>
int max_grid_k(int block) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_icsf<T, K>, block, 0);
  return sms * per;
}

}  // namespace

int icsf_max_levels() { return kIcsfMaxLev; }

cudaError_t launch_icsf_solve(const SolveArgs& a, int precision, int K, int block, int grid, cudaStream_t s) {
  if (a.nlev > kIcsfMaxLev || grid < 1 || block > 512) return cudaErrorInvalidValue;
  if (precision == CN_PREC_MIXED) {
    if (K == 1) return launch_k<float, 1>(a, block, grid, s);
    if (K == 3) return launch_k<float, 3>(a, block, grid, s);
  } else {
    if (K == 1) return launch_k<double, 1>(a, block, grid, s);
    if (K == 3) return launch_k<double, 3>(a, block, grid, s);
  }
  return cudaErrorInvalidValue;
}

int icsf_max_grid(int precision, int K, int block) {
  if (precision == CN_PREC_MIXED) {
    if (K == 1) return max_grid_k<float, 1>(block);
    if (K == 3) return max_grid_k<float, 3>(block);
  } else {
    if (K == 1) return max_grid_k<double, 1>(block);
    if (K == 3) return max_grid_k<double, 3>(block);
  }
  return 0;
}

}  // namespace cn
