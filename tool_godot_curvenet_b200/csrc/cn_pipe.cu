// cn_pipe.cu -- the row-cached persistent PCG solve (sm_100a): Jacobi or
// block SSOR, two CG forms.
//
// Same problem, right-hand sides, FP64 residual refinement and output as the
// level-scheduled persistent solve (cn_pcg.cu).  Each thread owns the rows
// b Qg B + q B + t (q < Qg) of its block b for the whole launch, and the
// block keeps its rows of A (column index and T value) in shared memory (one
// ELL slice per row slice, column-major, padding column -1) and, when it
// fits, their CG state, so a row costs one L2 round trip (the gathers of the
// vector its neighbours need) per phase.
//
// Pipelined form (Jacobi only): the preconditioned CG of Ghysels & Vanroose
// ("Hiding global synchronization latency in the preconditioned Conjugate
// Gradient algorithm", Parallel Computing 40, 2014, Alg. 4) with M = diag(A):
//
//   gamma = (r, u), delta = (w, u)               one reduction per iteration
//   m = M^-1 w ; n = A m                         overlaps that reduction
//   beta = gamma / gamma' ; alpha = gamma / (delta - beta gamma / alpha')
//   z = n + beta z ; s = w + beta s ; p = u + beta p
//   x += alpha p ; r -= alpha s ; w -= alpha z ; u = M^-1 r
//
// (with a diagonal M the recurrences u -= alpha q, q = m + beta q of the
// general form reduce to u = M^-1 r, so q is not kept).  An iteration is ONE
// phase between two team barriers: after the barrier a block issues the
// gathers of m (its rows' neighbours, written by their owners in the
// previous phase) and, in the same memory round trip, three warps sum the
// previous phase's partials (gamma, delta, ||r||^2 per column, a fixed
// order, so every block derives the same alpha, beta and stopping decision);
// the own rows update, store m' = M^-1 w' into the other copy of m, and the
// block's partial sums are written before the next barrier.
//
// Two-reduction form (Jacobi or block SSOR): phase S gathers z, forms
// p = z + beta p' and A p = A z + beta A p', (p, Ap); phase U updates x and
// r, applies z = M^-1 r (inline for Jacobi, by the block's colour sweeps in
// shared memory for block SSOR), (r, z) and ||r||^2.
//
// Single-reduction form (Jacobi or block SSOR; Chronopoulos & Gear, "s-step
// iterative methods for symmetric linear systems", J. Comput. Appl. Math. 25,
// 1989): one reduction of gamma = (r, z), delta = (z, A z) and ||r||^2 per
// iteration and ONE grid barrier; alpha = gamma / (delta - beta gamma /
// alpha'), beta = gamma / gamma', A p by s = A z + beta s'.  The exchange of
// z between the reduction's barriers is point to point: a block publishes
// its z with a release flag (an epoch count) and waits, with acquire loads,
// only for the flags of the blocks its rows couple to.
//
// Partial sums alternate between two slot groups by phase parity (a block
// may write phase i+1's partials while a slower block still reads phase i's);
// the gathered vectors alternate between two buffers for the same reason.
#include <algorithm>
#include <set>
#include <tuple>
#include <type_traits>
#include <vector>

#include "cn_pcg_body.cuh"

namespace cn {
namespace {

using namespace pcg;

// Row of m as gathered: K values padded to a multiple of 16 bytes.
template <typename T, int K>
struct MRow {
  static constexpr int W = ((K * (int)sizeof(T) + 15) / 16) * 16 / (int)sizeof(T);
  static constexpr int NC = W * (int)sizeof(T) / 16;
};

constexpr int kPipeSplits = 8;  // partial-sum read: up to 8 x 128 blocks
constexpr int kNbrWords = 64;        // single-reduction form: neighbour-block bitmap (up to 2048 blocks)
constexpr int kMaxNbrBlocks = 64;    // neighbour blocks a block waits for one by one
constexpr int kMaxColours = 64;   // block SSOR: colours of a block (greedy: at most the row length)
constexpr int kSweepRows = 4;     // block SSOR, tables in global memory: rows a thread sweeps at a time
// The pipelined recurrences in FP32 lose track of the true residual below
// about 1e-4 of the starting one, so each refinement step of the mixed solve
// asks the inner solve for at most this much reduction.
constexpr double kPipeInnerFloor = 1e-3;

template <int K>
struct PipeSmem {
  Smem<K> sm;
  double red2[kMaxWarps * 3 * K];
  double psum[3 * K][kPipeSplits];
  // single-reduction form: the other blocks whose rows this block's rows
  // couple to (bitmap over blocks, then the list; nbn < 0: more than
  // kMaxNbrBlocks, the z exchange then waits at a grid barrier)
  unsigned nbm[kNbrWords];
  int nbl[kMaxNbrBlocks];
  int nbn;
  int nbok;
  double tau2[K], stop[K], gprev[K], aprev[K], alpha[K], beta[K], rrprev[K];
  int use_pipe;
  int act[K];
  int flag;
  int wmax[kPipeSlices];
  int base[kPipeSlices + 1];
  int cached, own_s;
  // block SSOR: start of each colour's rows in the slot list, the widths of
  // the colour's lower / upper neighbour lists and where those lists start
  int coff[kMaxColours + 1];
  int wl[kMaxColours], wu[kMaxColours], loff[kMaxColours], uoff[kMaxColours];
  int lents;  // entries of the neighbour lists
  int ncb;    // colours of this block's rows
};

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

// Block SSOR list entry: a neighbour's list position (-1: padding) and its
// coefficient scaled by the row's 1 / A_ii (one 8- or 16-byte load)
template <typename T>
struct alignas(2 * sizeof(T)) LEnt {
  int j;
  T v;
};

template <typename T, int K>
__device__ __forceinline__ void load_m(const T* __restrict__ m, int j, T (&x)[K]) {
  constexpr int W = MRow<T, K>::W, NC = MRow<T, K>::NC;
  if (j < 0) {
#pragma unroll
    for (int c = 0; c < K; ++c) x[c] = (T)0;
    return;
  }
  const uint4* src = reinterpret_cast<const uint4*>(m + (size_t)j * W);
  T buf[W];
#pragma unroll
  for (int i = 0; i < NC; ++i) {
    const uint4 v = src[i];
    if constexpr (sizeof(T) == 4) {
      buf[4 * i + 0] = __uint_as_float(v.x);
      buf[4 * i + 1] = __uint_as_float(v.y);
      buf[4 * i + 2] = __uint_as_float(v.z);
      buf[4 * i + 3] = __uint_as_float(v.w);
    } else {
      buf[2 * i + 0] = __hiloint2double((int)v.y, (int)v.x);
      buf[2 * i + 1] = __hiloint2double((int)v.w, (int)v.z);
    }
  }
#pragma unroll
  for (int c = 0; c < K; ++c) x[c] = buf[c];
}

template <typename T, int K>
__device__ __forceinline__ void store_m(T* __restrict__ m, int j, const T (&x)[K]) {
  constexpr int W = MRow<T, K>::W, NC = MRow<T, K>::NC;
  T buf[W];
#pragma unroll
  for (int c = 0; c < W; ++c) buf[c] = c < K ? x[c] : (T)0;
  uint4* dst = reinterpret_cast<uint4*>(m + (size_t)j * W);
#pragma unroll
  for (int i = 0; i < NC; ++i) {
    uint4 v;
    if constexpr (sizeof(T) == 4) {
      v.x = __float_as_uint(buf[4 * i + 0]);
      v.y = __float_as_uint(buf[4 * i + 1]);
      v.z = __float_as_uint(buf[4 * i + 2]);
      v.w = __float_as_uint(buf[4 * i + 3]);
    } else {
      v.x = (unsigned)__double2loint(buf[2 * i + 0]);
      v.y = (unsigned)__double2hiint(buf[2 * i + 0]);
      v.z = (unsigned)__double2loint(buf[2 * i + 1]);
      v.w = (unsigned)__double2hiint(buf[2 * i + 1]);
    }
    dst[i] = v;
  }
}

// One row of A: entries at c[e * stride], v[e * stride] for e < len; a
// column index < 0 is padding.
template <typename T>
struct RowRef {
  const int* c;
  const T* v;
  int stride;
  int len;
};

// acc = sum_e v_e m(c_e): U entries' indices and values first, then their U
// row gathers, then the multiply-adds.
template <typename T, int K, int U>
__device__ __forceinline__ void gather_m(const RowRef<T>& rr, const T* __restrict__ m, T (&acc)[K]) {
#pragma unroll
  for (int c = 0; c < K; ++c) acc[c] = (T)0;
  for (int e = 0; e < rr.len; e += U) {
    int j[U];
    T v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const bool ok = e + u < rr.len;
      j[u] = ok ? rr.c[(e + u) * rr.stride] : -1;
      v[u] = ok ? rr.v[(e + u) * rr.stride] : (T)0;
    }
    T x[U][K];
#pragma unroll
    for (int u = 0; u < U; ++u) load_m<T, K>(m, j[u], x[u]);
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int c = 0; c < K; ++c) acc[c] += v[u] * x[u][c];
  }
}

// The gathers of QR rows at once (so all of their loads are in flight
// together): acc[q] = sum_e v_e m(c_e) over row q's entries, rows with
// ok[q] false give zero.
template <typename T, int K, int U, int QR>
__device__ __forceinline__ void gather_rows(const RowRef<T> (&rr)[QR], const bool (&ok)[QR],
                                            const T* __restrict__ m, T (&acc)[QR][K]) {
  int len = 0;
#pragma unroll
  for (int q = 0; q < QR; ++q) {
#pragma unroll
    for (int c = 0; c < K; ++c) acc[q][c] = (T)0;
    if (ok[q] && rr[q].len > len) len = rr[q].len;
  }
  for (int e = 0; e < len; e += U) {
    int j[QR][U];
    T v[QR][U];
#pragma unroll
    for (int q = 0; q < QR; ++q)
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const bool g = ok[q] && e + u < rr[q].len;
        j[q][u] = g ? rr[q].c[(e + u) * rr[q].stride] : -1;
        v[q][u] = g ? rr[q].v[(e + u) * rr[q].stride] : (T)0;
      }
    T x[QR][U][K];
#pragma unroll
    for (int q = 0; q < QR; ++q)
#pragma unroll
      for (int u = 0; u < U; ++u) load_m<T, K>(m, j[q][u], x[q][u]);
#pragma unroll
    for (int q = 0; q < QR; ++q)
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int c = 0; c < K; ++c) acc[q][c] += v[q][u] * x[q][u][c];
  }
}

// Sum v[0..N) over the block and store sum c at out[c * stride]: warp level
// in A (one shuffle per value for the FP32 solve), then thread c adds the
// warp sums of value c in FP64 in a fixed order.  The caller synchronises
// the block before `red` is written again.
template <int N, typename A>
__device__ void block_reduce_strided(const A (&v)[N], double* red, double* out, int stride) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int c = 0; c < N; ++c) {
    A t = v[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) red[warp * N + c] = (double)t;
  }
  __syncthreads();
  // thread c adds the warp sums of value c (independent shared loads)
  if ((int)threadIdx.x < N) {
    const int c = threadIdx.x;
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += red[w * N + c];
    out[(size_t)c * stride] = t;
  }
}

// Own-row state in T, one contiguous record of (6 + EX) K + 1 values per
// row: quantities r, w, z, s, p, x (K columns each), with EX = 2 also u and
// q (the pipelined form with block SSOR keeps u = M^-1 r and q = M^-1 s by
// recurrence), then 1/A_ii.  An odd record length keeps the shared-memory
// accesses of a warp on distinct banks.
enum { kQr = 0, kQw = 1, kQz = 2, kQs = 3, kQp = 4, kQx = 5, kQu = 6, kQq = 7 };
template <typename T, int K, int EX = 0>
struct OwnRef {
  static constexpr int kLen = (6 + EX) * K + 1;
  T* p;
  __device__ __forceinline__ T& operator()(int qy, int c) const { return p[qy * K + c]; }
  __device__ __forceinline__ T& minv() const { return p[kLen - 1]; }
};

// One own row's update of a pipelined iteration: z = n + beta z,
// s = w + beta s, p = M^-1 r + beta p, x += alpha p, r -= alpha s,
// w -= alpha z; m = M^-1 w to mnext; (r, M^-1 r) and (w, M^-1 r) into d2.
template <typename T, int K, class O>
__device__ __forceinline__ void pipe_update(const O& o, int row, const T (&nn)[K], const T (&alpha)[K],
                                            const T (&beta)[K], bool b0, T* __restrict__ mnext, T (&d2)[2 * K]) {
  const T mi = o.minv();
  T m[K];
#pragma unroll
  for (int c = 0; c < K; ++c) {
    const T r0 = o(kQr, c), w0 = o(kQw, c);
    const T zo = b0 ? (T)0 : o(kQz, c);
    const T so = b0 ? (T)0 : o(kQs, c);
    const T po = b0 ? (T)0 : o(kQp, c);
    const T z = nn[c] + beta[c] * zo;
    const T sx = w0 + beta[c] * so;
    const T p = mi * r0 + beta[c] * po;
    const T r = r0 - alpha[c] * sx;
    const T w = w0 - alpha[c] * z;
    o(kQx, c) += alpha[c] * p;
    o(kQz, c) = z;
    o(kQs, c) = sx;
    o(kQp, c) = p;
    o(kQr, c) = r;
    o(kQw, c) = w;
    m[c] = mi * w;
    const T u = mi * r;
    d2[c] += r * u;
    d2[K + c] += w * u;
  }
  store_m<T, K>(mnext, row, m);
}

// The block-SSOR sweeps over a block's colour lists when they live in global
// memory (a block whose shared memory cannot hold them): the same steps as
// the shared-memory sweeps of pipe_body, NR rows per thread at a time with
// their loads issued together (rows of one colour are not coupled, and a
// thread has several rows per step when a block holds many row slices).
// Kept out of line, so the kernel body holds the hot shared-memory loop only.
template <typename T, int K, int NR>
__device__ __noinline__ void ssor_sweeps_global(const PipeSmem<K>* s, const LEnt<T>* lent, T* sv, int t, int B) {
  const int nc = s->ncb;
  for (int pass = 0; pass < 2; ++pass) {
    const bool fwd = pass == 0;
    for (int step = 1; step < nc; ++step) {
      const int c = fwd ? step : nc - 1 - step;
      const int beg = s->coff[c], cnt = s->coff[c + 1] - beg;
      const int w = fwd ? s->wl[c] : s->wu[c];
      const LEnt<T>* le = lent + (fwd ? s->loff[c] : s->uoff[c]);
      for (int p0 = t; p0 < cnt; p0 += NR * B) {
        T x[NR][K];
        bool okr[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          okr[r] = p0 + r * B < cnt;
          load_m<T, K>(sv, okr[r] ? beg + p0 + r * B : -1, x[r]);
        }
        for (int e = 0; e < w; e += 2) {
          LEnt<T> e0[NR], e1[NR];
#pragma unroll
          for (int r = 0; r < NR; ++r) {
            const int p = p0 + r * B;
            e0[r] = okr[r] ? le[e * cnt + p] : LEnt<T>{-1, (T)0};
            e1[r] = okr[r] && e + 1 < w ? le[(e + 1) * cnt + p] : LEnt<T>{-1, (T)0};
          }
          T y0[NR][K], y1[NR][K];
#pragma unroll
          for (int r = 0; r < NR; ++r) {
            load_m<T, K>(sv, e0[r].j, y0[r]);
            load_m<T, K>(sv, e1[r].j, y1[r]);
          }
#pragma unroll
          for (int r = 0; r < NR; ++r)
#pragma unroll
            for (int cc = 0; cc < K; ++cc) x[r][cc] -= e0[r].v * y0[r][cc] + e1[r].v * y1[r][cc];
        }
#pragma unroll
        for (int r = 0; r < NR; ++r)
          if (okr[r]) store_m<T, K>(sv, beg + p0 + r * B, x[r]);
      }
      __syncthreads();
    }
  }
}

// The CG forms of a launch: FORM selects the code compiled into a kernel
// (each form keeps the registers of its own loop: one kernel holding all
// three spilled more in every one of them).
enum { kFormClassic = 0, kFormPipe = 1, kFormSingle = 2, kFormPipeSsor = 3 };
__host__ __device__ constexpr int form_of(int pipe_mode) {
  return pipe_mode == 3                      ? kFormSingle
         : (pipe_mode == 1 || pipe_mode == 2) ? kFormPipe
         : (pipe_mode == 4 || pipe_mode == 5) ? kFormPipeSsor
                                              : kFormClassic;
}

template <typename T, int K, int QR, int FORM, class Team>
__device__ void pipe_body(const SolveArgs& a, const Team& team, PipeSmem<K>* s, unsigned char* dyn) {
  // the pipelined form with block SSOR keeps u and q in the own-row records
  constexpr bool PS = FORM == kFormPipeSsor;
  using Own = OwnRef<T, K, PS ? 2 : 0>;
  // entries of a row gathered together (K values per neighbour in both forms)
  constexpr int UP = sizeof(T) == 4 ? 8 : 4;
  const T* Aval = (const T*)a.A_val;
  T* mb0 = (T*)a.m0;
  T* mb1 = (T*)a.m1;
  T* mb2 = (T*)a.m2;
  const int n = a.n, B = blockDim.x, t = threadIdx.x;
  // Block b owns the contiguous rows [b Qg B, (b + 1) Qg B): thread t the
  // rows b Qg B + q B + t, q < Qg (consecutive threads, consecutive rows;
  // a block's rows are neighbours on the mesh in natural order)
  const int Qg = (int)(((long long)n + (long long)team.size() * B - 1) / ((long long)team.size() * B));
  const int R = B;
  const int blk0 = team.rank() * Qg * B;
  const int row0 = blk0 + t;
  const int Qb = n > blk0 ? Qg : 0;  // row slices of this block
  const int tsize = team.size();
  const int warp = t >> 5, lane = t & 31, nw = B >> 5;
  double* part = a.partials;
  auto slot_ptr = [&](int slot) { return part + ((size_t)slot * tsize) * K; };
  // the pipelined partials (gamma, delta per column): parity g uses slots
  // 2 + 2g .. 3 + 2g as a [2K][blocks] table (quantity-major, so a warp reads
  // one quantity's partials with consecutive loads)
  auto pipe_ptr = [&](int g) { return part + ((size_t)(2 + 2 * g) * tsize) * K; };
  int status = CN_OK, total_iters = 0, refinements = 0;

  const unsigned char* bcol = a.bcolor;
  const bool bssor = bcol != nullptr;
  const int rb_n = n - blk0 < Qg * B ? n - blk0 : Qg * B;  // rows of this block
  // ---- shared memory: the block's rows of A, then (if it fits) the own-row
  // state and, for block SSOR, the colour lists
  {
    if (t < kPipeSlices) s->wmax[t] = 0;
    if (t < kMaxColours) s->wl[t] = s->wu[t] = 0;
    if (t <= kMaxColours) s->coff[t] = 0;
    __syncthreads();
    const int qc = Qb < kPipeSlices ? Qb : kPipeSlices;
    for (int q = 0; q < qc; ++q) {
      const int row = row0 + q * R;
      if (row < n) atomicMax(&s->wmax[q], a.A_ptr[row + 1] - a.A_ptr[row]);
    }
    if (bssor)  // rows per colour; lower / upper neighbours inside the block per row
      for (int q = 0; q < Qb; ++q) {
        const int row = row0 + q * R;
        if (row >= n) break;
        const int ci = (int)__ldg(bcol + row);
        int nl = 0, nu = 0;
        for (int e = a.A_ptr[row]; e < a.A_ptr[row + 1]; ++e) {
          const int j = a.A_col[e];
          if (j < blk0 || j >= blk0 + rb_n || j == row) continue;
          const int cj = (int)__ldg(bcol + j);
          nl += cj < ci;
          nu += cj > ci;
        }
        atomicAdd(&s->coff[ci + 1], 1);
        atomicMax(&s->wl[ci], nl);
        atomicMax(&s->wu[ci], nu);
      }
    __syncthreads();
    if (t == 0) {
      int ents = 0;
      for (int q = 0; q < qc; ++q) {
        s->base[q] = ents;
        ents += s->wmax[q] * B;
      }
      s->base[qc] = ents;
      const size_t need = align16((size_t)ents * sizeof(int)) + align16((size_t)ents * sizeof(T));
      // own-row state, plus for block SSOR the rows' colours and list
      // positions, the colours' neighbour lists and the sweep vector in
      // list order
      size_t own = align16((size_t)Own::kLen * Qb * B * sizeof(T));
      int lents = 0, ncb = 0;
      if (bssor) {
        for (int c = 0; c < kMaxColours; ++c) {
          const int cnt = s->coff[c + 1];
          if (cnt > 0) ncb = c + 1;
          s->coff[c + 1] += s->coff[c];
          s->loff[c] = lents;
          lents += cnt * s->wl[c];
          s->uoff[c] = lents;
          lents += cnt * s->wu[c];
        }
        own += align16((size_t)Qb * B) + 2 * align16((size_t)Qb * B * sizeof(short)) +
               align16((size_t)lents * sizeof(LEnt<T>)) + (size_t)Qb * B * MRow<T, K>::W * sizeof(T);
      }
      s->lents = lents;
      s->ncb = ncb;
      s->cached = (qc == Qb && Qb > 0 && need <= (size_t)a.cache_bytes) ? 1 : 0;
      s->own_s = (s->cached && need + own <= (size_t)a.cache_bytes) ? 1 : 0;
    }
    __syncthreads();
  }
  const bool cached = s->cached != 0, own_s = s->own_s != 0;
  const int ents = s->base[Qb < kPipeSlices ? Qb : kPipeSlices];
  int* ccol = (int*)dyn;
  T* cval = (T*)(dyn + align16((size_t)ents * sizeof(int)));
  T* os = (T*)(dyn + align16((size_t)ents * sizeof(int)) + align16((size_t)ents * sizeof(T)));
  // block SSOR, own state in shared memory: the block's rows are listed by
  // colour (in row order inside a colour); per slot (q B + t) its colour and
  // list position; per colour the lower- and higher-colour neighbours of its
  // rows inside the block, entry e of the colour's p-th row at
  // off + e * rows of the colour + p; the sweep vector v in list order, one
  // 16-byte-padded row per position (consecutive threads of a step touch
  // consecutive rows)
  const int nsl = Qb * B;
  unsigned char* srowc = (unsigned char*)os + align16((size_t)Own::kLen * nsl * sizeof(T));
  short* spos = (short*)(srowc + align16((size_t)nsl));
  const int lents = s->lents;
  short* const slist = (short*)((unsigned char*)spos + align16((size_t)nsl * sizeof(short)));  // position -> slot
  LEnt<T>* const lent = (LEnt<T>*)((unsigned char*)slist + align16((size_t)nsl * sizeof(short)));
  T* const sv = (T*)((unsigned char*)lent + align16((size_t)lents * sizeof(LEnt<T>)));  // 16-byte rows
  // the same tables in the global scratch a.bss_* (this block's share), for
  // blocks whose shared memory cannot hold them
  LEnt<T>* const lent_g = bssor ? (LEnt<T>*)a.bss_lent + a.bss_loff[team.rank()] : nullptr;
  T* const sv_g = bssor ? (T*)a.bss_v + (size_t)blk0 * MRow<T, K>::W : nullptr;
  T* pown = (T*)a.pown;
  auto own_ref = [&](int q, int row) {
    Own o;
    o.p = own_s ? os + ((size_t)q * B + t) * Own::kLen : pown + (size_t)row * Own::kLen;
    return o;
  };
  if (cached) {
    for (int q = 0; q < Qb; ++q) {
      const int row = row0 + q * R;
      const int e0 = row < n ? a.A_ptr[row] : 0;
      const int len = row < n ? a.A_ptr[row + 1] - e0 : 0;
      const int wq = s->wmax[q], bq = s->base[q];
      for (int e = 0; e < wq; ++e) {
        const int ix = bq + e * B + t;
        ccol[ix] = e < len ? a.A_col[e0 + e] : -1;
        cval[ix] = e < len ? Aval[e0 + e] : (T)0;
      }
    }
  }
  for (int q = 0; q < Qb; ++q) {
    const int row = row0 + q * R;
    if (row >= n) break;
    const double d = a.dinv64[row];
    own_ref(q, row).minv() = (T)(d * d);  // dinv = 1 / sqrt(A_ii) (the pivots of the empty factor)
  }
  __syncthreads();
  auto row_ref = [&](int q, int row) {
    RowRef<T> rr;
    if (cached) {
      const int bq = s->base[q];
      rr.c = ccol + bq + t;
      rr.v = cval + bq + t;
      rr.stride = B;
      rr.len = s->wmax[q];
    } else {
      const int e0 = a.A_ptr[row];
      rr.c = a.A_col + e0;
      rr.v = Aval + e0;
      rr.stride = 1;
      rr.len = a.A_ptr[row + 1] - e0;
    }
    return rr;
  };
  // ---- block SSOR (a.bcolor != null): M = (D + L) D^-1 (D + U) over the
  // block's own rows (the couplings to other blocks dropped), L / U in the
  // order of the block-local colours a.bcolor (rows of one colour are not
  // coupled).  z = M^-1 r: y = (D + L)^-1 r colour by colour upwards, then
  // z = y - D^-1 U z colour by colour downwards; one block barrier per
  // colour step.
  //
  // Own state in shared memory: the owners set v = M_ii^-1 r_i before the
  // barrier ahead of the sweeps; going up, v_i -= sum over lower neighbours
  // of (a_ij / a_ii) v_j turns v into y colour by colour (colour 0 has no
  // lower neighbour); going down, v_i -= sum over higher neighbours of
  // (a_ij / a_ii) v_j turns it into z (the top colour's z is its y).  A step
  // runs over the colour's list, one row per thread.
  // With fin (the inner iterations, at least two colours), the thread that
  // makes a row's z final (the top colour going up, the others going down)
  // also writes it to the row's record and to the gathered copy zn, and adds
  // the row's (r, z) and ||r||^2 to d2: no pass over the own rows afterwards.
  auto ssor_fast_fin = [&](bool fin, auto rec, T* zn, T* d2) {
    const int nc = s->ncb;
    for (int pass = 0; pass < 2; ++pass) {
      const bool fwd = pass == 0;
      for (int step = 1; step < nc; ++step) {
        const int c = fwd ? step : nc - 1 - step;
        const int beg = s->coff[c], cnt = s->coff[c + 1] - beg;
        const int w = fwd ? s->wl[c] : s->wu[c];
        const LEnt<T>* le = lent + (fwd ? s->loff[c] : s->uoff[c]);
        for (int p = t; p < cnt; p += B) {
          T x[K];
          load_m<T, K>(sv, beg + p, x);
          int e = 0;
          for (; e + 1 < w; e += 2) {
            const LEnt<T> e0 = le[e * cnt + p], e1 = le[(e + 1) * cnt + p];
            T y0[K], y1[K];
            load_m<T, K>(sv, e0.j, y0);
            load_m<T, K>(sv, e1.j, y1);
#pragma unroll
            for (int cc = 0; cc < K; ++cc) x[cc] -= e0.v * y0[cc] + e1.v * y1[cc];
          }
          if (e < w) {
            const LEnt<T> e0 = le[e * cnt + p];
            T y0[K];
            load_m<T, K>(sv, e0.j, y0);
#pragma unroll
            for (int cc = 0; cc < K; ++cc) x[cc] -= e0.v * y0[cc];
          }
          store_m<T, K>(sv, beg + p, x);
          if (fin && (!fwd || c == nc - 1)) {
            const int slot = slist[beg + p];
            if constexpr (decltype(rec)::value) {  // the two-reduction form: z's record and the dots too
              T* o = os + (size_t)slot * Own::kLen;
#pragma unroll
              for (int cc = 0; cc < K; ++cc) {
                const T r = o[kQr * K + cc];
                o[kQz * K + cc] = x[cc];
                d2[cc] += r * x[cc];
                d2[K + cc] += r * r;
              }
            }
            store_m<T, K>(zn, blk0 + slot, x);
          }
        }
        __syncthreads();
      }
    }
  };
  auto ssor_fast = [&]() { ssor_fast_fin(false, std::false_type{}, nullptr, nullptr); };
  // The tables in shared memory (beside the own state, when everything fits
  // there) or in the global scratch; the colours of the global case come
  // from a.bcolor, the list positions from a.bss_pos.
  const bool sm_ssor = bssor && own_s;
  int* const gpos = a.bss_pos;
  auto colour_of = [&](int slot) -> int {
    if (sm_ssor) return srowc[slot];
    return slot < rb_n ? (int)__ldg(bcol + blk0 + slot) : 255;
  };
  auto pos_of = [&](int slot) -> int { return sm_ssor ? (int)spos[slot] : gpos[blk0 + slot]; };
  auto ssor_apply = [&]() {
    if (sm_ssor) ssor_fast();
    else if (Qb <= 2) ssor_sweeps_global<T, K, 1>(s, lent_g, sv_g, t, B);
    else ssor_sweeps_global<T, K, kSweepRows>(s, lent_g, sv_g, t, B);
  };
  // a row's entry of the sweep vector, by slot
  auto sv_store = [&](int slot, const T (&x)[K]) {
    if (sm_ssor) store_m<T, K>(sv, spos[slot], x);
    else store_m<T, K>(sv_g, gpos[blk0 + slot], x);
  };
  auto sv_load = [&](int slot, T (&x)[K]) {
    if (sm_ssor) load_m<T, K>(sv, spos[slot], x);
    else load_m<T, K>(sv_g, gpos[blk0 + slot], x);
  };
  // The pipelined form with block SSOR: the sweeps turn the D^-1 w the own
  // rows left in the sweep vector into m = M^-1 w and write m to `out` for
  // the neighbours (in the sweep step that makes a row's m final when the
  // lists are in shared memory).
  auto ps_sweeps = [&](T* out) {
    if (sm_ssor && s->ncb >= 2) {
      ssor_fast_fin(true, std::false_type{}, out, nullptr);
      return;
    }
    ssor_apply();
    for (int q = 0; q < Qb; ++q) {
      const int row = row0 + q * R;
      if (row >= n) break;
      T m[K];
      sv_load(q * B + t, m);
      store_m<T, K>(out, row, m);
    }
  };
  if (bssor) {
    if (sm_ssor)
      for (int q = 0; q < Qb; ++q) {
        const int row = row0 + q * R;
        srowc[q * B + t] = row < n ? __ldg(bcol + row) : (unsigned char)255;
      }
    __syncthreads();
    // list positions in row order (warp w scans the block's slots for the
    // colours w, w + warps, ...; ballots give the positions) and the list
    // order's 1 / A_ii
    for (int c = warp; c < s->ncb; c += nw) {
      int pos0 = s->coff[c];
      for (int s0 = 0; s0 < nsl; s0 += 32) {
        const int slot = s0 + lane;
        const bool hit = slot < nsl && colour_of(slot) == c;
        const unsigned m = __ballot_sync(0xffffffffu, hit);
        if (hit) {
          const int pos = pos0 + __popc(m & ((1u << lane) - 1u));
          if (sm_ssor) {
            spos[slot] = (short)pos;
            slist[pos] = (short)slot;
          }
          else gpos[blk0 + slot] = pos;
        }
        pos0 += __popc(m);
      }
    }
    __syncthreads();
    // each row's column of its colour's lists
    for (int q = 0; q < Qb; ++q) {
      const int row = row0 + q * R;
      if (row >= n) break;
      const int slot = q * B + t, ci = colour_of(slot);
      const int p = pos_of(slot) - s->coff[ci], cnt = s->coff[ci + 1] - s->coff[ci];
      LEnt<T>* const lbase = sm_ssor ? lent : lent_g;
      LEnt<T>* ll = lbase + s->loff[ci] + p;
      LEnt<T>* lu = lbase + s->uoff[ci] + p;
      const T mi = own_ref(q, row).minv();
      const RowRef<T> rr = row_ref(q, row);
      int nl = 0, nu = 0;
      for (int e = 0; e < rr.len; ++e) {
        const int j = rr.c[e * rr.stride];
        if (j < blk0 || j >= blk0 + rb_n || j == row) continue;
        const int cj = colour_of(j - blk0);
        const LEnt<T> en{pos_of(j - blk0), mi * rr.v[e * rr.stride]};
        if (cj < ci) ll[(size_t)nl++ * cnt] = en;
        else if (cj > ci) lu[(size_t)nu++ * cnt] = en;
      }
      for (; nl < s->wl[ci]; ++nl) ll[(size_t)nl * cnt] = LEnt<T>{-1, (T)0};
      for (; nu < s->wu[ci]; ++nu) lu[(size_t)nu * cnt] = LEnt<T>{-1, (T)0};
    }
    __syncthreads();
  }

  // row slices q < QR: gathered together before the partial sums are needed
  bool okq[QR];
  RowRef<T> rrq[QR];
  Own ownq[QR];
#pragma unroll
  for (int q = 0; q < QR; ++q) {
    const int row = row0 + q * R;
    okq[q] = q < Qb && row < n;
    if (okq[q]) rrq[q] = row_ref(q, row);
    ownq[q] = own_ref(q, okq[q] ? row : 0);
  }

  // ---- single-reduction form: the blocks that own the columns of this
  // block's rows (their z is what this block gathers)
  if constexpr (FORM == kFormSingle) {
    for (int i = t; i < kNbrWords; i += B) s->nbm[i] = 0u;
    __syncthreads();
    const long long rows_per = (long long)Qg * B;
    for (int q = 0; q < Qb; ++q) {
      const int row = row0 + q * R;
      if (row >= n) break;
      const RowRef<T> rr = row_ref(q, row);
      for (int e = 0; e < rr.len; ++e) {
        const int j = rr.c[e * rr.stride];
        if (j < 0) continue;
        const int ob = (int)(j / rows_per);
        if (ob != team.rank() && ob < kNbrWords * 32) atomicOr(&s->nbm[ob >> 5], 1u << (ob & 31));
      }
    }
    __syncthreads();
    if (t == 0) {
      int cnt = 0;
      for (int w = 0; w < kNbrWords; ++w)
        for (unsigned m = s->nbm[w]; m; m &= m - 1) {
          if (cnt < kMaxNbrBlocks) s->nbl[cnt] = 32 * w + __ffs(m) - 1;
          ++cnt;
        }
      // more neighbours than the list holds (or blocks than the bitmap
      // covers): wait for every other block's flag
      s->nbn = (cnt > kMaxNbrBlocks || tsize > kNbrWords * 32) ? -1 : cnt;
    }
    __syncthreads();
  }
  unsigned epoch = 0;  // z publications of this launch (the host zeroes the flags)

  // ---- phase A: right-hand side (HarmonicSolve.lean:51-66 / DeformSolve.lean:123-135)
  {
    double bb[K];
#pragma unroll
    for (int c = 0; c < K; ++c) bb[c] = 0.0;
    for (int q = 0; q < Qb; ++q) {
      const int row = row0 + q * R;
      if (row >= n) break;
      double acc[K];
#pragma unroll
      for (int c = 0; c < K; ++c) acc[c] = 0.0;
      const int v = a.free_of[row];
      if (a.mode != CN_MODE_RHS) {
        const bool deform = a.mode == CN_MODE_DEFORM;
        gather_row<K, 1, 4>(a.K_ptr[v], a.K_ptr[v + 1], 0, a.K_col, a.K_val,
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
      for (int c = 0; c < K; ++c) {
        const double b = a.mode == CN_MODE_RHS ? a.targets[(size_t)row * K + c] : -acc[c];
        a.b64[(size_t)row * K + c] = b;
        bb[c] += b * b;
        if (!a.warm) a.x64[(size_t)row * K + c] = a.x0 ? a.x0[(size_t)v * K + c] : 0.0;
      }
    }
    block_reduce_store<K>(bb, s->sm.red, slot_ptr(kBB) + (size_t)team.rank() * K);
    if (!team.sync()) { status = CN_TIMEOUT; goto done; }
    team_sum<K>(slot_ptr(kBB), tsize, &s->sm);
    if (t < K) s->sm.bb[t] = s->sm.sum[t];
    __syncthreads();
  }

  for (int refine = 0;; ++refine) {
    // ---- phase R: FP64 residual r = b - A x; u = M^-1 r goes to m0 for the
    // first product w = A u
    {
      double rr[K];
#pragma unroll
      for (int c = 0; c < K; ++c) rr[c] = 0.0;
      for (int q = 0; q < Qb; ++q) {
        const int row = row0 + q * R;
        if (row >= n) break;
        double acc[K];
#pragma unroll
        for (int c = 0; c < K; ++c) acc[c] = 0.0;
        gather_row<K, 1, 4>(a.A_ptr[row], a.A_ptr[row + 1], 0, a.A_col, a.A_val64,
                            [&](int j, double* x) {
#pragma unroll
                              for (int c = 0; c < K; ++c) x[c] = a.x64[(size_t)j * K + c];
                            },
                            acc);
        const Own o = own_ref(q, row);
        const T mi = o.minv();
        T u[2 * K];
#pragma unroll
        for (int c = 0; c < K; ++c) {
          const double rv = a.b64[(size_t)row * K + c] - acc[c];
          const T rt = (T)rv;
          o(kQr, c) = rt;
          o(kQx, c) = (T)0;
          u[c] = mi * rt;
          u[K + c] = (T)0;
          o(kQz, c) = u[c];
          rr[c] += rv * rv;
        }
        if (bssor) {  // the block sweeps start from M^-1 r
          T v[K];
#pragma unroll
          for (int c = 0; c < K; ++c) v[c] = u[c];
          sv_store(q * B + t, v);
        }
        // both forms' first gathers: u = M^-1 r (pipelined, to m0) and
        // z = M^-1 r (classic, to m2; after the block sweeps with block SSOR)
        if (!bssor) {
          T m[K];
#pragma unroll
          for (int c = 0; c < K; ++c) m[c] = u[c];
          store_m<T, K>(mb0, row, m);
          store_m<T, K>(mb2, row, m);
        }
      }
      if (bssor) {
        __syncthreads();
        ssor_apply();
        for (int q = 0; q < Qb; ++q) {
          const int row = row0 + q * R;
          if (row >= n) break;
          const Own o = own_ref(q, row);
          T m[K];
          if (bssor) {
            sv_load(q * B + t, m);
#pragma unroll
            for (int c = 0; c < K; ++c) o(kQz, c) = m[c];
          } else {
#pragma unroll
            for (int c = 0; c < K; ++c) m[c] = o(kQz, c);
          }
          if constexpr (PS) {  // u = M^-1 r starts the pipelined recurrences
#pragma unroll
            for (int c = 0; c < K; ++c) o(kQu, c) = m[c];
          }
          store_m<T, K>(mb0, row, m);
          store_m<T, K>(mb2, row, m);
        }
      }
      block_reduce_store<K>(rr, s->sm.red, slot_ptr(kRR64) + (size_t)team.rank() * K);
      if (!team.sync()) { status = CN_TIMEOUT; goto done; }
      team_sum<K>(slot_ptr(kRR64), tsize, &s->sm);
      if (t == 0) {
        int any = 0, bad = 0;
        // the pipelined form falls back to the classic one (for the rest of
        // the solve) when its last inner solve cut the FP64 residual of some
        // column by less than 10x
        if (refine == 0)
          s->use_pipe = (FORM == kFormPipe && (a.pipe_mode == 1 || a.pipe_mode == 2)) ||
                        (PS && (a.pipe_mode == 4 || a.pipe_mode == 5));
        if (s->use_pipe && (a.pipe_mode == 2 || a.pipe_mode == 4) && refine > 0)
          for (int c = 0; c < K; ++c)
            if (s->rrprev[c] > 0.0 && !(s->sm.sum[c] <= 1e-2 * s->rrprev[c])) s->use_pipe = 0;
        for (int c = 0; c < K; ++c) {
          const double rr64 = s->sm.sum[c], bb = s->sm.bb[c];
          s->rrprev[c] = rr64;
          const double rel = bb > 0.0 ? sqrt(rr64 / bb) : sqrt(rr64);
          if (c < 32) a.stats->rel_residual[c] = rel;
          if (!(rel == rel)) bad = 1;
          const int act = rel > a.tol;
          s->act[c] = act;
          any |= act;
          // the inner solve stops when (r, M^-1 r) has fallen by tau^2
          const double want = bb > 0.0 ? 0.5 * a.tol * sqrt(bb / (rr64 > 0.0 ? rr64 : 1.0)) : 0.0;
          double tau = fmax(a.inner_tol, want);
          if (s->use_pipe && sizeof(T) == 4) tau = fmax(tau, kPipeInnerFloor);
          s->tau2[c] = tau * tau;
          s->stop[c] = tau * tau * rr64;  // the classic form tests ||r||^2
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

    bool pipe_failed = false;
    if ((FORM == kFormPipe || PS) && s->use_pipe) {
    // ---- phase I: w = A u, m = M^-1 w (to m1), gamma = (r, u), delta = (w, u)
    {
      T d2[2 * K];
#pragma unroll
      for (int c = 0; c < 2 * K; ++c) d2[c] = (T)0;
      for (int q = 0; q < Qb; ++q) {
        const int row = row0 + q * R;
        if (row >= n) break;
        T acc[K];
        gather_m<T, K, UP>(row_ref(q, row), mb0, acc);
        const Own o = own_ref(q, row);
        const T mi = o.minv();
        T m[K];
#pragma unroll
        for (int c = 0; c < K; ++c) {
          const T r = o(kQr, c), w = acc[c];
          T u;
          if constexpr (PS) u = o(kQu, c);
          else u = mi * r;
          o(kQw, c) = w;
          m[c] = mi * w;
          d2[c] += r * u;
          d2[K + c] += w * u;
        }
        if constexpr (PS) sv_store(q * B + t, m);  // the block sweeps start from D^-1 w
        else store_m<T, K>(mb1, row, m);
      }
      if constexpr (PS) {  // m = M^-1 w by the block sweeps, to m1 for the neighbours
        __syncthreads();
        ps_sweeps(mb1);
      }
      block_reduce_strided<2 * K, T>(d2, s->red2, pipe_ptr(0) + team.rank(), tsize);
      if (!team.sync()) { status = CN_TIMEOUT; goto done; }
    }

    // ---- the pipelined iterations, one team barrier each
    for (int it = 0;; ++it) {
      const int g = it & 1;
      const T* mcur = g ? mb0 : mb1;
      T* mnext = g ? mb1 : mb0;
      const bool b0 = it == 0;
      // (1) the previous phase's partials: item (quantity fc, split sp) sums
      // blocks [128 sp, 128 sp + 128); a warp's first item is loaded before
      // the gathers, so both round trips overlap
      const int ns = (tsize + 127) >> 7, items = 2 * K * ns;
      const double* pp = pipe_ptr(g);
      double pl[4];
      const bool item0 = warp < items;
      if (item0) {
        const int fc = warp / ns, sp = warp - fc * ns;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int b = sp * 128 + i * 32 + lane;
          pl[i] = b < tsize ? __ldcg(pp + (size_t)fc * tsize + b) : 0.0;
        }
      }
      // (2) row slices q < QR: the gathers of n = A m
      T nq[QR][K];
      gather_rows<T, K, UP, QR>(rrq, okq, mcur, nq);
      // (3) finish the partial sums
      auto reduce_item = [&](int item, const double (&v)[4]) {
        double x = (v[0] + v[1]) + (v[2] + v[3]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
        const int fc = item / ns;
        if (lane == 0) s->psum[fc][item - fc * ns] = x;
      };
      if (item0) reduce_item(warp, pl);
      for (int item = warp + nw; item < items; item += nw) {
        const int fc = item / ns, sp = item - fc * ns;
        double v[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int b = sp * 128 + i * 32 + lane;
          v[i] = b < tsize ? __ldcg(pp + (size_t)fc * tsize + b) : 0.0;
        }
        reduce_item(item, v);
      }
      __syncthreads();
      // (4) the scalars: lane c of warp 0 for column c
      if (warp == 0) {
        int act = 0, bad = 0;
        if (lane < K) {
          const int c = lane;
          double gam = 0.0, del = 0.0;
          for (int sp = 0; sp < ns; ++sp) {
            gam += s->psum[c][sp];
            del += s->psum[K + c][sp];
          }
          if (!(gam == gam) || !(del == del)) bad = 1;
          act = s->act[c];
          if (b0) s->stop[c] = s->tau2[c] * gam;
          else if (act && gam < s->stop[c]) act = 0;
          double be = 0.0, den = del;
          if (!b0) {
            const double gp = s->gprev[c];
            be = gp == 0.0 ? 0.0 : gam / gp;
            den = del - be * gam / s->aprev[c];
          }
          // a non-positive (p, Ap) ends this column's inner solve; the next
          // FP64 residual decides whether it restarts
          if (act && !(den > 0.0)) act = 0;
          const double al = act ? gam / den : 0.0;
          s->alpha[c] = al;
          s->beta[c] = act ? be : 0.0;
          s->act[c] = act;
          s->gprev[c] = gam;
          s->aprev[c] = act ? al : 1.0;
        }
        const int any = __any_sync(0xffffffffu, act), anybad = __any_sync(0xffffffffu, bad);
        if (lane == 0) s->flag = anybad ? 2 : (any ? 1 : 0);
      }
      __syncthreads();
      if (s->flag == 2) {
        if (a.pipe_mode == 2 || a.pipe_mode == 4) {  // drop this inner solve, continue in the classic form
          pipe_failed = true;
          break;
        }
        status = CN_NAN;
        goto done;
      }
      if (s->flag == 0 || it >= a.max_iter) break;
      T alpha[K], beta[K];
#pragma unroll
      for (int c = 0; c < K; ++c) {
        alpha[c] = (T)s->alpha[c];
        beta[c] = (T)s->beta[c];
      }
      // (5) the updates of the own rows
      T d2[2 * K];
#pragma unroll
      for (int c = 0; c < 2 * K; ++c) d2[c] = (T)0;
      if constexpr (PS) {
        // block SSOR: z = n + beta z, q = m + beta q, s = w + beta s,
        // p = u + beta p, x += alpha p, r -= alpha s, u -= alpha q,
        // w -= alpha z (m = M^-1 w of the last phase, still in the sweep
        // vector); the sweeps then turn D^-1 w into the next m
        auto ps_update = [&](const Own& o, int slot, const T (&nn)[K], T (&d)[2 * K]) {
          const T mi = o.minv();
          T mo[K], v[K];
          sv_load(slot, mo);
#pragma unroll
          for (int c = 0; c < K; ++c) {
            const T r0 = o(kQr, c), w0 = o(kQw, c), u0 = o(kQu, c);
            const T zo = b0 ? (T)0 : o(kQz, c);
            const T qo = b0 ? (T)0 : o(kQq, c);
            const T so = b0 ? (T)0 : o(kQs, c);
            const T po = b0 ? (T)0 : o(kQp, c);
            const T z = nn[c] + beta[c] * zo;
            const T qv = mo[c] + beta[c] * qo;
            const T sx = w0 + beta[c] * so;
            const T p = u0 + beta[c] * po;
            const T r = r0 - alpha[c] * sx;
            const T u = u0 - alpha[c] * qv;
            const T w = w0 - alpha[c] * z;
            o(kQx, c) += alpha[c] * p;
            o(kQz, c) = z;
            o(kQq, c) = qv;
            o(kQs, c) = sx;
            o(kQp, c) = p;
            o(kQr, c) = r;
            o(kQu, c) = u;
            o(kQw, c) = w;
            v[c] = mi * w;
            d[c] += r * u;
            d[K + c] += w * u;
          }
          sv_store(slot, v);
        };
#pragma unroll
        for (int q = 0; q < QR; ++q)
          if (okq[q]) ps_update(ownq[q], q * B + t, nq[q], d2);
        for (int q = QR; q < Qb; ++q) {
          const int row = row0 + q * R;
          if (row >= n) break;
          T nn[K];
          gather_m<T, K, UP>(row_ref(q, row), mcur, nn);
          ps_update(own_ref(q, row), q * B + t, nn, d2);
        }
        __syncthreads();
        ps_sweeps(mnext);
      } else {
#pragma unroll
        for (int q = 0; q < QR; ++q)
          if (okq[q]) pipe_update<T, K>(ownq[q], row0 + q * R, nq[q], alpha, beta, b0, mnext, d2);
        for (int q = QR; q < Qb; ++q) {
          const int row = row0 + q * R;
          if (row >= n) break;
          T nn[K];
          gather_m<T, K, UP>(row_ref(q, row), mcur, nn);
          pipe_update<T, K>(own_ref(q, row), row, nn, alpha, beta, b0, mnext, d2);
        }
      }
      block_reduce_strided<2 * K, T>(d2, s->red2, pipe_ptr(g ^ 1) + team.rank(), tsize);
      ++total_iters;
      if (!team.sync()) { status = CN_TIMEOUT; goto done; }
    }
    } else if (FORM == kFormSingle) {
    // ---- the single-reduction CG, one grid barrier per iteration:
    //   gamma, delta, ||r||^2 of the last phase -> stop?, beta, alpha;
    //   p = z + beta p'; s = w + beta s'; x += alpha p; r -= alpha s;
    //   z = M^-1 r (inline for Jacobi, the colour sweeps for block SSOR),
    //   (r, z), ||r||^2; publish z; wait for the neighbour blocks' z;
    //   w = A z, (z, w); this block's partial sums; grid barrier.
    // Partial tables [3K][blocks] (gamma, ||r||^2, delta) alternate by
    // parity at slots 2 and 5.
    double* const tR[2] = {part + (size_t)2 * tsize * K, part + (size_t)5 * tsize * K};
    const int ns = (tsize + 127) >> 7, items = 3 * K * ns;
    T* const zb[2] = {mb2, mb1};
    // prologue: w = A z for the z = M^-1 r of phase R (mb2, visible since its barrier)
    {
      T d3[3 * K];
#pragma unroll
      for (int c = 0; c < 3 * K; ++c) d3[c] = (T)0;
      for (int q = 0; q < Qb; ++q) {
        const int row = row0 + q * R;
        if (row >= n) break;
        RowRef<T> r1[1] = {row_ref(q, row)};
        const bool ok1[1] = {true};
        T acc1[1][K];
        gather_rows<T, K, UP, 1>(r1, ok1, mb2, acc1);
        const Own o = own_ref(q, row);
#pragma unroll
        for (int c = 0; c < K; ++c) {
          const T r = o(kQr, c), z = o(kQz, c), w = acc1[0][c];
          o(kQw, c) = w;
          d3[c] += r * z;
          d3[K + c] += r * r;
          d3[2 * K + c] += z * w;
        }
      }
      block_reduce_strided<3 * K, T>(d3, s->red2, tR[0] + team.rank(), tsize);
      if (!team.sync()) { status = CN_TIMEOUT; goto done; }
    }
    for (int it = 0;; ++it) {
      const int g = it & 1;
      T* const zn = zb[g ^ 1];
      for (int item = warp; item < items; item += nw) {
        const int fc = item / ns, sp = item - fc * ns;
        double v[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int b = sp * 128 + i * 32 + lane;
          v[i] = b < tsize ? __ldcg(tR[g] + (size_t)fc * tsize + b) : 0.0;
        }
        double x = (v[0] + v[1]) + (v[2] + v[3]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
        if (lane == 0) s->psum[fc][sp] = x;
      }
      __syncthreads();
      if (warp == 0) {
        int act = 0, bad = 0;
        if (lane < K) {
          const int c = lane;
          act = s->act[c];
          double ga = 0.0, rr = 0.0, de = 0.0;
          for (int sp = 0; sp < ns; ++sp) {
            ga += s->psum[c][sp];
            rr += s->psum[K + c][sp];
            de += s->psum[2 * K + c][sp];
          }
          if (!(ga == ga) || !(rr == rr) || !(de == de)) bad = 1;
          if (act && rr < s->stop[c]) act = 0;
          double be = 0.0, al = 0.0;
          if (act) {
            be = (it == 0 || s->gprev[c] == 0.0) ? 0.0 : ga / s->gprev[c];
            // (p, A p) = delta - beta gamma / alpha'; SparseLinAlg.lean:118
            // stops on pAp == 0: a non-positive value ends this column's
            // inner solve (the next FP64 residual decides)
            const double den = it == 0 ? de : de - be * ga / s->aprev[c];
            if (den > 0.0) al = ga / den;
            else act = 0;
          }
          s->beta[c] = act ? be : 0.0;
          s->alpha[c] = act ? al : 0.0;
          if (act) {
            s->gprev[c] = ga;
            s->aprev[c] = al;
          }
          s->act[c] = act;
        }
        const int any = __any_sync(0xffffffffu, act), anybad = __any_sync(0xffffffffu, bad);
        if (lane == 0) s->flag = anybad ? 2 : (any ? 1 : 0);
      }
      __syncthreads();
      if (s->flag == 2) { status = CN_NAN; goto done; }
      if (s->flag == 0 || it >= a.max_iter) break;
      {
        T alpha[K], beta[K];
#pragma unroll
        for (int c = 0; c < K; ++c) {
          alpha[c] = (T)s->alpha[c];
          beta[c] = (T)s->beta[c];
        }
        T d3[3 * K];
#pragma unroll
        for (int c = 0; c < 3 * K; ++c) d3[c] = (T)0;
        for (int q = 0; q < Qb; ++q) {
          const int row = row0 + q * R;
          if (row >= n) break;
          const Own o = own_ref(q, row);
          const T mi = o.minv();
          T rec[K];
#pragma unroll
          for (int c = 0; c < K; ++c) {
            // the first iteration reads no p', s' (the records may hold anything)
            const T p = it == 0 ? o(kQz, c) : o(kQz, c) + beta[c] * o(kQp, c);
            const T sv_ = it == 0 ? o(kQw, c) : o(kQw, c) + beta[c] * o(kQs, c);  // A p
            o(kQp, c) = p;
            o(kQs, c) = sv_;
            o(kQx, c) += alpha[c] * p;
            const T r = o(kQr, c) - alpha[c] * sv_;
            o(kQr, c) = r;
            if (!bssor) {
              const T z = mi * r;
              o(kQz, c) = z;
              rec[c] = z;
              d3[c] += r * z;
              d3[K + c] += r * r;
            } else {
              rec[c] = mi * r;  // block SSOR: the sweeps start from M^-1 r
            }
          }
          if (!bssor) store_m<T, K>(zn, row, rec);
          else sv_store(q * B + t, rec);
        }
        if (bssor && sm_ssor && s->ncb >= 2) {  // the sweeps also write the records, zn and the dots
          __syncthreads();
          ssor_fast_fin(true, std::true_type{}, zn, d3);
        } else if (bssor) {
          __syncthreads();
          ssor_apply();
          for (int q = 0; q < Qb; ++q) {
            const int row = row0 + q * R;
            if (row >= n) break;
            const Own o = own_ref(q, row);
            T zf[K];
            sv_load(q * B + t, zf);
#pragma unroll
            for (int c = 0; c < K; ++c) {
              const T r = o(kQr, c);
              o(kQz, c) = zf[c];
              d3[c] += r * zf[c];
              d3[K + c] += r * r;
            }
            store_m<T, K>(zn, row, zf);
          }
        }
        // publish z, then wait (bounded) for the z of the neighbour blocks
        __syncthreads();
        ++epoch;
        if (t == 0) {
          __threadfence();
          asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(a.nbflag + team.rank()), "r"(epoch) : "memory");
        }
        if (warp == 0) {
          const int nb = s->nbn < 0 ? tsize : s->nbn;
          int ok = 1;
          for (int i = lane; i < nb && ok; i += 32) {
            const int ob = s->nbn < 0 ? i : s->nbl[i];
            if (ob == team.rank()) continue;
            const unsigned* f = a.nbflag + ob;
            if (ld_acquire_u32(f) < epoch) {
              const unsigned long long t0 = global_ns();
              unsigned spins = 0;
              while (ld_acquire_u32(f) < epoch) {
                // the clock at the first poll and every 64th (as the grid barrier)
                const unsigned sp = spins++;
                if (sp == 0 || (sp & 63u) == 63u) {
                  if ((long long)(global_ns() - t0) > a.timeout_ns) {
                    atomicExch(&a.ctl->abort, 1);
                    ok = 0;
                    break;
                  }
                  if (sp != 0 && *(volatile int*)&a.ctl->abort) { ok = 0; break; }
                }
              }
            }
          }
          ok = __all_sync(0xffffffffu, ok);
          if (lane == 0) s->nbok = ok;
        }
        __syncthreads();
        if (!s->nbok) { status = CN_TIMEOUT; goto done; }
        // w = A z, (z, w)
        T accq[QR][K];
        gather_rows<T, K, UP, QR>(rrq, okq, zn, accq);
        auto take_w = [&](const Own& o, const T (&acc)[K]) {
#pragma unroll
          for (int c = 0; c < K; ++c) {
            o(kQw, c) = acc[c];
            d3[2 * K + c] += o(kQz, c) * acc[c];
          }
        };
#pragma unroll
        for (int q = 0; q < QR; ++q)
          if (okq[q]) take_w(ownq[q], accq[q]);
        for (int q = QR; q < Qb; ++q) {
          const int row = row0 + q * R;
          if (row >= n) break;
          RowRef<T> r1[1] = {row_ref(q, row)};
          const bool ok1[1] = {true};
          T acc1[1][K];
          gather_rows<T, K, UP, 1>(r1, ok1, zn, acc1);
          take_w(own_ref(q, row), acc1[0]);
        }
        block_reduce_strided<3 * K, T>(d3, s->red2, tR[g ^ 1] + team.rank(), tsize);
      }
      ++total_iters;
      if (!team.sync()) { status = CN_TIMEOUT; goto done; }
    }
    } else {
    // ---- the classic two-reduction CG in two phases per iteration:
    //   S: p = z + beta p'; A p = A z + beta A p' (each row gathers its
    //      neighbours' z, without waiting for beta), (p, Ap)
    //   U: alpha = (r, z) / (p, Ap); x += alpha p; r -= alpha Ap;
    //      z = M^-1 r for the next S; (r, z), ||r||^2
    // Partial tables [2K][blocks]: tS = (p.Ap, r.z) from S, tU = (r.z, r.r)
    // from U (each is read in the phase after the barrier that follows its
    // writes, and written again only after the next barrier).
    double* tS = part + (size_t)2 * tsize * K;
    double* tU = part + (size_t)4 * tsize * K;
    const int ns = (tsize + 127) >> 7, items = 2 * K * ns;
    auto load_item = [&](const double* tbl, int item, double (&v)[4]) {
      const int fc = item / ns, sp = item - fc * ns;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int b = sp * 128 + i * 32 + lane;
        v[i] = b < tsize ? __ldcg(tbl + (size_t)fc * tsize + b) : 0.0;
      }
    };
    auto reduce_item = [&](int item, const double (&v)[4]) {
      double x = (v[0] + v[1]) + (v[2] + v[3]);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
      const int fc = item / ns;
      if (lane == 0) s->psum[fc][item - fc * ns] = x;
    };
    for (int it = 0;; ++it) {
      const int g = it & 1;
      const T* rcur = g ? mb1 : mb2;
      T* rnext = g ? mb2 : mb1;
      const bool b0 = it == 0;
      // ---- phase S
      double pl[4];
      const bool item0 = !b0 && warp < items;
      if (item0) load_item(tU, warp, pl);
      T accq[QR][K];
      gather_rows<T, K, UP, QR>(rrq, okq, rcur, accq);
      if (item0) reduce_item(warp, pl);
      if (!b0)
        for (int item = warp + nw; item < items; item += nw) {
          double v[4];
          load_item(tU, item, v);
          reduce_item(item, v);
        }
      __syncthreads();
      if (warp == 0) {
        int act = 0, bad = 0;
        if (lane < K) {
          const int c = lane;
          act = s->act[c];
          double be = 0.0;
          if (!b0) {
            double rzn = 0.0, rr = 0.0;
            for (int sp = 0; sp < ns; ++sp) {
              rzn += s->psum[c][sp];
              rr += s->psum[K + c][sp];
            }
            if (!(rzn == rzn) || !(rr == rr)) bad = 1;
            if (act && rr < s->stop[c]) act = 0;
            be = s->gprev[c] == 0.0 ? 0.0 : (double)((T)rzn / (T)s->gprev[c]);
          }
          s->beta[c] = act ? be : 0.0;
          s->act[c] = act;
        }
        const int any = __any_sync(0xffffffffu, act), anybad = __any_sync(0xffffffffu, bad);
        if (lane == 0) s->flag = anybad ? 2 : (any ? 1 : 0);
      }
      __syncthreads();
      if (s->flag == 2) { status = CN_NAN; goto done; }
      if (s->flag == 0 || it >= a.max_iter) break;
      {
        T beta[K];
#pragma unroll
        for (int c = 0; c < K; ++c) beta[c] = (T)s->beta[c];
        T d2[2 * K];
#pragma unroll
        for (int c = 0; c < 2 * K; ++c) d2[c] = (T)0;
        auto form_p = [&](const Own& o, const T (&acc)[K]) {
#pragma unroll
          for (int c = 0; c < K; ++c) {
            const T z = o(kQz, c);
            const T po = b0 ? (T)0 : o(kQp, c);
            const T apo = b0 ? (T)0 : o(kQw, c);
            const T p = z + beta[c] * po;
            const T ap = acc[c] + beta[c] * apo;  // A p = A z + beta A p'
            o(kQp, c) = p;
            o(kQw, c) = ap;  // A p, for phase U and the next recurrence
            d2[c] += p * ap;
            d2[K + c] += o(kQr, c) * z;
          }
        };
#pragma unroll
        for (int q = 0; q < QR; ++q)
          if (okq[q]) form_p(ownq[q], accq[q]);
        for (int q = QR; q < Qb; ++q) {
          const int row = row0 + q * R;
          if (row >= n) break;
          RowRef<T> r1[1] = {row_ref(q, row)};
          const bool ok1[1] = {true};
          T acc1[1][K];
          gather_rows<T, K, UP, 1>(r1, ok1, rcur, acc1);
          form_p(own_ref(q, row), acc1[0]);
        }
        block_reduce_strided<2 * K, T>(d2, s->red2, tS + team.rank(), tsize);
      }
      if (!team.sync()) { status = CN_TIMEOUT; goto done; }
      // ---- phase U
      for (int item = warp; item < items; item += nw) {
        double v[4];
        load_item(tS, item, v);
        reduce_item(item, v);
      }
      __syncthreads();
      if (warp == 0 && lane < K) {
        const int c = lane;
        double pap = 0.0, rz = 0.0;
        for (int sp = 0; sp < ns; ++sp) {
          pap += s->psum[c][sp];
          rz += s->psum[K + c][sp];
        }
        int act = s->act[c];
        // SparseLinAlg.lean:118 stops on pAp == 0; a non-positive value ends
        // this column's inner solve (the next FP64 residual decides)
        if (act && !(pap > 0.0)) act = 0;
        s->alpha[c] = act ? (double)((T)rz / (T)pap) : 0.0;
        s->gprev[c] = rz;
        s->act[c] = act;
      }
      __syncthreads();
      {
        T alpha[K];
#pragma unroll
        for (int c = 0; c < K; ++c) alpha[c] = (T)s->alpha[c];
        T d2[2 * K];
#pragma unroll
        for (int c = 0; c < 2 * K; ++c) d2[c] = (T)0;
        for (int q = 0; q < Qb; ++q) {
          const int row = row0 + q * R;
          if (row >= n) break;
          const Own o = own_ref(q, row);
          const T mi = o.minv();
          T rec[K];
#pragma unroll
          for (int c = 0; c < K; ++c) {
            const T p = o(kQp, c);
            o(kQx, c) += alpha[c] * p;
            const T r = o(kQr, c) - alpha[c] * o(kQw, c);
            o(kQr, c) = r;
            if (!bssor) {
              const T z = mi * r;
              o(kQz, c) = z;
              rec[c] = z;
              d2[c] += r * z;
              d2[K + c] += r * r;
            } else {
              rec[c] = mi * r;  // block SSOR: the sweeps start from M^-1 r
            }
          }
          if (!bssor) store_m<T, K>(rnext, row, rec);
          else sv_store(q * B + t, rec);
        }
        if (bssor && sm_ssor && s->ncb >= 2) {  // the sweeps also write the records and the dots
          __syncthreads();
          ssor_fast_fin(true, std::true_type{}, rnext, d2);
        } else if (bssor) {  // z = M^-1 r by the block sweeps, then the records and the dots
          __syncthreads();
          ssor_apply();
          for (int q = 0; q < Qb; ++q) {
            const int row = row0 + q * R;
            if (row >= n) break;
            const Own o = own_ref(q, row);
            T zf[K];
            if (bssor) sv_load(q * B + t, zf);
            T rec[K];
#pragma unroll
            for (int c = 0; c < K; ++c) {
              const T r = o(kQr, c);
              if (bssor) o(kQz, c) = zf[c];
              const T z = o(kQz, c);
              rec[c] = z;
              d2[c] += r * z;
              d2[K + c] += r * r;
            }
            store_m<T, K>(rnext, row, rec);
          }
        }
        block_reduce_strided<2 * K, T>(d2, s->red2, tU + team.rank(), tsize);
      }
      ++total_iters;
      if (!team.sync()) { status = CN_TIMEOUT; goto done; }
    }
    }
    if (pipe_failed) {
      __syncthreads();
      if (t == 0) s->use_pipe = 0;
      continue;  // x64 unchanged: the next residual is this one again
    }
    // ---- x64 += x (FP64 accumulation of the correction)
    for (int q = 0; q < Qb; ++q) {
      const int row = row0 + q * R;
      if (row >= n) break;
      const Own o = own_ref(q, row);
#pragma unroll
      for (int c = 0; c < K; ++c) a.x64[(size_t)row * K + c] += (double)o(kQx, c);
    }
    if (!team.sync()) { status = CN_TIMEOUT; goto done; }
  }

  // ---- output: free rows, then the handle overlay (DeformSolve.lean:108-109)
  if (a.x_out) {
    for (int q = 0; q < Qb; ++q) {
      const int row = row0 + q * R;
      if (row >= n) break;
      const int v = a.free_of[row];
#pragma unroll
      for (int c = 0; c < K; ++c) a.x_out[(size_t)v * K + c] = a.x64[(size_t)row * K + c];
    }
    for (int h = team.rank() * B + t; h < a.nh; h += team.size() * B) {
      const int v = a.handles[h];
#pragma unroll
      for (int c = 0; c < K; ++c)
        a.x_out[(size_t)v * K + c] = a.mode == CN_MODE_RHS ? 0.0 : a.targets[(size_t)h * K + c];
    }
  }

done:
  if (team.rank() == 0 && t == 0) {
    a.stats->status = status;
    a.stats->iterations = total_iters;
    a.stats->refinements = refinements;
  }
}

// entries of a row gathered together: all of a mesh row in FP32, half of it in FP64
template <typename T>
constexpr int pipe_unroll() { return sizeof(T) == 4 ? 8 : 4; }

// QR = 1: one row per thread, up to 1024 threads; QR = 2: two rows per
// thread gathered together, up to 512 threads (twice the registers).
template <typename T, int K, int QR, int FORM>
__global__ void __launch_bounds__(1024 / QR, 1) k_pipe_grid(SolveArgs a) {
  __shared__ PipeSmem<K> s;
  extern __shared__ __align__(16) unsigned char dyn[];
  GridTeam team{a.ctl, a.timeout_ns, 0u};
  pipe_body<T, K, QR, FORM>(a, team, &s, dyn);
}

template <typename T, int K, int FORM>
__global__ void __launch_bounds__(1024, 1) k_pipe_cta(SolveArgs a) {
  __shared__ PipeSmem<K> s;
  extern __shared__ __align__(16) unsigned char dyn[];
  CtaTeam team;
  pipe_body<T, K, 1, FORM>(a, team, &s, dyn);
}

template <typename T, int K, int FORM>
cudaError_t launch_pkf(const SolveArgs& a, int block, int grid, int qr, cudaStream_t st) {
  const int dyn = a.cache_bytes;
  if (grid <= 1) {
    SolveArgs c = a;
    c.cache_bytes = 0;
    k_pipe_cta<T, K, FORM><<<1, block, 0, st>>>(c);
    return cudaGetLastError();
  }
  auto kern = qr == 2 ? k_pipe_grid<T, K, 2, FORM> : k_pipe_grid<T, K, 1, FORM>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
  if (e != cudaSuccess) return e;
  SolveArgs copy = a;
  void* args[] = {&copy};
  return cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(block), args, (size_t)dyn, st);
}

template <typename T, int K>
cudaError_t launch_pk(const SolveArgs& a, int block, int grid, int qr, cudaStream_t st) {
  switch (form_of(a.pipe_mode)) {
    case kFormPipe: return launch_pkf<T, K, kFormPipe>(a, block, grid, qr, st);
    case kFormSingle: return launch_pkf<T, K, kFormSingle>(a, block, grid, qr, st);
    case kFormPipeSsor:  // FP32 only (the host never asks for it in FP64)
      if constexpr (sizeof(T) == 4) return launch_pkf<T, K, kFormPipeSsor>(a, block, grid, qr, st);
      return cudaErrorInvalidValue;
    default: return launch_pkf<T, K, kFormClassic>(a, block, grid, qr, st);
  }
}

template <typename T, int K, int FORM>
int max_grid_pkf(int block, int dyn, int qr) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  auto kern = qr == 2 ? k_pipe_grid<T, K, 2, FORM> : k_pipe_grid<T, K, 1, FORM>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, block, dyn) != cudaSuccess) return 0;
  return sms * per;
}

template <typename T, int K>
int max_grid_pk(int block, int dyn, int qr, int pipe_mode) {
  switch (form_of(pipe_mode)) {
    case kFormPipe: return max_grid_pkf<T, K, kFormPipe>(block, dyn, qr);
    case kFormSingle: return max_grid_pkf<T, K, kFormSingle>(block, dyn, qr);
    case kFormPipeSsor:
      if constexpr (sizeof(T) == 4) return max_grid_pkf<T, K, kFormPipeSsor>(block, dyn, qr);
      return 0;
    default: return max_grid_pkf<T, K, kFormClassic>(block, dyn, qr);
  }
}

}  // namespace

cudaError_t launch_pipelined_solve(const SolveArgs& a, int precision, int K, int block, int grid, int qr,
                                   cudaStream_t s) {
  if (precision == CN_PREC_MIXED) {
    if (K == 1) return launch_pk<float, 1>(a, block, grid, qr, s);
    if (K == 3) return launch_pk<float, 3>(a, block, grid, qr, s);
    if (K == 9) return launch_pk<float, 9>(a, block, grid, qr, s);
  } else {
    if (K == 1) return launch_pk<double, 1>(a, block, grid, qr, s);
    if (K == 3) return launch_pk<double, 3>(a, block, grid, qr, s);
    if (K == 9) return launch_pk<double, 9>(a, block, grid, qr, s);
  }
  return cudaErrorInvalidValue;
}

int pipelined_max_grid(int precision, int K, int block, int cache_bytes, int qr, int pipe_mode) {
  if (precision == CN_PREC_MIXED) {
    if (K == 1) return max_grid_pk<float, 1>(block, cache_bytes, qr, pipe_mode);
    if (K == 3) return max_grid_pk<float, 3>(block, cache_bytes, qr, pipe_mode);
    if (K == 9) return max_grid_pk<float, 9>(block, cache_bytes, qr, pipe_mode);
  } else {
    if (K == 1) return max_grid_pk<double, 1>(block, cache_bytes, qr, pipe_mode);
    if (K == 3) return max_grid_pk<double, 3>(block, cache_bytes, qr, pipe_mode);
    if (K == 9) return max_grid_pk<double, 9>(block, cache_bytes, qr, pipe_mode);
  }
  return 0;
}

int block_colours(const int* A_ptr, const int* A_col, int n, int rb, unsigned char* col) {
  // DSatur inside each block: the next row is the uncoloured one with the
  // most distinct colours among its coloured neighbours (then the most
  // uncoloured neighbours, then the lowest index); it takes the lowest
  // colour none of them has.
  //
  // Then a top colour (beyond the third) of at most kFoldRows rows, which
  // would cost every sweep two block barriers (and, through the grid
  // barrier, every block) for a handful of rows, is folded into the lower
  // colour holding the fewest of each row's neighbours.  The couplings
  // between rows of one colour are left out of the block's L and U on both
  // sides (the kernel's list build skips them), so M = (D + L) D^-1 (D + L)^T
  // stays symmetric positive definite; a few of a block's thousands of
  // couplings are dropped.
  constexpr int kFoldRows = 8;
  int maxc = 0;
  std::vector<unsigned long long> used;
  std::vector<int> deg;
  for (int lo = 0; lo < n; lo += rb) {
    const int hi = std::min(n, lo + rb), m = hi - lo;
    used.assign((size_t)m, 0ull);
    deg.assign((size_t)m, 0);
    for (int i = lo; i < hi; ++i)
      for (int e = A_ptr[i]; e < A_ptr[i + 1]; ++e) {
        const int j = A_col[e];
        if (j >= lo && j < hi && j != i) ++deg[i - lo];
      }
    // key: (saturation, uncoloured neighbours, -index), largest first
    std::set<std::tuple<int, int, int>> pq;
    for (int r = 0; r < m; ++r) pq.insert({0, deg[r], -r});
    std::vector<char> done((size_t)m, 0);
    while (!pq.empty()) {
      const auto top = *pq.rbegin();
      pq.erase(std::prev(pq.end()));
      const int r = -std::get<2>(top), i = lo + r;
      int c = 0;
      while (c < kMaxColours - 1 && (used[r] >> c & 1ull)) ++c;
      col[i] = (unsigned char)c;
      done[r] = 1;
      maxc = std::max(maxc, c + 1);
      for (int e = A_ptr[i]; e < A_ptr[i + 1]; ++e) {
        const int j = A_col[e];
        if (j < lo || j >= hi || j == i || done[j - lo]) continue;
        const int q = j - lo;
        pq.erase({__builtin_popcountll(used[q]), deg[q], -q});
        used[q] |= 1ull << c;
        --deg[q];
        pq.insert({__builtin_popcountll(used[q]), deg[q], -q});
      }
    }
    for (;;) {
      int top = 0, ntop = 0;
      for (int i = lo; i < hi; ++i) top = std::max(top, (int)col[i]);
      for (int i = lo; i < hi; ++i) ntop += col[i] == top;
      if (top < 3 || ntop > kFoldRows) break;
      for (int i = lo; i < hi; ++i) {
        if (col[i] != top) continue;
        int cnt[kMaxColours] = {};
        for (int e = A_ptr[i]; e < A_ptr[i + 1]; ++e) {
          const int j = A_col[e];
          if (j >= lo && j < hi && j != i) ++cnt[col[j]];
        }
        int best = 0;
        for (int c = 1; c < top; ++c)
          if (cnt[c] < cnt[best]) best = c;
        col[i] = (unsigned char)best;
      }
    }
  }
  maxc = 0;
  for (int i = 0; i < n; ++i) maxc = std::max(maxc, (int)col[i] + 1);
  return maxc;
}

long long block_list_entries(const int* A_ptr, const int* A_col, const unsigned char* col, long long blk0,
                             long long rb_n) {
  int cnt[kMaxColours] = {}, wl[kMaxColours] = {}, wu[kMaxColours] = {};
  for (long long row = blk0; row < blk0 + rb_n; ++row) {
    const int ci = col[row];
    int nl = 0, nu = 0;
    for (int e = A_ptr[row]; e < A_ptr[row + 1]; ++e) {
      const int j = A_col[e];
      if (j < blk0 || j >= blk0 + rb_n || j == row) continue;
      nl += col[j] < ci;
      nu += col[j] > ci;
    }
    ++cnt[ci];
    wl[ci] = std::max(wl[ci], nl);
    wu[ci] = std::max(wu[ci], nu);
  }
  long long lents = 0;
  for (int k = 0; k < kMaxColours; ++k) lents += (long long)cnt[k] * (wl[k] + wu[k]);
  return lents;
}

void pipelined_smem_need(const int* A_ptr, const int* A_col, int n, int grid, int block, int precision, int K,
                         bool bssor, int rec_vectors, size_t* cache, size_t* full) {
  const size_t vs = precision == CN_PREC_MIXED ? sizeof(float) : sizeof(double);
  const long long Qg = ((long long)n + (long long)grid * block - 1) / ((long long)grid * block);
  const long long R = block;
  size_t wc = 0, wf = 0;
  *cache = *full = (size_t)-1;
  if (Qg > kPipeSlices) return;
  std::vector<unsigned char> col;
  if (bssor && n > 0) {  // the colours the solve will use for blocks of Qg x block rows
    col.resize((size_t)n);
    block_colours(A_ptr, A_col, n, (int)(Qg * block), col.data());
  }
  for (int b = 0; b < grid; ++b) {
    const long long blk0 = (long long)b * Qg * block;
    if (blk0 >= n) break;
    const long long Qb = Qg;
    const long long rb_n = std::min<long long>(n - blk0, Qg * block);
    size_t ents = 0;
    for (long long q = 0; q < Qb; ++q) {
      int w = 0;
      for (int t = 0; t < block; ++t) {
        const long long row = blk0 + t + q * R;
        if (row < n) w = std::max(w, A_ptr[row + 1] - A_ptr[row]);
      }
      ents += (size_t)w * block;
    }
    const size_t c = align16(ents * sizeof(int)) + align16(ents * vs);
    wc = std::max(wc, c);
    size_t extra = 0;
    if (bssor) {  // the kernel's colour lists: rows per colour x (lower + upper width)
      const size_t lents = (size_t)block_list_entries(A_ptr, A_col, col.data(), blk0, rb_n);
      // (LEnt: 8 bytes in FP32, 16 in FP64; the sweep vector padded to 16 bytes a row)
      const size_t wpad = ((size_t)K * vs + 15) / 16 * 16;
      extra = align16((size_t)Qb * block) + 2 * align16((size_t)Qb * block * sizeof(short)) + align16(lents * 2 * vs) +
              (size_t)Qb * (size_t)block * wpad;
    }
    wf = std::max(wf, c + align16((size_t)(rec_vectors * K + 1) * (size_t)Qb * (size_t)block * vs) + extra);
  }
  *cache = wc;
  *full = wf;
}

}  // namespace cn
