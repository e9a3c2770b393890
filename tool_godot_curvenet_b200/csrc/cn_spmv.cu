// cn_spmv.cu -- stand-alone SpMV / SpMM y = A X on the reduced matrix of a
// handle (sm_100a), the HBM-bound primitive of SparseLinAlg.lean:44-60 and
// SlangCodegen/SpmvMulti.lean:78-119 (X row-major n x k).
//
// Two kernels, chosen by the width of a row of X:
//
// * k_spmm_vec (k a multiple of a 16-byte chunk: FP32 k = 24, FP64 k = 24):
//   work item = three 16-byte chunks of one output row (2 threads a row in
//   FP32, 4 in FP64); the grid holds the blocks resident on the device at
//   once and walks the items grid-stride (one wave).  The threads of a row
//   take interleaved chunks (thread c: chunks c, c + T, c + 2T), so the store
//   of Y and each gather of a neighbour row of X are contiguous across them,
//   and the row's column indices and values are the same addresses for those
//   threads.  Two entries at a time, their 2 x 3 gathers in flight together,
//   60 registers (1,024 threads per SM; __launch_bounds__(256, 1) lets ptxas
//   keep them: bounded for occupancy it chose 40 registers and the same
//   kernel took 74 instead of 61 us).  Against one chunk per thread with
//   four entries at a time (32 registers, 2,048 threads per SM) on the
//   1.05M-row torus: FP32 69.6 -> 61.5 us, FP64 129 -> 109 us; fewer threads
//   each with three independent gathers per entry keep more bytes in flight
//   per load instruction, and each row's indices are loaded by a third as
//   many threads.
//
// * k_spmm_staged (FP32 k = 1 and 3: rows of X of 4 or 12 bytes): one thread
//   per row, tiles of kTileRows consecutive rows.  A producer warp per block
//   copies each tile's row pointers, column indices and values from HBM into
//   a ring of shared-memory stages with bulk asynchronous copies
//   (cp.async.bulk, completion counted on the stage's mbarrier), kStages - 1
//   tiles ahead; the consumer threads then read their row's entries from
//   shared memory and keep only the gathers of X (up to 8 entries x k values
//   in flight) on the critical path.  A stage is released to the producer by
//   an arrive of every consumer warp on the stage's second mbarrier.  Every
//   wait is bounded (kWaitNs); a wait that runs out (not expected: the
//   copies are this SM's own) raises *err and fills the rows of the
//   remaining tiles with NaN, so a failed product cannot pass as a result.
//   Against the grid-stride kernel it measured 20.5 us against 22.5 us at
//   FP32 k = 3 on the 1.05M-row torus (65 % of the measured copy bandwidth
//   against 59 %); for 16-byte chunks (k = 24) the staged form was slower in
//   every shape tried (one item per tile per thread waits a full memory
//   round trip per tile).
//
// The bulk copies start on 16-byte boundaries: a tile's ranges are rounded
// down to a 16-byte boundary and up to a multiple of 16 bytes, so a copy can
// read up to 12 bytes past the last row pointer or entry; the handle's
// row-pointer, column and value arrays are allocated with 4 elements to spare.
#include <algorithm>

#include "cn_internal.h"

namespace cn {
namespace {

template <typename T>
struct V16;
template <>
struct V16<float> {
  using type = float4;
  static constexpr int W = 4;
};
template <>
struct V16<double> {
  using type = double2;
  static constexpr int W = 2;
};

__device__ __forceinline__ void fma16(float4& acc, float a, const float4& x) {
  acc.x += a * x.x;
  acc.y += a * x.y;
  acc.z += a * x.z;
  acc.w += a * x.w;
}
__device__ __forceinline__ void fma16(double2& acc, double a, const double2& x) {
  acc.x += a * x.x;
  acc.y += a * x.y;
}

constexpr int kU = 4;

constexpr int kVecChunks = 3;   // 16-byte chunks of a row per thread
constexpr int kVecEntries = 2;  // entries of a row gathered together

// K a multiple of kVecChunks chunks: thread = (row, chunk group) for the
// items tid, tid + threads, ...; each item's loads are issued together: the
// row pointers, then two entries' indices and values, then their gathers,
// then the multiply-adds.
template <typename T, int K>
__global__ void __launch_bounds__(256, 1) k_spmm_vec(int n, const int* __restrict__ ptr, const int* __restrict__ col,
                                                  const T* __restrict__ val, const T* __restrict__ x,
                                                  T* __restrict__ y) {
  using V = typename V16<T>::type;
  constexpr int C = K / V16<T>::W;  // chunks per row
  constexpr int CW = kVecChunks, U = kVecEntries;
  static_assert(C % CW == 0, "a row's chunks split evenly over its threads");
  constexpr int CT = C / CW;  // threads per row
  const long long items = (long long)n * CT;
  const V* __restrict__ xv = reinterpret_cast<const V*>(x);
  for (long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x; it < items;
       it += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(it / CT), tc = (int)(it - (long long)row * CT);
    const int e0 = __ldg(ptr + row), e1 = __ldg(ptr + row + 1);
    V acc[CW];
#pragma unroll
    for (int w = 0; w < CW; ++w) {
      if constexpr (sizeof(T) == 4) acc[w] = make_float4(0.f, 0.f, 0.f, 0.f);
      else acc[w] = make_double2(0.0, 0.0);
    }
    for (int e = e0; e < e1; e += U) {
      int j[U];
      T a[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const bool g = e + u < e1;
        j[u] = g ? __ldg(col + e + u) : -1;
        a[u] = g ? __ldg(val + e + u) : (T)0;
      }
      V xs[U][CW];
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int w = 0; w < CW; ++w) {
          if (j[u] >= 0) xs[u][w] = __ldg(xv + (size_t)j[u] * C + tc + w * CT);
          else if constexpr (sizeof(T) == 4) xs[u][w] = make_float4(0.f, 0.f, 0.f, 0.f);
          else xs[u][w] = make_double2(0.0, 0.0);
        }
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int w = 0; w < CW; ++w) fma16(acc[w], a[u], xs[u][w]);
    }
#pragma unroll
    for (int w = 0; w < CW; ++w) reinterpret_cast<V*>(y)[(size_t)row * C + tc + w * CT] = acc[w];
  }
}

// Any K: thread = row.
template <typename T, int K>
__global__ void __launch_bounds__(256) k_spmm_row(int n, const int* __restrict__ ptr, const int* __restrict__ col,
                                                  const T* __restrict__ val, const T* __restrict__ x,
                                                  T* __restrict__ y) {
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    T acc[K];
#pragma unroll
    for (int c = 0; c < K; ++c) acc[c] = (T)0;
    const int e0 = ptr[row], e1 = ptr[row + 1];
    for (int e = e0; e < e1; e += kU) {
      int j[kU];
      T a[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const bool ok = e + u < e1;
        j[u] = ok ? __ldg(col + e + u) : -1;
        a[u] = ok ? __ldg(val + e + u) : (T)0;
      }
      T xs[kU][K];
#pragma unroll
      for (int u = 0; u < kU; ++u)
#pragma unroll
        for (int c = 0; c < K; ++c) xs[u][c] = j[u] >= 0 ? __ldg(x + (size_t)j[u] * K + c) : (T)0;
#pragma unroll
      for (int u = 0; u < kU; ++u)
#pragma unroll
        for (int c = 0; c < K; ++c) acc[c] += a[u] * xs[u][c];
    }
#pragma unroll
    for (int c = 0; c < K; ++c) y[(size_t)row * K + c] = acc[c];
  }
}

// ---- the staged kernel: mbarriers and bulk copies (PTX, sm_90 and later)
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long ns_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Wait for the completion of the phase of parity `parity`, bounded by limit_ns.
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity, long long limit_ns) {
  if (mbar_try_wait(b, parity)) return true;
  const unsigned long long t0 = ns_now();
  for (unsigned i = 1;; ++i) {
    if (mbar_try_wait(b, parity)) return true;
    if ((i & 15u) == 0 && (long long)(ns_now() - t0) > limit_ns) return false;
  }
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

constexpr int kTileRows = 256;  // rows of a tile = consumer threads of a block
constexpr int kStages = 3;      // shared-memory stages in the ring
constexpr int kGather = 8;      // entries of a row whose gathers are in flight together
constexpr long long kWaitNs = 2000000000LL;

// Stage layout: [row pointers | column indices | values], each 16-byte
// aligned and sized for `ents`, the most entries any tile holds.
struct StageGeo {
  static constexpr int kPtrBytes = ((kTileRows + 8) * 4 + 15) / 16 * 16;
  __host__ __device__ static int col_bytes(int ents) { return ((ents + 8) * 4 + 15) / 16 * 16; }
  __host__ __device__ static int val_bytes(int ents) { return ((ents + 8) * 4 + 15) / 16 * 16; }
  __host__ __device__ static int bytes(int ents) { return kPtrBytes + col_bytes(ents) + val_bytes(ents); }
};

template <int K>
__global__ void __launch_bounds__(kTileRows + 32) k_spmm_staged(int n, const int* __restrict__ ptr,
                                                                const int* __restrict__ col,
                                                                const float* __restrict__ val,
                                                                const float* __restrict__ x, float* __restrict__ y,
                                                                int ntiles, int ents, int* err) {
  extern __shared__ __align__(128) unsigned char dyn[];
  __shared__ __align__(8) unsigned long long full[kStages], empty[kStages];
  constexpr int NW = kTileRows / 32;
  const int sbytes = StageGeo::bytes(ents);
  const int t = threadIdx.x, lane = t & 31;
  if (t == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (t >= kTileRows) {  // the producer warp: one elected lane issues the copies
    if (lane == 0) {
      int i = 0;
      for (int tile = blockIdx.x; tile < ntiles; ++i, tile += gridDim.x) {
        const int s = i % kStages;
        // stage s is free once every consumer warp released its use i - kStages
        if (i >= kStages && !mbar_wait(&empty[s], ((unsigned)(i / kStages) & 1u) ^ 1u, kWaitNs)) {
          atomicExch(err, 1);
          break;
        }
        unsigned char* st = dyn + (size_t)s * sbytes;
        const int r0 = tile * kTileRows, r1 = min(r0 + kTileRows, n);
        const int e0 = __ldg(ptr + r0), e1 = __ldg(ptr + r1);
        const int r0a = r0 & ~3, c0 = e0 & ~3;
        const unsigned pb = (unsigned)(((r1 + 1 - r0a) * 4 + 15) & ~15);
        const unsigned cb = (unsigned)(((e1 - c0) * 4 + 15) & ~15);
        mbar_expect_tx(&full[s], pb + 2 * cb);
        bulk_g2s(st, ptr + r0a, pb, &full[s]);
        if (cb) {
          bulk_g2s(st + StageGeo::kPtrBytes, col + c0, cb, &full[s]);
          bulk_g2s(st + StageGeo::kPtrBytes + StageGeo::col_bytes(ents), val + c0, cb, &full[s]);
        }
      }
      // the copies still in flight land before the block may exit
      for (int q = max(0, i - kStages); q < i; ++q)
        if (!mbar_wait(&full[q % kStages], (unsigned)(q / kStages) & 1u, kWaitNs)) atomicExch(err, 1);
    }
    return;
  }
  bool failed = false;
  int i = 0;
  for (int tile = blockIdx.x; tile < ntiles; ++i, tile += gridDim.x) {
    const int row = tile * kTileRows + t;
    if (!failed) {
      const int s = i % kStages;
      const bool got = mbar_wait(&full[s], (unsigned)(i / kStages) & 1u, kWaitNs);
      if (!__all_sync(0xffffffffu, got)) {
        failed = true;
        if (lane == 0) atomicExch(err, 1);
      } else {
        const unsigned char* st = dyn + (size_t)s * sbytes;
        const int* sp = reinterpret_cast<const int*>(st);
        const int* sc = reinterpret_cast<const int*>(st + StageGeo::kPtrBytes);
        const float* sv = reinterpret_cast<const float*>(st + StageGeo::kPtrBytes + StageGeo::col_bytes(ents));
        const int r0a = (tile * kTileRows) & ~3;
        const int c0 = sp[tile * kTileRows - r0a] & ~3;
        const bool ok = row < n;
        const int eb = ok ? sp[row - r0a] : 0, ee = ok ? sp[row + 1 - r0a] : 0;
        float acc[K];
#pragma unroll
        for (int c = 0; c < K; ++c) acc[c] = 0.f;
        for (int e = eb; e < ee; e += kGather) {
          int j[kGather];
          float a[kGather];
#pragma unroll
          for (int u = 0; u < kGather; ++u) {
            const bool g = e + u < ee;
            j[u] = g ? sc[e + u - c0] : -1;
            a[u] = g ? sv[e + u - c0] : 0.f;
          }
          float xs[kGather][K];
#pragma unroll
          for (int u = 0; u < kGather; ++u)
#pragma unroll
            for (int c = 0; c < K; ++c) xs[u][c] = j[u] >= 0 ? __ldg(x + (size_t)j[u] * K + c) : 0.f;
#pragma unroll
          for (int u = 0; u < kGather; ++u)
#pragma unroll
            for (int c = 0; c < K; ++c) acc[c] += a[u] * xs[u][c];
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        if (ok)
#pragma unroll
          for (int c = 0; c < K; ++c) y[(size_t)row * K + c] = acc[c];
        continue;
      }
    }
    if (row < n)
#pragma unroll
      for (int c = 0; c < K; ++c) y[(size_t)row * K + c] = __int_as_float(0x7fc00000);
  }
}

// Blocks of `threads` resident on the whole device at once: the grid of the
// grid-stride and staged kernels (one wave, no tail of partly filled waves).
template <typename F>
int resident_blocks(F kern, int threads, size_t smem) {
  int dev = 0, sms = 148, per = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem) != cudaSuccess || per < 1) per = 1;
  return sms * per;
}

template <int K>
cudaError_t launch_staged(int n, const int* ptr, const int* col, const float* val, const float* x, float* y,
                          int ents, int* err, cudaStream_t s) {
  const int ntiles = (n + kTileRows - 1) / kTileRows;
  const size_t smem = (size_t)kStages * StageGeo::bytes(ents);
  auto kern = k_spmm_staged<K>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int slots = resident_blocks(kern, kTileRows + 32, smem);
  kern<<<std::min(ntiles, slots), kTileRows + 32, smem, s>>>(n, ptr, col, val, x, y, ntiles, ents, err);
  return cudaGetLastError();
}

template <typename T, int K>
cudaError_t launch_k(int n, const int* ptr, const int* col, const T* val, const T* x, T* y, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if constexpr (K % (V16<T>::W * kVecChunks) == 0) {
    const long long items = (long long)n * (K / V16<T>::W / kVecChunks);
    static const int slots = resident_blocks(k_spmm_vec<T, K>, 256, 0);
    const long long nb = std::min<long long>((items + 255) / 256, slots);
    k_spmm_vec<T, K><<<(unsigned)nb, 256, 0, s>>>(n, ptr, col, val, x, y);
  } else {
    static const int slots = resident_blocks(k_spmm_row<T, K>, 256, 0);
    const long long nb = std::min<long long>((n + 255) / 256, slots);
    k_spmm_row<T, K><<<(unsigned)nb, 256, 0, s>>>(n, ptr, col, val, x, y);
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_t(int n, int k, const int* ptr, const int* col, const T* val, const T* x, T* y,
                     cudaStream_t s) {
  switch (k) {
    case 1: return launch_k<T, 1>(n, ptr, col, val, x, y, s);
    case 3: return launch_k<T, 3>(n, ptr, col, val, x, y, s);
    case 9: return launch_k<T, 9>(n, ptr, col, val, x, y, s);
    case 24: return launch_k<T, 24>(n, ptr, col, val, x, y, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

int spmm_tile_entries(const int* hptr, int n) {
  int ents = 0;
  for (int r0 = 0; r0 < n; r0 += kTileRows) ents = std::max(ents, hptr[std::min(r0 + kTileRows, n)] - hptr[r0]);
  return ents;
}

cudaError_t launch_spmm(int n, int k, int precision, const int* ptr, const int* col, const void* val,
                        const void* x, void* y, int tile_ents, int* err, cudaStream_t s) {
  if (precision == CN_PREC_MIXED) {
    if (n > 0 && (k == 1 || k == 3) && tile_ents >= 0 && err) {
      const float* v = (const float*)val;
      return k == 1 ? launch_staged<1>(n, ptr, col, v, (const float*)x, (float*)y, tile_ents, err, s)
                    : launch_staged<3>(n, ptr, col, v, (const float*)x, (float*)y, tile_ents, err, s);
    }
    return launch_t<float>(n, k, ptr, col, (const float*)val, (const float*)x, (float*)y, s);
  }
  return launch_t<double>(n, k, ptr, col, (const double*)val, (const double*)x, (double*)y, s);
}

}  // namespace cn
