// cn_spmv.cu -- stand-alone SpMV / SpMM y = A X on the reduced matrix of a
// handle (sm_100a), the HBM-bound primitive of SparseLinAlg.lean:44-60 and
// SlangCodegen/SpmvMulti.lean:78-119 (X row-major n x k).
//
// Work item: one 16-byte chunk of one output row (4 FP32 or 2 FP64 columns)
// when k is a multiple of the chunk, else one whole row; the grid holds the
// blocks resident on the device at once and walks the items grid-stride
// (one wave: about 17 % faster than one thread per item at k = 24 in FP64).  Consecutive threads
// take consecutive chunks, so the store of Y and the gather of a neighbour
// row of X are contiguous across the threads of a row; the row's column
// indices and values are the same addresses for those threads (one L1
// transaction).  Four entries are in flight per thread (indices and values
// first, then the four gathers, then the multiply-adds): the kernel then fits
// in 32 registers, so every SM holds 2048 threads, which keeps more loads
// outstanding than eight entries per thread at 40-48 registers did
// (k = 24: 46 % -> 56 % of the copy bandwidth).
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

// K a multiple of the chunk width: thread = (row, chunk) for RPT items
// h, h + H, ... (H = items / RPT rounded up), all of whose loads are issued
// together: the row pointers, then every entry's index and value, then every
// gather, then the multiply-adds.
template <typename T, int K, int RPT>
__global__ void __launch_bounds__(256) k_spmm_vec(int n, const int* __restrict__ ptr, const int* __restrict__ col,
                                                  const T* __restrict__ val, const T* __restrict__ x,
                                                  T* __restrict__ y) {
  using V = typename V16<T>::type;
  constexpr int C = K / V16<T>::W;  // chunks per row
  const long long items = (long long)n * C;
  const long long H = (items + RPT - 1) / RPT;
  const V* __restrict__ xv = reinterpret_cast<const V*>(x);
  for (long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x; tid < H;
       tid += (long long)gridDim.x * blockDim.x) {
    int row[RPT], ch[RPT], e0[RPT], e1[RPT];
    bool ok[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const long long it = tid + q * H;
      ok[q] = it < items;
      row[q] = ok[q] ? (int)(it / C) : 0;
      ch[q] = ok[q] ? (int)(it - (long long)row[q] * C) : 0;
    }
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      e0[q] = ok[q] ? __ldg(ptr + row[q]) : 0;
      e1[q] = ok[q] ? __ldg(ptr + row[q] + 1) : 0;
    }
    V acc[RPT];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      if constexpr (sizeof(T) == 4) acc[q] = make_float4(0.f, 0.f, 0.f, 0.f);
      else acc[q] = make_double2(0.0, 0.0);
    }
    int len = 0;
#pragma unroll
    for (int q = 0; q < RPT; ++q) len = max(len, e1[q] - e0[q]);
    for (int e = 0; e < len; e += kU) {
      int j[RPT][kU];
      T a[RPT][kU];
#pragma unroll
      for (int q = 0; q < RPT; ++q)
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          const bool g = e0[q] + e + u < e1[q];
          j[q][u] = g ? __ldg(col + e0[q] + e + u) : -1;
          a[q][u] = g ? __ldg(val + e0[q] + e + u) : (T)0;
        }
      V xs[RPT][kU];
#pragma unroll
      for (int q = 0; q < RPT; ++q)
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          if (j[q][u] >= 0) xs[q][u] = __ldg(xv + (size_t)j[q][u] * C + ch[q]);
          else if constexpr (sizeof(T) == 4) xs[q][u] = make_float4(0.f, 0.f, 0.f, 0.f);
          else xs[q][u] = make_double2(0.0, 0.0);
        }
#pragma unroll
      for (int q = 0; q < RPT; ++q)
#pragma unroll
        for (int u = 0; u < kU; ++u) fma16(acc[q], a[q][u], xs[q][u]);
    }
#pragma unroll
    for (int q = 0; q < RPT; ++q)
      if (ok[q]) reinterpret_cast<V*>(y)[(size_t)row[q] * C + ch[q]] = acc[q];
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

// Blocks of 256 threads resident on the whole device at once: the grid of
// the grid-stride kernels (one wave, no tail of partly filled waves).
template <typename F>
int resident_blocks(F kern) {
  int dev = 0, sms = 148, per = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 256, 0) != cudaSuccess || per < 1) per = 1;
  return sms * per;
}

template <typename T, int K>
cudaError_t launch_k(int n, const int* ptr, const int* col, const T* val, const T* x, T* y, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  if constexpr (K % V16<T>::W == 0) {
    constexpr int RPT = 1;
    const long long items = (long long)n * (K / V16<T>::W);
    const long long threads = (items + RPT - 1) / RPT;
    static const int slots = resident_blocks(k_spmm_vec<T, K, RPT>);
    const long long nb = std::min<long long>((threads + 255) / 256, slots);
    k_spmm_vec<T, K, RPT><<<(unsigned)nb, 256, 0, s>>>(n, ptr, col, val, x, y);
  } else {
    static const int slots = resident_blocks(k_spmm_row<T, K>);
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

cudaError_t launch_spmm(int n, int k, int precision, const int* ptr, const int* col, const void* val,
                        const void* x, void* y, cudaStream_t s) {
  if (precision == CN_PREC_MIXED)
    return launch_t<float>(n, k, ptr, col, (const float*)val, (const float*)x, (float*)y, s);
  return launch_t<double>(n, k, ptr, col, (const double*)val, (const double*)x, (double*)y, s);
}

}  // namespace cn
