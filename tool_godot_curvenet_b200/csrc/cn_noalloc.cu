// cn_noalloc.cu -- cn_pcg_csr_noalloc: the persistent FP64 Jacobi-PCG solve on
// a caller-owned device CSR matrix, for callers that must not allocate GPU
// memory while they run (a frame loop of a real-time engine with a fixed
// memory budget, code recording a CUDA stream, a host that forbids
// cudaMalloc after start-up).  The caller passes the matrix, the right-hand
// sides and the solution buffer; every temporary lives in one file-scope
// device array of fixed size, so the call itself allocates nothing.
//
// Limits: at most kNaMaxRows unknowns and kNaMaxRowsTimesRhs unknowns times
// right-hand sides; about 14 MB of device memory per GPU that loads the
// library, held until the process exits.  The array is shared by every call
// and keeps the last call's contents: each call rewrites what it needs
// before use, and calls that overlap on the GPU (two streams, two threads)
// race on it.  Every call looks up the array's device address on the
// current device (cudaGetSymbolAddress; the first lookup on a device loads
// the module, so make the first call before any stream capture).  A call
// without a statistics pointer does not synchronise; its results stay in the
// scratch until the next call and cn_pcg_csr_noalloc_last_stats reads them
// once the caller has synchronised.
#include <cstdio>
#include <cstring>

#include "cn_pcg_body.cuh"

namespace cn {
namespace {

using namespace pcg;

constexpr int kNaMaxRows = 65536;
constexpr int kNaMaxRowsTimesRhs = 196608;
constexpr int kNaBlock = 512;
constexpr int kNaLanes = 2;
constexpr int kNaMaxGrid = 296;
constexpr int kNaMaxK = 9;

constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kOffCtl = 0;
constexpr size_t kOffStats = 256;
constexpr size_t kOffPart = align256(kOffStats + sizeof(DevStats));
constexpr size_t kOffDinv = align256(kOffPart + sizeof(double) * kSlots * kNaMaxGrid * kNaMaxK);
constexpr size_t kOffIdent = align256(kOffDinv + sizeof(double) * kNaMaxRows);
constexpr size_t kOffZero = align256(kOffIdent + sizeof(int) * (kNaMaxRows + 1));
constexpr size_t kOffLev = align256(kOffZero + sizeof(int) * (kNaMaxRows + 1));
constexpr size_t kOffVec = align256(kOffLev + sizeof(int) * 2);
constexpr int kNaVectors = 8;  // r, y, z, p0, p1, Ap, xin, b
constexpr size_t kVecBytes = sizeof(double) * kNaMaxRowsTimesRhs;
constexpr size_t kScratchBytes = kOffVec + kNaVectors * kVecBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Per-call preparation: the control block and statistics start at zero (the
// right-hand-side count goes in the statistics' spare word), the
// Jacobi scale 1/sqrt(A_ii) (a zero diagonal maps to 0 as in
// SparseLinAlg.lean:92-97), the identity row map, the empty strictly-lower
// pattern and the single level [0, n).
__global__ void k_na_prepare(int n, int k, const int* rowptr, const int* colidx, const double* vals,
                             unsigned char* base) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double* dinv = (double*)(base + kOffDinv);
  int* ident = (int*)(base + kOffIdent);
  int* zero = (int*)(base + kOffZero);
  if (i == 0) {
    Control* c = (Control*)(base + kOffCtl);
    c->bar_count = 0; c->bar_gen = 0; c->abort = 0; c->status = 0;
    DevStats* st = (DevStats*)(base + kOffStats);
    st->status = 0; st->iterations = 0; st->refinements = 0; st->pad = k;
    for (int c = 0; c < 32; ++c) st->rel_residual[c] = 0.0;
    int* lev = (int*)(base + kOffLev);
    lev[0] = 0;
    lev[1] = n;
  }
  if (i <= n) {
    ident[i] = i;
    zero[i] = 0;
  }
  if (i < n) {
    double d = 0.0;
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e)
      if (colidx[e] == i) { d = vals[e]; break; }
    dinv[i] = d > 0.0 ? 1.0 / sqrt(d) : 0.0;
  }
}

template <int K>
__global__ void __launch_bounds__(1024) k_na_grid(SolveArgs a) {
  __shared__ Smem<K> s;
  GridTeam team{a.ctl, a.timeout_ns, 0u};
  solve_body<double, K, kNaLanes>(a, team, &s);
}

template <int K>
__global__ void __launch_bounds__(1024) k_na_cta(SolveArgs a) {
  __shared__ Smem<K> s;
  CtaTeam team;
  solve_body<double, K, kNaLanes>(a, team, &s);
}

template <int K>
cudaError_t na_launch(const SolveArgs& a, int n, cudaStream_t st) {
  if (n <= 12288) {
    k_na_cta<K><<<1, kNaBlock, 0, st>>>(a);
    return cudaGetLastError();
  }
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_na_grid<K>, kNaBlock, 0);
  int grid = sms < kNaMaxGrid ? sms : kNaMaxGrid;
  if (per < 1) return cudaErrorLaunchOutOfResources;
  SolveArgs copy = a;
  void* args[] = {&copy};
  return cudaLaunchCooperativeKernel((const void*)k_na_grid<K>, dim3(grid), dim3(kNaBlock), args, 0, st);
}

thread_local char g_na_err[256];

// The message becomes the text of cn_last_error() on this thread.
cn_status na_fail(cn_status s) {
  set_last_error_text(g_na_err);
  return s;
}

// Device address of the scratch on the current device, looked up on every
// call (a cached address would outlive a context reset).
cn_status na_base(unsigned char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    snprintf(g_na_err, sizeof g_na_err, "cudaGetSymbolAddress of the scratch failed: %s", cudaGetErrorString(e));
    return na_fail(CN_CUDA_ERROR);
  }
  *out = (unsigned char*)p;
  return CN_OK;
}

cn_status na_stats(const DevStats& ds, cn_solve_stats* stats) {
  memset(stats, 0, sizeof *stats);
  stats->status = ds.status;
  stats->iterations = ds.iterations;
  stats->refinements = ds.refinements;
  stats->k = ds.pad;
  double mx = 0.0;
  for (int c = 0; c < ds.pad && c < 32; ++c) {
    stats->rel_residual[c] = ds.rel_residual[c];
    mx = mx > ds.rel_residual[c] ? mx : ds.rel_residual[c];
  }
  stats->max_rel_residual = mx;
  return (cn_status)ds.status;
}

}  // namespace
}  // namespace cn

extern "C" cn_status cn_pcg_csr_noalloc(int32_t n, const int32_t* d_rowptr, const int32_t* d_colidx,
                                        const double* d_vals, int32_t k, const double* d_b, double* d_x,
                                        double tol, int32_t max_iter, void* stream,
                                        cn_solve_stats* stats) {
  using namespace cn;
  g_na_err[0] = 0;
  set_last_error_text("");
  if (n < 1 || n > kNaMaxRows) {
    snprintf(g_na_err, sizeof g_na_err, "n = %d is outside 1..%d, the limit of the static scratch", n,
             kNaMaxRows);
    return na_fail(CN_BAD_INPUT);
  }
  if (k != 1 && k != 3 && k != 9) {
    snprintf(g_na_err, sizeof g_na_err, "k = %d: supported right-hand-side counts are 1, 3 and 9", k);
    return na_fail(CN_BAD_INPUT);
  }
  if ((long long)n * k > kNaMaxRowsTimesRhs) {
    snprintf(g_na_err, sizeof g_na_err, "n * k = %lld exceeds %d, the limit of the static scratch",
             (long long)n * k, kNaMaxRowsTimesRhs);
    return na_fail(CN_BAD_INPUT);
  }
  if (!d_rowptr || !d_colidx || !d_vals || !d_b || !d_x || !(tol > 0.0) || max_iter < 0) {
    snprintf(g_na_err, sizeof g_na_err, "null pointer or bad tolerance / iteration limit");
    return na_fail(CN_BAD_INPUT);
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    snprintf(g_na_err, sizeof g_na_err, "no current CUDA device");
    return na_fail(CN_NO_DEVICE);
  }
  unsigned char* B = nullptr;
  if (na_base(&B) != CN_OK) return CN_CUDA_ERROR;
  cudaStream_t st = (cudaStream_t)stream;
  k_na_prepare<<<(n + 1 + 255) / 256, 256, 0, st>>>(n, k, d_rowptr, d_colidx, d_vals, B);
  SolveArgs a{};
  a.n = n;
  a.nlev = 1;
  a.lev_ptr = (const int*)(B + kOffLev);
  a.A_ptr = d_rowptr; a.A_col = d_colidx; a.A_val = d_vals; a.A_val64 = d_vals;
  a.L_ptr = (const int*)(B + kOffZero); a.L_col = (const int*)(B + kOffZero); a.L_val = d_vals;
  a.U_ptr = (const int*)(B + kOffZero); a.U_col = (const int*)(B + kOffZero); a.U_val = d_vals;
  a.dinv = (const void*)(B + kOffDinv);
  a.nv = n; a.nh = 0;
  a.free_of = (const int*)(B + kOffIdent);
  a.mode = CN_MODE_RHS; a.targets = d_b; a.x_out = nullptr; a.x0 = nullptr; a.warm = 1;
  double* vec = (double*)(B + kOffVec);
  const size_t stride = kNaMaxRowsTimesRhs;
  a.r = vec; a.y = vec + stride; a.z = vec + 2 * stride; a.p0 = vec + 3 * stride;
  a.p1 = vec + 4 * stride; a.Ap = vec + 5 * stride; a.xin = vec + 6 * stride;
  a.b64 = vec + 7 * stride;
  a.x64 = d_x;
  a.partials = (double*)(B + kOffPart);
  a.tol = tol; a.inner_tol = 0.0; a.max_iter = max_iter; a.max_refine = 4;
  a.ctl = (Control*)(B + kOffCtl);
  a.stats = (DevStats*)(B + kOffStats);
  a.timeout_ns = 2000000000LL;
  cudaError_t e = k == 1 ? na_launch<1>(a, n, st) : (k == 3 ? na_launch<3>(a, n, st) : na_launch<9>(a, n, st));
  if (e != cudaSuccess) {
    snprintf(g_na_err, sizeof g_na_err, "launch failed: %s", cudaGetErrorString(e));
    return na_fail(CN_CUDA_ERROR);
  }
  if (!stats) return CN_OK;
  DevStats ds;
  e = cudaMemcpyAsync(&ds, B + kOffStats, sizeof ds, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    snprintf(g_na_err, sizeof g_na_err, "solve failed: %s", cudaGetErrorString(e));
    return na_fail(CN_CUDA_ERROR);
  }
  return na_stats(ds, stats);
}

extern "C" cn_status cn_pcg_csr_noalloc_last_stats(cn_solve_stats* stats) {
  using namespace cn;
  g_na_err[0] = 0;
  set_last_error_text("");
  if (!stats) {
    snprintf(g_na_err, sizeof g_na_err, "null statistics pointer");
    return na_fail(CN_BAD_INPUT);
  }
  DevStats ds;
  const cudaError_t e = cudaMemcpyFromSymbol(&ds, g_noalloc_scratch, sizeof ds, kOffStats, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    snprintf(g_na_err, sizeof g_na_err, "reading the statistics failed: %s", cudaGetErrorString(e));
    return na_fail(CN_CUDA_ERROR);
  }
  return na_stats(ds, stats);
}
