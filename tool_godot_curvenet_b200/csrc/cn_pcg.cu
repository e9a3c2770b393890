// cn_pcg.cu -- the persistent preconditioned-CG solve (sm_100a).
//
// One launch performs a whole solve of the handle-constrained system
//   A x = b,  A = K[free, free],  b = -(K diff)_free
// for K right-hand sides: right-hand-side assembly, FP64 residual
// refinement around an inner PCG in T (float for mixed precision, double for
// plain FP64), the IC(0) (or Jacobi) preconditioner applied as level-scheduled
// forward/backward sweeps, and the scatter of the result with the handle
// values overlaid.
//
// Algorithm per inner iteration (SparseLinAlg.lean:137-163 cgWithGuess, with
// the IC(0) apply of IncompleteCholesky.lean:83-101 in place of Jacobi, and
// one colour/level per sweep step as SlangCodegen/IncompleteCholesky.lean:9-12
// schedules it):
//   SPMV  p' = z + beta p ; Ap = A p'            ; pAp        -> barrier
//   FWD_l x += alpha p' ; r -= alpha Ap ; y_l = (r - L y)/L_ll ; rr   -> barrier
//         (the last level also finishes z = y / L_ll)
//   BWD_l z_l = (y - L^T z)/L_ll ; rz                          -> barrier
// so an iteration costs 2 * n_levels team barriers.  The per-column scalars
// (alpha, beta, the stopping test) are reduced deterministically: each block
// writes its partial sums, and after the barrier every block adds all
// partials in the same order, so every block takes the same branch.
//
// The team barrier is a bounded spin on a generation counter (the launch is
// cooperative, so all blocks are co-resident); a wait that runs past
// timeout_ns sets ctl->abort and every block leaves the kernel with status
// CN_TIMEOUT.
#include "cn_pcg_body.cuh"

namespace cn {
namespace {

using namespace pcg;

template <typename T, int K, int G>
__global__ void __launch_bounds__(1024) k_solve_grid(SolveArgs a) {
  __shared__ Smem<K> s;
  GridTeam team{a.ctl, a.timeout_ns, 0u};
  solve_body<T, K, G>(a, team, &s);
}

// One block solving alone.  With a.cache_bytes > 0 the two vectors the
// sweeps and the product gather (y of the forward sweep, z of the backward
// sweep and the SpMV) live in dynamic shared memory for the whole launch, so
// the dependent chain of a level step is a shared-memory round trip instead
// of an L2 one.
template <typename T, int K, int G>
__global__ void __launch_bounds__(1024) k_solve_cta(SolveArgs a) {
  __shared__ Smem<K> s;
  extern __shared__ __align__(16) unsigned char dyn[];
  CtaTeam team;
  if (a.cache_bytes > 0) {
    const size_t half = (((size_t)a.n * K * sizeof(T)) + 15) & ~(size_t)15;
    a.y = dyn;
    a.z = dyn + half;
  }
  solve_body<T, K, G>(a, team, &s);
}

template <typename T, int K, int G>
cudaError_t launch_tg(const SolveArgs& a, int block, int grid, cudaStream_t st) {
  if (grid <= 1) {
    const int dyn = a.cache_bytes;
    if (dyn > 0) {
      const cudaError_t e = cudaFuncSetAttribute(k_solve_cta<T, K, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 dyn);
      if (e != cudaSuccess) return e;
    }
    k_solve_cta<T, K, G><<<1, block, dyn, st>>>(a);
    return cudaGetLastError();
  }
  SolveArgs copy = a;
  void* args[] = {&copy};
  return cudaLaunchCooperativeKernel((const void*)k_solve_grid<T, K, G>, dim3(grid), dim3(block),
                                     args, 0, st);
}

template <typename T, int K, int G>
int max_grid_tg(int block) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_solve_grid<T, K, G>, block, 0);
  return sms * per;
}

template <typename T, int K>
cudaError_t launch_t(const SolveArgs& a, int lanes, int block, int grid, cudaStream_t st) {
  switch (lanes) {
    case 1: return launch_tg<T, K, 1>(a, block, grid, st);
    case 2: return launch_tg<T, K, 2>(a, block, grid, st);
    case 4: return launch_tg<T, K, 4>(a, block, grid, st);
    case 8: return launch_tg<T, K, 8>(a, block, grid, st);
    case 16: return launch_tg<T, K, 16>(a, block, grid, st);
    default: return cudaErrorInvalidValue;
  }
}

template <typename T, int K>
int max_grid_t(int lanes, int block) {
  switch (lanes) {
    case 1: return max_grid_tg<T, K, 1>(block);
    case 2: return max_grid_tg<T, K, 2>(block);
    case 4: return max_grid_tg<T, K, 4>(block);
    case 8: return max_grid_tg<T, K, 8>(block);
    case 16: return max_grid_tg<T, K, 16>(block);
    default: return 0;
  }
}

}  // namespace

cudaError_t launch_persistent_solve(const SolveArgs& a, int precision, int K, int lanes,
                                    int block, int grid, cudaStream_t s) {
  if (precision == CN_PREC_MIXED) {
    if (K == 1) return launch_t<float, 1>(a, lanes, block, grid, s);
    if (K == 3) return launch_t<float, 3>(a, lanes, block, grid, s);
    if (K == 9) return launch_t<float, 9>(a, lanes, block, grid, s);
  } else {
    if (K == 1) return launch_t<double, 1>(a, lanes, block, grid, s);
    if (K == 3) return launch_t<double, 3>(a, lanes, block, grid, s);
    if (K == 9) return launch_t<double, 9>(a, lanes, block, grid, s);
  }
  return cudaErrorInvalidValue;
}

int persistent_max_grid(int precision, int K, int lanes, int block) {
  if (precision == CN_PREC_MIXED) {
    if (K == 1) return max_grid_t<float, 1>(lanes, block);
    if (K == 3) return max_grid_t<float, 3>(lanes, block);
    if (K == 9) return max_grid_t<float, 9>(lanes, block);
  } else {
    if (K == 1) return max_grid_t<double, 1>(lanes, block);
    if (K == 3) return max_grid_t<double, 3>(lanes, block);
    if (K == 9) return max_grid_t<double, 9>(lanes, block);
  }
  return 0;
}

}  // namespace cn
