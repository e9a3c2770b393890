// cn_batch.h -- the batched persistent solve (cn_batch.cu) and its launch.
// Not part of the public ABI.
#pragma once

#include "cn_internal.h"

namespace cn {

struct BatchArgs {
  const SolveArgs* meshes;   // per mesh: matrix, maps, mode, tolerances (vectors unset)
  const int* order;          // processing order (largest first)
  const long long* tgt_off;  // per mesh: offset of its targets in `targets`
  const long long* out_off;  // per mesh: offset of its positions in `x_out`
  const double* targets;     // concatenated handle targets (n_handles_m x K per mesh)
  double* x_out;             // concatenated positions (n_verts_m x K per mesh)
  int n_meshes;
  int* queue;                // work counter, zero at launch
  void* vec_T;               // per cluster: 7 vectors of `stride` elements of the inner type
  double* vec_64;            // per cluster: 2 vectors of `stride` doubles
  size_t stride;             // max rows x K
  DevStats* stats;           // per mesh
  int cluster_base;          // first per-cluster scratch slot of this launch
};

// lanes: lanes per row (K = 24: 8 or 4; K = 3: 1)
cudaError_t launch_batch(const BatchArgs& ba, int precision, int K, int lanes, int csize, int nclusters, int block,
                         cudaStream_t st);
// Co-resident clusters of the batch kernel for this configuration (0 if none).
int batch_max_clusters(int precision, int K, int lanes, int csize, int block);

}  // namespace cn
