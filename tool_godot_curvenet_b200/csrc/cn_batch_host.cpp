// cn_batch_host.cpp -- the batch handle of the C ABI: many meshes built into
// one device allocation, solved by one persistent, CUDA-graph-captured launch
// of the cluster kernel (cn_batch.cu).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

#include "cn_batch.h"
#include "cn_mesh.h"

using cn::BatchArgs;
using cn::DevStats;
using cn::MeshDev;
using cn::MeshHost;
using cn::SolveArgs;
using cn::set_err;

#define CN_CUDA(call)                                                          \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      set_err("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                       \
      return CN_CUDA_ERROR;                                                    \
    }                                                                          \
  } while (0)

struct cn_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cn_build_opts opts{};
  int K = 24, csize = 4, nclusters = 0, block = 512, max_n = 0, nm = 0;
  int ncl_prec[2] = {0, 0};  // clusters launched per precision (CN_PREC_*), <= nclusters (the scratch)
  std::vector<MeshHost> H;
  std::vector<MeshDev> D;
  std::vector<long long> tgt_off, out_off;
  char* buf = nullptr;
  size_t bytes = 0;
  SolveArgs* d_args = nullptr;
  int* d_order = nullptr;
  long long *d_tgt_off = nullptr, *d_out_off = nullptr;
  int* d_queue = nullptr;
  DevStats* d_stats = nullptr;
  int* d_status = nullptr;
  void* d_vecT = nullptr;
  double* d_vec64 = nullptr;
  size_t stride = 0;
  double *d_targets = nullptr, *d_xout = nullptr;
  // captured graph of the last (buffers, options)
  cudaGraphExec_t gexec = nullptr;
  const double* g_t = nullptr;
  double* g_x = nullptr;
  cn_solve_opts g_o{};
  bool have_graph = false;
  std::vector<DevStats> h_stats;
  std::vector<int> lanes;  // lanes per row of each mesh (K = 24: 4 or 8)
  std::vector<int> order_h;  // processing order (largest first)
  cudaStream_t side = nullptr;  // second branch of the captured graph (the 4-lane kernel)
  cudaEvent_t fork = nullptr, join = nullptr;
};

namespace {

void layout_batch(cn::Bump& b, cn_batch* B) {
  for (int m = 0; m < B->nm; ++m) cn::layout(b, B->H[m], B->D[m]);
  B->d_args = b.take<SolveArgs>(B->nm);
  B->d_order = b.take<int>(B->nm);
  B->d_tgt_off = b.take<long long>(B->nm + 1);
  B->d_out_off = b.take<long long>(B->nm + 1);
  B->d_queue = b.take<int>(2);
  B->d_stats = b.take<DevStats>(B->nm);
  B->d_status = b.take<int>(1);
  B->d_vecT = b.take<double>((size_t)B->nclusters * 7 * B->stride);
  B->d_vec64 = b.take<double>((size_t)B->nclusters * 2 * B->stride);
  B->d_targets = b.take<double>(B->tgt_off[B->nm] + 1);
  B->d_xout = b.take<double>(B->out_off[B->nm] + 1);
}

bool same_opts(const cn_solve_opts& a, const cn_solve_opts& b) {
  return a.precision == b.precision && a.mode == b.mode && a.tol == b.tol && a.max_iter == b.max_iter &&
         a.max_refine == b.max_refine && a.inner_tol == b.inner_tol;
}

}  // namespace

extern "C" {

cn_status cn_build_batch(const cn_mesh_desc* meshes, int32_t n_meshes, const cn_build_opts* opts, int32_t k,
                         int32_t cluster_size, int32_t n_clusters, cn_batch_handle* out) {
  cn::set_last_error_text("");
  if (!out || !meshes || n_meshes < 1) {
    set_err("null argument or no meshes");
    return CN_BAD_INPUT;
  }
  *out = nullptr;
  if (k != 3 && k != 24) {
    set_err("batch right-hand-side count k must be 3 or 24 (8 poses x 3)");
    return CN_BAD_INPUT;
  }
  if (cluster_size != 0 && (cluster_size < 1 || cluster_size > 16)) {
    set_err("cluster_size must be 1..16");
    return CN_BAD_INPUT;
  }
  cn_build_opts o;
  if (opts) o = *opts;
  else cn_default_build_opts(&o);
  if (o.precond != CN_PRECOND_IC0 && o.precond != CN_PRECOND_JACOBI) {
    set_err("unsupported preconditioner %d", o.precond);
    return CN_BAD_INPUT;
  }
  for (int m = 0; m < n_meshes; ++m) {
    cn_status st = cn::check_mesh(&meshes[m]);
    if (st != CN_OK) return st;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_err("no CUDA device");
    return CN_NO_DEVICE;
  }
  if (o.device < 0 || o.device >= ndev || cudaSetDevice(o.device) != cudaSuccess) {
    set_err("device %d unavailable", o.device);
    return CN_BAD_INPUT;
  }
  cn_batch* B = new cn_batch;
  B->opts = o;
  B->device = o.device;
  B->K = k;
  B->nm = n_meshes;
  auto fail = [&](cn_status s) {
    cn_destroy_batch(B);
    return s;
  };
  // host structure of every mesh, in parallel
  B->H.resize(n_meshes);
  B->D.resize(n_meshes);
  std::vector<cn_status> st(n_meshes, CN_OK);
  std::vector<std::string> msg(n_meshes);
  {
    std::atomic<int> next(0);
    auto work = [&]() {
      for (int m; (m = next.fetch_add(1)) < n_meshes;) {
        st[m] = cn::build_host(&meshes[m], o, B->H[m]);
        if (st[m] != CN_OK) msg[m] = cn::last_err();
      }
    };
    const int nt = std::max(1, std::min<int>(std::thread::hardware_concurrency(), 32));
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
  }
  for (int m = 0; m < n_meshes; ++m)
    if (st[m] != CN_OK) {
      set_err("mesh %d: %s", m, msg[m].c_str());
      return fail(st[m]);
    }
  B->tgt_off.assign(n_meshes + 1, 0);
  B->out_off.assign(n_meshes + 1, 0);
  for (int m = 0; m < n_meshes; ++m) {
    B->tgt_off[m + 1] = B->tgt_off[m] + (long long)B->H[m].nh * k;
    B->out_off[m + 1] = B->out_off[m] + (long long)B->H[m].nv * k;
    B->max_n = std::max(B->max_n, B->H[m].n);
  }
  B->stride = (size_t)std::max(B->max_n, 1) * k;
  // launch shape: clusters of csize blocks, as many as are co-resident
  B->block = o.block > 0 ? o.block : 512;
  B->csize = cluster_size > 0 ? cluster_size : 4;
  // each precision launches as many clusters as are co-resident for its kernel
  // (FP32 fits more per SM); the per-cluster scratch is sized for the larger
  const int l0 = k == 24 ? 8 : 1;
  const int mc64 = cn::batch_max_clusters(CN_PREC_FP64, k, l0, B->csize, B->block);
  const int mc32 = cn::batch_max_clusters(CN_PREC_MIXED, k, l0, B->csize, B->block);
  if (mc64 <= 0 || mc32 <= 0) {
    set_err("no co-resident cluster of %d x %d threads fits this device", B->csize, B->block);
    return fail(CN_CUDA_ERROR);
  }
  B->ncl_prec[CN_PREC_FP64] = n_clusters > 0 ? std::min(n_clusters, mc64) : mc64;
  B->ncl_prec[CN_PREC_MIXED] = n_clusters > 0 ? std::min(n_clusters, mc32) : mc32;
  B->nclusters = std::max(B->ncl_prec[CN_PREC_FP64], B->ncl_prec[CN_PREC_MIXED]);
  if (cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&B->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&B->join, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreate(&B->ev0) != cudaSuccess || cudaEventCreate(&B->ev1) != cudaSuccess) {
    set_err("stream/event creation failed");
    return fail(CN_CUDA_ERROR);
  }
  cn::Bump sizing;
  layout_batch(sizing, B);
  if (cudaMalloc((void**)&B->buf, sizing.off) != cudaSuccess) {
    set_err("device allocation of %zu bytes failed", sizing.off);
    return fail(CN_CUDA_ERROR);
  }
  B->bytes = sizing.off;
  cn::Bump real;
  real.base = B->buf;
  layout_batch(real, B);
  if (cudaMemsetAsync(B->buf, 0, B->bytes, B->stream) != cudaSuccess) {
    set_err("device memset failed");
    return fail(CN_CUDA_ERROR);
  }
  for (int m = 0; m < n_meshes; ++m) {
    cn_status s = cn::upload(B->H[m], B->D[m], B->stream);
    if (s == CN_OK) s = cn::assemble_factor(B->H[m], B->D[m], o, B->d_status, B->stream, nullptr);
    if (s != CN_OK) {
      const std::string e = cn::last_err();
      set_err("mesh %d: %s", m, e.c_str());
      return fail(s);
    }
  }
  // largest systems first (longest-processing-time order over the clusters)
  std::vector<int> order(n_meshes);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const long long ca = (long long)B->H[a].nnzA + 2LL * B->H[a].nnzL;
    const long long cb = (long long)B->H[b].nnzA + 2LL * B->H[b].nnzL;
    return ca > cb;
  });
  B->order_h = order;
  if (cudaMemcpyAsync(B->d_order, order.data(), sizeof(int) * n_meshes, cudaMemcpyHostToDevice, B->stream) ||
      cudaMemcpyAsync(B->d_tgt_off, B->tgt_off.data(), sizeof(long long) * (n_meshes + 1),
                      cudaMemcpyHostToDevice, B->stream) ||
      cudaMemcpyAsync(B->d_out_off, B->out_off.data(), sizeof(long long) * (n_meshes + 1),
                      cudaMemcpyHostToDevice, B->stream) ||
      cudaStreamSynchronize(B->stream)) {
    set_err("batch tables upload failed");
    return fail(CN_CUDA_ERROR);
  }
  B->h_stats.resize(n_meshes);
  B->lanes.assign(n_meshes, k == 24 ? 8 : 1);
  *out = B;
  return CN_OK;
}

cn_status cn_batch_set_lanes(cn_batch_handle B, int32_t n_classes, const int32_t* class_max_rows,
                             const int32_t* lanes) {
  if (!B || n_classes < 1 || !class_max_rows || !lanes) {
    set_err("null argument or no size class");
    return CN_BAD_INPUT;
  }
  for (int c = 0; c < n_classes; ++c) {
    const bool ok = B->K == 24 ? (lanes[c] == 4 || lanes[c] == 8) : lanes[c] == 1;
    if (!ok || (c > 0 && class_max_rows[c] <= class_max_rows[c - 1])) {
      set_err("size class %d: lanes per row must be 4 or 8 for k = 24 (1 for k = 3) and the bounds must rise", c);
      return CN_BAD_INPUT;
    }
  }
  for (int m = 0; m < B->nm; ++m) {
    int c = 0;
    while (c < n_classes - 1 && B->H[m].n > class_max_rows[c]) ++c;
    B->lanes[m] = lanes[c];
  }
  B->have_graph = false;  // the per-mesh arguments change: capture again
  return CN_OK;
}

cn_status cn_batch_lanes(cn_batch_handle B, int32_t* lanes) {
  if (!B || !lanes) return CN_BAD_INPUT;
  for (int m = 0; m < B->nm; ++m) lanes[m] = B->lanes[m];
  return CN_OK;
}

void cn_destroy_batch(cn_batch_handle B) {
  if (!B) return;
  cudaSetDevice(B->device);
  if (B->stream) cudaStreamSynchronize(B->stream);
  if (B->gexec) cudaGraphExecDestroy(B->gexec);
  if (B->buf) cudaFree(B->buf);
  if (B->ev0) cudaEventDestroy(B->ev0);
  if (B->ev1) cudaEventDestroy(B->ev1);
  if (B->stream) cudaStreamDestroy(B->stream);
  if (B->side) cudaStreamDestroy(B->side);
  if (B->fork) cudaEventDestroy(B->fork);
  if (B->join) cudaEventDestroy(B->join);
  delete B;
}

void* cn_batch_stream(cn_batch_handle B) { return B ? (void*)B->stream : nullptr; }

cn_status cn_batch_info(cn_batch_handle B, int64_t* info) {
  if (!B || !info) return CN_BAD_INPUT;
  int64_t nv = 0, nh = 0, nf = 0, na = 0, nl = 0;
  for (const MeshHost& h : B->H) { nv += h.nv; nh += h.nh; nf += h.n; na += h.nnzA; nl += h.nnzL; }
  int64_t v[12] = {B->nm, B->K, nv, nh, nf, na, nl, B->csize, B->nclusters, B->block, B->max_n,
                   (int64_t)B->bytes};
  std::memcpy(info, v, sizeof v);
  return CN_OK;
}

cn_status cn_batch_offsets(cn_batch_handle B, int64_t* tgt_off, int64_t* out_off) {
  if (!B) return CN_BAD_INPUT;
  for (int m = 0; m <= B->nm; ++m) {
    if (tgt_off) tgt_off[m] = B->tgt_off[m];
    if (out_off) out_off[m] = B->out_off[m];
  }
  return CN_OK;
}

cn_status cn_batch_mesh_stats(cn_batch_handle B, int32_t* status, int32_t* iterations, double* max_rel,
                              int32_t* refinements) {
  if (!B) return CN_BAD_INPUT;
  for (int m = 0; m < B->nm; ++m) {
    const DevStats& d = B->h_stats[m];
    if (status) status[m] = d.status;
    if (iterations) iterations[m] = d.iterations;
    if (refinements) refinements[m] = d.refinements;
    if (max_rel) {
      double mx = 0.0;
      for (int c = 0; c < B->K && c < 32; ++c) mx = std::max(mx, d.rel_residual[c]);
      max_rel[m] = mx;
    }
  }
  return CN_OK;
}

cn_status cn_solve_batch_device(cn_batch_handle B, const double* d_targets, double* d_x_out,
                                const cn_solve_opts* opts, cn_batch_stats* stats) {
  if (!B || !d_targets) {
    set_err("null argument");
    return CN_BAD_INPUT;
  }
  cn_solve_opts o;
  if (opts) o = *opts;
  else cn_default_solve_opts(&o);
  if (!(o.tol > 0.0) || o.max_iter < 0 || o.max_refine < 1 || o.algo == CN_ALGO_PLAIN) {
    set_err("bad solve options for a batch");
    return CN_BAD_INPUT;
  }
  CN_CUDA(cudaSetDevice(B->device));
  const bool mixed = o.precision == CN_PREC_MIXED;
  if (!B->have_graph || B->g_t != d_targets || B->g_x != d_x_out || !same_opts(B->g_o, o)) {
    std::vector<SolveArgs> args(B->nm);
    for (int m = 0; m < B->nm; ++m) {
      SolveArgs a = cn::solve_args(B->H[m], B->D[m], mixed);
      a.mode = o.mode;
      a.warm = 0;
      a.tol = o.tol;
      a.inner_tol = mixed ? o.inner_tol : 0.0;
      a.max_iter = o.max_iter;
      a.max_refine = o.max_refine;
      args[m] = a;
    }
    CN_CUDA(cudaMemcpyAsync(B->d_args, args.data(), sizeof(SolveArgs) * B->nm, cudaMemcpyHostToDevice,
                            B->stream));
    CN_CUDA(cudaStreamSynchronize(B->stream));
    // the meshes of each lanes value in processing order: group 0 (8 lanes,
    // or 1 for k = 3) first, group 1 (4 lanes) after it in d_order
    std::vector<int> grp[2];
    double cost[2] = {0.0, 0.0};
    for (int m : B->order_h) {
      const int gi = B->lanes[m] == 4 ? 1 : 0;
      grp[gi].push_back(m);
      cost[gi] += (double)B->H[m].nnzA + 2.0 * B->H[m].nnzL + 4.0 * B->H[m].n;
    }
    std::vector<int> ord(grp[0]);
    ord.insert(ord.end(), grp[1].begin(), grp[1].end());
    CN_CUDA(cudaMemcpyAsync(B->d_order, ord.data(), sizeof(int) * B->nm, cudaMemcpyHostToDevice, B->stream));
    CN_CUDA(cudaStreamSynchronize(B->stream));
    // clusters of each kernel: the co-resident total, split by work
    const int total = B->ncl_prec[o.precision == CN_PREC_MIXED];
    int ncl[2] = {total, 0};
    bool side_by_side = true;  // else the 4-lane kernel runs after the 8-lane one
    if (!grp[1].empty()) {
      const int mc4 = cn::batch_max_clusters(o.precision, B->K, 4, B->csize, B->block);
      const int tot = std::min(total, mc4 > 0 ? mc4 : total);
      if (grp[0].empty()) {
        ncl[0] = 0;
        ncl[1] = tot;
      } else if (tot >= 2) {
        ncl[1] = std::max(1, std::min(tot - 1, (int)std::lround(tot * cost[1] / (cost[0] + cost[1]))));
        ncl[0] = tot - ncl[1];
      } else {
        side_by_side = false;
        ncl[0] = ncl[1] = tot;
      }
    }
    BatchArgs ba[2] = {};
    for (int gi = 0; gi < 2; ++gi) {
      BatchArgs& b = ba[gi];
      b.meshes = B->d_args;
      b.order = B->d_order + (gi ? grp[0].size() : 0);
      b.tgt_off = B->d_tgt_off;
      b.out_off = B->d_out_off;
      b.targets = d_targets;
      b.x_out = d_x_out;
      b.n_meshes = (int)grp[gi].size();
      b.queue = B->d_queue + gi;
      b.vec_T = B->d_vecT;
      b.vec_64 = B->d_vec64;
      b.stride = B->stride;
      b.stats = B->d_stats;
      b.cluster_base = gi && side_by_side ? ncl[0] : 0;
    }
    if (B->gexec) {
      cudaGraphExecDestroy(B->gexec);
      B->gexec = nullptr;
    }
    cudaGraph_t g = nullptr;
    CN_CUDA(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e1 = cudaMemsetAsync(B->d_queue, 0, 2 * sizeof(int), B->stream);
    cudaError_t e2 = cudaSuccess;
    const bool fork = ncl[1] > 0 && side_by_side;
    if (fork) {  // the 4-lane kernel on a parallel branch of the graph
      if (e2 == cudaSuccess) e2 = cudaEventRecord(B->fork, B->stream);
      if (e2 == cudaSuccess) e2 = cudaStreamWaitEvent(B->side, B->fork, 0);
      if (e2 == cudaSuccess) e2 = cn::launch_batch(ba[1], o.precision, B->K, 4, B->csize, ncl[1], B->block, B->side);
      if (e2 == cudaSuccess) e2 = cudaEventRecord(B->join, B->side);
    }
    if (e2 == cudaSuccess && ncl[0] > 0)
      e2 = cn::launch_batch(ba[0], o.precision, B->K, B->K == 24 ? 8 : 1, B->csize, ncl[0], B->block, B->stream);
    if (e2 == cudaSuccess && ncl[1] > 0 && !side_by_side)
      e2 = cn::launch_batch(ba[1], o.precision, B->K, 4, B->csize, ncl[1], B->block, B->stream);
    if (e2 == cudaSuccess && fork) e2 = cudaStreamWaitEvent(B->stream, B->join, 0);
    cudaError_t e3 = cudaStreamEndCapture(B->stream, &g);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
      set_err("graph capture failed: %s / %s / %s", cudaGetErrorString(e1), cudaGetErrorString(e2),
              cudaGetErrorString(e3));
      if (g) cudaGraphDestroy(g);
      return CN_CUDA_ERROR;
    }
    cudaError_t e4 = cudaGraphInstantiate(&B->gexec, g, 0);
    cudaGraphDestroy(g);
    if (e4 != cudaSuccess) {
      set_err("graph instantiation failed: %s", cudaGetErrorString(e4));
      return CN_CUDA_ERROR;
    }
    B->have_graph = true;
    B->g_t = d_targets;
    B->g_x = d_x_out;
    B->g_o = o;
  }
  CN_CUDA(cudaEventRecord(B->ev0, B->stream));
  CN_CUDA(cudaGraphLaunch(B->gexec, B->stream));
  CN_CUDA(cudaEventRecord(B->ev1, B->stream));
  if (!stats) return CN_OK;
  CN_CUDA(cudaMemcpyAsync(B->h_stats.data(), B->d_stats, sizeof(DevStats) * B->nm, cudaMemcpyDeviceToHost,
                          B->stream));
  CN_CUDA(cudaStreamSynchronize(B->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, B->ev0, B->ev1);
  std::memset(stats, 0, sizeof *stats);
  stats->n_meshes = B->nm;
  stats->device_ms = ms;
  int worst = CN_OK;
  for (int m = 0; m < B->nm; ++m) {
    const DevStats& d = B->h_stats[m];
    if (d.status != CN_OK) {
      stats->n_failed++;
      if (worst == CN_OK || d.status > worst) worst = d.status;
    }
    stats->max_iterations = std::max(stats->max_iterations, d.iterations);
    stats->total_iterations += d.iterations;
    for (int c = 0; c < B->K && c < 32; ++c) stats->max_rel_residual = std::max(stats->max_rel_residual, d.rel_residual[c]);
  }
  stats->status = worst;
  return (cn_status)worst;
}

cn_status cn_solve_batch(cn_batch_handle B, const double* targets, double* x_out, const cn_solve_opts* opts,
                         cn_batch_stats* stats) {
  if (!B || !targets || !x_out) {
    set_err("null argument");
    return CN_BAD_INPUT;
  }
  CN_CUDA(cudaSetDevice(B->device));
  const long long nt = B->tgt_off[B->nm], no = B->out_off[B->nm];
  for (long long i = 0; i < nt; ++i)
    if (!std::isfinite(targets[i])) {
      set_err("target %lld is not finite", i);
      return CN_NAN;
    }
  CN_CUDA(cudaMemcpyAsync(B->d_targets, targets, sizeof(double) * nt, cudaMemcpyHostToDevice, B->stream));
  cn_batch_stats local;
  cn_status st = cn_solve_batch_device(B, B->d_targets, B->d_xout, opts, stats ? stats : &local);
  if (st != CN_OK && st != CN_MAX_ITER) return st;
  CN_CUDA(cudaMemcpyAsync(x_out, B->d_xout, sizeof(double) * no, cudaMemcpyDeviceToHost, B->stream));
  CN_CUDA(cudaStreamSynchronize(B->stream));
  return st;
}

}  // extern "C"
