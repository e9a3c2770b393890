// cn_cutmesh.cu -- cut-mesh construction on the GPU: the halfedge structure of
// a triangle soup (HalfedgeBuilder.lean:34-90), the seam cut along closed
// profile-curve loops, and batches of the cut surgery operations
// subdivideEdge / splitFace / insertCrack (CutAlgorithm.lean:49-255).
//
// Halfedge records are 4 int32: target, twin (-1: none), next, face (-1: the
// outer face).  The builder reproduces the specification's numbering: the
// interior halfedges 3f, 3f+1, 3f+2 of face f run t0->t1, t1->t2, t2->t0;
// the twin of an interior halfedge is the lowest interior index with the
// reversed (source, target) (the spec's first-match scan, here a hash table
// of directed edges keeping the minimum index); every interior halfedge
// without one gets a boundary halfedge, appended in interior index order (a
// prefix sum over the orphan flags); a boundary halfedge's next is the lowest
// boundary index whose source is its target (itself if none).
//
// A batch of surgery operations equals the same operations applied one after
// another in batch order (new vertex, face and halfedge indices are assigned
// by position in the batch) because the host admits only batches whose
// operations touch disjoint records: distinct edges (and twins) for
// subdivideEdge, distinct faces for splitFace, distinct anchors for
// insertCrack.
#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "cn_mesh.h"

namespace cn {
namespace {

constexpr unsigned long long kEmptyKey = ~0ull;
constexpr int kUnset = 0x7f7f7f7f;  // what a 0x7f byte fill leaves: above every index

__device__ __forceinline__ unsigned long long edge_key(int src, int tgt) {
  return ((unsigned long long)(unsigned)src << 32) | (unsigned)tgt;
}

__device__ __forceinline__ unsigned hash_slot(unsigned long long k, unsigned mask) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return (unsigned)k & mask;
}

// keep the minimum value per key (linear probing; the table is at least
// twice the number of keys, so a probe always ends)
__device__ void table_insert(unsigned long long* keys, int* vals, unsigned mask, unsigned long long k, int v) {
  unsigned s = hash_slot(k, mask);
  for (unsigned probe = 0; probe <= mask; ++probe) {
    const unsigned long long prev = atomicCAS(keys + s, kEmptyKey, k);
    if (prev == kEmptyKey || prev == k) {
      atomicMin(vals + s, v);
      return;
    }
    s = (s + 1) & mask;
  }
}

__device__ int table_find(const unsigned long long* keys, const int* vals, unsigned mask, unsigned long long k) {
  unsigned s = hash_slot(k, mask);
  for (unsigned probe = 0; probe <= mask; ++probe) {
    const unsigned long long cur = keys[s];
    if (cur == k) return vals[s];
    if (cur == kEmptyKey) return -1;
    s = (s + 1) & mask;
  }
  return -1;
}

__device__ __forceinline__ int src_of(const int* tris, int h) { return tris[h]; }
__device__ __forceinline__ int tgt_of(const int* tris, int h) { return tris[3 * (h / 3) + (h % 3 + 1) % 3]; }

__global__ void k_he_insert(int nint, const int* tris, unsigned long long* keys, int* vals, unsigned mask) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < nint) table_insert(keys, vals, mask, edge_key(src_of(tris, j), tgt_of(tris, j)), j);
}

// interior records (HalfedgeBuilder.lean:40-47) and twins (:49-61)
__global__ void k_he_interior(int nint, const int* tris, const unsigned long long* keys, const int* vals,
                              unsigned mask, int* he, int* orphan) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nint) return;
  const int f = i / 3, l = i % 3;
  const int tw = table_find(keys, vals, mask, edge_key(tgt_of(tris, i), src_of(tris, i)));
  int* r = he + 4 * (size_t)i;
  r[0] = tgt_of(tris, i);
  r[1] = tw;
  r[2] = 3 * f + (l + 1) % 3;
  r[3] = f;
  orphan[i] = tw < 0 ? 1 : 0;
}

// boundary halfedges (:62-70): bh = nint + rank of the orphan
__global__ void k_he_boundary(int nint, const int* tris, const int* orphan, const int* rank, int* he,
                              int* first_by_src) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nint || !orphan[i]) return;
  const int bh = nint + rank[i];
  int* r = he + 4 * (size_t)bh;
  r[0] = src_of(tris, i);
  r[1] = i;
  r[3] = -1;
  he[4 * (size_t)i + 1] = bh;
  atomicMin(first_by_src + tgt_of(tris, i), bh);  // the source of bh is the target of i
}

// boundary loop links (:71-87)
__global__ void k_he_boundary_next(int nint, int nb, const int* first_by_src, int* he) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nb) return;
  const int bh = nint + k;
  const int nx = first_by_src[he[4 * (size_t)bh]];
  he[4 * (size_t)bh + 2] = nx == kUnset ? bh : nx;
}

// Exclusive prefix sum of int flags: per block of 1024 x 4 elements, then
// the block totals in one block, then the offsets.
constexpr int kScanPer = 4096;

__global__ void k_scan_block(int n, const int* in, int* out, int* totals) {
  __shared__ int warp_sums[32];
  const int base = blockIdx.x * kScanPer + threadIdx.x * 4;
  int v[4], s = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    v[i] = base + i < n ? in[base + i] : 0;
    s += v[i];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = warp_sums[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    warp_sums[lane] = w;
  }
  __syncthreads();
  int run = x - s + (warp > 0 ? warp_sums[warp - 1] : 0);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (base + i < n) out[base + i] = run;
    run += v[i];
  }
  if (threadIdx.x == blockDim.x - 1) totals[blockIdx.x] = run;
}

__global__ void k_scan_totals(int nblk, int* totals, int* grand) {
  if (threadIdx.x == 0) {
    int run = 0;
    for (int b = 0; b < nblk; ++b) {
      const int t = totals[b];
      totals[b] = run;
      run += t;
    }
    *grand = run;
  }
}

__global__ void k_scan_add(int n, int* out, const int* totals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += totals[i / kScanPer];
}

// The seam cut: one thread per loop vertex (flat index i over all loops);
// its copy is n_verts + i.  Faces swept counter-clockwise around v from the
// one holding the interior halfedge v -> next up to, not including, the one
// holding v -> prev take the copy at v's corner.  The sweep steps to
// twin(prev(h)), the rotation the spec's surgery preserves.
__global__ void k_cut(int nv, int nint, int total, const int* loop_ptr, const int* loop_of, const int* lv,
                      const int* tris, const int* he, const unsigned long long* keys, const int* vals,
                      unsigned mask, int nhe, int* tris_out, int* parent, int* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int l = loop_of[i], lo = loop_ptr[l], m = loop_ptr[l + 1] - lo, p = i - lo;
  const int v = lv[i], vn = lv[lo + (p + 1) % m], vp = lv[lo + (p - 1 + m) % m];
  const int copy = nv + i;
  parent[copy] = v;
  int h = table_find(keys, vals, mask, edge_key(v, vn));
  if (h < 0) {
    atomicExch(err, 1);
    return;
  }
  for (int guard = 0;; ) {
    if (h >= nint || ++guard > nhe) {  // a halfedge of the outer face: the fan is open
      atomicExch(err, 1);
      return;
    }
    const int f = h / 3;
    for (int c = 0; c < 3; ++c)
      if (tris[3 * f + c] == v) tris_out[3 * f + c] = copy;
    const int pv = 3 * f + (h % 3 + 2) % 3;
    const int t = he[4 * (size_t)pv + 1];
    if (t < 0) {
      atomicExch(err, 1);
      return;
    }
    if (he[4 * (size_t)t] == vp) break;
    h = t;
  }
}

// CutAlgorithm.lean:49-100 subdivideEdge, op k of a batch
__global__ void k_subdivide(int m, const int* edges, int nv, int nh, int* he) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const int h = edges[k];
  int o[4], t[4];
  for (int q = 0; q < 4; ++q) o[q] = he[4 * (size_t)h + q];
  const int twin = o[1] >= 0 ? o[1] : h;
  for (int q = 0; q < 4; ++q) t[q] = he[4 * (size_t)twin + q];
  const int c = nv + k, hnew = nh + 2 * k, tnew = nh + 2 * k + 1;
  const int H[4] = {c, tnew, hnew, o[3]};
  const int Hn[4] = {o[0], twin, o[2], o[3]};
  const int Tw[4] = {c, hnew, tnew, t[3]};
  const int Tn[4] = {t[0], h, t[2], t[3]};
  for (int q = 0; q < 4; ++q) he[4 * (size_t)h + q] = H[q];
  for (int q = 0; q < 4; ++q) he[4 * (size_t)twin + q] = Tw[q];
  for (int q = 0; q < 4; ++q) he[4 * (size_t)hnew + q] = Hn[q];
  for (int q = 0; q < 4; ++q) he[4 * (size_t)tnew + q] = Tn[q];
}

// CutAlgorithm.lean:125-170 splitFace, op k of a batch (faces distinct)
__global__ void k_split(int m, const int* as, const int* bs, int nf, int nh, int* he) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const int a = as[k], b = bs[k];
  int A[4], B[4];
  for (int q = 0; q < 4; ++q) {
    A[q] = he[4 * (size_t)a + q];
    B[q] = he[4 * (size_t)b + q];
  }
  const int nhk = nh + 2 * k;  // the halfedge count when this op runs in batch order
  const int fp = nf + k, hAB = nhk, hBA = nhk + 1;
  int cur = B[2], steps = 0;
  while (cur != a && steps < nhk) {
    he[4 * (size_t)cur + 3] = fp;
    cur = he[4 * (size_t)cur + 2];
    ++steps;
  }
  he[4 * (size_t)a + 3] = fp;
  he[4 * (size_t)a + 2] = hAB;
  he[4 * (size_t)b + 2] = hBA;
  const int AB[4] = {B[0], hBA, B[2], fp};
  const int BA[4] = {A[0], hAB, A[2], A[3]};
  for (int q = 0; q < 4; ++q) he[4 * (size_t)hAB + q] = AB[q];
  for (int q = 0; q < 4; ++q) he[4 * (size_t)hBA + q] = BA[q];
}

// CutAlgorithm.lean:225-251 insertCrack, op k of a batch (anchors distinct)
__global__ void k_crack(int m, const int* anchors, int nv, int nh, int* he) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const int a = anchors[k];
  int An[4];
  for (int q = 0; q < 4; ++q) An[q] = he[4 * (size_t)a + q];
  const int c = nv + k, hout = nh + 2 * k, hin = nh + 2 * k + 1;
  he[4 * (size_t)a + 2] = hout;
  const int O[4] = {c, hin, hin, An[3]};
  const int I[4] = {An[0], hout, An[2], An[3]};
  for (int q = 0; q < 4; ++q) he[4 * (size_t)hout + q] = O[q];
  for (int q = 0; q < 4; ++q) he[4 * (size_t)hin + q] = I[q];
}

int blocks_for(long long n, int b) { return (int)((n + b - 1) / b); }

// Device buffers of one call, freed on every return path.
struct Scratch {
  std::vector<void*> ptrs;
  ~Scratch() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <class Tp>
  cudaError_t get(Tp** p, size_t n) {
    *p = nullptr;
    const cudaError_t e = cudaMalloc((void**)p, sizeof(Tp) * (n > 0 ? n : 1));
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
};

#define CM_CUDA(call)                                                                      \
  do {                                                                                     \
    const cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                               \
      set_err("%s failed: %s", #call, cudaGetErrorString(e_));                             \
      return CN_CUDA_ERROR;                                                                \
    }                                                                                      \
  } while (0)

cn_status need_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    set_err("no CUDA device");
    return CN_NO_DEVICE;
  }
  return CN_OK;
}

// The halfedge records of a triangle soup on the device (d_he capacity
// 6 nt x 4), plus the directed-edge table the cut reuses.
struct HeBuild {
  unsigned long long* keys = nullptr;
  int* vals = nullptr;
  unsigned mask = 0;
  int n_he = 0;
};

cn_status build_halfedges_dev(Scratch& sc, int nv, int nt, const int* d_tris, int* d_he, HeBuild* out) {
  const int nint = 3 * nt;
  unsigned cap = 1024;
  while (cap < 2u * (unsigned)nint) cap <<= 1;
  HeBuild& b = *out;
  b.mask = cap - 1;
  int *orphan = nullptr, *rank = nullptr, *totals = nullptr, *grand = nullptr, *first = nullptr;
  const int nblk = blocks_for(nint, kScanPer);
  CM_CUDA(sc.get(&b.keys, cap));
  CM_CUDA(sc.get(&b.vals, cap));
  CM_CUDA(sc.get(&orphan, nint));
  CM_CUDA(sc.get(&rank, nint));
  CM_CUDA(sc.get(&totals, nblk));
  CM_CUDA(sc.get(&grand, 1));
  CM_CUDA(sc.get(&first, nv));
  CM_CUDA(cudaMemset(b.keys, 0xff, sizeof(unsigned long long) * cap));
  CM_CUDA(cudaMemset(b.vals, 0x7f, sizeof(int) * cap));
  CM_CUDA(cudaMemset(first, 0x7f, sizeof(int) * (size_t)(nv > 0 ? nv : 1)));
  CM_CUDA(cudaMemset(grand, 0, sizeof(int)));
  if (nint > 0) {
    k_he_insert<<<blocks_for(nint, 256), 256>>>(nint, d_tris, b.keys, b.vals, b.mask);
    k_he_interior<<<blocks_for(nint, 256), 256>>>(nint, d_tris, b.keys, b.vals, b.mask, d_he, orphan);
    k_scan_block<<<nblk, 1024>>>(nint, orphan, rank, totals);
    k_scan_totals<<<1, 32>>>(nblk, totals, grand);
    k_scan_add<<<blocks_for(nint, 256), 256>>>(nint, rank, totals);
  }
  CM_CUDA(cudaGetLastError());
  int nb = 0;
  CM_CUDA(cudaMemcpy(&nb, grand, sizeof(int), cudaMemcpyDeviceToHost));
  if (nint > 0) {
    k_he_boundary<<<blocks_for(nint, 256), 256>>>(nint, d_tris, orphan, rank, d_he, first);
    if (nb > 0) k_he_boundary_next<<<blocks_for(nb, 256), 256>>>(nint, nb, first, d_he);
  }
  CM_CUDA(cudaGetLastError());
  CM_CUDA(cudaDeviceSynchronize());
  b.n_he = nint + nb;
  return CN_OK;
}

cn_status check_tris(int nv, int nt, const int* tris) {
  if (nv < 0 || nt < 0 || (nt > 0 && !tris)) {
    set_err("bad arguments");
    return CN_BAD_INPUT;
  }
  if ((long long)nt * 3 > INT_MAX / 4) {
    set_err("too many triangles");
    return CN_BAD_INPUT;
  }
  for (long long i = 0; i < 3LL * nt; ++i)
    if (tris[i] < 0 || tris[i] >= nv) {
      set_err("triangle vertex out of range");
      return CN_BAD_INPUT;
    }
  return CN_OK;
}

// Counts and halfedge checks shared by the surgery batches.
cn_status check_surgery(const int32_t* counts, const int32_t* he, int m) {
  if (!counts || !he || m < 0) {
    set_err("null argument or negative batch size");
    return CN_BAD_INPUT;
  }
  if (counts[0] < 0 || counts[1] < 0 || counts[2] < 0 || (long long)counts[2] + 2LL * m > INT_MAX / 4) {
    set_err("bad counts");
    return CN_BAD_INPUT;
  }
  return CN_OK;
}

}  // namespace
}  // namespace cn

using cn::set_err;

extern "C" {

cn_status cn_halfedges(int32_t n_verts, int32_t n_tris, const int32_t* tris, int32_t* he_out, int32_t* n_he_out) {
  cn::set_last_error_text("");
  if (!he_out || !n_he_out) {
    set_err("null argument");
    return CN_BAD_INPUT;
  }
  cn_status st = cn::check_tris(n_verts, n_tris, tris);
  if (st != CN_OK) return st;
  if ((st = cn::need_device()) != CN_OK) return st;
  cn::Scratch sc;
  int *d_tris = nullptr, *d_he = nullptr;
  CM_CUDA(sc.get(&d_tris, 3 * (size_t)n_tris));
  CM_CUDA(sc.get(&d_he, 4 * 6 * (size_t)n_tris));
  if (n_tris) CM_CUDA(cudaMemcpy(d_tris, tris, sizeof(int) * 3 * (size_t)n_tris, cudaMemcpyHostToDevice));
  cn::HeBuild b;
  if ((st = cn::build_halfedges_dev(sc, n_verts, n_tris, d_tris, d_he, &b)) != CN_OK) return st;
  if (b.n_he) CM_CUDA(cudaMemcpy(he_out, d_he, sizeof(int) * 4 * (size_t)b.n_he, cudaMemcpyDeviceToHost));
  *n_he_out = b.n_he;
  return CN_OK;
}

cn_status cn_cut_mesh_gpu(int32_t n_verts, int32_t n_tris, const int32_t* tris, int32_t n_loops,
                          const int32_t* loop_ptr, const int32_t* loop_verts, int32_t* tris_out,
                          int32_t* parent_out, int32_t* n_verts_out) {
  cn::set_last_error_text("");
  if (n_loops < 0 || !tris_out || !parent_out || !n_verts_out || (n_loops > 0 && (!loop_ptr || !loop_verts))) {
    set_err("bad arguments");
    return CN_BAD_INPUT;
  }
  cn_status st = cn::check_tris(n_verts, n_tris, tris);
  if (st != CN_OK) return st;
  // loops: at least 3 vertices, in range, no vertex in two loops (or twice)
  const int total = n_loops > 0 ? loop_ptr[n_loops] : 0;
  std::vector<int> loop_of((size_t)(total > 0 ? total : 1));
  std::vector<char> seen((size_t)(n_verts > 0 ? n_verts : 1), 0);
  if (n_loops > 0 && loop_ptr[0] != 0) {
    set_err("loop_ptr[0] must be 0");
    return CN_BAD_INPUT;
  }
  for (int l = 0; l < n_loops; ++l) {
    const int lo = loop_ptr[l], hi = loop_ptr[l + 1];
    if (hi - lo < 3) {
      set_err("loop %d has fewer than 3 vertices", l);
      return CN_BAD_INPUT;
    }
    for (int i = lo; i < hi; ++i) {
      const int v = loop_verts[i];
      if (v < 0 || v >= n_verts || seen[v]) {
        set_err("loop vertex %d out of range or in two loops", v);
        return CN_BAD_INPUT;
      }
      seen[v] = 1;
      loop_of[i] = l;
    }
  }
  if ((st = cn::need_device()) != CN_OK) return st;
  cn::Scratch sc;
  int *d_tris = nullptr, *d_he = nullptr, *d_out = nullptr, *d_parent = nullptr, *d_lp = nullptr,
      *d_lof = nullptr, *d_lv = nullptr, *d_err = nullptr;
  CM_CUDA(sc.get(&d_tris, 3 * (size_t)n_tris));
  CM_CUDA(sc.get(&d_he, 4 * 6 * (size_t)n_tris));
  CM_CUDA(sc.get(&d_out, 3 * (size_t)n_tris));
  CM_CUDA(sc.get(&d_parent, (size_t)n_verts + total));
  CM_CUDA(sc.get(&d_lp, (size_t)n_loops + 1));
  CM_CUDA(sc.get(&d_lof, (size_t)total));
  CM_CUDA(sc.get(&d_lv, (size_t)total));
  CM_CUDA(sc.get(&d_err, 1));
  if (n_tris) {
    CM_CUDA(cudaMemcpy(d_tris, tris, sizeof(int) * 3 * (size_t)n_tris, cudaMemcpyHostToDevice));
    CM_CUDA(cudaMemcpy(d_out, tris, sizeof(int) * 3 * (size_t)n_tris, cudaMemcpyHostToDevice));
  }
  if (total > 0) {
    CM_CUDA(cudaMemcpy(d_lp, loop_ptr, sizeof(int) * ((size_t)n_loops + 1), cudaMemcpyHostToDevice));
    CM_CUDA(cudaMemcpy(d_lof, loop_of.data(), sizeof(int) * (size_t)total, cudaMemcpyHostToDevice));
    CM_CUDA(cudaMemcpy(d_lv, loop_verts, sizeof(int) * (size_t)total, cudaMemcpyHostToDevice));
  }
  CM_CUDA(cudaMemset(d_err, 0, sizeof(int)));
  cn::HeBuild b;
  if ((st = cn::build_halfedges_dev(sc, n_verts, n_tris, d_tris, d_he, &b)) != CN_OK) return st;
  if (total > 0)
    cn::k_cut<<<cn::blocks_for(total, 128), 128>>>(n_verts, 3 * n_tris, total, d_lp, d_lof, d_lv, d_tris, d_he,
                                                   b.keys, b.vals, b.mask, b.n_he, d_out, d_parent, d_err);
  CM_CUDA(cudaGetLastError());
  int err = 0;
  CM_CUDA(cudaMemcpy(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    set_err("a loop edge has no face on its left or a loop vertex's fan is open");
    return CN_BAD_INPUT;
  }
  if (n_tris) CM_CUDA(cudaMemcpy(tris_out, d_out, sizeof(int) * 3 * (size_t)n_tris, cudaMemcpyDeviceToHost));
  for (int v = 0; v < n_verts; ++v) parent_out[v] = v;
  if (total > 0)
    CM_CUDA(cudaMemcpy(parent_out + n_verts, d_parent + n_verts, sizeof(int) * (size_t)total,
                       cudaMemcpyDeviceToHost));
  *n_verts_out = n_verts + total;
  return CN_OK;
}

cn_status cn_subdivide_edges(int32_t* counts, int32_t* he, int32_t m, const int32_t* edges) {
  cn::set_last_error_text("");
  cn_status st = cn::check_surgery(counts, he, m);
  if (st != CN_OK) return st;
  if (m > 0 && !edges) {
    set_err("null edges");
    return CN_BAD_INPUT;
  }
  const int nh = counts[2];
  std::vector<char> used((size_t)(nh > 0 ? nh : 1), 0);
  for (int k = 0; k < m; ++k) {
    const int h = edges[k];
    if (h < 0 || h >= nh) {
      set_err("edge %d: halfedge %d out of range", k, h);
      return CN_BAD_INPUT;
    }
    const int tw = he[4 * (size_t)h + 1] >= 0 ? he[4 * (size_t)h + 1] : h;
    if (tw >= nh || used[h] || (tw != h && used[tw])) {
      set_err("edge %d: the batch touches halfedge %d (or its twin) twice", k, h);
      return CN_BAD_INPUT;
    }
    used[h] = 1;
    used[tw] = 1;
  }
  if ((st = cn::need_device()) != CN_OK) return st;
  cn::Scratch sc;
  int *d_he = nullptr, *d_e = nullptr;
  CM_CUDA(sc.get(&d_he, 4 * ((size_t)nh + 2 * (size_t)m)));
  CM_CUDA(sc.get(&d_e, (size_t)m));
  if (nh) CM_CUDA(cudaMemcpy(d_he, he, sizeof(int) * 4 * (size_t)nh, cudaMemcpyHostToDevice));
  if (m) CM_CUDA(cudaMemcpy(d_e, edges, sizeof(int) * (size_t)m, cudaMemcpyHostToDevice));
  if (m) cn::k_subdivide<<<cn::blocks_for(m, 128), 128>>>(m, d_e, counts[0], nh, d_he);
  CM_CUDA(cudaGetLastError());
  CM_CUDA(cudaMemcpy(he, d_he, sizeof(int) * 4 * ((size_t)nh + 2 * (size_t)m), cudaMemcpyDeviceToHost));
  counts[0] += m;
  counts[2] += 2 * m;
  return CN_OK;
}

cn_status cn_split_faces(int32_t* counts, int32_t* he, int32_t m, const int32_t* a, const int32_t* b) {
  cn::set_last_error_text("");
  cn_status st = cn::check_surgery(counts, he, m);
  if (st != CN_OK) return st;
  if (m > 0 && (!a || !b)) {
    set_err("null halfedge lists");
    return CN_BAD_INPUT;
  }
  const int nh = counts[2];
  std::vector<int> faces;
  for (int k = 0; k < m; ++k) {
    if (a[k] < 0 || a[k] >= nh || b[k] < 0 || b[k] >= nh || a[k] == b[k]) {
      set_err("split %d: halfedges out of range or equal", k);
      return CN_BAD_INPUT;
    }
    const int fa = he[4 * (size_t)a[k] + 3], fb = he[4 * (size_t)b[k] + 3];
    if (fa < 0 || fa != fb) {
      set_err("split %d: the halfedges are not in one face", k);
      return CN_BAD_INPUT;
    }
    faces.push_back(fa);
  }
  std::vector<int> sorted(faces);
  std::sort(sorted.begin(), sorted.end());
  if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end()) {
    set_err("a batch of face splits must touch each face once");
    return CN_BAD_INPUT;
  }
  if ((st = cn::need_device()) != CN_OK) return st;
  cn::Scratch sc;
  int *d_he = nullptr, *d_a = nullptr, *d_b = nullptr;
  CM_CUDA(sc.get(&d_he, 4 * ((size_t)nh + 2 * (size_t)m)));
  CM_CUDA(sc.get(&d_a, (size_t)m));
  CM_CUDA(sc.get(&d_b, (size_t)m));
  if (nh) CM_CUDA(cudaMemcpy(d_he, he, sizeof(int) * 4 * (size_t)nh, cudaMemcpyHostToDevice));
  if (m) {
    CM_CUDA(cudaMemcpy(d_a, a, sizeof(int) * (size_t)m, cudaMemcpyHostToDevice));
    CM_CUDA(cudaMemcpy(d_b, b, sizeof(int) * (size_t)m, cudaMemcpyHostToDevice));
    cn::k_split<<<cn::blocks_for(m, 128), 128>>>(m, d_a, d_b, counts[1], nh, d_he);
  }
  CM_CUDA(cudaGetLastError());
  CM_CUDA(cudaMemcpy(he, d_he, sizeof(int) * 4 * ((size_t)nh + 2 * (size_t)m), cudaMemcpyDeviceToHost));
  counts[1] += m;
  counts[2] += 2 * m;
  return CN_OK;
}

cn_status cn_insert_cracks(int32_t* counts, int32_t* he, int32_t m, const int32_t* anchors) {
  cn::set_last_error_text("");
  cn_status st = cn::check_surgery(counts, he, m);
  if (st != CN_OK) return st;
  if (m > 0 && !anchors) {
    set_err("null anchors");
    return CN_BAD_INPUT;
  }
  const int nh = counts[2];
  std::vector<char> used((size_t)(nh > 0 ? nh : 1), 0);
  for (int k = 0; k < m; ++k) {
    const int h = anchors[k];
    if (h < 0 || h >= nh || used[h]) {
      set_err("crack %d: anchor %d out of range or used twice", k, h);
      return CN_BAD_INPUT;
    }
    used[h] = 1;
  }
  if ((st = cn::need_device()) != CN_OK) return st;
  cn::Scratch sc;
  int *d_he = nullptr, *d_a = nullptr;
  CM_CUDA(sc.get(&d_he, 4 * ((size_t)nh + 2 * (size_t)m)));
  CM_CUDA(sc.get(&d_a, (size_t)m));
  if (nh) CM_CUDA(cudaMemcpy(d_he, he, sizeof(int) * 4 * (size_t)nh, cudaMemcpyHostToDevice));
  if (m) {
    CM_CUDA(cudaMemcpy(d_a, anchors, sizeof(int) * (size_t)m, cudaMemcpyHostToDevice));
    cn::k_crack<<<cn::blocks_for(m, 128), 128>>>(m, d_a, counts[0], nh, d_he);
  }
  CM_CUDA(cudaGetLastError());
  CM_CUDA(cudaMemcpy(he, d_he, sizeof(int) * 4 * ((size_t)nh + 2 * (size_t)m), cudaMemcpyDeviceToHost));
  counts[0] += m;
  counts[2] += 2 * m;
  return CN_OK;
}

}  // extern "C"
