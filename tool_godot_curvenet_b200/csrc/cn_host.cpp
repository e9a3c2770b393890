// cn_host.cpp -- host side of the C ABI: input checks, the seam cut, the CSR
// pattern of K and of the reduced system, the elimination order (greedy
// colouring + level sets), the IC(0) task lists, device buffers, and the
// solve dispatch.  All floating-point work runs on the GPU; the host builds
// integer structure only.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "cn_internal.h"

using cn::BuildArgs;
using cn::Control;
using cn::DevStats;
using cn::SolveArgs;

namespace {

thread_local std::string g_err;

void set_err(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
}

#define CN_CUDA(call)                                                          \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      set_err("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                       \
      return CN_CUDA_ERROR;                                                    \
    }                                                                          \
  } while (0)

// Device allocation list owned by a handle.
struct DevArena {
  std::vector<void*> ptrs;
  size_t bytes = 0;
  template <class T>
  cudaError_t alloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * count);
    if (e == cudaSuccess) { ptrs.push_back(*p); bytes += sizeof(T) * count; }
    return e;
  }
  template <class T>
  cudaError_t upload(T** p, const std::vector<T>& h) {
    cudaError_t e = alloc(p, h.size());
    if (e != cudaSuccess) return e;
    if (!h.empty()) e = cudaMemcpy(*p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
    return e;
  }
  void release() {
    for (void* p : ptrs) cudaFree(p);
    ptrs.clear();
    bytes = 0;
  }
};

// Union-find over vertices.
struct Dsu {
  std::vector<int> p;
  explicit Dsu(int n) : p(n) { std::iota(p.begin(), p.end(), 0); }
  int find(int a) {
    while (p[a] != a) { p[a] = p[p[a]]; a = p[a]; }
    return a;
  }
  void unite(int a, int b) { p[find(a)] = find(b); }
};

}  // namespace

void cn::set_last_error_text(const char* msg) { g_err = msg; }

// ---------------------------------------------------------------------------
struct cn_system {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cn_build_opts opts{};
  int nv = 0, nt = 0, nh = 0, n = 0, nlev = 0, ncolors = 0, kmax = 3;
  int nnzK = 0, nnzA = 0, nnzL = 0;
  int lanes = 4, block = 512, grid = 0;
  double shift_used = 0.0;
  // host structure (exports)
  std::vector<int> K_ptr, K_col, free_of, A_ptr, A_col, L_ptr, L_col, lev_ptr, handles;
  // device
  DevArena mem;
  double *d_pos = nullptr, *d_face_m = nullptr, *d_K_val = nullptr;
  int *d_tris = nullptr, *d_K_ptr = nullptr, *d_K_col = nullptr, *d_K_cptr = nullptr,
      *d_K_contrib = nullptr;
  int *d_hidx = nullptr, *d_free_of = nullptr, *d_handles = nullptr;
  int *d_A_ptr = nullptr, *d_A_col = nullptr, *d_A_src = nullptr, *d_A_diag = nullptr,
      *d_lev_ptr = nullptr;
  double* d_A64 = nullptr;
  float* d_A32 = nullptr;
  int *d_L_ptr = nullptr, *d_L_col = nullptr, *d_L_src = nullptr, *d_T_ptr = nullptr,
      *d_T_a = nullptr, *d_T_b = nullptr;
  int *d_U_ptr = nullptr, *d_U_col = nullptr, *d_U_src = nullptr;
  double *d_L64 = nullptr, *d_U64 = nullptr, *d_Ld64 = nullptr, *d_dinv64 = nullptr;
  float *d_L32 = nullptr, *d_U32 = nullptr, *d_dinv32 = nullptr;
  int* d_status = nullptr;
  // solve state
  double *d_b64 = nullptr, *d_x64 = nullptr, *d_partials = nullptr;
  double* d_w64[7] = {};
  float* d_w32[7] = {};
  Control* d_ctl = nullptr;
  DevStats* d_stats = nullptr;
  double *d_targets = nullptr, *d_x0 = nullptr, *d_xout = nullptr, *d_scal = nullptr;
  int max_grid_alloc = 0;
  bool have_solution = false;
};

namespace {

const char* kStatusText[] = {"ok", "max_iter", "singular_component", "nonpositive_pivot",
                             "nan", "breakdown", "timeout", "bad_input", "cuda_error",
                             "no_device"};

int local_of(int corner) { return (corner + 2) % 3; }  // t0,t1,t2 -> faceLoop slots 2,0,1
int off_slot(int a, int b) {
  if (a > b) std::swap(a, b);
  return a == 0 ? (b == 1 ? 3 : 4) : 5;
}

// Vertex -> incident faces (ascending face id), with the corner of the vertex.
void vertex_faces(int nv, int nt, const int* tris, std::vector<int>& ptr, std::vector<int>& face,
                  std::vector<int>& corner) {
  ptr.assign(nv + 1, 0);
  for (int i = 0; i < 3 * nt; ++i) ptr[tris[i] + 1]++;
  for (int v = 0; v < nv; ++v) ptr[v + 1] += ptr[v];
  face.resize(3 * (size_t)nt);
  corner.resize(3 * (size_t)nt);
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (int f = 0; f < nt; ++f)
    for (int c = 0; c < 3; ++c) {
      int v = tris[3 * f + c];
      face[fill[v]] = f;
      corner[fill[v]] = c;
      fill[v]++;
    }
}

cn_status build_structure(cn_system* S, const cn_mesh_desc* m, std::vector<int>& K_cptr,
                          std::vector<int>& K_contrib, std::vector<int>& hidx,
                          std::vector<int>& A_src, std::vector<int>& A_diag,
                          std::vector<int>& L_src, std::vector<int>& T_ptr, std::vector<int>& T_a,
                          std::vector<int>& T_b, std::vector<int>& U_ptr, std::vector<int>& U_col,
                          std::vector<int>& U_src) {
  const int nv = m->n_verts, nt = m->n_tris;
  const int* tris = m->tris;
  // --- K pattern and the face contributions of every entry
  std::vector<int> vf_ptr, vf_face, vf_corner;
  vertex_faces(nv, nt, tris, vf_ptr, vf_face, vf_corner);
  S->K_ptr.assign(nv + 1, 0);
  S->K_col.clear();
  S->K_col.reserve((size_t)nv * 8);
  std::vector<int> nb;
  for (int u = 0; u < nv; ++u) {
    nb.clear();
    nb.push_back(u);
    for (int q = vf_ptr[u]; q < vf_ptr[u + 1]; ++q) {
      int f = vf_face[q];
      for (int c = 0; c < 3; ++c) nb.push_back(tris[3 * f + c]);
    }
    std::sort(nb.begin(), nb.end());
    nb.erase(std::unique(nb.begin(), nb.end()), nb.end());
    S->K_col.insert(S->K_col.end(), nb.begin(), nb.end());
    S->K_ptr[u + 1] = (int)S->K_col.size();
  }
  S->nnzK = (int)S->K_col.size();
  K_cptr.assign(S->nnzK + 1, 0);
  auto entry = [&](int u, int v) {
    int lo = S->K_ptr[u], hi = S->K_ptr[u + 1];
    return (int)(std::lower_bound(S->K_col.begin() + lo, S->K_col.begin() + hi, v) - S->K_col.begin());
  };
  for (int pass = 0; pass < 2; ++pass) {
    std::vector<int> fill;
    if (pass == 1) {
      for (int e = 0; e < S->nnzK; ++e) K_cptr[e + 1] += K_cptr[e];
      K_contrib.assign(K_cptr[S->nnzK], 0);
      fill.assign(K_cptr.begin(), K_cptr.end() - 1);
    }
    for (int u = 0; u < nv; ++u)
      for (int q = vf_ptr[u]; q < vf_ptr[u + 1]; ++q) {  // ascending face
        const int f = vf_face[q], cu = vf_corner[q], a = local_of(cu);
        for (int c = 0; c < 3; ++c) {
          const int v = tris[3 * f + c], b = local_of(c);
          const int e = entry(u, v);
          const int slot = c == cu ? a : off_slot(a, b);
          if (pass == 0) K_cptr[e + 1]++;
          else K_contrib[fill[e]++] = 6 * f + slot;
        }
      }
  }
  // --- handles, components (every component needs a handle)
  hidx.assign(nv, -1);
  for (int h = 0; h < m->n_handles; ++h) {
    const int v = m->handles[h];
    if (v < 0 || v >= nv || hidx[v] >= 0) {
      set_err("handle %d: vertex %d out of range or repeated", h, v);
      return CN_BAD_INPUT;
    }
    hidx[v] = h;
  }
  {
    Dsu dsu(nv);
    for (int f = 0; f < nt; ++f) {
      dsu.unite(tris[3 * f], tris[3 * f + 1]);
      dsu.unite(tris[3 * f], tris[3 * f + 2]);
    }
    std::vector<char> has(nv, 0);
    for (int h = 0; h < m->n_handles; ++h) has[dsu.find(m->handles[h])] = 1;
    for (int v = 0; v < nv; ++v)
      if (!has[dsu.find(v)]) {
        set_err("vertex %d lies in a connected component without a handle", v);
        return CN_SINGULAR_COMPONENT;
      }
  }
  // --- free unknowns in vertex order; A_nat = K[free, free]
  std::vector<int> fidx(nv, -1), fverts;
  for (int v = 0; v < nv; ++v)
    if (hidx[v] < 0) { fidx[v] = (int)fverts.size(); fverts.push_back(v); }
  const int n = (int)fverts.size();
  S->n = n;
  std::vector<int> Nptr(n + 1, 0), Ncol, Nsrc;
  Ncol.reserve(S->nnzK);
  Nsrc.reserve(S->nnzK);
  for (int i = 0; i < n; ++i) {
    const int v = fverts[i];
    for (int e = S->K_ptr[v]; e < S->K_ptr[v + 1]; ++e)
      if (fidx[S->K_col[e]] >= 0) { Ncol.push_back(fidx[S->K_col[e]]); Nsrc.push_back(e); }
    Nptr[i + 1] = (int)Ncol.size();
  }
  // --- elimination order: natural, or greedy colour (GraphColoring.lean:41-56)
  std::vector<int> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::vector<int> color(n, 0);
  {
    std::vector<int> mark;
    int nc = n ? 1 : 0;
    for (int i = 0; i < n; ++i) {
      mark.assign(Nptr[i + 1] - Nptr[i] + 2, 0);
      for (int p = Nptr[i]; p < Nptr[i + 1]; ++p) {
        const int j = Ncol[p];
        if (j < i && color[j] < (int)mark.size()) mark[color[j]] = 1;
      }
      int c = 0;
      while (c < (int)mark.size() && mark[c]) ++c;
      color[i] = c;
      nc = std::max(nc, c + 1);
    }
    S->ncolors = nc;
  }
  if (S->opts.ordering == CN_ORDER_COLOR)
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return color[a] < color[b]; });
  // level of every unknown in that order; rows sorted by level
  std::vector<int> posn(n), level(n, 0);
  for (int i = 0; i < n; ++i) posn[ord[i]] = i;
  int nlev = n ? 1 : 0;
  if (S->opts.precond == CN_PRECOND_IC0) {
    for (int i = 0; i < n; ++i) {
      const int v = ord[i];
      int l = 0;
      for (int p = Nptr[v]; p < Nptr[v + 1]; ++p) {
        const int u = Ncol[p];
        if (posn[u] < i) l = std::max(l, level[u] + 1);
      }
      level[v] = l;
      nlev = std::max(nlev, l + 1);
    }
  }
  std::vector<int> perm = ord;
  std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return level[a] < level[b]; });
  std::vector<int> inv(n);
  for (int i = 0; i < n; ++i) inv[perm[i]] = i;
  S->nlev = nlev;
  S->lev_ptr.assign(nlev + 1, 0);
  for (int i = 0; i < n; ++i) S->lev_ptr[level[perm[i]] + 1]++;
  for (int l = 0; l < nlev; ++l) S->lev_ptr[l + 1] += S->lev_ptr[l];
  S->free_of.resize(n);
  for (int i = 0; i < n; ++i) S->free_of[i] = fverts[perm[i]];
  // --- permuted A with its source entries in K
  S->A_ptr.assign(n + 1, 0);
  S->A_col.resize(Ncol.size());
  A_src.resize(Ncol.size());
  A_diag.assign(n, -1);
  std::vector<std::pair<int, int>> row;
  for (int i = 0; i < n; ++i) {
    const int o = perm[i];
    row.clear();
    for (int p = Nptr[o]; p < Nptr[o + 1]; ++p) row.push_back({inv[Ncol[p]], Nsrc[p]});
    std::sort(row.begin(), row.end());
    const int base = S->A_ptr[i];
    for (size_t q = 0; q < row.size(); ++q) {
      S->A_col[base + q] = row[q].first;
      A_src[base + q] = row[q].second;
      if (row[q].first == i) A_diag[i] = base + (int)q;
    }
    S->A_ptr[i + 1] = base + (int)row.size();
    if (A_diag[i] < 0) {
      set_err("row %d has no diagonal entry", i);
      return CN_BAD_INPUT;
    }
  }
  S->nnzA = (int)S->A_col.size();
  // --- strictly-lower L pattern (IC(0): no fill), its tasks, and U = L^T
  S->L_ptr.assign(n + 1, 0);
  S->L_col.clear();
  L_src.clear();
  if (S->opts.precond == CN_PRECOND_IC0) {
    for (int i = 0; i < n; ++i) {
      for (int e = S->A_ptr[i]; e < S->A_ptr[i + 1]; ++e)
        if (S->A_col[e] < i) { S->L_col.push_back(S->A_col[e]); L_src.push_back(e); }
      S->L_ptr[i + 1] = (int)S->L_col.size();
    }
  }
  S->nnzL = (int)S->L_col.size();
  T_ptr.assign(S->nnzL + 1, 0);
  T_a.clear();
  T_b.clear();
  for (int i = 0; i < n; ++i)
    for (int e = S->L_ptr[i]; e < S->L_ptr[i + 1]; ++e) {
      const int j = S->L_col[e];
      int a = S->L_ptr[i], b = S->L_ptr[j];
      const int bhi = S->L_ptr[j + 1];
      while (a < e && b < bhi) {  // common k < j, ascending
        if (S->L_col[a] == S->L_col[b]) { T_a.push_back(a); T_b.push_back(b); ++a; ++b; }
        else if (S->L_col[a] < S->L_col[b]) ++a;
        else ++b;
      }
      T_ptr[e + 1] = (int)T_a.size();
    }
  U_ptr.assign(n + 1, 0);
  for (int e = 0; e < S->nnzL; ++e) U_ptr[S->L_col[e] + 1]++;
  for (int i = 0; i < n; ++i) U_ptr[i + 1] += U_ptr[i];
  U_col.resize(S->nnzL);
  U_src.resize(S->nnzL);
  {
    std::vector<int> fill(U_ptr.begin(), U_ptr.end() - 1);
    for (int i = 0; i < n; ++i)
      for (int e = S->L_ptr[i]; e < S->L_ptr[i + 1]; ++e) {
        const int j = S->L_col[e];
        U_col[fill[j]] = i;
        U_src[fill[j]] = e;
        fill[j]++;
      }
  }
  return CN_OK;
}

cn_status check_mesh(const cn_mesh_desc* m) {
  if (!m || m->n_verts < 0 || m->n_tris < 0 || m->n_handles < 0) {
    set_err("negative sizes");
    return CN_BAD_INPUT;
  }
  if ((m->n_verts && !m->positions) || (m->n_tris && !m->tris) || (m->n_handles && !m->handles)) {
    set_err("null array");
    return CN_BAD_INPUT;
  }
  for (long long i = 0; i < 3LL * m->n_verts; ++i)
    if (!std::isfinite(m->positions[i])) {
      set_err("position %lld is not finite", i / 3);
      return CN_NAN;
    }
  for (int f = 0; f < m->n_tris; ++f) {
    const int a = m->tris[3 * f], b = m->tris[3 * f + 1], c = m->tris[3 * f + 2];
    if (a < 0 || b < 0 || c < 0 || a >= m->n_verts || b >= m->n_verts || c >= m->n_verts ||
        a == b || b == c || a == c) {
      set_err("triangle %d has an out-of-range or repeated vertex", f);
      return CN_BAD_INPUT;
    }
  }
  return CN_OK;
}

cn_status alloc_solve_state(cn_system* S) {
  const size_t nk = (size_t)std::max(S->n, 1) * S->kmax;
  CN_CUDA(S->mem.alloc(&S->d_b64, nk));
  CN_CUDA(S->mem.alloc(&S->d_x64, nk));
  CN_CUDA(cudaMemset(S->d_x64, 0, sizeof(double) * nk));
  for (int i = 0; i < 7; ++i) {
    CN_CUDA(S->mem.alloc(&S->d_w64[i], nk));
    CN_CUDA(S->mem.alloc(&S->d_w32[i], nk));
    CN_CUDA(cudaMemset(S->d_w64[i], 0, sizeof(double) * nk));
    CN_CUDA(cudaMemset(S->d_w32[i], 0, sizeof(float) * nk));
  }
  int sms = 0;
  CN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, S->device));
  S->max_grid_alloc = std::max(sms * 8, 1024);
  CN_CUDA(S->mem.alloc(&S->d_partials, (size_t)cn::kSlots * S->max_grid_alloc * S->kmax));
  CN_CUDA(S->mem.alloc(&S->d_scal, 64));
  CN_CUDA(S->mem.alloc(&S->d_ctl, 1));
  CN_CUDA(S->mem.alloc(&S->d_stats, 1));
  CN_CUDA(S->mem.alloc(&S->d_targets, (size_t)std::max(S->nh, S->n) * S->kmax + 1));
  CN_CUDA(S->mem.alloc(&S->d_x0, (size_t)S->nv * S->kmax + 1));
  CN_CUDA(S->mem.alloc(&S->d_xout, (size_t)S->nv * S->kmax + 1));
  return CN_OK;
}

void choose_launch(cn_system* S) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, S->device);
  S->lanes = S->opts.lanes > 0 ? S->opts.lanes : 2;
  if (S->n <= 12288) {
    S->block = S->opts.block > 0 ? S->opts.block : 1024;
    S->grid = S->opts.grid > 0 ? S->opts.grid : 1;
  } else {
    S->block = S->opts.block > 0 ? S->opts.block : 512;
    S->grid = S->opts.grid > 0 ? S->opts.grid : sms;
  }
}

}  // namespace

// ===========================================================================
extern "C" {

void cn_default_build_opts(cn_build_opts* o) {
  std::memset(o, 0, sizeof *o);
  o->precond = CN_PRECOND_IC0;
  o->ordering = CN_ORDER_COLOR;
  o->laplacian = CN_LAPLACIAN_COT;
  o->mollify_delta = 1e-4;
  o->device = 0;
  o->max_rhs = 3;
}

void cn_default_solve_opts(cn_solve_opts* o) {
  std::memset(o, 0, sizeof *o);
  o->precision = CN_PREC_MIXED;
  o->mode = CN_MODE_DEFORM;
  o->algo = CN_ALGO_FUSED;
  o->tol = 1e-8;
  o->max_iter = 2000;
  o->max_refine = 8;
  o->inner_tol = 1e-5;
  o->warm_start = 0;
}

const char* cn_status_string(int32_t s) {
  if (s < 0 || s > 9) return "unknown";
  return kStatusText[s];
}

const char* cn_last_error(void) { return g_err.c_str(); }

cn_status cn_cut_mesh(int32_t nv, int32_t nt, const int32_t* tris, int32_t nloops,
                      const int32_t* loop_ptr, const int32_t* loop_verts, int32_t* tris_out,
                      int32_t* parent_out, int32_t* nv_out) {
  if (nv < 0 || nt < 0 || nloops < 0 || !tris_out || !parent_out || !nv_out) {
    set_err("bad arguments");
    return CN_BAD_INPUT;
  }
  for (int i = 0; i < 3 * nt; ++i)
    if (tris[i] < 0 || tris[i] >= nv) {
      set_err("triangle vertex out of range");
      return CN_BAD_INPUT;
    }
  std::vector<int> vf_ptr, vf_face, vf_corner;
  vertex_faces(nv, nt, tris, vf_ptr, vf_face, vf_corner);
  std::memcpy(tris_out, tris, sizeof(int32_t) * 3 * (size_t)nt);
  for (int v = 0; v < nv; ++v) parent_out[v] = v;
  std::vector<char> seen(nv, 0);
  int next_id = nv;
  for (int l = 0; l < nloops; ++l) {
    const int lo = loop_ptr[l], hi = loop_ptr[l + 1], m = hi - lo;
    if (m < 3) {
      set_err("loop %d has fewer than 3 vertices", l);
      return CN_BAD_INPUT;
    }
    for (int i = 0; i < m; ++i) {
      const int v = loop_verts[lo + i];
      const int vn = loop_verts[lo + (i + 1) % m], vp = loop_verts[lo + (i - 1 + m) % m];
      if (v < 0 || v >= nv || seen[v]) {
        set_err("loop vertex %d out of range or in two loops", v);
        return CN_BAD_INPUT;
      }
      seen[v] = 1;
      const int copy = next_id++;
      parent_out[copy] = v;
      // Sweep the fan of v counter-clockwise from the face with edge (v, vn):
      // in face (v, a, b) the next face is the one holding (v, b, .).
      int a = vn, guard = 0;
      const int deg = vf_ptr[v + 1] - vf_ptr[v];
      while (true) {
        int f = -1, cf = -1;
        for (int q = vf_ptr[v]; q < vf_ptr[v + 1]; ++q) {
          const int ff = vf_face[q], c = vf_corner[q];
          if (tris[3 * ff + (c + 1) % 3] == a) { f = ff; cf = c; break; }
        }
        if (f < 0 || ++guard > deg) {
          set_err("loop %d: the fan of vertex %d is open or not a disc", l, v);
          return CN_BAD_INPUT;
        }
        tris_out[3 * f + cf] = copy;
        const int b = tris[3 * f + (cf + 2) % 3];
        if (b == vp) break;
        a = b;
      }
    }
  }
  *nv_out = next_id;
  return CN_OK;
}

cn_status cn_build(const cn_mesh_desc* mesh, const cn_build_opts* opts, cn_handle* out) {
  g_err.clear();
  if (!out) {
    set_err("out is NULL");
    return CN_BAD_INPUT;
  }
  *out = nullptr;
  cn_status st = check_mesh(mesh);
  if (st != CN_OK) return st;
  cn_build_opts o;
  if (opts) o = *opts;
  else cn_default_build_opts(&o);
  if (o.max_rhs != 1 && o.max_rhs != 3 && o.max_rhs != 9) {
    set_err("max_rhs must be 1, 3 or 9");
    return CN_BAD_INPUT;
  }
  if (o.precond != CN_PRECOND_IC0 && o.precond != CN_PRECOND_JACOBI) {
    set_err("unsupported preconditioner %d", o.precond);
    return CN_BAD_INPUT;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_err("no CUDA device");
    return CN_NO_DEVICE;
  }
  if (o.device < 0 || o.device >= ndev) {
    set_err("device %d out of range", o.device);
    return CN_BAD_INPUT;
  }
  if (cudaSetDevice(o.device) != cudaSuccess) {
    set_err("cudaSetDevice(%d) failed", o.device);
    return CN_CUDA_ERROR;
  }
  cn_system* S = new cn_system;
  S->opts = o;
  S->device = o.device;
  S->kmax = o.max_rhs;
  S->nv = mesh->n_verts;
  S->nt = mesh->n_tris;
  S->nh = mesh->n_handles;
  S->handles.assign(mesh->handles, mesh->handles + mesh->n_handles);
  auto fail = [&](cn_status s) {
    cn_destroy(S);
    return s;
  };
  std::vector<int> K_cptr, K_contrib, hidx, A_src, A_diag, L_src, T_ptr, T_a, T_b, U_ptr, U_col,
      U_src;
  st = build_structure(S, mesh, K_cptr, K_contrib, hidx, A_src, A_diag, L_src, T_ptr, T_a, T_b,
                       U_ptr, U_col, U_src);
  if (st != CN_OK) return fail(st);
  if (cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&S->ev0) != cudaSuccess || cudaEventCreate(&S->ev1) != cudaSuccess) {
    set_err("stream/event creation failed");
    return fail(CN_CUDA_ERROR);
  }
  DevArena& M = S->mem;
  std::vector<double> pos(mesh->positions, mesh->positions + 3 * (size_t)S->nv);
  std::vector<int> tris(mesh->tris, mesh->tris + 3 * (size_t)S->nt);
#define UP(dst, vec)                                     \
  if (M.upload(&(dst), (vec)) != cudaSuccess) {          \
    set_err("device allocation/upload of " #vec " failed"); \
    return fail(CN_CUDA_ERROR);                          \
  }
  UP(S->d_pos, pos);
  UP(S->d_tris, tris);
  UP(S->d_K_ptr, S->K_ptr);
  UP(S->d_K_col, S->K_col);
  UP(S->d_K_cptr, K_cptr);
  UP(S->d_K_contrib, K_contrib);
  UP(S->d_hidx, hidx);
  UP(S->d_free_of, S->free_of);
  UP(S->d_handles, S->handles);
  UP(S->d_A_ptr, S->A_ptr);
  UP(S->d_A_col, S->A_col);
  UP(S->d_A_src, A_src);
  UP(S->d_A_diag, A_diag);
  UP(S->d_lev_ptr, S->lev_ptr);
  UP(S->d_L_ptr, S->L_ptr);
  UP(S->d_L_col, S->L_col);
  UP(S->d_L_src, L_src);
  UP(S->d_T_ptr, T_ptr);
  UP(S->d_T_a, T_a);
  UP(S->d_T_b, T_b);
  UP(S->d_U_ptr, U_ptr);
  UP(S->d_U_col, U_col);
  UP(S->d_U_src, U_src);
#undef UP
  if (M.alloc(&S->d_face_m, 6 * (size_t)S->nt) || M.alloc(&S->d_K_val, S->nnzK) ||
      M.alloc(&S->d_A64, S->nnzA) || M.alloc(&S->d_A32, S->nnzA) ||
      M.alloc(&S->d_L64, S->nnzL) || M.alloc(&S->d_L32, S->nnzL) ||
      M.alloc(&S->d_U64, S->nnzL) || M.alloc(&S->d_U32, S->nnzL) ||
      M.alloc(&S->d_Ld64, S->n) || M.alloc(&S->d_dinv64, S->n) || M.alloc(&S->d_dinv32, S->n) ||
      M.alloc(&S->d_status, 1)) {
    set_err("device allocation failed");
    return fail(CN_CUDA_ERROR);
  }
  st = alloc_solve_state(S);
  if (st != CN_OK) return fail(st);

  BuildArgs b{};
  b.nv = S->nv; b.nt = S->nt; b.nnzK = S->nnzK; b.n = S->n; b.nnzA = S->nnzA;
  b.nnzL = S->nnzL; b.nlev = S->nlev;
  b.pos = S->d_pos; b.tris = S->d_tris; b.lap_kind = o.laplacian; b.delta = o.mollify_delta;
  b.face_m = S->d_face_m; b.K_cptr = S->d_K_cptr; b.K_contrib = S->d_K_contrib; b.K_val = S->d_K_val;
  b.A_src = S->d_A_src; b.A_val64 = S->d_A64; b.A_val32 = S->d_A32; b.A_diag = S->d_A_diag;
  b.lev_ptr = S->d_lev_ptr; b.h_lev_ptr = S->lev_ptr.data();
  b.L_ptr = S->d_L_ptr; b.L_src = S->d_L_src; b.L_col = S->d_L_col;
  b.T_ptr = S->d_T_ptr; b.T_a = S->d_T_a; b.T_b = S->d_T_b;
  b.L_val64 = S->d_L64; b.L_val32 = S->d_L32; b.Ld64 = S->d_Ld64;
  b.dinv64 = S->d_dinv64; b.dinv32 = S->d_dinv32;
  b.U_src = S->d_U_src; b.U_val64 = S->d_U64; b.U_val32 = S->d_U32;
  b.status = S->d_status; b.precond = o.precond;
  if (cn::launch_assemble(b, S->stream) != cudaSuccess) {
    set_err("assembly launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    return fail(CN_CUDA_ERROR);
  }
  // IC(0) with Manteuffel diagonal-shift retries on a non-positive pivot.
  const double shifts[] = {0.0, 1e-3, 1e-2, 1e-1};
  int bad = -1;
  for (double sh : shifts) {
    const int ok = 0x7fffffff;
    if (cudaMemcpyAsync(S->d_status, &ok, sizeof ok, cudaMemcpyHostToDevice, S->stream) != cudaSuccess) {
      set_err("status reset failed");
      return fail(CN_CUDA_ERROR);
    }
    b.shift = sh;
    if (cn::launch_factor(b, S->stream) != cudaSuccess) {
      set_err("factor launch failed");
      return fail(CN_CUDA_ERROR);
    }
    int h_status = 0;
    if (cudaMemcpyAsync(&h_status, S->d_status, sizeof h_status, cudaMemcpyDeviceToHost, S->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(S->stream) != cudaSuccess) {
      set_err("factor failed: %s", cudaGetErrorString(cudaGetLastError()));
      return fail(CN_CUDA_ERROR);
    }
    bad = h_status == ok ? -1 : h_status;
    S->shift_used = sh;
    if (bad < 0) break;
  }
  if (bad >= 0) {
    set_err("IC(0) pivot of row %d is not positive", bad);
    return fail(CN_NONPOS_PIVOT);
  }
  choose_launch(S);
  *out = S;
  return CN_OK;
}

void cn_destroy(cn_handle S) {
  if (!S) return;
  cudaSetDevice(S->device);
  if (S->stream) cudaStreamSynchronize(S->stream);
  S->mem.release();
  if (S->ev0) cudaEventDestroy(S->ev0);
  if (S->ev1) cudaEventDestroy(S->ev1);
  if (S->stream) cudaStreamDestroy(S->stream);
  delete S;
}

void* cn_stream(cn_handle S) { return S ? (void*)S->stream : nullptr; }

cn_status cn_system_info(cn_handle S, int64_t* info) {
  if (!S || !info) return CN_BAD_INPUT;
  int64_t v[12] = {S->n, S->nnzA, S->nnzL, S->nlev, S->nnzK, S->nv, S->nh,
                   S->grid, S->block, S->lanes, S->ncolors, (int64_t)S->mem.bytes};
  std::memcpy(info, v, sizeof v);
  return CN_OK;
}

static cn_status solve_plain(cn_handle S, int k, const double* d_targets, double* d_xout,
                             const cn_solve_opts* o, cn_solve_stats* stats);

static cn_status fill_stats(cn_handle S, int k, cn_solve_stats* stats) {
  DevStats ds;
  CN_CUDA(cudaMemcpyAsync(&ds, S->d_stats, sizeof ds, cudaMemcpyDeviceToHost, S->stream));
  CN_CUDA(cudaStreamSynchronize(S->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, S->ev0, S->ev1);
  std::memset(stats, 0, sizeof *stats);
  stats->status = ds.status;
  stats->iterations = ds.iterations;
  stats->refinements = ds.refinements;
  stats->k = k;
  stats->device_ms = ms;
  double mx = 0.0;
  for (int c = 0; c < k && c < 32; ++c) {
    stats->rel_residual[c] = ds.rel_residual[c];
    mx = std::max(mx, ds.rel_residual[c]);
  }
  stats->max_rel_residual = mx;
  return (cn_status)ds.status;
}

cn_status cn_solve_device(cn_handle S, int32_t k, const double* d_targets, double* d_xout,
                          const cn_solve_opts* opts, cn_solve_stats* stats) {
  if (!S) return CN_BAD_INPUT;
  cn_solve_opts o;
  if (opts) o = *opts;
  else cn_default_solve_opts(&o);
  if (k != 1 && k != 3 && k != 9) {
    set_err("k must be 1, 3 or 9");
    return CN_BAD_INPUT;
  }
  if (k > S->kmax) {
    set_err("k = %d exceeds the build's max_rhs = %d", k, S->kmax);
    return CN_BAD_INPUT;
  }
  if (o.mode == CN_MODE_DEFORM && k % 3 != 0) {
    set_err("deform mode needs k a multiple of 3");
    return CN_BAD_INPUT;
  }
  if (!(o.tol > 0.0) || o.max_iter < 0 || o.max_refine < 1) {
    set_err("bad solve options");
    return CN_BAD_INPUT;
  }
  CN_CUDA(cudaSetDevice(S->device));
  if (o.algo == CN_ALGO_PLAIN) return solve_plain(S, k, d_targets, d_xout, &o, stats);
  const bool mixed = o.precision == CN_PREC_MIXED;
  SolveArgs a{};
  a.n = S->n; a.nlev = S->nlev; a.lev_ptr = S->d_lev_ptr;
  a.A_ptr = S->d_A_ptr; a.A_col = S->d_A_col;
  a.A_val = mixed ? (const void*)S->d_A32 : (const void*)S->d_A64;
  a.A_val64 = S->d_A64;
  a.L_ptr = S->d_L_ptr; a.L_col = S->d_L_col;
  a.L_val = mixed ? (const void*)S->d_L32 : (const void*)S->d_L64;
  a.U_ptr = S->d_U_ptr; a.U_col = S->d_U_col;
  a.U_val = mixed ? (const void*)S->d_U32 : (const void*)S->d_U64;
  a.dinv = mixed ? (const void*)S->d_dinv32 : (const void*)S->d_dinv64;
  a.nv = S->nv; a.nh = S->nh;
  a.K_ptr = S->d_K_ptr; a.K_col = S->d_K_col; a.K_val = S->d_K_val;
  a.free_of = S->d_free_of; a.hidx = S->d_hidx; a.handles = S->d_handles; a.pos = S->d_pos;
  a.mode = o.mode; a.targets = d_targets; a.x_out = d_xout; a.x0 = nullptr;
  a.warm = o.warm_start && S->have_solution ? 1 : 0;
  a.b64 = S->d_b64; a.x64 = S->d_x64;
  void** w = mixed ? (void**)S->d_w32 : (void**)S->d_w64;
  a.r = w[0]; a.y = w[1]; a.z = w[2]; a.p0 = w[3]; a.p1 = w[4]; a.Ap = w[5]; a.xin = w[6];
  a.partials = S->d_partials;
  a.tol = o.tol;
  a.inner_tol = mixed ? o.inner_tol : 0.0;
  a.max_iter = o.max_iter;
  a.max_refine = o.max_refine;
  a.ctl = S->d_ctl; a.stats = S->d_stats;
  a.timeout_ns = 2000000000LL;
  int grid = S->grid;
  if (grid > 1) {
    const int mg = cn::persistent_max_grid(o.precision, k, S->lanes, S->block);
    if (mg <= 0) {
      set_err("the persistent solve does not fit on this device (lanes %d, block %d)", S->lanes, S->block);
      return CN_CUDA_ERROR;
    }
    grid = std::min(std::min(grid, mg), S->max_grid_alloc);
  }
  CN_CUDA(cudaMemsetAsync(S->d_ctl, 0, sizeof(Control), S->stream));
  CN_CUDA(cudaEventRecord(S->ev0, S->stream));
  CN_CUDA(cn::launch_persistent_solve(a, o.precision, k, S->lanes, S->block, grid, S->stream));
  CN_CUDA(cudaEventRecord(S->ev1, S->stream));
  S->have_solution = true;
  if (!stats) return CN_OK;
  return fill_stats(S, k, stats);
}

cn_status cn_solve(cn_handle S, int32_t k, const double* targets, const double* x0,
                   double* x_out, const cn_solve_opts* opts, cn_solve_stats* stats) {
  if (!S || !x_out || (k > 0 && !targets)) {
    set_err("null argument");
    return CN_BAD_INPUT;
  }
  if (k < 1 || k > S->kmax) {
    set_err("k out of range");
    return CN_BAD_INPUT;
  }
  cn_solve_opts o;
  if (opts) o = *opts;
  else cn_default_solve_opts(&o);
  CN_CUDA(cudaSetDevice(S->device));
  const size_t nt = (size_t)(o.mode == CN_MODE_RHS ? S->n : S->nh) * k;
  for (size_t i = 0; i < nt; ++i)
    if (!std::isfinite(targets[i])) {
      set_err("target %zu is not finite", i);
      return CN_NAN;
    }
  if (nt) CN_CUDA(cudaMemcpyAsync(S->d_targets, targets, sizeof(double) * nt, cudaMemcpyHostToDevice, S->stream));
  if (x0) {
    // the initial guess enters as the warm-start state, gathered to solve order
    std::vector<double> xs((size_t)S->n * k);
    for (int i = 0; i < S->n; ++i)
      for (int c = 0; c < k; ++c) xs[(size_t)i * k + c] = x0[(size_t)S->free_of[i] * k + c];
    CN_CUDA(cudaMemcpyAsync(S->d_x64, xs.data(), sizeof(double) * xs.size(), cudaMemcpyHostToDevice,
                            S->stream));
    CN_CUDA(cudaStreamSynchronize(S->stream));
    S->have_solution = true;
    o.warm_start = 1;
  }
  cn_solve_stats local;
  cn_status st = cn_solve_device(S, k, S->d_targets, S->d_xout, &o, stats ? stats : &local);
  if (st != CN_OK && st != CN_MAX_ITER) return st;
  CN_CUDA(cudaMemcpyAsync(x_out, S->d_xout, sizeof(double) * (size_t)S->nv * k, cudaMemcpyDeviceToHost,
                          S->stream));
  CN_CUDA(cudaStreamSynchronize(S->stream));
  return st;
}

// Plain FP64 Jacobi-PCG: one kernel per primitive, the dots folded on the host
// every iteration (SlangCodegen/SparseLinAlg.lean:11-15,
// SlangCodegen/DotReduceMulti.lean:8-11), absolute-to-relative test as cn_solve.
static cn_status solve_plain(cn_handle S, int k, const double* d_targets, double* d_xout,
                             const cn_solve_opts* o, cn_solve_stats* stats) {
  cn::PlainArgs p{};
  p.n = S->n; p.K = k;
  p.A_ptr = S->d_A_ptr; p.A_col = S->d_A_col; p.A_val = S->d_A64; p.A_diag = S->d_A_diag;
  p.b = S->d_b64; p.x = S->d_x64;
  p.r = S->d_w64[0]; p.z = S->d_w64[1]; p.p = S->d_w64[2]; p.Ap = S->d_w64[3];
  p.blocks = 120;
  p.partials = S->d_partials;
  double* d_scal = S->d_scal;
  SolveArgs sa{};
  sa.nv = S->nv; sa.nh = S->nh; sa.K_ptr = S->d_K_ptr; sa.K_col = S->d_K_col; sa.K_val = S->d_K_val;
  sa.free_of = S->d_free_of; sa.hidx = S->d_hidx; sa.handles = S->d_handles; sa.pos = S->d_pos;
  sa.mode = o->mode; sa.targets = d_targets; sa.x_out = d_xout; sa.x0 = nullptr;
  std::vector<double> part((size_t)p.blocks * k), alpha(k), beta(k), rz(k), bb(k), rr(k);
  std::vector<int> active(k, 1);
  auto host_dot = [&](const double* u, const double* v, std::vector<double>& out) -> cn_status {
    CN_CUDA(cn::plain_dot(p, u, v, S->stream));
    CN_CUDA(cudaMemcpyAsync(part.data(), p.partials, sizeof(double) * part.size(), cudaMemcpyDeviceToHost,
                            S->stream));
    CN_CUDA(cudaStreamSynchronize(S->stream));
    for (int c = 0; c < k; ++c) {
      double s = 0.0;
      for (int b = 0; b < p.blocks; ++b) s += part[(size_t)b * k + c];
      out[c] = s;
    }
    return CN_OK;
  };
  CN_CUDA(cudaEventRecord(S->ev0, S->stream));
  CN_CUDA(cn::plain_rhs_and_init(sa, p, S->stream));
  CN_CUDA(cn::plain_residual(p, S->stream));
  cn_status st;
  if ((st = host_dot(p.b, p.b, bb)) != CN_OK) return st;
  CN_CUDA(cn::plain_jacobi(p, S->stream));
  CN_CUDA(cudaMemcpyAsync(p.p, p.z, sizeof(double) * (size_t)p.n * k, cudaMemcpyDeviceToDevice, S->stream));
  if ((st = host_dot(p.r, p.z, rz)) != CN_OK) return st;
  int it = 0;
  for (; it < o->max_iter; ++it) {
    CN_CUDA(cn::plain_spmv(p, p.p, p.Ap, S->stream));
    std::vector<double> pap(k);
    if ((st = host_dot(p.p, p.Ap, pap)) != CN_OK) return st;
    for (int c = 0; c < k; ++c) {
      if (active[c] && !(pap[c] > 0.0)) active[c] = 0;
      alpha[c] = active[c] ? rz[c] / pap[c] : 0.0;
    }
    CN_CUDA(cn::plain_set_scalars(d_scal, alpha.data(), k, S->stream));
    CN_CUDA(cn::plain_axpy2(p, d_scal, S->stream));
    if ((st = host_dot(p.r, p.r, rr)) != CN_OK) return st;
    bool any = false;
    for (int c = 0; c < k; ++c) {
      if (active[c] && rr[c] < o->tol * o->tol * bb[c]) active[c] = 0;
      any = any || active[c];
    }
    if (!any) { ++it; break; }
    CN_CUDA(cn::plain_jacobi(p, S->stream));
    std::vector<double> rzn(k);
    if ((st = host_dot(p.r, p.z, rzn)) != CN_OK) return st;
    for (int c = 0; c < k; ++c) {
      beta[c] = active[c] ? (rz[c] == 0.0 ? 0.0 : rzn[c] / rz[c]) : 0.0;
      rz[c] = rzn[c];
    }
    CN_CUDA(cn::plain_set_scalars(d_scal + k, beta.data(), k, S->stream));
    CN_CUDA(cn::plain_saxpby(p, d_scal + k, S->stream));
  }
  CN_CUDA(cn::plain_residual(p, S->stream));
  if ((st = host_dot(p.r, p.r, rr)) != CN_OK) return st;
  CN_CUDA(cn::plain_output(sa, p, S->stream));
  CN_CUDA(cudaEventRecord(S->ev1, S->stream));
  CN_CUDA(cudaStreamSynchronize(S->stream));
  S->have_solution = false;  // the plain path does not keep the warm-start layout
  CN_CUDA(cudaMemsetAsync(S->d_x64, 0, sizeof(double) * (size_t)S->n * S->kmax, S->stream));
  double mx = 0.0;
  cn_status res = CN_OK;
  cn_solve_stats local{};
  cn_solve_stats* out = stats ? stats : &local;
  std::memset(out, 0, sizeof *out);
  for (int c = 0; c < k; ++c) {
    const double rel = bb[c] > 0 ? std::sqrt(rr[c] / bb[c]) : std::sqrt(rr[c]);
    if (c < 32) out->rel_residual[c] = rel;
    mx = std::max(mx, rel);
    if (!(rel <= o->tol)) res = CN_MAX_ITER;
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, S->ev0, S->ev1);
  out->status = res;
  out->iterations = it;
  out->refinements = 1;
  out->k = k;
  out->max_rel_residual = mx;
  out->device_ms = ms;
  return res;
}

cn_status cn_export_csr(cn_handle S, int32_t* free_of, int32_t* rowptr, int32_t* colidx,
                        double* vals) {
  if (!S) return CN_BAD_INPUT;
  CN_CUDA(cudaSetDevice(S->device));
  if (free_of) std::memcpy(free_of, S->free_of.data(), sizeof(int) * S->n);
  if (rowptr) std::memcpy(rowptr, S->A_ptr.data(), sizeof(int) * (S->n + 1));
  if (colidx) std::memcpy(colidx, S->A_col.data(), sizeof(int) * S->nnzA);
  if (vals) CN_CUDA(cudaMemcpy(vals, S->d_A64, sizeof(double) * S->nnzA, cudaMemcpyDeviceToHost));
  return CN_OK;
}

cn_status cn_export_factor(cn_handle S, int32_t* rowptr, int32_t* colidx, double* vals) {
  if (!S) return CN_BAD_INPUT;
  CN_CUDA(cudaSetDevice(S->device));
  std::vector<double> L(S->nnzL), d(S->n);
  if (S->nnzL) CN_CUDA(cudaMemcpy(L.data(), S->d_L64, sizeof(double) * S->nnzL, cudaMemcpyDeviceToHost));
  if (S->n) CN_CUDA(cudaMemcpy(d.data(), S->d_Ld64, sizeof(double) * S->n, cudaMemcpyDeviceToHost));
  int q = 0;
  if (rowptr) rowptr[0] = 0;
  for (int i = 0; i < S->n; ++i) {
    for (int e = S->L_ptr[i]; e < S->L_ptr[i + 1]; ++e, ++q) {
      if (colidx) colidx[q] = S->L_col[e];
      if (vals) vals[q] = L[e];
    }
    if (colidx) colidx[q] = i;
    if (vals) vals[q] = d[i];
    ++q;
    if (rowptr) rowptr[i + 1] = q;
  }
  return CN_OK;
}

cn_status cn_export_k(cn_handle S, int32_t* rowptr, int32_t* colidx, double* vals) {
  if (!S) return CN_BAD_INPUT;
  CN_CUDA(cudaSetDevice(S->device));
  if (rowptr) std::memcpy(rowptr, S->K_ptr.data(), sizeof(int) * (S->nv + 1));
  if (colidx) std::memcpy(colidx, S->K_col.data(), sizeof(int) * S->nnzK);
  if (vals) CN_CUDA(cudaMemcpy(vals, S->d_K_val, sizeof(double) * S->nnzK, cudaMemcpyDeviceToHost));
  return CN_OK;
}

}  // extern "C"
