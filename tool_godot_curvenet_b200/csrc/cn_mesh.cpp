// cn_mesh.cpp -- per-mesh host structure (K pattern and face contributions,
// handle checks, elimination order, IC(0) pattern and task lists), its device
// layout and upload, and the GPU assembly + factor with shift retries.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "cn_mesh.h"

namespace cn {
namespace {

thread_local std::string g_err;

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

int local_of(int corner) { return (corner + 2) % 3; }  // t0,t1,t2 -> faceLoop slots 2,0,1
int off_slot(int a, int b) {
  if (a > b) std::swap(a, b);
  return a == 0 ? (b == 1 ? 3 : 4) : 5;
}

}  // namespace

void set_err(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
}

const char* last_err() { return g_err.c_str(); }

void set_last_error_text(const char* msg) { g_err = msg; }

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

cn_status build_host(const cn_mesh_desc* m, const cn_build_opts& o, MeshHost& H) {
  MeshHost* S = &H;
  std::vector<int>& K_cptr = H.K_cptr;
  std::vector<int>& K_contrib = H.K_contrib;
  std::vector<int>& hidx = H.hidx;
  std::vector<int>& A_src = H.A_src;
  std::vector<int>& A_diag = H.A_diag;
  std::vector<int>& L_src = H.L_src;
  std::vector<int>& T_ptr = H.T_ptr;
  std::vector<int>& T_a = H.T_a;
  std::vector<int>& T_b = H.T_b;
  std::vector<int>& U_ptr = H.U_ptr;
  std::vector<int>& U_col = H.U_col;
  std::vector<int>& U_src = H.U_src;
  H.nv = m->n_verts;
  H.nt = m->n_tris;
  H.nh = m->n_handles;
  H.pos.assign(m->positions, m->positions + 3 * (size_t)m->n_verts);
  H.tris.assign(m->tris, m->tris + 3 * (size_t)m->n_tris);
  H.handles.assign(m->handles, m->handles + m->n_handles);
  const int nv = m->n_verts, nt = m->n_tris;
  const int* tris = m->tris;
  // --- K pattern and the face contributions of every entry
  std::vector<int>& vf_ptr = H.vf_ptr;
  std::vector<int>& vf_face = H.vf_face;
  std::vector<int>& vf_corner = H.vf_corner;
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
  const bool by_color = o.ordering == CN_ORDER_COLOR || (o.ordering == CN_ORDER_AUTO && o.precond == CN_PRECOND_IC0);
  if (by_color)
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return color[a] < color[b]; });
  // level of every unknown in that order; rows sorted by level
  std::vector<int> posn(n), level(n, 0);
  for (int i = 0; i < n; ++i) posn[ord[i]] = i;
  int nlev = n ? 1 : 0;
  if (o.precond == CN_PRECOND_IC0) {
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
  if (o.precond == CN_PRECOND_IC0) {
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

void layout(Bump& b, const MeshHost& H, MeshDev& D) {
  D.pos = b.take<double>(H.pos.size());
  D.tris = b.take<int>(H.tris.size());
  D.K_ptr = b.take<int>(H.K_ptr.size());
  D.K_col = b.take<int>(H.K_col.size());
  D.K_cptr = b.take<int>(H.K_cptr.size());
  D.K_contrib = b.take<int>(H.K_contrib.size());
  D.hidx = b.take<int>(H.hidx.size());
  D.free_of = b.take<int>(H.free_of.size());
  D.handles = b.take<int>(H.handles.size());
  // 4 elements to spare: the staged SpMV's bulk copies round up to 16 bytes
  D.A_ptr = b.take<int>(H.A_ptr.size() + 4);
  D.A_col = b.take<int>(H.A_col.size() + 4);
  D.A_src = b.take<int>(H.A_src.size());
  D.A_diag = b.take<int>(H.A_diag.size());
  D.lev_ptr = b.take<int>(H.lev_ptr.size());
  D.L_ptr = b.take<int>(H.L_ptr.size());
  D.L_col = b.take<int>(H.L_col.size());
  D.L_src = b.take<int>(H.L_src.size());
  D.T_ptr = b.take<int>(H.T_ptr.size());
  D.T_a = b.take<int>(H.T_a.size());
  D.T_b = b.take<int>(H.T_b.size());
  D.U_ptr = b.take<int>(H.U_ptr.size());
  D.U_col = b.take<int>(H.U_col.size());
  D.U_src = b.take<int>(H.U_src.size());
  D.face_m = b.take<double>(6 * (size_t)H.nt);
  D.K_val = b.take<double>(H.nnzK);
  D.A64 = b.take<double>(H.nnzA + 4);
  D.A32 = b.take<float>(H.nnzA + 4);
  D.L64 = b.take<double>(H.nnzL);
  D.L32 = b.take<float>(H.nnzL);
  D.U64 = b.take<double>(H.nnzL);
  D.U32 = b.take<float>(H.nnzL);
  D.Ld64 = b.take<double>(H.n);
  D.dinv64 = b.take<double>(H.n);
  D.dinv32 = b.take<float>(H.n);
}

cn_status upload(const MeshHost& H, const MeshDev& D, cudaStream_t s) {
  auto up = [&](void* dst, const void* src, size_t bytes) {
    return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s) : cudaSuccess;
  };
#define UPV(field, vec) \
  if (up(D.field, H.vec.data(), sizeof(H.vec[0]) * H.vec.size()) != cudaSuccess) { set_err("upload of " #vec " failed"); return CN_CUDA_ERROR; }
  UPV(pos, pos) UPV(tris, tris) UPV(K_ptr, K_ptr) UPV(K_col, K_col) UPV(K_cptr, K_cptr)
  UPV(K_contrib, K_contrib) UPV(hidx, hidx) UPV(free_of, free_of) UPV(handles, handles)
  UPV(A_ptr, A_ptr) UPV(A_col, A_col) UPV(A_src, A_src) UPV(A_diag, A_diag) UPV(lev_ptr, lev_ptr)
  UPV(L_ptr, L_ptr) UPV(L_col, L_col) UPV(L_src, L_src) UPV(T_ptr, T_ptr) UPV(T_a, T_a)
  UPV(T_b, T_b) UPV(U_ptr, U_ptr) UPV(U_col, U_col) UPV(U_src, U_src)
#undef UPV
  return CN_OK;
}

cn_status assemble_factor(const MeshHost& H, const MeshDev& D, const cn_build_opts& o, int* d_status,
                          cudaStream_t s, double* shift_used) {
  BuildArgs b{};
  b.nv = H.nv; b.nt = H.nt; b.nnzK = H.nnzK; b.n = H.n; b.nnzA = H.nnzA; b.nnzL = H.nnzL; b.nlev = H.nlev;
  b.pos = D.pos; b.tris = D.tris; b.lap_kind = o.laplacian; b.delta = o.mollify_delta;
  b.face_m = D.face_m; b.K_cptr = D.K_cptr; b.K_contrib = D.K_contrib; b.K_val = D.K_val;
  b.A_src = D.A_src; b.A_val64 = D.A64; b.A_val32 = D.A32; b.A_diag = D.A_diag;
  b.lev_ptr = D.lev_ptr; b.h_lev_ptr = H.lev_ptr.data();
  b.L_ptr = D.L_ptr; b.L_src = D.L_src; b.L_col = D.L_col;
  b.T_ptr = D.T_ptr; b.T_a = D.T_a; b.T_b = D.T_b;
  b.L_val64 = D.L64; b.L_val32 = D.L32; b.Ld64 = D.Ld64;
  b.dinv64 = D.dinv64; b.dinv32 = D.dinv32;
  b.U_src = D.U_src; b.U_val64 = D.U64; b.U_val32 = D.U32;
  b.status = d_status; b.precond = o.precond;
  if (launch_assemble(b, s) != cudaSuccess) {
    set_err("assembly launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    return CN_CUDA_ERROR;
  }
  // IC(0) with Manteuffel diagonal-shift retries on a non-positive pivot.
  const double shifts[] = {0.0, 1e-3, 1e-2, 1e-1};
  int bad = -1;
  for (double sh : shifts) {
    const int ok = 0x7fffffff;
    if (cudaMemcpyAsync(d_status, &ok, sizeof ok, cudaMemcpyHostToDevice, s) != cudaSuccess) {
      set_err("status reset failed");
      return CN_CUDA_ERROR;
    }
    b.shift = sh;
    if (launch_factor(b, s) != cudaSuccess) {
      set_err("factor launch failed");
      return CN_CUDA_ERROR;
    }
    int h_status = 0;
    if (cudaMemcpyAsync(&h_status, d_status, sizeof h_status, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      set_err("factor failed: %s", cudaGetErrorString(cudaGetLastError()));
      return CN_CUDA_ERROR;
    }
    bad = h_status == ok ? -1 : h_status;
    if (shift_used) *shift_used = sh;
    if (bad < 0) break;
  }
  if (bad >= 0) {
    set_err("IC(0) pivot of row %d is not positive", bad);
    return CN_NONPOS_PIVOT;
  }
  return CN_OK;
}

void permute_solve_order(MeshHost& H, const std::vector<int>& order) {
  const int n = H.n;
  std::vector<int> pos_of(n);
  for (int p = 0; p < n; ++p) pos_of[order[p]] = p;
  std::vector<int> ptr(n + 1, 0), col(H.nnzA), src(H.nnzA), diag(n, -1), free_of(n);
  std::vector<std::pair<int, int>> row;
  for (int p = 0; p < n; ++p) {
    const int o = order[p];
    free_of[p] = H.free_of[o];
    row.clear();
    for (int e = H.A_ptr[o]; e < H.A_ptr[o + 1]; ++e) row.push_back({pos_of[H.A_col[e]], H.A_src[e]});
    std::sort(row.begin(), row.end());
    for (size_t q = 0; q < row.size(); ++q) {
      col[ptr[p] + q] = row[q].first;
      src[ptr[p] + q] = row[q].second;
      if (row[q].first == p) diag[p] = ptr[p] + (int)q;
    }
    ptr[p + 1] = ptr[p] + (int)row.size();
  }
  H.A_ptr.swap(ptr);
  H.A_col.swap(col);
  H.A_src.swap(src);
  H.A_diag.swap(diag);
  H.free_of.swap(free_of);
}

SolveArgs solve_args(const MeshHost& H, const MeshDev& D, bool mixed) {
  SolveArgs a{};
  a.n = H.n; a.nlev = H.nlev; a.lev_ptr = D.lev_ptr;
  a.A_ptr = D.A_ptr; a.A_col = D.A_col;
  a.A_val = mixed ? (const void*)D.A32 : (const void*)D.A64;
  a.A_val64 = D.A64;
  a.L_ptr = D.L_ptr; a.L_col = D.L_col;
  a.L_val = mixed ? (const void*)D.L32 : (const void*)D.L64;
  a.U_ptr = D.U_ptr; a.U_col = D.U_col;
  a.U_val = mixed ? (const void*)D.U32 : (const void*)D.U64;
  a.dinv = mixed ? (const void*)D.dinv32 : (const void*)D.dinv64;
  a.nv = H.nv; a.nh = H.nh;
  a.K_ptr = D.K_ptr; a.K_col = D.K_col; a.K_val = D.K_val;
  a.free_of = D.free_of; a.hidx = D.hidx; a.handles = D.handles; a.pos = D.pos;
  return a;
}

}  // namespace cn
