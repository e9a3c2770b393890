// curvenet_oracle.cpp -- CPU FP64 restatement of the reference's Lean
// specification of the profile-curves deformer's sparse solve.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker: it is linked by the
// tests, by __graft_entry__.smoke() and by bench.py's cpu_baseline / reference
// arm, and by nothing else.  The product (tool_godot_curvenet_b200) never
// calls into it.
//
// Every function cites the Lean file:line (relative to the reference project
// root) whose arithmetic it restates.  Floating point follows Lean core
// `Float` (IEEE binary64): the build uses -ffp-contract=off so a*b+c is two
// roundings, exactly as Lean evaluates it, and sums run in the spec's order.
//
// Conventions of the C ABI (ctypes-friendly):
//   * halfedge meshes are int32 [nhe][4] = (target, twin, next, face), with
//     -1 standing for Lean's `none`;
//   * matrices are row-major double arrays; CSR uses int32 row pointers.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// PolygonLaplacian.lean:32-40  cotAtVertex
double cot_at_vertex(const double* apex, const double* o1, const double* o2) {
  double ax = o1[0] - apex[0], ay = o1[1] - apex[1], az = o1[2] - apex[2];
  double bx = o2[0] - apex[0], by = o2[1] - apex[1], bz = o2[2] - apex[2];
  double dot = ax * bx + ay * by + az * bz;
  double cx = ay * bz - az * by;
  double cy = az * bx - ax * bz;
  double cz = ax * by - ay * bx;
  double cross_len = std::sqrt(cx * cx + cy * cy + cz * cz);
  return dot / cross_len;
}

// PolygonLaplacian.lean:56-71  triangleCotLaplacian (row-major 3x3)
void triangle_cot_laplacian(const double* a, const double* b, const double* c,
                            double* m) {
  double cotA = cot_at_vertex(a, b, c);
  double cotB = cot_at_vertex(b, a, c);
  double cotC = cot_at_vertex(c, a, b);
  double w_bc = cotA * 0.5, w_ac = cotB * 0.5, w_ab = cotC * 0.5;
  for (int i = 0; i < 9; ++i) m[i] = 0.0;
  m[0 * 3 + 1] = -w_ab; m[1 * 3 + 0] = -w_ab;
  m[0 * 3 + 2] = -w_ac; m[2 * 3 + 0] = -w_ac;
  m[1 * 3 + 2] = -w_bc; m[2 * 3 + 1] = -w_bc;
  m[0] = w_ab + w_ac;
  m[4] = w_ab + w_bc;
  m[8] = w_ac + w_bc;
}

// RobustLaplacian.lean:66-72 edgeLengthsFromTriangle (eA=|b-c|, eB=|a-c|, eC=|a-b|)
void edge_lengths(const double* a, const double* b, const double* c, double* e) {
  auto d = [](const double* u, const double* v) {
    double dx = u[0] - v[0], dy = u[1] - v[1], dz = u[2] - v[2];
    return std::sqrt(dx * dx + dy * dy + dz * dz);
  };
  e[0] = d(b, c); e[1] = d(a, c); e[2] = d(a, b);
}

// RobustLaplacian.lean:83-89 mollifyTriangle
double mollify_triangle(double delta, const double* e) {
  double ra = delta + e[0] - e[1] - e[2];
  double rb = delta + e[1] - e[0] - e[2];
  double rc = delta + e[2] - e[0] - e[1];
  double m = std::max(ra, std::max(rb, rc));
  return std::max(0.0, m);
}

// RobustLaplacian.lean:106-109 cotFromLengths
double cot_from_lengths(double eo, double e1, double e2) {
  double s = (eo + e1 + e2) * 0.5;
  double area = std::sqrt(s * (s - eo) * (s - e1) * (s - e2));
  return (e1 * e1 + e2 * e2 - eo * eo) / (4.0 * area);
}

// RobustLaplacian.lean:114-140 robustTriangleCotLaplacian
void robust_triangle_cot_laplacian(double delta, const double* a, const double* b,
                                   const double* c, double* m) {
  double e[3];
  edge_lengths(a, b, c, e);
  double eps = mollify_triangle(delta, e);
  e[0] += eps; e[1] += eps; e[2] += eps;
  double cotA = cot_from_lengths(e[0], e[1], e[2]);
  double cotB = cot_from_lengths(e[1], e[0], e[2]);
  double cotC = cot_from_lengths(e[2], e[0], e[1]);
  double w_bc = cotA * 0.5, w_ac = cotB * 0.5, w_ab = cotC * 0.5;
  for (int i = 0; i < 9; ++i) m[i] = 0.0;
  m[1] = -w_ab; m[3] = -w_ab;
  m[2] = -w_ac; m[6] = -w_ac;
  m[5] = -w_bc; m[7] = -w_bc;
  m[0] = w_ab + w_ac;
  m[4] = w_ab + w_bc;
  m[8] = w_ac + w_bc;
}

// Per-triangle 3x3 in the chosen discretisation (0 = embedded cot, 1 = robust).
void tri_laplacian(int kind, double delta, const double* a, const double* b,
                   const double* c, double* m) {
  if (kind == 1) robust_triangle_cot_laplacian(delta, a, b, c, m);
  else triangle_cot_laplacian(a, b, c, m);
}

// PolygonLaplacian.lean:77-93 polygonCotLaplacian (fan from vertex 0)
void polygon_cot_laplacian(int kind, double delta, int n, const double* pts,
                           double* m) {
  for (int i = 0; i < n * n; ++i) m[i] = 0.0;
  if (n < 3) return;
  for (int i = 1; i < n - 1; ++i) {
    double t[9];
    tri_laplacian(kind, delta, pts, pts + 3 * i, pts + 3 * (i + 1), t);
    int idx[3] = {0, i, i + 1};
    for (int li = 0; li < 3; ++li)
      for (int lj = 0; lj < 3; ++lj)
        m[idx[li] * n + idx[lj]] = m[idx[li] * n + idx[lj]] + t[li * 3 + lj];
  }
}

struct HE { int target, twin, next, face; };

// CutMeshLaplacian.lean:29-46 faceLoop (scan for the first halfedge of the face)
std::vector<int> face_loop(const std::vector<HE>& hes, int f) {
  int nh = (int)hes.size();
  int start = -1;
  for (int h = 0; h < nh; ++h)
    if (hes[h].face == f) { start = h; break; }
  std::vector<int> acc;
  if (start < 0) return acc;
  acc.push_back(start);
  int cur = hes[start].next, steps = 0;
  while (cur != start && steps < nh) {
    acc.push_back(cur);
    cur = hes[cur].next;
    ++steps;
  }
  return acc;
}

}  // namespace

extern "C" {

// ===========================================================================
// Per-element geometry
// ===========================================================================
double orc_cot_at_vertex(const double* apex, const double* o1, const double* o2) {
  return cot_at_vertex(apex, o1, o2);
}
void orc_triangle_cot_laplacian(const double* a, const double* b, const double* c,
                                double* out9) {
  triangle_cot_laplacian(a, b, c, out9);
}
void orc_polygon_cot_laplacian(int n, const double* pts, double* out) {
  polygon_cot_laplacian(0, 0.0, n, pts, out);
}
void orc_edge_lengths(const double* a, const double* b, const double* c, double* e3) {
  edge_lengths(a, b, c, e3);
}
double orc_mollify_triangle(double delta, const double* e3) {
  return mollify_triangle(delta, e3);
}
double orc_cot_from_lengths(double eo, double e1, double e2) {
  return cot_from_lengths(eo, e1, e2);
}
void orc_robust_triangle_cot_laplacian(double delta, const double* a, const double* b,
                                       const double* c, double* out9) {
  robust_triangle_cot_laplacian(delta, a, b, c, out9);
}

// ===========================================================================
// Halfedge layer
// ===========================================================================

// HalfedgeBuilder.lean:34-90 fromTriangles.  The O(n^2) twin scan of the spec
// (:53-56) is replaced by a map to the lowest matching index, which is the
// same "first match" the linear scan returns.  Output capacity 6*nt.
int orc_halfedges_from_triangles(int nv, int nt, const int* tris, int* he_out) {
  (void)nv;
  int nint = 3 * nt;
  std::vector<HE> hes(nint);
  auto src_of = [&](int h) { int f = h / 3, l = h % 3; return tris[3 * f + l]; };
  for (int f = 0; f < nt; ++f) {
    int t0 = tris[3 * f], t1 = tris[3 * f + 1], t2 = tris[3 * f + 2];
    hes[3 * f + 0] = {t1, -1, 3 * f + 1, f};
    hes[3 * f + 1] = {t2, -1, 3 * f + 2, f};
    hes[3 * f + 2] = {t0, -1, 3 * f + 0, f};
  }
  std::unordered_map<uint64_t, int> first;  // (src,tgt) -> lowest interior index
  first.reserve(nint * 2);
  for (int j = 0; j < nint; ++j) {
    uint64_t key = ((uint64_t)(uint32_t)src_of(j) << 32) | (uint32_t)hes[j].target;
    if (!first.count(key)) first[key] = j;
  }
  std::vector<int> need;
  for (int i = 0; i < nint; ++i) {
    uint64_t key = ((uint64_t)(uint32_t)hes[i].target << 32) | (uint32_t)src_of(i);
    auto it = first.find(key);
    if (it != first.end()) hes[i].twin = it->second;
    else need.push_back(i);
  }
  int bstart = (int)hes.size();
  for (int i : need) {
    int bh = (int)hes.size();
    hes.push_back({src_of(i), i, 0, -1});
    hes[i].twin = bh;
  }
  int n = (int)hes.size();
  // step 4: next = first boundary halfedge (index order) whose source == my target
  std::unordered_map<int, int> first_by_src;
  for (int j = bstart; j < n; ++j) {
    int srcj = hes[hes[j].twin].target;
    if (!first_by_src.count(srcj)) first_by_src[srcj] = j;
  }
  for (int i = bstart; i < n; ++i) {
    auto it = first_by_src.find(hes[i].target);
    hes[i].next = it == first_by_src.end() ? i : it->second;
  }
  for (int h = 0; h < n; ++h) {
    he_out[4 * h] = hes[h].target; he_out[4 * h + 1] = hes[h].twin;
    he_out[4 * h + 2] = hes[h].next; he_out[4 * h + 3] = hes[h].face;
  }
  return n;
}

// Halfedge.lean:253-331 manifold? = indicesInRange && twinInvolutive &&
// twinsAreOpposite && faceLoopsClose.  Returns 1/0.
int orc_manifold(int nv, int nf, int nhe, const int* he) {
  auto T = [&](int h) { return he[4 * h]; };
  auto W = [&](int h) { return he[4 * h + 1]; };
  auto N = [&](int h) { return he[4 * h + 2]; };
  auto F = [&](int h) { return he[4 * h + 3]; };
  for (int i = 0; i < nhe; ++i) {  // :253-265
    if (T(i) >= nv || T(i) < 0) return 0;
    if (N(i) >= nhe || N(i) < 0) return 0;
    if (W(i) >= nhe) return 0;
    if (F(i) >= nf) return 0;
  }
  for (int i = 0; i < nhe; ++i) {  // :268-278
    int t = W(i);
    if (t < 0) continue;
    if (W(t) != i) return 0;
  }
  std::vector<int> prev(nhe, 0);  // :286-302
  for (int i = 0; i < nhe; ++i) prev[N(i)] = i;
  for (int i = 0; i < nhe; ++i) {
    int t = W(i);
    if (t < 0) continue;
    if (T(prev[i]) != T(t)) return 0;
  }
  for (int s = 0; s < nhe; ++s) {  // :307-326
    int f0 = F(s);
    if (f0 < 0) continue;
    int cur = N(s), steps = 0;
    bool closed = false;
    while (steps < nhe) {
      if (cur == s) { closed = true; break; }
      if (F(cur) != f0) return 0;
      cur = N(cur);
      ++steps;
    }
    if (!closed) return 0;
  }
  return 1;
}

// CutAlgorithm.lean:49-99 subdivideEdge.  he_out has capacity nhe+2.
// counts = {nv, nf, nhe} updated in place.
void orc_subdivide_edge(int* counts, const int* he_in, int h, int* he_out) {
  int nv = counts[0], nh = counts[2];
  std::memcpy(he_out, he_in, sizeof(int) * 4 * nh);
  const int* o = he_in + 4 * h;
  int twin = o[1] >= 0 ? o[1] : h;
  const int* t = he_in + 4 * twin;
  int c = nv, hnew = nh, tnew = nh + 1;
  int H[4] = {c, tnew, hnew, o[3]};
  int Hn[4] = {o[0], twin, o[2], o[3]};
  int Tw[4] = {c, hnew, tnew, t[3]};
  int Tn[4] = {t[0], h, t[2], t[3]};
  std::memcpy(he_out + 4 * h, H, sizeof H);
  std::memcpy(he_out + 4 * twin, Tw, sizeof Tw);
  std::memcpy(he_out + 4 * hnew, Hn, sizeof Hn);
  std::memcpy(he_out + 4 * tnew, Tn, sizeof Tn);
  counts[0] = nv + 1;
  counts[2] = nh + 2;
}

// CutAlgorithm.lean:125-170 splitFace
void orc_split_face(int* counts, const int* he_in, int a, int b, int* he_out) {
  int nh = counts[2], nf = counts[1];
  std::memcpy(he_out, he_in, sizeof(int) * 4 * nh);
  int A[4], B[4];
  std::memcpy(A, he_in + 4 * a, sizeof A);
  std::memcpy(B, he_in + 4 * b, sizeof B);
  int oldNextA = A[2], oldNextB = B[2];
  int fp = nf, hAB = nh, hBA = nh + 1;
  int cur = oldNextB, steps = 0;
  while (cur != a && steps < nh) {
    he_out[4 * cur + 3] = fp;
    cur = he_out[4 * cur + 2];
    ++steps;
  }
  he_out[4 * a + 3] = fp; he_out[4 * a + 2] = hAB;
  he_out[4 * b + 2] = hBA;
  int AB[4] = {B[0], hBA, oldNextB, fp};
  int BA[4] = {A[0], hAB, oldNextA, A[3]};
  std::memcpy(he_out + 4 * hAB, AB, sizeof AB);
  std::memcpy(he_out + 4 * hBA, BA, sizeof BA);
  counts[1] = nf + 1;
  counts[2] = nh + 2;
}

// CutAlgorithm.lean:225-251 insertCrack
void orc_insert_crack(int* counts, const int* he_in, int h_anchor, int* he_out) {
  int nh = counts[2], nv = counts[0];
  std::memcpy(he_out, he_in, sizeof(int) * 4 * nh);
  int An[4];
  std::memcpy(An, he_in + 4 * h_anchor, sizeof An);
  int vb = An[0], oldNext = An[2], c = nv, hout = nh, hin = nh + 1;
  he_out[4 * h_anchor + 2] = hout;
  int O[4] = {c, hin, hin, An[3]};
  int I[4] = {vb, hout, oldNext, An[3]};
  std::memcpy(he_out + 4 * hout, O, sizeof O);
  std::memcpy(he_out + 4 * hin, I, sizeof I);
  counts[0] = nv + 1;
  counts[2] = nh + 2;
}

// Length of the `next` loop through halfedge h (the walks in CutAlgorithm.lean's
// examples, e.g. :281-290).
int orc_loop_length(int nhe, const int* he, int h) {
  int cur = he[4 * h + 2], steps = 1;
  while (cur != h && steps < nhe) { cur = he[4 * cur + 2]; ++steps; }
  return steps;
}

// CutMesh.lean:83-103 partitionOfUnity / VtCIsZero.  vkind: 0 = meshVertex,
// 1 = sample, 2 = edgeIntersection.  Returns 1 when every halfedge maps to
// exactly one of V or C.
int orc_partition_of_unity(int nhe, const int* he, const int* vkind) {
  for (int h = 0; h < nhe; ++h) {
    int k = vkind[he[4 * h]];
    bool v = k == 0, c = k == 1;
    if (v == c) return 0;
  }
  return 1;
}

// ===========================================================================
// Seam cut of a triangle mesh along closed vertex loops (the build's A2 cut).
// For each loop vertex v (loops in order, positions in order) a copy with id
// nv + running index is created, and every face swept counter-clockwise
// around v from the outgoing loop edge (v -> next) up to, not including, the
// face of the halfedge (v -> prev) is re-pointed to the copy.  The sweep walks
// the halfedge structure of HalfedgeBuilder.lean:34-90 (prev(h) then twin),
// which is the rotation the spec's CutAlgorithm surgery preserves.
// Returns the new vertex count, or -1 on a loop edge without a left face or
// an open fan, -2 on a vertex appearing in two loops.
int orc_cut_mesh(int nv, int nt, const int* tris, int nloops, const int* loop_ptr,
                 const int* loop_verts, int* tris_out, int* parent_out) {
  std::vector<int> he(4 * 6 * (size_t)nt);
  int nhe = orc_halfedges_from_triangles(nv, nt, tris, he.data());
  auto T = [&](int h) { return he[4 * h]; };
  auto W = [&](int h) { return he[4 * h + 1]; };
  auto N = [&](int h) { return he[4 * h + 2]; };
  auto F = [&](int h) { return he[4 * h + 3]; };
  // interior halfedge lookup by (src, tgt); src(h) = target of prev(h)
  std::unordered_map<uint64_t, int> by_edge;
  by_edge.reserve(3 * nt * 2);
  for (int h = 0; h < 3 * nt; ++h) {
    int src = tris[3 * (h / 3) + h % 3];
    by_edge[((uint64_t)(uint32_t)src << 32) | (uint32_t)T(h)] = h;
  }
  std::memcpy(tris_out, tris, sizeof(int) * 3 * nt);
  std::vector<char> seen(nv, 0);
  int next_id = nv;
  for (int v = 0; v < nv; ++v) parent_out[v] = v;
  for (int l = 0; l < nloops; ++l) {
    int lo = loop_ptr[l], hi = loop_ptr[l + 1], m = hi - lo;
    for (int i = 0; i < m; ++i) {
      int v = loop_verts[lo + i];
      int vn = loop_verts[lo + (i + 1) % m];
      int vp = loop_verts[lo + (i - 1 + m) % m];
      if (seen[v]) return -2;
      seen[v] = 1;
      int copy = next_id++;
      parent_out[copy] = v;
      auto it = by_edge.find(((uint64_t)(uint32_t)v << 32) | (uint32_t)vn);
      if (it == by_edge.end()) return -1;
      int h = it->second;
      int guard = 0;
      while (true) {
        int f = F(h);
        if (f < 0 || ++guard > nhe) return -1;
        for (int c = 0; c < 3; ++c)
          if (tris[3 * f + c] == v) tris_out[3 * f + c] = copy;
        // prev(h) in a triangle loop is next(next(h)); its twin leaves v
        int pv = N(N(h));
        int t = W(pv);
        if (t < 0) return -1;
        if (T(t) == vp) break;
        h = t;
      }
    }
  }
  return next_id;
}

// ===========================================================================
// Dense, literal DeGoes22 assembly (CutMeshLaplacian.lean:56-93)
// ===========================================================================

// CutMeshLaplacian.lean:56-71 assembleLh, :75-83 assembleV, :86-93 assembleVtLhV.
// vkind[v] == 0 marks mesh vertices (columns of V).  out: nv*nv.
// Dense O(nhe^2) memory: small meshes only.
void orc_assemble_vtlhv_dense(int nv, int nf, int nhe, const int* he, const int* vkind,
                              const double* pos, int lap_kind, double delta, double* out) {
  std::vector<HE> hes(nhe);
  for (int h = 0; h < nhe; ++h) hes[h] = {he[4 * h], he[4 * h + 1], he[4 * h + 2], he[4 * h + 3]};
  size_t nh = nhe;
  std::vector<double> L(nh * nh, 0.0);
  for (int f = 0; f < nf; ++f) {
    std::vector<int> loop = face_loop(hes, f);
    int n = (int)loop.size();
    if (n < 3) continue;
    std::vector<double> poly(3 * n), Lf(n * n);
    for (int i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) poly[3 * i + d] = pos[3 * hes[loop[i]].target + d];
    polygon_cot_laplacian(lap_kind, delta, n, poly.data(), Lf.data());
    for (int li = 0; li < n; ++li)
      for (int lj = 0; lj < n; ++lj) {
        size_t gi = loop[li], gj = loop[lj];
        L[gi * nh + gj] = L[gi * nh + gj] + Lf[li * n + lj];
      }
  }
  // V[h, target(h)] = 1 for mesh-vertex targets.  LhV = L V; VtLhV = Vt (L V),
  // both as the spec's matMul (sum from 0.0 over the inner index in order).
  std::vector<int> vcol(nhe);
  for (int h = 0; h < nhe; ++h) vcol[h] = vkind[hes[h].target] == 0 ? hes[h].target : -1;
  std::vector<double> LV(nh * (size_t)nv, 0.0);
  for (size_t i = 0; i < nh; ++i)
    for (int j = 0; j < nv; ++j) {
      double s = 0.0;
      for (size_t p = 0; p < nh; ++p) s = s + L[i * nh + p] * (vcol[p] == j ? 1.0 : 0.0);
      LV[i * nv + j] = s;
    }
  for (int i = 0; i < nv; ++i)
    for (int j = 0; j < nv; ++j) {
      double s = 0.0;
      for (size_t p = 0; p < nh; ++p) s = s + (vcol[p] == i ? 1.0 : 0.0) * LV[p * nv + j];
      out[(size_t)i * nv + j] = s;
    }
}

// DenseLinAlg.lean:70-109 solve (Gaussian elimination, partial pivoting; a
// zero pivot is skipped and its unknown returns 0).
void orc_dense_solve(int n, const double* A, const double* b, double* x) {
  int m = n + 1;
  std::vector<double> aug((size_t)n * m);
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) aug[(size_t)i * m + j] = A[(size_t)i * n + j];
    aug[(size_t)i * m + n] = b[i];
  }
  for (int k = 0; k < n; ++k) {
    int piv = k;
    double best = std::fabs(aug[(size_t)k * m + k]);
    for (int r = k + 1; r < n; ++r) {
      double v = std::fabs(aug[(size_t)r * m + k]);
      if (v > best) { best = v; piv = r; }
    }
    if (piv != k)
      for (int j = 0; j < m; ++j) std::swap(aug[(size_t)k * m + j], aug[(size_t)piv * m + j]);
    double pivot = aug[(size_t)k * m + k];
    if (pivot == 0.0) continue;
    for (int r = k + 1; r < n; ++r) {
      double factor = aug[(size_t)r * m + k] / pivot;
      for (int j = k; j < m; ++j)
        aug[(size_t)r * m + j] = aug[(size_t)r * m + j] - factor * aug[(size_t)k * m + j];
    }
  }
  for (int i = 0; i < n; ++i) {
    int row = n - 1 - i;
    double s = aug[(size_t)row * m + n];
    for (int j = row + 1; j < n; ++j) s = s - aug[(size_t)row * m + j] * x[j];
    double pivot = aug[(size_t)row * m + row];
    x[row] = pivot == 0.0 ? 0.0 : s / pivot;
  }
}

// DenseLinAlg.lean:122-131 solveMulti (column by column)
void orc_dense_solve_multi(int n, int k, const double* A, const double* B, double* X) {
  std::vector<double> bc(n), xc(n);
  for (int c = 0; c < k; ++c) {
    for (int i = 0; i < n; ++i) bc[i] = B[(size_t)i * k + c];
    orc_dense_solve(n, A, bc.data(), xc.data());
    for (int i = 0; i < n; ++i) X[(size_t)i * k + c] = xc[i];
  }
}

// DenseLinAlg.lean:145-176 factorizeLU + :179-205 solveWithLU
void orc_lu_solve(int n, const double* Ain, const double* b, double* x) {
  std::vector<double> a(Ain, Ain + (size_t)n * n);
  std::vector<int> piv(n);
  for (int i = 0; i < n; ++i) piv[i] = i;
  for (int k = 0; k < n; ++k) {
    int pr = k;
    double best = std::fabs(a[(size_t)k * n + k]);
    for (int r = k + 1; r < n; ++r) {
      double v = std::fabs(a[(size_t)r * n + k]);
      if (v > best) { best = v; pr = r; }
    }
    if (pr != k) {
      for (int j = 0; j < n; ++j) std::swap(a[(size_t)k * n + j], a[(size_t)pr * n + j]);
      std::swap(piv[k], piv[pr]);
    }
    double pivot = a[(size_t)k * n + k];
    if (pivot == 0.0) continue;
    for (int r = k + 1; r < n; ++r) {
      double factor = a[(size_t)r * n + k] / pivot;
      a[(size_t)r * n + k] = factor;
      for (int j = k + 1; j < n; ++j)
        a[(size_t)r * n + j] = a[(size_t)r * n + j] - factor * a[(size_t)k * n + j];
    }
  }
  std::vector<double> y(n);
  for (int i = 0; i < n; ++i) y[i] = b[piv[i]];
  for (int i = 0; i < n; ++i) {
    double s = y[i];
    for (int j = 0; j < i; ++j) s = s - a[(size_t)i * n + j] * y[j];
    y[i] = s;
  }
  for (int i = 0; i < n; ++i) {
    int row = n - 1 - i;
    double s = y[row];
    for (int j = row + 1; j < n; ++j) s = s - a[(size_t)row * n + j] * x[j];
    double pivot = a[(size_t)row * n + row];
    x[row] = pivot == 0.0 ? 0.0 : s / pivot;
  }
}

// DenseLinAlg.lean:242-260 choleskyFactor
void orc_cholesky_factor(int n, const double* A, double* L) {
  for (int i = 0; i < n * n; ++i) L[i] = 0.0;
  for (int j = 0; j < n; ++j) {
    double s = 0.0;
    for (int k = 0; k < j; ++k) { double v = L[(size_t)j * n + k]; s = s + v * v; }
    double diag = std::sqrt(A[(size_t)j * n + j] - s);
    L[(size_t)j * n + j] = diag;
    for (int i = j + 1; i < n; ++i) {
      double t = 0.0;
      for (int k = 0; k < j; ++k) t = t + L[(size_t)i * n + k] * L[(size_t)j * n + k];
      L[(size_t)i * n + j] = (A[(size_t)i * n + j] - t) / diag;
    }
  }
}

// DenseLinAlg.lean:263-290 forwardSolve / backwardSolve / solveWithCholesky
void orc_cholesky_solve(int n, const double* L, const double* b, double* x) {
  std::vector<double> y(n);
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int j = 0; j < i; ++j) s = s + L[(size_t)i * n + j] * y[j];
    y[i] = (b[i] - s) / L[(size_t)i * n + i];
  }
  for (int ii = 0; ii < n; ++ii) {
    int i = n - 1 - ii;
    double s = 0.0;
    for (int j = i + 1; j < n; ++j) s = s + L[(size_t)j * n + i] * x[j];
    x[i] = (y[i] - s) / L[(size_t)i * n + i];
  }
}

// ---------------------------------------------------------------------------
// HarmonicSolve.lean:35-66 solveMulti (literal dense path).  sample_col[v] is
// the C column of vertex v (-1 for mesh vertices); Fc is nc x k.  Xv: nv x k.
void orc_harmonic_solve_multi(int nv, int nf, int nhe, const int* he,
                              const int* sample_col, const double* pos, int nc,
                              const double* Fc, int k, double* Xv) {
  (void)nc;
  std::vector<int> vkind(nv);
  for (int v = 0; v < nv; ++v) vkind[v] = sample_col[v] >= 0 ? 1 : 0;
  std::vector<HE> hes(nhe);
  for (int h = 0; h < nhe; ++h) hes[h] = {he[4 * h], he[4 * h + 1], he[4 * h + 2], he[4 * h + 3]};
  size_t nh = nhe;
  std::vector<double> L(nh * nh, 0.0);
  for (int f = 0; f < nf; ++f) {
    std::vector<int> loop = face_loop(hes, f);
    int n = (int)loop.size();
    if (n < 3) continue;
    std::vector<double> poly(3 * n), Lf(n * n);
    for (int i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) poly[3 * i + d] = pos[3 * hes[loop[i]].target + d];
    polygon_cot_laplacian(0, 0.0, n, poly.data(), Lf.data());
    for (int li = 0; li < n; ++li)
      for (int lj = 0; lj < n; ++lj) {
        size_t gi = loop[li], gj = loop[lj];
        L[gi * nh + gj] = L[gi * nh + gj] + Lf[li * n + lj];
      }
  }
  std::vector<double> lhs((size_t)nv * nv);
  orc_assemble_vtlhv_dense(nv, nf, nhe, he, vkind.data(), pos, 0, 0.0, lhs.data());
  // CFc (nh x k), LhCFc = Lh CFc, VtLhCFc = Vt LhCFc, rhs = -VtLhCFc
  std::vector<double> CF(nh * k, 0.0), LCF(nh * k, 0.0), rhs((size_t)nv * k, 0.0);
  for (size_t h = 0; h < nh; ++h) {
    int c = sample_col[hes[h].target];
    if (c >= 0)
      for (int j = 0; j < k; ++j) CF[h * k + j] = Fc[(size_t)c * k + j];
  }
  for (size_t i = 0; i < nh; ++i)
    for (int j = 0; j < k; ++j) {
      double s = 0.0;
      for (size_t p = 0; p < nh; ++p) s = s + L[i * nh + p] * CF[p * k + j];
      LCF[i * k + j] = s;
    }
  for (int v = 0; v < nv; ++v)
    for (int j = 0; j < k; ++j) {
      double s = 0.0;
      for (size_t p = 0; p < nh; ++p) {
        double vt = (vkind[hes[p].target] == 0 && hes[p].target == v) ? 1.0 : 0.0;
        s = s + vt * LCF[p * k + j];
      }
      rhs[(size_t)v * k + j] = -s;
    }
  orc_dense_solve_multi(nv, k, lhs.data(), rhs.data(), Xv);
}

// DeformSolve.lean:110-135 solveDeformation (Stage 1 k=9, Eq.3 bridge,
// face average :57-70, y_h :75-97, Stage 2 k=3).  Fc: nc x 9, Xc: nc x 3,
// out: nv x 3 (promoted slots 0, as in the spec).
void orc_solve_deformation(int nv, int nf, int nhe, const int* he, const int* sample_col,
                           const double* pos, int nc, const double* Fc, const double* Xc,
                           double* out) {
  std::vector<HE> hes(nhe);
  for (int h = 0; h < nhe; ++h) hes[h] = {he[4 * h], he[4 * h + 1], he[4 * h + 2], he[4 * h + 3]};
  size_t nh = nhe;
  std::vector<double> Fv((size_t)nv * 9);
  orc_harmonic_solve_multi(nv, nf, nhe, he, sample_col, pos, nc, Fc, 9, Fv.data());
  // computeFh (:40-53)
  std::vector<double> Fh(nh * 9, 0.0);
  for (size_t h = 0; h < nh; ++h) {
    int t = hes[h].target;
    if (sample_col[t] < 0)
      for (int j = 0; j < 9; ++j) Fh[h * 9 + j] = Fv[(size_t)t * 9 + j];
    else
      for (int j = 0; j < 9; ++j) Fh[h * 9 + j] = Fc[(size_t)sample_col[t] * 9 + j];
  }
  // averageOverFaces (:57-70)
  std::vector<double> Ff((size_t)nf * 9, 0.0);
  for (int f = 0; f < nf; ++f) {
    std::vector<int> loop = face_loop(hes, f);
    int n = (int)loop.size();
    if (n == 0) continue;
    double invN = 1.0 / (double)n;
    for (int j = 0; j < 9; ++j) {
      double s = 0.0;
      for (int i = 0; i < n; ++i) s = s + Fh[(size_t)loop[i] * 9 + j];
      Ff[(size_t)f * 9 + j] = s * invN;
    }
  }
  // computeYh (:75-97)
  std::vector<double> yh(nh * 3, 0.0);
  for (size_t h = 0; h < nh; ++h) {
    int f = hes[h].face;
    if (f < 0) continue;
    const double* p = pos + 3 * hes[h].target;
    const double* F = Ff.data() + (size_t)f * 9;
    yh[h * 3 + 0] = p[0] * F[0] + p[1] * F[1] + p[2] * F[2];
    yh[h * 3 + 1] = p[0] * F[3] + p[1] * F[4] + p[2] * F[5];
    yh[h * 3 + 2] = p[0] * F[6] + p[1] * F[7] + p[2] * F[8];
  }
  // Stage 2 (:123-135): rhs = -Vt Lh (C Xc - yh)
  std::vector<int> vkind(nv);
  for (int v = 0; v < nv; ++v) vkind[v] = sample_col[v] >= 0 ? 1 : 0;
  std::vector<double> L(nh * nh, 0.0);
  for (int f = 0; f < nf; ++f) {
    std::vector<int> loop = face_loop(hes, f);
    int n = (int)loop.size();
    if (n < 3) continue;
    std::vector<double> poly(3 * n), Lf(n * n);
    for (int i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) poly[3 * i + d] = pos[3 * hes[loop[i]].target + d];
    polygon_cot_laplacian(0, 0.0, n, poly.data(), Lf.data());
    for (int li = 0; li < n; ++li)
      for (int lj = 0; lj < n; ++lj) {
        size_t gi = loop[li], gj = loop[lj];
        L[gi * nh + gj] = L[gi * nh + gj] + Lf[li * n + lj];
      }
  }
  std::vector<double> diff(nh * 3, 0.0);
  for (size_t h = 0; h < nh; ++h) {
    int c = sample_col[hes[h].target];
    for (int j = 0; j < 3; ++j) {
      double cx = c >= 0 ? Xc[(size_t)c * 3 + j] : 0.0;
      diff[h * 3 + j] = cx - yh[h * 3 + j];
    }
  }
  std::vector<double> Ld(nh * 3, 0.0), rhs((size_t)nv * 3, 0.0);
  for (size_t i = 0; i < nh; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (size_t p = 0; p < nh; ++p) s = s + L[i * nh + p] * diff[p * 3 + j];
      Ld[i * 3 + j] = s;
    }
  for (int v = 0; v < nv; ++v)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (size_t p = 0; p < nh; ++p) {
        double vt = (vkind[hes[p].target] == 0 && hes[p].target == v) ? 1.0 : 0.0;
        s = s + vt * Ld[p * 3 + j];
      }
      rhs[(size_t)v * 3 + j] = -s;
    }
  std::vector<double> lhs((size_t)nv * nv);
  orc_assemble_vtlhv_dense(nv, nf, nhe, he, vkind.data(), pos, 0, 0.0, lhs.data());
  orc_dense_solve_multi(nv, 3, lhs.data(), rhs.data(), out);
}

}  // extern "C"
