// cn_curvenet.cu -- the curve side of the deformer on the GPU: per pose, the
// constraint deformation gradients F_c and targets X_c of the handles from
// the posed profile curves (DeGoes22 section 3 as the reference specifies it):
//
//   * samples of each composite cubic Bezier at fixed parameters
//     (EndToEndExample.lean:52-60 bezier3 per segment), a polyline of
//     segments between consecutive samples (a closed curve's last segment
//     joins its last sample to its first);
//   * per segment the tangent and length, rest and posed
//     (ScaledFrames.lean:40-45 tangentLength);
//   * isolated curves (closed, or no intersection at either end): both sides
//     get F = (l / l_rest) R(t_rest, t) (ScaledFrames.lean:71-98
//     smallestRotation / isolatedSegmentGradient; SegmentGradient.lean:40-47);
//   * curves that end at intersections: at every intersection the outgoing
//     segments in counter-clockwise order give corner vectors, corner normals
//     (with the T-junction fallback) and per-side widths
//     (IntersectionFrames.lean:65-143), rest and posed; the per-side data of a
//     curve's end segments are interpolated linearly along the curve
//     (CurveInterp.lean:45-60 interpAlongCurve), each segment side gets the
//     scaled frame B S = [t l | (n x t) w | n sqrt(l w)]
//     (IntersectionFrames.lean:160-170 scaledFrame), and
//     F^+- = (B S)_posed (B S)_rest^-1 (ScaledFrames.lean:120-170
//     mat3Inv / deformationGradient; SegmentGradient.lean:49-58
//     intersectionPair);
//   * a handle bound to (curve, sample, side) takes F of the segment that
//     starts at the sample (the last segment for an open curve's last
//     sample) on its side, and X_c = the posed sample point
//     (EndToEndExample.lean:140-142).
//
// The rules that join these pieces (outgoing segment of a curve end, the
// side swap at a curve's far end, constant extension when only one end is at
// an intersection, the segment a handle takes) are this library's own: the
// reference states the pieces, not the assembly.  The file is compiled
// without FMA contraction and every expression keeps the reference's order,
// so the results equal the FP64 oracle's bit for bit.
#include "cn_internal.h"

namespace cn {
namespace {

struct V3 {
  double x, y, z;
};

__device__ __forceinline__ V3 ld3(const double* p) { return V3{p[0], p[1], p[2]}; }

__device__ __forceinline__ V3 cross3(V3 a, V3 b) {
  return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

__device__ __forceinline__ double norm3(V3 v) { return sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }

// EndToEndExample.lean:52-60 on segment s of a composite curve at tau
// (s = min(floor(tau), S - 1), t = tau - s).
__device__ V3 eval_curve(const double* P, int S, double tau) {
  int s = (int)floor(tau);
  if (s > S - 1) s = S - 1;
  if (s < 0) s = 0;
  const double t = tau - (double)s;
  const double* q = P + 9 * s;
  const double u = 1.0 - t;
  const double c0 = u * u * u;
  const double c1 = 3.0 * u * u * t;
  const double c2 = 3.0 * u * t * t;
  const double c3 = t * t * t;
  return V3{c0 * q[0] + c1 * q[3] + c2 * q[6] + c3 * q[9], c0 * q[1] + c1 * q[4] + c2 * q[7] + c3 * q[10],
            c0 * q[2] + c1 * q[5] + c2 * q[8] + c3 * q[11]};
}

// ScaledFrames.lean:40-45
__device__ double tangent_length(V3 p, V3 q, V3* t) {
  const V3 d{q.x - p.x, q.y - p.y, q.z - p.z};
  const double l = sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
  const double inv = l == 0.0 ? 0.0 : 1.0 / l;
  *t = V3{d.x * inv, d.y * inv, d.z * inv};
  return l;
}

// ScaledFrames.lean:71-98: r R(from, to), R = (I + K) + K^2 / (1 + cos)
__device__ void isolated_gradient(V3 f, double lf, V3 to, double lt, double* F) {
  const double r = lf == 0.0 ? 0.0 : lt / lf;
  const double cx = f.y * to.z - f.z * to.y;
  const double cy = f.z * to.x - f.x * to.z;
  const double cz = f.x * to.y - f.y * to.x;
  const double cosT = f.x * to.x + f.y * to.y + f.z * to.z;
  const double K[9] = {0.0, -cz, cy, cz, 0.0, -cx, -cy, cx, 0.0};
  const double denom = 1.0 + cosT;
  const double invd = denom == 0.0 ? 0.0 : 1.0 / denom;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double k2 = K[i * 3 + 0] * K[0 * 3 + j] + K[i * 3 + 1] * K[1 * 3 + j] + K[i * 3 + 2] * K[2 * 3 + j];
      const double id = i == j ? 1.0 : 0.0;
      F[i * 3 + j] = r * ((id + K[i * 3 + j]) + invd * k2);
    }
}

// IntersectionFrames.lean:160-170
__device__ void scaled_frame(V3 t, V3 n, double l, double w, double* M) {
  const double bx = n.y * t.z - n.z * t.y;
  const double by = n.z * t.x - n.x * t.z;
  const double bz = n.x * t.y - n.y * t.x;
  const double h = sqrt(l * w);
  M[0] = t.x * l; M[1] = bx * w; M[2] = n.x * h;
  M[3] = t.y * l; M[4] = by * w; M[5] = n.y * h;
  M[6] = t.z * l; M[7] = bz * w; M[8] = n.z * h;
}

// ScaledFrames.lean:139-160 mat3Inv (adjugate; a singular input gives 0)
__device__ void mat3_inv(const double* m, double* o) {
  const double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
  const double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
  const double inv = det == 0.0 ? 0.0 : 1.0 / det;
  o[0] = inv * (e * i - f * h); o[1] = inv * (c * h - b * i); o[2] = inv * (b * f - c * e);
  o[3] = inv * (f * g - d * i); o[4] = inv * (a * i - c * g); o[5] = inv * (c * d - a * f);
  o[6] = inv * (d * h - e * g); o[7] = inv * (b * g - a * h); o[8] = inv * (a * e - b * d);
}

// ScaledFrames.lean:59-65 mat3Mul
__device__ void mat3_mul(const double* a, const double* b, double* o) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) o[i * 3 + j] = a[i * 3 + 0] * b[0 * 3 + j] + a[i * 3 + 1] * b[1 * 3 + j] +
                                               a[i * 3 + 2] * b[2 * 3 + j];
}

// Segment records: per pose and global segment, rest tangent + length and
// posed tangent + length (8 doubles).
__global__ void k_cnet_segments(CurvenetArgs a, int n_poses, const double* posed_cp) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n_poses * a.total_segs) return;
  const int pose = (int)(idx / a.total_segs);
  const int g = (int)(idx % a.total_segs);
  // curve of global segment g: the last c with seg_off[c] <= g
  int lo = 0, hi = a.n_curves - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a.seg_off[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  const int c = lo;
  const int i = g - a.seg_off[c];
  const int M = a.n_samples;
  const int j = i + 1 < M ? i + 1 : 0;  // a closed curve's last segment returns to sample 0
  const size_t np = 3 * (size_t)a.n_segments + 1;
  const double* R = a.rest_cp + (size_t)c * np * 3;
  const double* P = posed_cp + ((size_t)pose * a.n_curves + c) * np * 3;
  const double ti = a.sample_tau[(size_t)c * M + i], tj = a.sample_tau[(size_t)c * M + j];
  V3 tr, tp;
  const double lr = tangent_length(eval_curve(R, a.n_segments, ti), eval_curve(R, a.n_segments, tj), &tr);
  const double lp = tangent_length(eval_curve(P, a.n_segments, ti), eval_curve(P, a.n_segments, tj), &tp);
  double* o = a.seg + ((size_t)pose * a.total_segs + g) * 8;
  o[0] = tr.x; o[1] = tr.y; o[2] = tr.z; o[3] = lr;
  o[4] = tp.x; o[5] = tp.y; o[6] = tp.z; o[7] = lp;
}

// One thread per (pose, intersection): the outgoing segments of its curve
// ends (a start leaves along segment 0, an end along the reversed last
// segment), corner vectors and normals (IntersectionFrames.lean:65-110),
// per-side widths (:120-143), rest (cfg 0) and posed (cfg 1).  Writes each
// curve end's per-side data in the curve's own direction: at a start,
// plus = (m_i, w_i^+), minus = (m_{i-1}, w_i^-); at an end the two sides swap.
__global__ void k_cnet_nodes(CurvenetArgs a, int n_poses) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_poses * a.n_nodes) return;
  const int pose = idx / a.n_nodes;
  const int node = idx % a.n_nodes;
  const int b = a.node_ptr[node];
  const int n = a.node_ptr[node + 1] - b;
  const double eps = 1.0e-12;
  for (int cfg = 0; cfg < 2; ++cfg) {
    V3 t[kCnetMaxNodeDegree], cv[kCnetMaxNodeDegree];
    double l[kCnetMaxNodeDegree];
    for (int q = 0; q < n; ++q) {
      const int e = a.node_ends[b + q];
      const int c = e >> 1;
      const int seg = (e & 1) ? a.seg_off[c + 1] - 1 : a.seg_off[c];
      const double* s = a.seg + ((size_t)pose * a.total_segs + seg) * 8 + 4 * cfg;
      t[q] = (e & 1) ? V3{-s[0], -s[1], -s[2]} : V3{s[0], s[1], s[2]};
      l[q] = s[3];
    }
    for (int q = 0; q < n; ++q) cv[q] = cross3(t[q], t[(q + 1) % n]);
    V3 m[kCnetMaxNodeDegree];
    for (int q = 0; q < n; ++q) {
      const V3 cc = cv[q];
      const double nrm = norm3(cc);
      if (nrm > eps) {
        const double s = 1.0 / nrm;
        m[q] = V3{s * cc.x, s * cc.y, s * cc.z};
      } else {
        const V3 cP = cv[(q + 1) % n], cM = cv[(q + n - 1) % n];
        const V3 sum{cP.x + cM.x, cP.y + cM.y, cP.z + cM.z};
        const double sn = norm3(sum);
        if (sn > eps) {
          const double s = 1.0 / sn;
          m[q] = V3{s * sum.x, s * sum.y, s * sum.z};
        } else {
          m[q] = V3{0.0, 0.0, 0.0};
        }
      }
    }
    for (int q = 0; q < n; ++q) {
      const double li = l[q], liP = l[(q + 1) % n], liM = l[(q + n - 1) % n];
      const double cMag = norm3(cv[q]), cMagM = norm3(cv[(q + n - 1) % n]);
      const double wP = li + cMag * (liP - li);
      const double wM = li + cMagM * (liM - li);
      const V3 nP = m[q], nM = m[(q + n - 1) % n];
      const int e = a.node_ends[b + q];
      // record: [cfg][plus n, plus w, minus n, minus w] in the curve's direction
      double* o = a.ends + (((size_t)pose * a.n_curves + (e >> 1)) * 2 + (e & 1)) * 16 + 8 * cfg;
      const bool swap = (e & 1) != 0;
      const V3 np_ = swap ? nM : nP, nm_ = swap ? nP : nM;
      o[0] = np_.x; o[1] = np_.y; o[2] = np_.z; o[3] = swap ? wM : wP;
      o[4] = nm_.x; o[5] = nm_.y; o[6] = nm_.z; o[7] = swap ? wP : wM;
    }
  }
}

// One thread per (pose, handle): F_c (9, row-major) and X_c (3).
__global__ void k_cnet_handles(CurvenetArgs a, int n_poses, const double* posed_cp, double* Fc, double* Xc) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_poses * a.nh) return;
  const int pose = idx / a.nh;
  const int h = idx % a.nh;
  double* F = Fc + (size_t)idx * 9;
  double* X = Xc + (size_t)idx * 3;
  const int c = a.h_curve[h];
  if (c < 0) {
    for (int k = 0; k < 9; ++k) F[k] = (k % 4 == 0) ? 1.0 : 0.0;
    const double* p = a.pos + 3 * (size_t)a.handles[h];
    X[0] = p[0]; X[1] = p[1]; X[2] = p[2];
    return;
  }
  const int i = a.h_sample[h];
  const int side = a.h_side[h];
  const int nseg = a.seg_off[c + 1] - a.seg_off[c];
  const int si = i < nseg ? i : nseg - 1;
  const double* s = a.seg + ((size_t)pose * a.total_segs + a.seg_off[c] + si) * 8;
  const int kind = a.curve_kind[c];  // 0 isolated; 1 start node only; 2 end node only; 3 both
  if (kind == 0) {
    isolated_gradient(ld3(s), s[3], ld3(s + 4), s[7], F);
  } else {
    const double* E = a.ends + ((size_t)pose * a.n_curves + c) * 2 * 16;
    const double* first = (kind & 1) ? E : E + 16;
    const double* last = (kind & 2) ? E + 16 : E;
    double fr[2][9];
    for (int cfg = 0; cfg < 2; ++cfg) {
      const double* f = first + 8 * cfg + 4 * side;
      const double* g = last + 8 * cfg + 4 * side;
      V3 nn;
      double ww;
      if (nseg == 1) {  // CurveInterp.lean:49: one segment keeps `first`
        nn = ld3(f);
        ww = f[3];
      } else {
        const double tt = (double)si / (double)(nseg - 1);
        nn = V3{(1.0 - tt) * f[0] + tt * g[0], (1.0 - tt) * f[1] + tt * g[1], (1.0 - tt) * f[2] + tt * g[2]};
        ww = (1.0 - tt) * f[3] + tt * g[3];
      }
      scaled_frame(ld3(s + 4 * cfg), nn, s[4 * cfg + 3], ww, fr[cfg]);
    }
    double inv[9];
    mat3_inv(fr[0], inv);
    mat3_mul(fr[1], inv, F);
  }
  const int M = a.n_samples;
  const size_t np = 3 * (size_t)a.n_segments + 1;
  const V3 x = eval_curve(posed_cp + ((size_t)pose * a.n_curves + c) * np * 3, a.n_segments,
                          a.sample_tau[(size_t)c * M + i]);
  X[0] = x.x; X[1] = x.y; X[2] = x.z;
}

// x[handles[h]] = X_c(h) (DeformSolve.lean:108-109 overlay), n_verts x 3.
__global__ void k_cnet_overlay(int nh, const int* handles, const double* Xc, double* x) {
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= nh) return;
  for (int d = 0; d < 3; ++d) x[3 * (size_t)handles[h] + d] = Xc[3 * (size_t)h + d];
}

}  // namespace

cudaError_t launch_curvenet_constraints(const CurvenetArgs& a, int n_poses, const double* posed_cp, double* Fc,
                                        double* Xc, cudaStream_t s) {
  const long long nseg = (long long)n_poses * a.total_segs;
  if (nseg > 0) k_cnet_segments<<<(unsigned)((nseg + 127) / 128), 128, 0, s>>>(a, n_poses, posed_cp);
  const int nn = n_poses * a.n_nodes;
  if (nn > 0) k_cnet_nodes<<<(nn + 63) / 64, 64, 0, s>>>(a, n_poses);
  const int nh = n_poses * a.nh;
  if (nh > 0) k_cnet_handles<<<(nh + 127) / 128, 128, 0, s>>>(a, n_poses, posed_cp, Fc, Xc);
  return cudaGetLastError();
}

cudaError_t launch_curvenet_overlay(int nh, const int* handles, const double* Xc, double* x, cudaStream_t s) {
  if (nh > 0) k_cnet_overlay<<<(nh + 127) / 128, 128, 0, s>>>(nh, handles, Xc, x);
  return cudaGetLastError();
}

}  // namespace cn
