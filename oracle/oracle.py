"""ctypes wrapper of the CPU FP64 oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY.  The oracle restates the reference's Lean
specification (see the file:line citations in curvenet_oracle*.cpp).  Only
tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference arm
import it; the product never does.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None

_I = C.POINTER(C.c_int32)
_D = C.POINTER(C.c_double)
_P = C.c_void_p


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        sig = {
            "orc_cot_at_vertex": (C.c_double, [_D, _D, _D]),
            "orc_apply_transform4x4": (None, [_D, C.c_double, C.c_double, C.c_double, _D]),
            "orc_lbs_matvec": (None, [_D, C.c_int, _I, _D, C.c_double, C.c_double, C.c_double, _D]),
            "orc_lbs_matvec_csr": (None, [C.c_int, _D, _D, _I, _I, _D, _D]),
            "orc_smooth_weights": (None, [C.c_int, C.c_int, _D, _I, _I, C.c_int, C.c_double, _D]),
            "orc_sparsify_topk": (None, [C.c_int, C.c_int, _D, C.c_int, _I, _D]),
            "orc_triangle_cot_laplacian": (None, [_D, _D, _D, _D]),
            "orc_polygon_cot_laplacian": (None, [C.c_int, _D, _D]),
            "orc_edge_lengths": (None, [_D, _D, _D, _D]),
            "orc_mollify_triangle": (C.c_double, [C.c_double, _D]),
            "orc_cot_from_lengths": (C.c_double, [C.c_double, C.c_double, C.c_double]),
            "orc_robust_triangle_cot_laplacian": (None, [C.c_double, _D, _D, _D, _D]),
            "orc_halfedges_from_triangles": (C.c_int, [C.c_int, C.c_int, _I, _I]),
            "orc_manifold": (C.c_int, [C.c_int, C.c_int, C.c_int, _I]),
            "orc_subdivide_edge": (None, [_I, _I, C.c_int, _I]),
            "orc_split_face": (None, [_I, _I, C.c_int, C.c_int, _I]),
            "orc_insert_crack": (None, [_I, _I, C.c_int, _I]),
            "orc_loop_length": (C.c_int, [C.c_int, _I, C.c_int]),
            "orc_partition_of_unity": (C.c_int, [C.c_int, _I, _I]),
            "orc_cut_mesh": (C.c_int, [C.c_int, C.c_int, _I, C.c_int, _I, _I, _I, _I]),
            "orc_assemble_vtlhv_dense": (None, [C.c_int, C.c_int, C.c_int, _I, _I, _D, C.c_int, C.c_double, _D]),
            "orc_dense_solve": (None, [C.c_int, _D, _D, _D]),
            "orc_dense_solve_multi": (None, [C.c_int, C.c_int, _D, _D, _D]),
            "orc_lu_solve": (None, [C.c_int, _D, _D, _D]),
            "orc_cholesky_factor": (None, [C.c_int, _D, _D]),
            "orc_cholesky_solve": (None, [C.c_int, _D, _D, _D]),
            "orc_harmonic_solve_multi": (None, [C.c_int, C.c_int, C.c_int, _I, _I, _D, C.c_int, _D, C.c_int, _D]),
            "orc_solve_deformation": (None, [C.c_int, C.c_int, C.c_int, _I, _I, _D, C.c_int, _D, _D, _D]),
            "orc_assemble_csr": (C.c_longlong, [C.c_int, C.c_int, _I, _D, C.c_int, C.c_double, _I, _I, _D]),
            "orc_greedy_color": (None, [C.c_int, _I, _I, _I]),
            "orc_ic0_factor": (C.c_int, [C.c_int, _I, _I, _D, _I, _I, _D]),
            "orc_cg_ref": (C.c_int, [C.c_int, _I, _I, _D, _D, _D, C.c_int, C.c_double, _D]),
            "orc_hsc_eliminate": (C.c_int, [C.c_int, _I, _I, _D, C.c_int, _I, _I, _D]),
            "orc_system_create": (_P, [C.c_int, C.c_int, _I, _D, C.c_int, _I, C.c_int, C.c_double, C.c_int, C.c_int]),
            "orc_system_free": (None, [_P]),
            "orc_system_sizes": (None, [_P, C.POINTER(C.c_longlong)]),
            "orc_system_export": (None, [_P, _I, _I, _I, _D, _I, _I, _D]),
            "orc_system_solve": (C.c_int, [_P, C.c_int, _D, C.c_int, C.c_double, C.c_int, C.c_int, _D, _D, _I, _D]),
            "orc_system_rhs": (None, [_P, C.c_int, _D, C.c_int, _D]),
            "orc_bezier3": (None, [_D, C.c_double, _D]),
            "orc_isolated_segment_gradient": (None, [_D, _D, _D, _D, _D]),
            "orc_curve_targets": (None, [C.c_int, C.c_int, _D, _D, _D, C.c_int, _I, _I, _D, _D, _D]),
            "orc_tangent_length": (C.c_double, [_D, _D, _D]),
            "orc_smallest_rotation": (None, [_D, _D, _D]),
            "orc_mat3_mul": (None, [_D, _D, _D]),
            "orc_mat3_det": (C.c_double, [_D]),
            "orc_mat3_inv": (None, [_D, _D]),
            "orc_deformation_gradient": (None, [_D, _D, _D]),
            "orc_corner_normals": (None, [C.c_int, _D, _D, _D]),
            "orc_per_side_widths": (None, [C.c_int, _D, _D, _D, _D]),
            "orc_scaled_frame": (None, [_D, _D, C.c_double, C.c_double, _D]),
            "orc_interp_along_curve": (None, [_D, _D, C.c_int, _D]),
            "orc_curvenet_constraints": (C.c_int, [C.c_int, C.c_int, C.c_int, _D, _D, _I, C.c_int, _I, _I, C.c_int,
                                                   _I, _I, _I, _I, _D, C.c_int, _D, _D, _D]),
            "orc_deform_adjoint": (C.c_double, [_P, C.c_int, _I, _I, _D, C.c_int, _I, C.c_int, C.c_int, _D, _D, _D,
                                                C.c_int, _I, _I, _D, _D, _D, C.c_double, C.c_int, _D, _D, _D]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def ip(a):
    return a.ctypes.data_as(_I)


def dp(a):
    return a.ctypes.data_as(_D)


# --------------------------------------------------------------------- geometry
def triangle_cot_laplacian(a, b, c):
    out = np.empty(9)
    lib().orc_triangle_cot_laplacian(dp(f64(a)), dp(f64(b)), dp(f64(c)), dp(out))
    return out.reshape(3, 3)


def polygon_cot_laplacian(pts):
    pts = f64(pts)
    n = pts.shape[0]
    out = np.empty(n * n)
    lib().orc_polygon_cot_laplacian(n, dp(pts), dp(out))
    return out.reshape(n, n)


def robust_triangle_cot_laplacian(delta, a, b, c):
    out = np.empty(9)
    lib().orc_robust_triangle_cot_laplacian(delta, dp(f64(a)), dp(f64(b)), dp(f64(c)), dp(out))
    return out.reshape(3, 3)


def mollify_triangle(delta, e):
    return lib().orc_mollify_triangle(delta, dp(f64(e)))


def cot_from_lengths(eo, e1, e2):
    return lib().orc_cot_from_lengths(eo, e1, e2)


# --------------------------------------------------------------------- topology
def halfedges_from_triangles(nv, tris):
    tris = i32(tris).reshape(-1, 3)
    out = np.empty((6 * tris.shape[0], 4), np.int32)
    n = lib().orc_halfedges_from_triangles(nv, tris.shape[0], ip(tris), ip(out))
    return out[:n].copy()


def manifold(nv, nf, he):
    he = i32(he)
    return bool(lib().orc_manifold(nv, nf, he.shape[0], ip(he)))


def _surgery(fn, counts, he, *args):
    counts = i32(counts).copy()
    he = i32(he)
    out = np.empty((he.shape[0] + 2, 4), np.int32)
    fn(ip(counts), ip(he), *args, ip(out))
    return counts, out


def subdivide_edge(counts, he, h):
    return _surgery(lib().orc_subdivide_edge, counts, he, h)


def split_face(counts, he, a, b):
    return _surgery(lib().orc_split_face, counts, he, a, b)


def insert_crack(counts, he, h):
    return _surgery(lib().orc_insert_crack, counts, he, h)


def loop_length(he, h):
    he = i32(he)
    return lib().orc_loop_length(he.shape[0], ip(he), h)


def partition_of_unity(he, vkind):
    he = i32(he)
    return bool(lib().orc_partition_of_unity(he.shape[0], ip(he), ip(i32(vkind))))


def cut_mesh(nv, tris, loops):
    tris = i32(tris).reshape(-1, 3)
    ptr = np.zeros(len(loops) + 1, np.int32)
    for i, l in enumerate(loops):
        ptr[i + 1] = ptr[i] + len(l)
    verts = i32(np.concatenate(loops)) if loops else np.zeros(0, np.int32)
    out = np.empty_like(tris)
    parent = np.empty(nv + verts.size, np.int32)
    r = lib().orc_cut_mesh(nv, tris.shape[0], ip(tris), len(loops), ip(ptr), ip(verts), ip(out), ip(parent))
    if r < 0:
        raise ValueError(f"orc_cut_mesh failed ({r})")
    return out, parent[:r]


# --------------------------------------------------------------------- assembly
def assemble_vtlhv_dense(nv, nf, he, vkind, pos, kind=0, delta=0.0):
    he = i32(he)
    out = np.empty(nv * nv)
    lib().orc_assemble_vtlhv_dense(nv, nf, he.shape[0], ip(he), ip(i32(vkind)), dp(f64(pos)), kind, delta, dp(out))
    return out.reshape(nv, nv)


def assemble_csr(nv, tris, pos, kind=0, delta=0.0):
    tris = i32(tris).reshape(-1, 3)
    pos = f64(pos)
    nnz = lib().orc_assemble_csr(nv, tris.shape[0], ip(tris), dp(pos), kind, delta, None, None, None)
    ptr = np.empty(nv + 1, np.int32)
    col = np.empty(nnz, np.int32)
    val = np.empty(nnz)
    lib().orc_assemble_csr(nv, tris.shape[0], ip(tris), dp(pos), kind, delta, ip(ptr), ip(col), dp(val))
    return ptr, col, val


# --------------------------------------------------------------------- dense LA
def dense_solve(A, b):
    A = f64(A)
    n = A.shape[0]
    x = np.empty(n)
    lib().orc_dense_solve(n, dp(A), dp(f64(b)), dp(x))
    return x


def lu_solve(A, b):
    A = f64(A)
    n = A.shape[0]
    x = np.empty(n)
    lib().orc_lu_solve(n, dp(A), dp(f64(b)), dp(x))
    return x


def cholesky_factor(A):
    A = f64(A)
    n = A.shape[0]
    Lm = np.empty(n * n)
    lib().orc_cholesky_factor(n, dp(A), dp(Lm))
    return Lm.reshape(n, n)


def cholesky_solve(Lm, b):
    Lm = f64(Lm)
    n = Lm.shape[0]
    x = np.empty(n)
    lib().orc_cholesky_solve(n, dp(Lm), dp(f64(b)), dp(x))
    return x


def harmonic_solve_multi(nv, nf, he, sample_col, pos, Fc, k):
    he = i32(he)
    Fc = f64(Fc)
    out = np.empty(nv * k)
    lib().orc_harmonic_solve_multi(nv, nf, he.shape[0], ip(he), ip(i32(sample_col)), dp(f64(pos)),
                                   Fc.size // k, dp(Fc), k, dp(out))
    return out.reshape(nv, k)


def solve_deformation(nv, nf, he, sample_col, pos, Fc, Xc):
    he = i32(he)
    Fc = f64(Fc)
    out = np.empty(nv * 3)
    lib().orc_solve_deformation(nv, nf, he.shape[0], ip(he), ip(i32(sample_col)), dp(f64(pos)),
                                Fc.size // 9, dp(Fc), dp(f64(Xc)), dp(out))
    return out.reshape(nv, 3)


# --------------------------------------------------------------------- sparse
def greedy_color(adj):
    n = len(adj)
    ptr = np.zeros(n + 1, np.int32)
    for i, a in enumerate(adj):
        ptr[i + 1] = ptr[i] + len(a)
    col = i32(np.concatenate([np.asarray(a, np.int32) for a in adj]) if n else [])
    out = np.empty(n, np.int32)
    lib().orc_greedy_color(n, ip(ptr), ip(col), ip(out))
    return out


def ic0_factor(ptr, col, val):
    ptr, col, val = i32(ptr), i32(col), f64(val)
    n = ptr.size - 1
    Lp = np.empty(n + 1, np.int32)
    st = lib().orc_ic0_factor(n, ip(ptr), ip(col), dp(val), ip(Lp), None, None)
    Lc = np.empty(Lp[-1], np.int32)
    Lv = np.empty(Lp[-1])
    st = lib().orc_ic0_factor(n, ip(ptr), ip(col), dp(val), ip(Lp), ip(Lc), dp(Lv))
    return st, Lp, Lc, Lv


def cg_ref(ptr, col, val, b, max_iter, tol, x0=None):
    ptr, col, val, b = i32(ptr), i32(col), f64(val), f64(b)
    n = ptr.size - 1
    x = np.empty(n)
    it = lib().orc_cg_ref(n, ip(ptr), ip(col), dp(val), dp(b), dp(f64(x0)) if x0 is not None else None,
                          max_iter, tol, dp(x))
    return x, it


def hsc_eliminate(edges, v):
    eu = i32([e[0] for e in edges])
    ev = i32([e[1] for e in edges])
    ew = f64([e[2] for e in edges])
    deg = sum(1 for e in edges if v in (e[0], e[1]))
    cap = len(edges) + deg * deg + 1
    ou, ov, ow = np.empty(cap, np.int32), np.empty(cap, np.int32), np.empty(cap)
    m = lib().orc_hsc_eliminate(len(edges), ip(eu), ip(ev), dp(ew), v, ip(ou), ip(ov), dp(ow))
    return [(int(ou[i]), int(ov[i]), float(ow[i])) for i in range(m)]


class System:
    """Oracle system of one cut mesh: K, the reduced A in solve order, IC(0)."""

    def __init__(self, positions, tris, handles, kind=0, delta=0.0, ordering=1, precond=1):
        self.positions = f64(positions).reshape(-1, 3)
        self.tris = i32(tris).reshape(-1, 3)
        self.handles = i32(handles)
        self.nv = self.positions.shape[0]
        self._h = lib().orc_system_create(self.nv, self.tris.shape[0], ip(self.tris), dp(self.positions),
                                          self.handles.size, ip(self.handles), kind, delta, ordering, precond)
        s = (C.c_longlong * 7)()
        lib().orc_system_sizes(self._h, s)
        self.status, self.n, self.nnz_A, self.nnz_L, self.n_levels, self.nnz_K = [int(v) for v in s[:6]]
        self.shift = s[6] * 1e-6

    def close(self):
        if self._h:
            lib().orc_system_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def export(self):
        free_of = np.empty(self.n, np.int32)
        Ap = np.empty(self.n + 1, np.int32)
        Ac = np.empty(max(self.nnz_A, 1), np.int32)
        Av = np.empty(max(self.nnz_A, 1))
        Lp = np.empty(self.n + 1, np.int32)
        Lc = np.empty(max(self.nnz_L, 1), np.int32)
        Lv = np.empty(max(self.nnz_L, 1))
        lib().orc_system_export(self._h, ip(free_of), ip(Ap), ip(Ac), dp(Av), ip(Lp), ip(Lc), dp(Lv))
        return dict(free_of=free_of, A=(Ap, Ac[: self.nnz_A], Av[: self.nnz_A]),
                    L=(Lp, Lc[: self.nnz_L], Lv[: self.nnz_L]))

    def rhs(self, targets, mode=1):
        t = f64(targets)
        k = t.shape[1]
        b = np.empty((self.n, k))
        lib().orc_system_rhs(self._h, k, dp(t), mode, dp(b))
        return b

    def solve(self, targets, mode=1, tol=1e-10, max_iter=100000, threads=1, x0=None):
        t = f64(targets)
        t = t.reshape(t.shape[0], -1)
        k = t.shape[1]
        x = np.empty((self.nv, k))
        it = np.zeros(k, np.int32)
        rel = np.zeros(k)
        st = lib().orc_system_solve(self._h, k, dp(t), mode, tol, max_iter, threads,
                                    dp(f64(x0)) if x0 is not None else None, dp(x), ip(it), dp(rel))
        return st, x, it, rel


# --------------------------------------------------------------------- curvenet (DeGoes22 section 3)
def tangent_length(p, q):
    t = np.empty(3)
    l = lib().orc_tangent_length(dp(f64(p)), dp(f64(q)), dp(t))
    return t, l


def smallest_rotation(a, b):
    R = np.empty(9)
    lib().orc_smallest_rotation(dp(f64(a)), dp(f64(b)), dp(R))
    return R.reshape(3, 3)


def isolated_segment_gradient(rp, rq, pp, pq):
    F = np.empty(9)
    lib().orc_isolated_segment_gradient(dp(f64(rp)), dp(f64(rq)), dp(f64(pp)), dp(f64(pq)), dp(F))
    return F.reshape(3, 3)


def mat3_mul(a, b):
    o = np.empty(9)
    lib().orc_mat3_mul(dp(f64(a).ravel()), dp(f64(b).ravel()), dp(o))
    return o.reshape(3, 3)


def mat3_det(m):
    return lib().orc_mat3_det(dp(f64(m).ravel()))


def mat3_inv(m):
    o = np.empty(9)
    lib().orc_mat3_inv(dp(f64(m).ravel()), dp(o))
    return o.reshape(3, 3)


def deformation_gradient(rest, posed):
    o = np.empty(9)
    lib().orc_deformation_gradient(dp(f64(rest).ravel()), dp(f64(posed).ravel()), dp(o))
    return o.reshape(3, 3)


def corner_normals(tangents):
    t = f64(tangents).reshape(-1, 3)
    cv, m = np.empty_like(t), np.empty_like(t)
    lib().orc_corner_normals(t.shape[0], dp(t), dp(cv), dp(m))
    return cv, m


def per_side_widths(tangents, lengths):
    t = f64(tangents).reshape(-1, 3)
    wp, wm = np.empty(t.shape[0]), np.empty(t.shape[0])
    lib().orc_per_side_widths(t.shape[0], dp(t), dp(f64(lengths)), dp(wp), dp(wm))
    return wp, wm


def scaled_frame(t, n, l, w):
    o = np.empty(9)
    lib().orc_scaled_frame(dp(f64(t)), dp(f64(n)), l, w, dp(o))
    return o.reshape(3, 3)


def interp_along_curve(first, last, n):
    """first / last: 8 doubles (plus n, plus w, minus n, minus w); (n, 8)."""
    out = np.empty((max(n, 1), 8))
    lib().orc_interp_along_curve(dp(f64(first)), dp(f64(last)), n, dp(out))
    return out[:n]


def curvenet_constraints(net, rest_positions, handles, posed_cp):
    """F_c (poses, nh, 3, 3) and X_c (poses, nh, 3) of a curvenet dict with the
    fields of cn_curvenet_desc (rest_cp, sample_tau, closed, node_ptr,
    node_ends, handle_curve, handle_sample, handle_side)."""
    rest_cp = f64(net["rest_cp"])
    C, npts, _ = rest_cp.shape
    S = (npts - 1) // 3
    tau = f64(net["sample_tau"])
    M = tau.shape[1]
    closed = i32(net.get("closed", np.zeros(C)))
    node_ptr = i32(net.get("node_ptr", [0]))
    node_ends = i32(net.get("node_ends", [0]) if len(net.get("node_ends", [])) else [0])
    hc, hs, hd = i32(net["handle_curve"]), i32(net["handle_sample"]), i32(net["handle_side"])
    P = f64(posed_cp).reshape(-1, C, npts, 3)
    nh = hc.size
    F = np.empty((P.shape[0], nh, 9))
    X = np.empty((P.shape[0], nh, 3))
    r = lib().orc_curvenet_constraints(C, S, M, dp(rest_cp), dp(tau), ip(closed), node_ptr.size - 1, ip(node_ptr),
                                       ip(node_ends), nh, ip(hc), ip(hs), ip(hd), ip(i32(handles)),
                                       dp(f64(rest_positions)), P.shape[0], dp(P), dp(F), dp(X))
    if r != 0:
        raise ValueError("malformed curvenet")
    return F.reshape(P.shape[0], nh, 3, 3), X


# --------------------------------------------------------------------- Direct Delta Mush
def lbs_matvec(transforms, infl, rest):
    """DirectDeltaMush.lean:84-102 for one vertex; infl = [(handle, w), ...]."""
    T = f64(transforms).reshape(-1, 16)
    idx = i32([i for i, _ in infl]) if infl else np.zeros(1, np.int32)
    w = f64([x for _, x in infl]) if infl else np.zeros(1)
    out = np.empty(3)
    lib().orc_lbs_matvec(dp(T), len(infl), ip(idx), dp(w), float(rest[0]), float(rest[1]), float(rest[2]), dp(out))
    return out


def lbs_matvec_csr(rest, transforms, start, idx, w):
    rest = f64(rest).reshape(-1, 3)
    out = np.empty_like(rest)
    lib().orc_lbs_matvec_csr(rest.shape[0], dp(rest), dp(f64(transforms).reshape(-1, 16)), ip(i32(start)),
                             ip(i32(idx)), dp(f64(w)), dp(out))
    return out


def smooth_weights(W, adj, nu, omega):
    """DirectDeltaMushBind.lean:72-94; adj = list of neighbour lists."""
    W = f64(W)
    n, nh = W.shape
    ptr = np.zeros(n + 1, np.int32)
    for v, nb in enumerate(adj):
        ptr[v + 1] = ptr[v] + len(nb)
    idx = i32([u for nb in adj for u in nb]) if ptr[-1] else np.zeros(1, np.int32)
    out = np.empty_like(W)
    lib().orc_smooth_weights(n, nh, dp(W), ip(ptr), ip(idx), nu, omega, dp(out))
    return out


def sparsify_topk(W, K):
    """DirectDeltaMushBind.lean:104-133: (idx, w) arrays of n x min(K, nh)."""
    W = f64(W)
    n, nh = W.shape
    take = min(K, nh)
    idx = np.empty((n, max(take, 1)), np.int32)
    w = np.empty((n, max(take, 1)))
    lib().orc_sparsify_topk(n, nh, dp(W), K, ip(idx), dp(w))
    return idx[:, :take], w[:, :take]
