"""Host-side mirror of the reference runtime's build / solve / deform entry
points for the sparse solve, over the C ABI (include/curvenet_b200.h).

Names follow the reference: `cut_mesh` is the seam cut of CutAlgorithm.lean /
CutMesh.lean, `CutMeshSolver` holds the assembled V^T L_h V
(CutMeshLaplacian.lean:86-93) with its factor, `solve_multi` is
HarmonicSolve.lean:51-66 and `solve_deformation` is the Stage-2 solve of
DeformSolve.lean:110-135 with F_f = I.  Failures raise CnError carrying the
status code (the reference's silent "degenerate -> 0" results are reported as
statuses instead).
"""
import ctypes as C

import numpy as np

from . import _lib as L


class CnError(RuntimeError):
    def __init__(self, status, where):
        self.status = int(status)
        super().__init__(f"{where}: {L.status_string(status)} ({self.status}): {L.last_error()}")


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


_PRECOND = {"jacobi": L.PRECOND_JACOBI, "ic0": L.PRECOND_IC0, "hsc": L.PRECOND_HSC, "bssor": L.PRECOND_BSSOR}
_ORDER = {"natural": L.ORDER_NATURAL, "color": L.ORDER_COLOR, "auto": L.ORDER_AUTO}
_LAP = {"cot": L.LAPLACIAN_COT, "robust": L.LAPLACIAN_ROBUST}
_PREC = {"fp64": L.PREC_FP64, "mixed": L.PREC_MIXED}
_MODE = {"harmonic": L.MODE_HARMONIC, "deform": L.MODE_DEFORM, "rhs": L.MODE_RHS}
_ALGO = {"fused": L.ALGO_FUSED, "plain": L.ALGO_PLAIN, "classic": L.ALGO_CLASSIC,
         "pipelined": L.ALGO_PIPELINED, "single": L.ALGO_SINGLE}


def cut_mesh(n_verts, tris, loops):
    """Duplicate the vertices of each closed loop; faces on the loop's left move
    to the copies.  Returns (tris_cut, parent) with parent[v] the uncut vertex."""
    tris = _i32(tris).reshape(-1, 3)
    ptr = np.zeros(len(loops) + 1, np.int32)
    for i, l in enumerate(loops):
        ptr[i + 1] = ptr[i] + len(l)
    verts = _i32(np.concatenate(loops)) if loops else np.zeros(0, np.int32)
    out = np.empty_like(tris)
    parent = np.empty(n_verts + verts.size, np.int32)
    nv_out = C.c_int32(0)
    st = L.lib().cn_cut_mesh(n_verts, tris.shape[0], _ip(tris), len(loops), _ip(ptr), _ip(verts),
                             _ip(out), _ip(parent), C.byref(nv_out))
    if st != L.CN_OK:
        raise CnError(st, "cn_cut_mesh")
    return out, parent[: nv_out.value]


class SolveResult:
    def __init__(self, x, stats):
        self.x = x
        self.status = stats.status
        self.iterations = stats.iterations
        self.refinements = stats.refinements
        self.rel_residual = np.array(stats.rel_residual[: max(1, min(stats.k, 32))])
        self.device_ms = stats.device_ms


class CutMeshSolver:
    """Assembled and factored system of one cut mesh on one GPU."""

    def __init__(self, positions, tris, handles, precond="ic0", ordering="auto",
                 laplacian="cot", mollify_delta=1e-4, max_rhs=3, device=0, lanes=0,
                 block=0, grid=0, hsc_tail_rows=0, hsc_theta=0.0):
        self.positions = _f64(positions).reshape(-1, 3)
        self.tris = _i32(tris).reshape(-1, 3)
        self.handles = _i32(handles).reshape(-1)
        self.n_verts = self.positions.shape[0]
        desc = L.MeshDesc(self.n_verts, self.tris.shape[0], _dp(self.positions), _ip(self.tris),
                          self.handles.size, _ip(self.handles))
        opts = L.BuildOpts()
        L.lib().cn_default_build_opts(C.byref(opts))
        opts.precond = _PRECOND[precond]
        opts.ordering = _ORDER[ordering]
        opts.laplacian = _LAP[laplacian]
        opts.mollify_delta = mollify_delta
        opts.max_rhs = max_rhs
        opts.device = device
        opts.lanes, opts.block, opts.grid = lanes, block, grid
        opts.hsc_tail_rows, opts.hsc_theta = hsc_tail_rows, hsc_theta
        h = C.c_void_p()
        st = L.lib().cn_build(C.byref(desc), C.byref(opts), C.byref(h))
        if st != L.CN_OK:
            raise CnError(st, "cn_build")
        self._h = h
        self.max_rhs = max_rhs

    # -- lifetime
    def close(self):
        if getattr(self, "_h", None):
            L.lib().cn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- introspection
    def info(self):
        v = (C.c_int64 * 12)()
        L.lib().cn_system_info(self._h, v)
        keys = ["n_free", "nnz_A", "nnz_L", "n_levels", "nnz_K", "n_verts", "n_handles", "grid",
                "block", "lanes", "n_colors", "device_bytes"]
        return dict(zip(keys, list(v)))

    def stream(self):
        return L.lib().cn_stream(self._h)

    def hsc_info(self):
        """(n_levels, tail, n_coarse, level_off, order) of an HSC handle."""
        i = self.info()
        nl, tail, nc = C.c_int32(), C.c_int32(), C.c_int32()
        off = np.zeros(65, np.int32)
        order = np.zeros(i["n_free"], np.int32)
        st = L.lib().cn_hsc_info(self._h, C.byref(nl), C.byref(tail), C.byref(nc), _ip(off), _ip(order))
        if st != L.CN_OK:
            raise CnError(st, "cn_hsc_info")
        return nl.value, tail.value, nc.value, off[: nl.value + 1].copy(), order

    def export_csr(self):
        i = self.info()
        n, nnz = i["n_free"], i["nnz_A"]
        free_of = np.empty(n, np.int32)
        ptr = np.empty(n + 1, np.int32)
        col = np.empty(max(nnz, 1), np.int32)
        val = np.empty(max(nnz, 1), np.float64)
        st = L.lib().cn_export_csr(self._h, _ip(free_of), _ip(ptr), _ip(col), _dp(val))
        if st != L.CN_OK:
            raise CnError(st, "cn_export_csr")
        return free_of, ptr, col[:nnz], val[:nnz]

    def export_factor(self):
        i = self.info()
        n, nnz = i["n_free"], i["nnz_L"] + i["n_free"]
        ptr = np.empty(n + 1, np.int32)
        col = np.empty(max(nnz, 1), np.int32)
        val = np.empty(max(nnz, 1), np.float64)
        st = L.lib().cn_export_factor(self._h, _ip(ptr), _ip(col), _dp(val))
        if st != L.CN_OK:
            raise CnError(st, "cn_export_factor")
        return ptr, col[:nnz], val[:nnz]

    def export_k(self):
        i = self.info()
        nv, nnz = i["n_verts"], i["nnz_K"]
        ptr = np.empty(nv + 1, np.int32)
        col = np.empty(max(nnz, 1), np.int32)
        val = np.empty(max(nnz, 1), np.float64)
        st = L.lib().cn_export_k(self._h, _ip(ptr), _ip(col), _dp(val))
        if st != L.CN_OK:
            raise CnError(st, "cn_export_k")
        return ptr, col[:nnz], val[:nnz]

    # -- solves
    @staticmethod
    def make_opts(mode="deform", precision="mixed", tol=1e-8, max_iter=2000, max_refine=8,
                  inner_tol=1e-5, warm_start=False, algo="fused", wait_limit_ms=None):
        o = L.SolveOpts()
        L.lib().cn_default_solve_opts(C.byref(o))
        o.mode, o.precision, o.algo = _MODE[mode], _PREC[precision], _ALGO[algo]
        o.tol, o.max_iter, o.max_refine, o.inner_tol = tol, max_iter, max_refine, inner_tol
        o.warm_start = int(bool(warm_start))
        if wait_limit_ms is not None:
            o.wait_limit_ms = wait_limit_ms
        return o

    def solve(self, targets, x0=None, check=True, **kw):
        """targets: (n_handles, k) for harmonic/deform, (n_free, k) in solve
        order for mode='rhs'.  Returns SolveResult with x (n_verts, k)."""
        t = _f64(targets)
        t = t.reshape(t.shape[0], -1)
        k = t.shape[1]
        o = self.make_opts(**kw)
        x = np.empty((self.n_verts, k), np.float64)
        stats = L.SolveStats()
        x0p = _dp(_f64(x0).reshape(self.n_verts, k)) if x0 is not None else None
        st = L.lib().cn_solve(self._h, k, _dp(t), x0p, _dp(x), C.byref(o), C.byref(stats))
        if check and st not in (L.CN_OK,):
            raise CnError(st, "cn_solve")
        return SolveResult(x, stats)

    def solve_deformation(self, Fc, Xc, **kw):
        """DeformSolve.lean:110-135: Stage 1 (F), the Eq.(3) bridge, Stage 2
        (positions).  Fc: (n_handles, 9) row-major 3x3; Xc: (n_handles, 3)."""
        Fc = _f64(Fc).reshape(-1, 9)
        Xc = _f64(Xc).reshape(-1, 3)
        x = np.empty((self.n_verts, 3))
        o = self.make_opts(**kw)
        stats = L.SolveStats()
        st = L.lib().cn_solve_deformation(self._h, _dp(Fc), _dp(Xc), _dp(x), C.byref(o), C.byref(stats))
        if st != L.CN_OK:
            raise CnError(st, "cn_solve_deformation")
        return SolveResult(x, stats)

    # -- profile curvenet (DeGoes22 section 3 on the GPU)
    def bind_curvenet(self, rest_cp, sample_tau, handle_curve, handle_sample, handle_side, closed=None,
                      node_ptr=None, node_ends=None):
        """Bind curves to the handles (cn_bind_curvenet).  rest_cp:
        (n_curves, 3S+1, 3); sample_tau: (n_curves, n_samples); per handle its
        curve (-1: none), sample and side (0 plus, 1 minus); closed: per curve;
        node_ptr / node_ends: intersections as lists of curve ends (2 c + end)
        in counter-clockwise order."""
        rest_cp = _f64(rest_cp)
        C_, npts, _ = rest_cp.shape
        tau = _f64(sample_tau)
        self._cnet_keep = [rest_cp, tau, _i32(handle_curve), _i32(handle_sample), _i32(handle_side),
                           _i32(closed if closed is not None else np.zeros(C_)),
                           _i32(node_ptr if node_ptr is not None else [0]),
                           _i32(node_ends if node_ends is not None and len(node_ends) else [0])]
        rc, tu, hc, hs, hd, cl, npt, ne = self._cnet_keep
        d = L.CurvenetDesc(C_, (npts - 1) // 3, tau.shape[1], _dp(rc), _dp(tu), _ip(cl), npt.size - 1, _ip(npt),
                           _ip(ne), _ip(hc), _ip(hs), _ip(hd))
        st = L.lib().cn_bind_curvenet(self._h, C.byref(d))
        if st != L.CN_OK:
            raise CnError(st, "cn_bind_curvenet")
        self._cnet_shape = (C_, npts)

    def curvenet_constraints(self, posed_cp):
        """F_c (poses, n_handles, 3, 3) and X_c (poses, n_handles, 3) from
        posed control points (poses, n_curves, 3S+1, 3), on the GPU."""
        P = _f64(posed_cp).reshape(-1, *self._cnet_shape, 3)
        nh = self.handles.size
        F = np.empty((P.shape[0], nh, 9))
        X = np.empty((P.shape[0], nh, 3))
        st = L.lib().cn_curvenet_constraints(self._h, P.shape[0], _dp(P), _dp(F), _dp(X))
        if st != L.CN_OK:
            raise CnError(st, "cn_curvenet_constraints")
        return F.reshape(P.shape[0], nh, 3, 3), X

    def deform_curvenet(self, posed_cp, **kw):
        """Curves to deformed positions in one call (F_c, X_c on the GPU, then
        the two-stage solve of DeformSolve.lean:110-135).  Needs max_rhs=9."""
        P = _f64(posed_cp)
        x = np.empty((self.n_verts, 3))
        o = self.make_opts(**kw)
        stats = L.SolveStats()
        st = L.lib().cn_deform_curvenet(self._h, _dp(P), _dp(x), C.byref(o), C.byref(stats))
        if st != L.CN_OK:
            raise CnError(st, "cn_deform_curvenet")
        return SolveResult(x, stats)

    def ddm_bind(self, nu=2, omega=0.5, top_k=4, **kw):
        """Direct Delta Mush influences (DirectDeltaMushBind.lean:6-40):
        (idx, w), each (n_verts, min(top_k, n_handles)); row v's entries are
        vertex v's influences, largest |w| first.  Needs max_rhs=9."""
        take = min(top_k, self.handles.size)
        idx = np.empty((self.n_verts, take), np.int32)
        w = np.empty((self.n_verts, take))
        o = self.make_opts(mode="harmonic", **kw)
        st = L.lib().cn_ddm_bind(self._h, nu, omega, top_k, C.byref(o), _ip(idx), _dp(w))
        if st != L.CN_OK:
            raise CnError(st, "cn_ddm_bind")
        return idx, w

    def spmv_device(self, k, d_x, d_y, precision="mixed"):
        """y = A x on the reduced matrix in solve order (device pointers,
        [n_free][k], FP32 for "mixed", FP64 for "fp64"), on the handle's
        stream."""
        st = L.lib().cn_spmv_device(self._h, k, _PREC[precision], C.c_void_p(d_x), C.c_void_p(d_y))
        if st != L.CN_OK:
            raise CnError(st, "cn_spmv_device")

    def solve_device(self, k, d_targets, d_x_out, stats=True, **kw):
        """Device-pointer solve on the handle's stream (ints are device addresses)."""
        o = self.make_opts(**kw)
        s = L.SolveStats()
        st = L.lib().cn_solve_device(self._h, k, C.c_void_p(d_targets), C.c_void_p(d_x_out),
                                     C.byref(o), C.byref(s) if stats else None)
        if st != L.CN_OK:
            raise CnError(st, "cn_solve_device")
        return s if stats else None


def solve_multi(positions, tris, handles, Fc, **kw):
    """HarmonicSolve.lean:51-66: (V^T L_h V) X_v = -V^T L_h (C F_c); the handle
    rows carry F_c (the reference returns 0 there and the caller overlays)."""
    Fc = _f64(Fc)
    Fc = Fc.reshape(Fc.shape[0], -1)
    k = Fc.shape[1]
    with CutMeshSolver(positions, tris, handles, max_rhs=k if k in (1, 3, 9) else 9) as s:
        return s.solve(Fc, mode="harmonic", **kw).x


def solve_deformation(positions, tris, handles, Xc, **kw):
    """DeformSolve.lean:123-135 Stage 2 with F_f = I: the displacement-harmonic
    solve that reproduces the rest pose when X_c is the rest handle position."""
    with CutMeshSolver(positions, tris, handles, max_rhs=3) as s:
        return s.solve(_f64(Xc).reshape(-1, 3), mode="deform", **kw).x


class BatchSolver:
    """Many cut meshes solved together: one persistent, CUDA-graph-captured
    launch per solve of all meshes x k right-hand sides (cn_build_batch /
    cn_solve_batch).  meshes: list of (positions, tris, handles)."""

    def __init__(self, meshes, k=24, precond="ic0", ordering="auto", laplacian="cot",
                 mollify_delta=1e-4, device=0, cluster_size=0, n_clusters=0, block=0):
        self.k = k
        self._keep = []
        descs = (L.MeshDesc * len(meshes))()
        self.n_verts = []
        self.n_handles = []
        for i, (pos, tris, h) in enumerate(meshes):
            pos = _f64(pos).reshape(-1, 3)
            tris = _i32(tris).reshape(-1, 3)
            h = _i32(h).reshape(-1)
            self._keep += [pos, tris, h]
            descs[i] = L.MeshDesc(pos.shape[0], tris.shape[0], _dp(pos), _ip(tris), h.size, _ip(h))
            self.n_verts.append(pos.shape[0])
            self.n_handles.append(h.size)
        opts = L.BuildOpts()
        L.lib().cn_default_build_opts(C.byref(opts))
        opts.precond = _PRECOND[precond]
        opts.ordering = _ORDER[ordering]
        opts.laplacian = _LAP[laplacian]
        opts.mollify_delta = mollify_delta
        opts.device = device
        opts.block = block
        h = C.c_void_p()
        st = L.lib().cn_build_batch(descs, len(meshes), C.byref(opts), k, cluster_size, n_clusters, C.byref(h))
        self._keep = []
        if st != L.CN_OK:
            raise CnError(st, "cn_build_batch")
        self._h = h
        self.n_meshes = len(meshes)
        t = (C.c_int64 * (self.n_meshes + 1))()
        o = (C.c_int64 * (self.n_meshes + 1))()
        L.lib().cn_batch_offsets(self._h, t, o)
        self.tgt_off = np.array(list(t), np.int64)
        self.out_off = np.array(list(o), np.int64)

    def close(self):
        if getattr(self, "_h", None):
            L.lib().cn_destroy_batch(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def info(self):
        v = (C.c_int64 * 12)()
        L.lib().cn_batch_info(self._h, v)
        keys = ["n_meshes", "k", "n_verts", "n_handles", "n_free", "nnz_A", "nnz_L", "cluster_size",
                "n_clusters", "block", "max_free", "device_bytes"]
        return dict(zip(keys, list(v)))

    def stream(self):
        return L.lib().cn_batch_stream(self._h)

    def mesh_stats(self, refinements=False):
        """(status, iterations, max relative residual[, refinements]) per mesh
        of the last solve with statistics."""
        st = np.zeros(self.n_meshes, np.int32)
        it = np.zeros(self.n_meshes, np.int32)
        rel = np.zeros(self.n_meshes)
        ref = np.zeros(self.n_meshes, np.int32)
        L.lib().cn_batch_mesh_stats(self._h, _ip(st), _ip(it), _dp(rel), _ip(ref))
        return (st, it, rel, ref) if refinements else (st, it, rel)

    def set_lanes(self, class_max_rows, lanes):
        """Lanes per row by size class (cn_batch_set_lanes)."""
        cm, ln = _i32(class_max_rows), _i32(lanes)
        st = L.lib().cn_batch_set_lanes(self._h, cm.size, _ip(cm), _ip(ln))
        if st != L.CN_OK:
            raise CnError(st, "cn_batch_set_lanes")

    def lanes(self):
        out = np.zeros(self.n_meshes, np.int32)
        L.lib().cn_batch_lanes(self._h, _ip(out))
        return out

    def solve(self, targets, check=True, **kw):
        """targets: list of (n_handles_m, k) arrays.  Returns (list of
        (n_verts_m, k) arrays, BatchStats)."""
        flat = np.concatenate([_f64(t).reshape(-1) for t in targets])
        assert flat.size == self.tgt_off[-1]
        x = np.empty(int(self.out_off[-1]), np.float64)
        o = CutMeshSolver.make_opts(**kw)
        stats = L.BatchStats()
        st = L.lib().cn_solve_batch(self._h, _dp(flat), _dp(x), C.byref(o), C.byref(stats))
        if check and st != L.CN_OK:
            raise CnError(st, "cn_solve_batch")
        xs = [x[self.out_off[m]:self.out_off[m + 1]].reshape(-1, self.k) for m in range(self.n_meshes)]
        return xs, stats

    def solve_device(self, d_targets, d_x_out, stats=True, **kw):
        o = CutMeshSolver.make_opts(**kw)
        s = L.BatchStats()
        st = L.lib().cn_solve_batch_device(self._h, C.c_void_p(d_targets), C.c_void_p(d_x_out), C.byref(o),
                                           C.byref(s) if stats else None)
        if st != L.CN_OK:
            raise CnError(st, "cn_solve_batch_device")
        return s if stats else None


def lbs_matvec_device(n_verts, d_rest, d_transforms, d_start, d_idx, d_w, d_out, precision="mixed", stream=0):
    """Runtime Direct Delta Mush (DirectDeltaMush.lean:84-102) on device
    pointers (ints): rest/out n_verts x 3, transforms n_handles x 16,
    CSR influences start/idx/w; FP32 for "mixed", FP64 for "fp64"."""
    st = L.lib().cn_lbs_matvec_device(n_verts, _PREC[precision], C.c_void_p(d_rest), C.c_void_p(d_transforms),
                                      C.c_void_p(d_start), C.c_void_p(d_idx), C.c_void_p(d_w), C.c_void_p(d_out),
                                      C.c_void_p(stream))
    if st != L.CN_OK:
        raise CnError(st, "cn_lbs_matvec_device")
