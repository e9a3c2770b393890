"""Pins the CPU FP64 oracle to the reference's own known answers: every
`native_decide` example of the Lean specification on the sparse-solve path
(tests/golden/known_answers.json, written by make_known_answers.py)."""
import json
import math
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "known_answers.json")))

HE_BASE = {}


def _bases():
    from tests.golden.make_known_answers import HE_QUAD, HE_STRIP, HE_TRIANGLE
    return {"triangle": ([3, 1, 6], HE_TRIANGLE), "quad": ([4, 1, 8], HE_QUAD), "strip": ([4, 2, 10], HE_STRIP)}


def csr(A):
    return np.array(A["rowPtr"], np.int32), np.array(A["colIdx"], np.int32), np.array(A["values"])


def dense_of(A):
    p, c, v = csr(A)
    n = p.size - 1
    D = np.zeros((n, n))
    for i in range(n):
        D[i, c[p[i]:p[i + 1]]] = v[p[i]:p[i + 1]]
    return D


def fid(f):
    return f"{f['src']}:{f['kind']}"


CURVENET_KINDS = ("isolated_gradient", "rotate_vector", "gradient_displacement", "smallest_rotation", "det",
                  "inv", "inv_times", "times_inv", "inv_inv", "deformation_gradient", "gradient_pair_isolated",
                  "gradient_pair_intersection", "corner_normals", "per_side_normals", "corner_normals_z", "widths",
                  "scaled_frame", "per_side_frames", "corner_vector", "normal_unit", "normals_reflect",
                  "widths_equal", "frame_homogeneous", "interp", "interp_size")


def check_curvenet_fixture(O, f):
    """ScaledFrames.lean, SegmentGradient.lean, IntersectionFrames.lean and
    CurveInterp.lean examples against the oracle's primitives."""
    k = f["kind"]
    eps = f.get("eps", 0.0)

    def close(a, b, e=eps):
        return np.all(np.abs(np.asarray(a, float).ravel() - np.asarray(b, float).ravel()) < e)

    def m3(x):
        return np.asarray(x, float).reshape(3, 3)
    if k == "isolated_gradient":
        assert close(O.isolated_segment_gradient(*f["seg"]), f["F"])
    elif k == "rotate_vector":
        assert close(m3(O.smallest_rotation(f["a"], f["b"])) @ np.asarray(f["v"]), f["expected"])
    elif k == "gradient_displacement":
        F = O.isolated_segment_gradient(*f["seg"])
        assert close(F @ np.asarray(f["v"]), f["expected"])
    elif k == "smallest_rotation":
        assert close(O.smallest_rotation(f["a"], f["b"]), f["R"])
    elif k == "det":
        assert abs(O.mat3_det(f["M"]) - f["expected"]) < eps
    elif k == "inv":
        assert close(O.mat3_inv(f["M"]), f["expected"])
    elif k == "inv_times":
        assert close(O.mat3_mul(O.mat3_inv(f["M"]), f["M"]), f["expected"])
    elif k == "times_inv":
        assert close(O.mat3_mul(f["M"], O.mat3_inv(f["M"])), f["expected"])
    elif k == "inv_inv":
        assert close(O.mat3_inv(O.mat3_inv(f["M"])), f["expected"])
    elif k == "deformation_gradient":
        assert close(O.deformation_gradient(f["rest"], f["posed"]), f["F"])
    elif k == "gradient_pair_isolated":  # both sides take the isolated gradient
        F = O.isolated_segment_gradient(*f["seg"])
        assert close(F, f["Fp"]) and close(F, f["Fm"])
    elif k == "gradient_pair_intersection":
        assert close(O.deformation_gradient(f["rp"], f["pp"]), f["Fp"])
        assert close(O.deformation_gradient(f["rm"], f["pm"]), f["Fm"])
    elif k == "corner_normals":
        assert close(O.corner_normals(f["t"])[1], f["m"])
    elif k == "per_side_normals":
        m = O.corner_normals(f["t"])[1]
        i, n = f["seg"], len(f["t"])
        assert close(m[i], f["np"]) and close(m[(i + n - 1) % n], f["nm"])
    elif k == "corner_normals_z":
        assert close(O.corner_normals(f["t"])[1][:, 2], f["z"])
    elif k == "widths":
        wp, wm = O.per_side_widths(f["t"], f["l"])
        assert abs(wp[f["seg"]] - f["wp"]) < eps and abs(wm[f["seg"]] - f["wm"]) < eps
    elif k == "scaled_frame":
        assert close(O.scaled_frame(f["t"], f["n"], f["l"], f["w"]), f["M"])
    elif k == "per_side_frames":
        t = np.asarray(f["t"], float)
        m = O.corner_normals(t)[1]
        wp, wm = O.per_side_widths(t, f["l"])
        i, n = f["seg"], t.shape[0]
        Bp = O.scaled_frame(t[i], m[i], f["l"][i], wp[i]).ravel()
        Bm = O.scaled_frame(t[i], m[(i + n - 1) % n], f["l"][i], wm[i]).ravel()
        for side, idx, want in f["entries"]:
            assert abs((Bp if side == "p" else Bm)[idx] - want) < eps
    elif k == "corner_vector":
        assert close(O.corner_normals(f["t"])[0][f["i"]], f["expected"])
    elif k == "normal_unit":
        assert abs(np.linalg.norm(O.corner_normals(f["t"])[1][f["i"]]) - 1.0) < eps
    elif k == "normals_reflect":
        m = O.corner_normals(f["t"])[1]
        n = m.shape[0]
        for i in range(n):
            assert close(m[i] + m[(i + n - 1) % n], np.zeros(3))
    elif k == "widths_equal":
        wp, wm = O.per_side_widths(f["t"], f["l"])
        assert close(wp, wm)
    elif k == "frame_homogeneous":
        a = O.scaled_frame(f["t"], f["n"], f["l"], f["l"])
        b = O.scaled_frame(f["t"], f["n"], f["s"] * f["l"], f["s"] * f["l"])
        assert close(b, f["s"] * a)
    elif k == "interp":
        arr = O.interp_along_curve(f["first"], f["last"], f["n"])
        for i, j, want in f["entries"]:
            assert abs(arr[i, j] - want) < eps
    elif k == "interp_size":
        assert O.interp_along_curve(f["first"], f["last"], f["n"]).shape[0] == f["size"]


@pytest.mark.parametrize("f", FIX, ids=[fid(f) for f in FIX])
def test_known_answer(f, oracle):
    O = oracle
    k = f["kind"]
    eps = f.get("eps", 0.0)
    if k in ("tri_rowsum", "tri_symmetric", "tri_offdiag01"):
        Lm = O.triangle_cot_laplacian(*f["pts"])
        if k == "tri_rowsum":
            assert np.all(np.abs(Lm.sum(1)) < eps)
        elif k == "tri_symmetric":
            assert np.all(np.abs(Lm - Lm.T) < eps)
        else:
            assert abs(Lm[0, 1] - f["expected"]) < eps
    elif k in ("poly_rowsum", "poly_symmetric"):
        Lm = O.polygon_cot_laplacian(f["pts"])
        if k == "poly_rowsum":
            assert np.all(np.abs(Lm.sum(1)) < eps)
        else:
            assert np.all(np.abs(Lm - Lm.T) < eps)
    elif k == "mollify_zero":
        assert abs(O.mollify_triangle(f["delta"], f["e"])) < eps
    elif k == "mollify_positive":
        assert O.mollify_triangle(f["delta"], f["e"]) > 0.0
    elif k == "mollify_margin":
        d = f["delta"]
        e = np.array(f["e"]) + O.mollify_triangle(d, f["e"])
        t = f["tol"]
        assert e[1] + e[2] > e[0] + d - t and e[0] + e[2] > e[1] + d - t and e[0] + e[1] > e[2] + d - t
    elif k == "cot_from_lengths":
        assert abs(O.cot_from_lengths(*f["e"]) - f["expected"]) < eps
    elif k == "robust_equals_embedded":
        a = O.robust_triangle_cot_laplacian(f["delta"], *f["pts"])
        b = O.triangle_cot_laplacian(*f["pts"])
        assert np.all(np.abs(a - b) < eps)
    elif k == "robust_rowsum":
        a = O.robust_triangle_cot_laplacian(f["delta"], *f["pts"])
        assert np.all(np.abs(a.sum(1)) < eps)
    elif k == "robust_symmetric":
        a = O.robust_triangle_cot_laplacian(f["delta"], *f["pts"])
        assert np.all(np.abs(a - a.T) < eps)
    elif k == "robust_finite":
        a = O.robust_triangle_cot_laplacian(f["delta"], *f["pts"])
        assert np.all(np.isfinite(a))
    elif k == "manifold":
        assert O.manifold(f["nv"], f["nf"], np.array(f["he"], np.int32))
    elif k == "builder":
        he = O.halfedges_from_triangles(f["nv"], f["tris"])
        assert he.shape[0] == f["n_he"]
        assert O.manifold(f["nv"], f["nf"], he)
        if f.get("all_twins"):
            assert np.all(he[:, 1] >= 0) and np.all(he[he[:, 1], 1] == np.arange(he.shape[0]))
    elif k == "surgery":
        counts, he = _bases()[f["base"]]
        he = np.array(he, np.int32)
        counts = np.array(counts, np.int32)
        for op in f["ops"]:
            if op[0] == "subdivide":
                counts, he = O.subdivide_edge(counts, he, op[1])
            elif op[0] == "split":
                counts, he = O.split_face(counts, he, op[1], op[2])
            else:
                counts, he = O.insert_crack(counts, he, op[1])
        assert (counts[0], counts[2], counts[1]) == (f["nv"], f["n_he"], f["nf"])
        assert O.manifold(int(counts[0]), int(counts[1]), he)
        for h, length in f.get("loops", []):
            assert O.loop_length(he, h) == length
        if "crack" in f:
            a, b = f["crack"]
            assert he[a, 3] == 0 and he[b, 3] == 0 and he[a, 1] == b and he[b, 1] == a
    elif k == "partition":
        assert O.partition_of_unity(np.array(f["he"], np.int32), f["vkind"]) == f["expected"]
    elif k == "vtlhv":
        M = O.assemble_vtlhv_dense(f["nv"], f["nf"], np.array(f["he"], np.int32), f["vkind"], f["pos"])
        assert M.shape == (f["nv"], f["nv"])
        if "eps_rowsum" in f:
            assert np.all(np.abs(M.sum(1)) < f["eps_rowsum"])
        assert np.all(np.abs(M - M.T) < f["eps_sym"])
    elif k == "dense_solve":
        n = len(f["b"])
        x = O.dense_solve(np.array(f["A"], float).reshape(n, n), f["b"])
        assert np.all(np.abs(x - f["x"]) < eps)
    elif k == "dense_residual":
        n = len(f["b"])
        A = np.array(f["A"], float).reshape(n, n)
        x = O.dense_solve(A, f["b"])
        assert np.all(np.abs(A @ x - f["b"]) < eps)
    elif k == "lu_solve":
        n = len(f["b"])
        x = O.lu_solve(np.array(f["A"], float).reshape(n, n), f["b"])
        assert np.all(np.abs(x - f["x"]) < eps)
    elif k == "lu_vs_ge":
        n = len(f["b"])
        A = np.array(f["A"], float).reshape(n, n)
        assert np.all(np.abs(O.lu_solve(A, f["b"]) - O.dense_solve(A, f["b"])) < eps)
    elif k == "cholesky":
        n = int(math.isqrt(len(f["A"])))
        Lm = O.cholesky_factor(np.array(f["A"], float).reshape(n, n))
        assert np.all(np.abs(Lm - np.array(f["L"]).reshape(n, n)) < eps)
        assert np.all(np.abs(Lm @ Lm.T - np.array(f["A"]).reshape(n, n)) < eps)
    elif k == "cholesky_solve":
        n = len(f["b"])
        Lm = O.cholesky_factor(np.array(f["A"], float).reshape(n, n))
        assert np.all(np.abs(O.cholesky_solve(Lm, f["b"]) - f["x"]) < eps)
    elif k == "cholesky_vs_ge":
        n = len(f["b"])
        A = np.array(f["A"], float).reshape(n, n)
        Lm = O.cholesky_factor(A)
        assert np.all(np.abs(O.cholesky_solve(Lm, f["b"]) - O.dense_solve(A, f["b"])) < eps)
    elif k == "spmv":
        assert np.all(np.abs(dense_of(f["A"]) @ np.array(f["x"]) - f["y"]) < eps)
    elif k == "cg":
        x, _ = O.cg_ref(*csr(f["A"]), f["b"], f["max_iter"], f["tol"])
        assert np.all(np.abs(x - f["x"]) < eps)
    elif k == "cg_vs_dense":
        x, _ = O.cg_ref(*csr(f["A"]), f["b"], f["max_iter"], f["tol"])
        xd = O.dense_solve(np.array(f["A_dense"]).reshape(len(f["b"]), -1), f["b"])
        assert np.all(np.abs(x - xd) < eps)
    elif k == "cg_warm_vs_cold":
        xc, _ = O.cg_ref(*csr(f["A"]), f["b"], f["max_iter"], f["tol"])
        xw, _ = O.cg_ref(*csr(f["A"]), f["b"], f["max_iter"], f["tol"], x0=f["x0"])
        assert np.all(np.abs(xc - xw) < eps)
    elif k == "cg_warm_exact":
        xw, it = O.cg_ref(*csr(f["A"]), f["b"], f["max_iter"], f["tol"], x0=f["x0"])
        assert it == 0 and np.all(np.abs(xw - f["x0"]) < eps)
    elif k == "cg_residual":
        x, _ = O.cg_ref(*csr(f["A"]), f["b"], f["max_iter"], f["tol"])
        r = np.array(f["b"]) - dense_of(f["A"]) @ x
        assert float(r @ r) < f["rr_max"]
    elif k in ("ic0_llt", "ic0_solve"):
        st, Lp, Lc, Lv = O.ic0_factor(*csr(f["A"]))
        assert st == 0
        n = Lp.size - 1
        Lm = np.zeros((n, n))
        for i in range(n):
            Lm[i, Lc[Lp[i]:Lp[i + 1]]] = Lv[Lp[i]:Lp[i + 1]]
        assert np.all(np.triu(Lm, 1) == 0.0)
        A = dense_of(f["A"])
        if k == "ic0_llt":
            assert np.all(np.abs(Lm @ Lm.T - A) < eps)
        else:
            y = np.linalg.solve(Lm, f["b"])
            x = np.linalg.solve(Lm.T, y)
            assert np.all(np.abs(A @ x - f["b"]) < eps)
    elif k == "hsc":
        g = [tuple(e) for e in f["edges"]]
        for v in f["elim"]:
            g = O.hsc_eliminate(g, v)
        if "n_edges" in f:
            assert len(g) == f["n_edges"]
        for a, b, w in f.get("weights", []):
            got = [e[2] for e in g if (e[0], e[1]) == (a, b)]
            assert got and abs(got[0] - w) < eps
        if "degree" in f:
            v, d = f["degree"]
            assert abs(sum(e[2] for e in g if v in (e[0], e[1])) - d) < eps
    elif k == "color":
        c = O.greedy_color(f["adj"])
        assert all(c[i] != c[j] for i, a in enumerate(f["adj"]) for j in a)
        assert int(c.max()) + 1 == f["n_colors"]
    elif k == "harmonic":
        X = O.harmonic_solve_multi(f["nv"], f["nf"], np.array(f["he"], np.int32), f["sample_col"], f["pos"],
                                   f["Fc"], f["k"])
        for r, want in f["rows"].items():
            assert np.all(np.abs(X[int(r)] - want) < eps)
    elif k == "deform":
        X = O.solve_deformation(f["nv"], f["nf"], np.array(f["he"], np.int32), f["sample_col"], f["pos"],
                                f["Fc"], f["Xc"])
        for r, want in f["rows"].items():
            assert np.all(np.abs(X[int(r)] - want) < eps)
    elif k == "bezier":
        out = np.empty(3)
        O.lib().orc_bezier3(O.dp(O.f64(f["P"])), f["t"], O.dp(out))
        assert np.all(np.abs(out - f["expected"]) < eps)
    elif k in ("segment_gradient", "curve_deform"):
        def bez(P, t):
            out = np.empty(3)
            O.lib().orc_bezier3(O.dp(O.f64(P)), t, O.dp(out))
            return out
        rp, rq = bez(f["P_rest"], f["t"]), bez(f["P_rest"], f["t_fwd"])
        pp, pq = bez(f["P_posed"], f["t"]), bez(f["P_posed"], f["t_fwd"])
        F = np.empty(9)
        O.lib().orc_isolated_segment_gradient(O.dp(rp), O.dp(rq), O.dp(pp), O.dp(pq), O.dp(F))
        if k == "segment_gradient":
            assert np.all(np.abs(F - f["F"]) < eps)
        else:
            X = O.solve_deformation(f["nv"], f["nf"], np.array(f["he"], np.int32), f["sample_col"], f["pos"], F, pp)
            for r, want in f["rows"].items():
                assert np.all(np.abs(X[int(r)] - want) < eps)
    elif k == "lbs":
        got = O.lbs_matvec(f["T"], [tuple(x) for x in f["infl"]], f["rest"])
        assert np.all(np.abs(got - f["expected"]) < eps)
    elif k == "pou":
        assert np.all(np.abs(np.sum(f["W"], axis=1) - 1.0) < eps)
    elif k in ("smooth_entries", "smooth_pou"):
        W = O.smooth_weights(f["W"], f["adj"], f["nu"], f["omega"])
        if k == "smooth_pou":
            assert np.all(np.abs(W.sum(axis=1) - 1.0) < eps)
        else:
            for v, i, want in f["entries"]:
                assert abs(W[v, i] - want) < eps
    elif k in ("topk_size", "topk_rowsum", "topk_values"):
        idx, w = O.sparsify_topk(f["W"], f["K"])
        if k == "topk_size":
            assert idx.shape[1] == f["size"]
        elif k == "topk_rowsum":
            assert abs(w[0].sum() - 1.0) < eps
        else:
            assert np.all(np.abs(w[0] - f["values"]) < eps)
    elif k == "smooth_topk_pou":
        W = O.smooth_weights(f["W"], f["adj"], f["nu"], f["omega"])
        idx, w = O.sparsify_topk(W, f["K"])
        dense = np.zeros_like(W)
        np.put_along_axis(dense, idx, w, axis=1)
        assert np.all(np.abs(dense.sum(axis=1) - 1.0) < eps)
    elif k in CURVENET_KINDS:
        check_curvenet_fixture(O, f)
    else:
        pytest.fail(f"unknown fixture kind {k}")


def test_composed_deformation_matches_dense_oracle():
    """The composition used by the GPU deform tests on larger meshes agrees
    with the dense restatement of DeformSolve.lean:110-135 on the free rows."""
    from oracle import oracle as O
    from tests.helpers import composed_deformation, random_gradients, rel_err, sample_col, workload
    O.build()
    pos, tris, h, t = workload("cyl_tiny")
    nv = pos.shape[0]
    Fc = random_gradients(h.size, 3)
    he = O.halfedges_from_triangles(nv, tris)
    want = O.solve_deformation(nv, tris.shape[0], he, sample_col(nv, h), pos, Fc, t)
    got = composed_deformation(O, pos, tris, h, Fc, t)
    free = np.setdiff1d(np.arange(nv), h)
    assert rel_err(got[free], want[free]) < 1e-12
    assert np.array_equal(got[h], t)
