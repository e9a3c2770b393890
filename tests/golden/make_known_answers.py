"""Writes tests/golden/known_answers.json: the known-answer fixtures of the
reference's own `native_decide` examples for the sparse-solve path.

Each record carries the Lean file:line it comes from (relative to the
reference project root), its inputs, the expected values and the tolerance
the example states.  Values that the Lean examples state analytically
(1/sqrt 3, sqrt 3 / 2, ...) are computed here in binary64.  Run:

    python tests/golden/make_known_answers.py
"""
import json
import math
import os

S3 = math.sqrt(3.0)
TRI = [[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.5, 0.0, 0.8660254037844386]]
SQUARE = [[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [1.0, 0.0, 1.0], [0.0, 0.0, 1.0]]
PENT = [[math.cos(6.283185307179586 * k / 5.0), 0.0, math.sin(6.283185307179586 * k / 5.0)] for k in range(5)]
STRIP = [[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.5, 0.0, 0.8660254037844386], [1.5, 0.0, 0.8660254037844386]]

# Halfedge.lean:345-396 (target, twin, next, face); -1 = none
HE_TRIANGLE = [[1, 5, 1, 0], [2, 4, 2, 0], [0, 3, 0, 0], [2, 2, 4, -1], [1, 1, 5, -1], [0, 0, 3, -1]]
HE_QUAD = [[1, 7, 1, 0], [2, 6, 2, 0], [3, 5, 3, 0], [0, 4, 0, 0],
           [3, 3, 5, -1], [2, 2, 6, -1], [1, 1, 7, -1], [0, 0, 4, -1]]
HE_STRIP = [[1, 7, 1, 0], [2, 3, 2, 0], [0, 6, 0, 0], [1, 1, 4, 1], [3, 9, 5, 1], [2, 8, 3, 1],
            [2, 2, 8, -1], [0, 0, 6, -1], [3, 5, 9, -1], [1, 4, 7, -1]]

LAP4 = dict(rowPtr=[0, 2, 5, 8, 10], colIdx=[0, 1, 0, 1, 2, 1, 2, 3, 2, 3],
            values=[2.0, -1.0, -1.0, 2.0, -1.0, -1.0, 2.0, -1.0, -1.0, 2.0])
LAP4_DENSE = [2.0, -1.0, 0.0, 0.0, -1.0, 2.0, -1.0, 0.0, 0.0, -1.0, 2.0, -1.0, 0.0, 0.0, -1.0, 2.0]


def rec(src, kind, **kw):
    d = dict(src=src, kind=kind)
    d.update(kw)
    return d


def main():
    out = []
    # ---------------------------------------------------------------- Laplacians
    out += [
        rec("PolygonLaplacian.lean:144-147", "tri_rowsum", pts=TRI, eps=1e-12),
        rec("PolygonLaplacian.lean:149-152", "tri_symmetric", pts=TRI, eps=1e-12),
        rec("PolygonLaplacian.lean:154-158", "tri_offdiag01", pts=TRI, expected=-1.0 / (2.0 * S3), eps=1e-12),
        rec("PolygonLaplacian.lean:160-163", "poly_rowsum", pts=SQUARE, eps=1e-12),
        rec("PolygonLaplacian.lean:165-168", "poly_symmetric", pts=SQUARE, eps=1e-12),
        rec("PolygonLaplacian.lean:170-173", "poly_rowsum", pts=PENT, eps=1e-9),
        rec("PolygonLaplacian.lean:175-178", "poly_symmetric", pts=PENT, eps=1e-9),
        rec("RobustLaplacian.lean:168-170", "mollify_zero", delta=0.0, e=[1.0, 1.0, 1.0], eps=1e-12),
        rec("RobustLaplacian.lean:172-175", "mollify_zero", delta=0.01, e=[1.0, 1.0, 1.0], eps=1e-12),
        rec("RobustLaplacian.lean:177-186", "mollify_positive", delta=0.05, e=[1.0, 1.0, 1.99]),
        rec("RobustLaplacian.lean:188-202", "mollify_margin", delta=0.05, e=[1.0, 1.0, 1.99], tol=1e-12),
        rec("RobustLaplacian.lean:204-209", "cot_from_lengths", e=[1.0, 1.0, 1.0], expected=1.0 / S3, eps=1e-12),
        rec("RobustLaplacian.lean:211-216", "cot_from_lengths", e=[1.0, S3, 2.0], expected=S3, eps=1e-9),
        rec("RobustLaplacian.lean:218-223", "cot_from_lengths", e=[S3, 1.0, 2.0], expected=1.0 / S3, eps=1e-9),
        rec("RobustLaplacian.lean:225-229", "cot_from_lengths", e=[2.0, 1.0, S3], expected=0.0, eps=1e-9),
        rec("RobustLaplacian.lean:231-244", "robust_equals_embedded", pts=TRI, delta=0.0, eps=1e-12),
        rec("RobustLaplacian.lean:246-250", "robust_rowsum", pts=TRI, delta=0.0, eps=1e-12),
        rec("RobustLaplacian.lean:252-256", "robust_symmetric", pts=TRI, delta=0.0, eps=1e-12),
        rec("RobustLaplacian.lean:258-276", "robust_finite",
            pts=[[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [1.999999, 0.0, 0.0]], delta=0.01),
    ]
    # ---------------------------------------------------------------- topology
    out += [
        rec("Halfedge.lean:402-404", "manifold", nv=3, nf=1, he=HE_TRIANGLE),
        rec("Halfedge.lean:402-404", "manifold", nv=4, nf=1, he=HE_QUAD),
        rec("Halfedge.lean:402-404", "manifold", nv=4, nf=2, he=HE_STRIP),
        rec("HalfedgeBuilder.lean:115-119", "builder", nv=3, tris=[[0, 1, 2]], n_he=6, nf=1),
        rec("HalfedgeBuilder.lean:121-126", "builder", nv=4, tris=[[0, 1, 2], [2, 1, 3]], n_he=10, nf=2),
        rec("HalfedgeBuilder.lean:128-136", "builder", nv=4, tris=[[0, 1, 2], [0, 2, 3], [0, 3, 1], [1, 3, 2]],
            n_he=12, nf=4, all_twins=True),
        rec("CutAlgorithm.lean:270-291", "surgery", base="triangle", ops=[["subdivide", 0]],
            nv=4, n_he=8, nf=1, loops=[[0, 4]]),
        rec("CutAlgorithm.lean:293-298", "surgery", base="quad", ops=[["subdivide", 0]], nv=5, n_he=10, nf=1),
        rec("CutAlgorithm.lean:300-306", "surgery", base="triangle", ops=[["subdivide", 0], ["subdivide", 1]],
            nv=5, n_he=10, nf=1),
        rec("CutAlgorithm.lean:323-351", "surgery", base="quad", ops=[["split", 0, 2]],
            nv=4, n_he=10, nf=2, loops=[[1, 3], [0, 3]]),
        rec("CutAlgorithm.lean:362-370", "surgery", base="quad", ops=[["subdivide", 0], ["split", 1, 3]],
            nv=5, n_he=12, nf=2),
        rec("CutAlgorithm.lean:420-456", "surgery", base="triangle", ops=[["crack", 0]],
            nv=4, n_he=8, nf=1, loops=[[0, 5]], crack=[6, 7]),
        rec("CutAlgorithm.lean:462-507", "surgery", base="strip", ops=[["subdivide", 1], ["split", 2, 1], ["split", 3, 4]],
            nv=5, n_he=16, nf=4, loops=[[0, 3]]),
        rec("CutMesh.lean:157-164", "partition", he=HE_TRIANGLE, vkind=[0, 0, 0], expected=True),
        rec("CutMesh.lean:157-164", "partition", he=HE_QUAD, vkind=[0, 0, 0, 0], expected=True),
        rec("CutMesh.lean:187-188", "partition", he=HE_TRIANGLE, vkind=[1, 0, 0], expected=True),
    ]
    # ---------------------------------------------------------------- V^T L_h V
    out += [
        rec("CutMeshLaplacian.lean:305-316", "vtlhv", he=HE_TRIANGLE, nv=3, nf=1, vkind=[0, 0, 0], pos=TRI,
            eps_rowsum=1e-12, eps_sym=1e-12),
        rec("CutMeshLaplacian.lean:318-329", "vtlhv", he=HE_QUAD, nv=4, nf=1, vkind=[0, 0, 0, 0], pos=SQUARE,
            eps_rowsum=1e-12, eps_sym=1e-12),
        rec("CutMeshLaplacian.lean:339-350", "vtlhv", he=HE_STRIP, nv=4, nf=2, vkind=[0, 0, 0, 0], pos=STRIP,
            eps_rowsum=1e-10, eps_sym=1e-10),
        rec("CutMeshLaplacian.lean:352-361", "vtlhv", he=HE_TRIANGLE, nv=3, nf=1, vkind=[1, 0, 0], pos=TRI,
            eps_sym=1e-10),
    ]
    # ---------------------------------------------------------------- dense LA
    out += [
        rec("DenseLinAlg.lean:297-302", "dense_solve", A=[1, 0, 0, 0, 1, 0, 0, 0, 1], b=[1, 2, 3], x=[1, 2, 3], eps=1e-12),
        rec("DenseLinAlg.lean:305-312", "dense_solve", A=[2, 0, 0, 0, 3, 0, 0, 0, 4], b=[4, 9, 16], x=[2, 3, 4], eps=1e-12),
        rec("DenseLinAlg.lean:314-319", "dense_solve", A=[2, 1, 1, 2], b=[3, 3], x=[1, 1], eps=1e-12),
        rec("DenseLinAlg.lean:321-327", "dense_solve", A=[0, 1, 1, 0], b=[2, 3], x=[3, 2], eps=1e-12),
        rec("DenseLinAlg.lean:329-338", "dense_residual", A=[2, 0, 1, 0, 3, 0, 1, 0, 4], b=[5, 6, 9], eps=1e-10),
        rec("DenseLinAlg.lean:365-404", "lu_solve", A=[2, 1, 1, 2], b=[3, 3], x=[1, 1], eps=1e-12),
        rec("DenseLinAlg.lean:396-404", "lu_solve", A=[0, 1, 1, 0], b=[2, 3], x=[3, 2], eps=1e-12),
        rec("DenseLinAlg.lean:431-442", "lu_vs_ge", A=[4, 3, 0, 6, 3, 0, 0, 0, 1], b=[7, 9, 1], eps=1e-10),
        rec("DenseLinAlg.lean:444-452", "cholesky", A=[4, 2, 2, 3], L=[2, 0, 1, math.sqrt(2.0)], eps=1e-12),
        rec("DenseLinAlg.lean:463-472", "cholesky_solve", A=[4, 2, 2, 3], b=[10, 8], x=[1.75, 1.5], eps=1e-12),
        rec("DenseLinAlg.lean:486-490", "cholesky_solve", A=[4, 2, 2, 3], b=[4, 3], x=[0.75, 0.5], eps=1e-12),
        rec("DenseLinAlg.lean:474-483", "cholesky_vs_ge", A=LAP4_DENSE, b=[1, 0, 0, 0], eps=1e-10),
    ]
    # ---------------------------------------------------------------- CG (SparseLinAlg)
    I3 = dict(rowPtr=[0, 1, 2, 3], colIdx=[0, 1, 2], values=[1.0, 1.0, 1.0])
    D234 = dict(rowPtr=[0, 1, 2, 3], colIdx=[0, 1, 2], values=[2.0, 3.0, 4.0])
    SPD2 = dict(rowPtr=[0, 2, 4], colIdx=[0, 1, 0, 1], values=[2.0, 1.0, 1.0, 2.0])
    F07 = dict(rowPtr=[0, 2, 5, 7], colIdx=[0, 1, 0, 1, 2, 1, 2], values=[4.0, -1.0, -1.0, 4.0, -1.0, -1.0, 4.0])
    out += [
        rec("SparseLinAlg.lean:183-186", "spmv", A=I3, x=[1.0, 2.0, 3.0], y=[1.0, 2.0, 3.0], eps=1e-12),
        rec("SparseLinAlg.lean:189-192", "cg", A=I3, b=[1.0, 2.0, 3.0], max_iter=10, tol=1e-12, x=[1.0, 2.0, 3.0], eps=1e-9),
        rec("SparseLinAlg.lean:203-206", "cg", A=D234, b=[4.0, 9.0, 16.0], max_iter=10, tol=1e-12, x=[2.0, 3.0, 4.0], eps=1e-9),
        rec("SparseLinAlg.lean:217-220", "cg", A=SPD2, b=[3.0, 3.0], max_iter=50, tol=1e-12, x=[1.0, 1.0], eps=1e-8),
        rec("SparseLinAlg.lean:243-246", "cg", A=LAP4, b=[1.0, 0.0, 0.0, 0.0], max_iter=200, tol=1e-12,
            x=[0.8, 0.6, 0.4, 0.2], eps=1e-7),
        rec("SparseLinAlg.lean:251-260", "cg_vs_dense", A=LAP4, A_dense=LAP4_DENSE, b=[1.0, 2.0, 3.0, 4.0],
            max_iter=200, tol=1e-12, eps=1e-7),
        rec("SparseLinAlg.lean:265-269", "cg_warm_vs_cold", A=LAP4, b=[1.0, 2.0, 3.0, 4.0], x0=[0.0, 0.0, 0.0, 0.0],
            max_iter=200, tol=1e-12, eps=1e-9),
        rec("SparseLinAlg.lean:275-279", "cg_warm_exact", A=LAP4, b=[1.0, 0.0, 0.0, 0.0], x0=[0.8, 0.6, 0.4, 0.2],
            max_iter=0, tol=1e-9, eps=1e-9),
        rec("SparseLinAlg.lean:283-287", "cg_warm_vs_cold", A=LAP4, b=[1.0, 2.0, 3.0, 4.0], x0=[3.9, 6.9, 8.9, 6.9],
            max_iter=200, tol=1e-12, eps=1e-7),
        rec("Features/KnownKnowns/SolverKernels.lean:9-18", "cg_residual", A=F07, b=[1.0, 0.0, -1.0], max_iter=100,
            tol=1e-12, rr_max=1e-9),
    ]
    # ---------------------------------------------------------------- IC(0)
    ATRI = dict(rowPtr=[0, 2, 5, 7], colIdx=[0, 1, 0, 1, 2, 1, 2], values=[4.0, -1.0, -1.0, 4.0, -1.0, -1.0, 4.0])
    AWIDE = dict(rowPtr=[0, 2, 5, 7], colIdx=[0, 1, 0, 1, 2, 1, 2],
                 values=[1.0e-2, 1.0e-3, 1.0e-3, 1.0e0, 1.0e-2, 1.0e-2, 1.0e4])
    out += [
        rec("IncompleteCholesky.lean:142-151", "ic0_llt", A=ATRI, eps=1e-12),
        rec("IncompleteCholesky.lean:153-166", "ic0_solve", A=ATRI, b=[3.0, 2.0, 5.0], eps=1e-10),
        rec("IncompleteCholesky.lean:182-186", "ic0_llt", A=AWIDE, eps=1e-9),
    ]
    # ---------------------------------------------------------------- HSC
    path3 = [[0, 1, 1.0], [1, 2, 2.0]]
    star4 = [[0, 1, 1.0], [0, 2, 2.0], [0, 3, 3.0]]
    tpl = [[0, 1, 1.0], [0, 2, 1.0], [1, 2, 1.0], [0, 3, 4.0]]
    out += [
        rec("HierarchicalSparsifyCompensate.lean:404-411", "hsc", edges=path3, elim=[1], n_edges=1,
            weights=[[0, 2, 2.0 / 3.0]], eps=1e-12),
        rec("HierarchicalSparsifyCompensate.lean:425-439", "hsc", edges=star4, elim=[0], n_edges=3,
            weights=[[1, 2, 1.0 / 3.0], [1, 3, 0.5], [2, 3, 1.0]], eps=1e-12),
        rec("HierarchicalSparsifyCompensate.lean:454-460", "hsc", edges=tpl, elim=[0],
            weights=[[1, 2, 1.0 + 1.0 / 6.0], [1, 3, 4.0 / 6.0]], eps=1e-12),
        rec("HierarchicalSparsifyCompensate.lean:466-470", "hsc", edges=[[0, 1, 1.5]], elim=[2], n_edges=1,
            weights=[[0, 1, 1.5]], eps=1e-12),
        rec("HierarchicalSparsifyCompensate.lean:475-479", "hsc", edges=path3, elim=[1, 0], n_edges=0, eps=1e-12),
        rec("HierarchicalSparsifyCompensate.lean:485-488", "hsc", edges=star4, elim=[0], degree=[1, 5.0 / 6.0], eps=1e-12),
    ]
    # ---------------------------------------------------------------- colouring
    out += [
        rec("GraphColoring.lean:363-370", "color", adj=[[1, 2], [0, 2], [0, 1]], n_colors=3),
        rec("GraphColoring.lean:372-379", "color", adj=[[1, 3], [0, 2], [1, 3], [0, 2]], n_colors=2),
        rec("GraphColoring.lean:381-388", "color", adj=[[1], [0, 2], [1, 3], [2, 4], [3]], n_colors=2),
        rec("GraphColoring.lean:390-397", "color", adj=[[1, 2, 3, 4], [0], [0], [0], [0]], n_colors=2),
    ]
    # ---------------------------------------------------------------- harmonic / deform solves
    I9 = [1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0]
    RZ = [0.0, -1.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0]
    S2 = [2.0, 0.0, 0.0, 0.0, 2.0, 0.0, 0.0, 0.0, 2.0]
    tws = dict(he=HE_TRIANGLE, nv=3, nf=1, tris=[[0, 1, 2]], sample_col=[0, -1, -1], pos=TRI, handles=[0])
    out += [
        rec("HarmonicSolve.lean:284-293", "harmonic", Fc=[5.0, 10.0, 15.0], k=3,
            rows={"1": [5.0, 10.0, 15.0], "2": [5.0, 10.0, 15.0]}, eps=1e-9, **tws),
        rec("HarmonicSolve.lean:298-309", "harmonic", Fc=I9, k=9, rows={"1": I9}, eps=1e-9, **tws),
        rec("HarmonicSolve.lean:313-319", "harmonic", Fc=[7.0], k=1, rows={"1": [7.0], "2": [7.0]}, eps=1e-9, **tws),
        rec("HarmonicSolve.lean:323-330", "harmonic", Fc=[1.0, 2.0, 3.0], k=3,
            rows={"1": [1.0, 2.0, 3.0], "2": [1.0, 2.0, 3.0]}, eps=1e-9, **tws),
        rec("HarmonicSolve.lean:334-344", "harmonic", Fc=RZ, k=9, rows={"1": RZ}, eps=1e-9, **tws),
        rec("DeformSolve.lean:167-184", "deform", Fc=I9, Xc=[5.0, 0.0, 0.0],
            rows={"1": [6.0, 0.0, 0.0], "2": [5.5, 0.0, 0.8660254037844386]}, eps=1e-9, **tws),
        rec("DeformSolve.lean:187-195", "deform", Fc=I9, Xc=[0.0, 2.0, 0.0], rows={"1": [1.0, 2.0, 0.0]}, eps=1e-9, **tws),
        rec("DeformSolve.lean:208-226", "deform", Fc=RZ, Xc=[0.0, 0.0, 0.0],
            rows={"1": [0.0, 1.0, 0.0], "2": [0.0, 0.5, 0.8660254037844386]}, eps=1e-9, **tws),
        rec("DeformSolve.lean:235-253", "deform", Fc=S2, Xc=[0.0, 0.0, 0.0],
            rows={"1": [2.0, 0.0, 0.0], "2": [1.0, 0.0, 1.7320508075688772]}, eps=1e-9, **tws),
    ]
    # ---------------------------------------------------------------- curve-derived inputs
    prest = [[-1.5, 0.0, 0.0], [-0.5, 0.0, 0.0], [0.5, 0.0, 0.0], [1.5, 0.0, 0.0]]
    pposed = [[p[0] + 5.0, p[1], p[2]] for p in prest]
    prot = [[-p[1], p[0], p[2]] for p in prest]
    out += [
        rec("EndToEndExample.lean:94-100", "bezier", P=prest, t=0.5, expected=[0.0, 0.0, 0.0], eps=1e-12),
        rec("EndToEndExample.lean:98-100", "bezier", P=pposed, t=0.5, expected=[5.0, 0.0, 0.0], eps=1e-12),
        rec("EndToEndExample.lean:108-112", "segment_gradient", P_rest=prest, P_posed=pposed, t=0.5, t_fwd=0.6,
            F=I9, eps=1e-12),
        rec("EndToEndExample.lean:182-190", "segment_gradient", P_rest=prest, P_posed=prot, t=0.5, t_fwd=0.6,
            F=RZ, eps=1e-12),
        rec("EndToEndExample.lean:144-152", "curve_deform", P_rest=prest, P_posed=pposed, t=0.5, t_fwd=0.6,
            rows={"1": [6.0, 0.0, 0.0], "2": [5.5, 0.0, 0.8660254037844386]}, eps=1e-9, **tws),
        rec("EndToEndExample.lean:202-211", "curve_deform", P_rest=prest, P_posed=prot, t=0.5, t_fwd=0.6,
            rows={"1": [0.0, 1.0, 0.0], "2": [0.0, 0.5, 0.8660254037844386]}, eps=1e-9, **tws),
    ]
    # ---------------------------------------------------------------- curvenet frames (DeGoes22 section 3)
    O3, X1, Y1 = [0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]
    D234 = [2.0, 0.0, 0.0, 0.0, 3.0, 0.0, 0.0, 0.0, 4.0]
    M121 = [2.0, 1.0, 0.0, 1.0, 2.0, 1.0, 0.0, 1.0, 2.0]
    M123 = [1.0, 2.0, 3.0, 0.0, 1.0, 4.0, 5.0, 6.0, 0.0]
    out += [
        rec("ScaledFrames.lean:163-165", "isolated_gradient", seg=[O3, X1, O3, X1], F=I9, eps=1e-12),
        rec("ScaledFrames.lean:168-171", "isolated_gradient", seg=[O3, X1, O3, Y1], F=RZ, eps=1e-12),
        rec("ScaledFrames.lean:174-178", "rotate_vector", a=X1, b=Y1, v=X1, expected=[0.0, 1.0, 0.0], eps=1e-12),
        rec("ScaledFrames.lean:182-185", "isolated_gradient", seg=[O3, X1, O3, [2.0, 0.0, 0.0]], F=S2, eps=1e-12),
        rec("ScaledFrames.lean:190-195", "gradient_displacement", seg=[O3, X1, O3, [0.0, 3.0, 0.0]], v=X1,
            expected=[0.0, 3.0, 0.0], eps=1e-12),
        rec("ScaledFrames.lean:198-199", "smallest_rotation", a=X1, b=X1, R=I9, eps=1e-12),
        rec("ScaledFrames.lean:207", "det", M=I9, expected=1.0, eps=1e-12),
        rec("ScaledFrames.lean:210-212", "det", M=D234, expected=24.0, eps=1e-12),
        rec("ScaledFrames.lean:215-216", "inv", M=I9, expected=I9, eps=1e-12),
        rec("ScaledFrames.lean:219-222", "inv", M=D234,
            expected=[0.5, 0.0, 0.0, 0.0, 1.0 / 3.0, 0.0, 0.0, 0.0, 0.25], eps=1e-12),
        rec("ScaledFrames.lean:225-227", "inv_times", M=M121, expected=I9, eps=1e-10),
        rec("ScaledFrames.lean:230-231", "deformation_gradient", rest=I9, posed=I9, F=I9, eps=1e-12),
        rec("ScaledFrames.lean:234-236", "deformation_gradient", rest=I9, posed=D234, F=D234, eps=1e-12),
        rec("ScaledFrames.lean:239-241", "deformation_gradient", rest=M121, posed=M121, F=I9, eps=1e-10),
        rec("ScaledFrames.lean:244-246", "times_inv", M=M121, expected=I9, eps=1e-10),
        rec("ScaledFrames.lean:249-251", "times_inv", M=M123, expected=I9, eps=1e-10),
        rec("ScaledFrames.lean:254-256", "inv_times", M=M123, expected=I9, eps=1e-10),
        rec("ScaledFrames.lean:259-261", "inv_inv", M=M121, expected=M121, eps=1e-9),
        rec("ScaledFrames.lean:264-266", "times_inv", M=RZ, expected=I9, eps=1e-12),
        rec("SegmentGradient.lean:88-93", "gradient_pair_isolated", seg=[O3, X1, O3, X1], Fp=I9, Fm=I9, eps=1e-12),
        rec("SegmentGradient.lean:95-102", "gradient_pair_isolated", seg=[O3, X1, O3, Y1], Fp=RZ, Fm=RZ, eps=1e-12),
        rec("SegmentGradient.lean:104-113", "gradient_pair_intersection", rp=I9, pp=I9, rm=I9, pm=I9, Fp=I9, Fm=I9,
            eps=1e-12),
        rec("SegmentGradient.lean:115-133", "gradient_pair_intersection", rp=I9,
            pp=[1.0, 0.0, 0.0, 0.0, 2.0, 0.0, 0.0, 0.0, 1.0], rm=I9, pm=I9,
            Fp=[1.0, 0.0, 0.0, 0.0, 2.0, 0.0, 0.0, 0.0, 1.0], Fm=I9, eps=1e-12),
    ]
    perp = [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0]]
    s60, c60 = 0.8660254037844386, 0.5
    trij = [[1.0, 0.0, 0.0], [-c60, s60, 0.0], [-c60, -s60, 0.0]]
    tj = [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [-1.0, 0.0, 0.0]]
    out += [
        rec("IntersectionFrames.lean:189-197", "corner_normals", t=perp, m=[[0.0, 0.0, 1.0], [0.0, 0.0, -1.0]],
            eps=1e-12),
        rec("IntersectionFrames.lean:199-205", "per_side_normals", t=perp, seg=0, np=[0.0, 0.0, 1.0],
            nm=[0.0, 0.0, -1.0], eps=1e-12),
        rec("IntersectionFrames.lean:215-222", "corner_normals_z", t=trij, z=[1.0, 1.0, 1.0], eps=1e-12),
        rec("IntersectionFrames.lean:226-231", "widths", t=trij, l=[1.0, 1.0, 1.0], seg=0, wp=1.0, wm=1.0,
            eps=1e-12),
        rec("IntersectionFrames.lean:240-244", "widths", t=perp, l=[1.0, 3.0], seg=0, wp=3.0, wm=3.0, eps=1e-12),
        rec("IntersectionFrames.lean:257-259", "scaled_frame", t=X1, n=[0.0, 0.0, 1.0], l=1.0, w=1.0, M=I9,
            eps=1e-12),
        rec("IntersectionFrames.lean:263-271", "scaled_frame", t=X1, n=[0.0, 0.0, 1.0], l=2.0, w=3.0,
            M=[2.0, 0.0, 0.0, 0.0, 3.0, 0.0, 0.0, 0.0, math.sqrt(6.0)], eps=1e-12),
        rec("IntersectionFrames.lean:275-282", "per_side_frames", t=perp, l=[1.0, 1.0], seg=0,
            entries=[["p", 0, 1.0], ["p", 8, 1.0], ["m", 0, 1.0], ["m", 8, -1.0]], eps=1e-12),
        rec("IntersectionFrames.lean:301-305", "corner_vector", t=tj, i=2, expected=[0.0, 0.0, 0.0], eps=1e-12),
        rec("IntersectionFrames.lean:309-314", "corner_normals_z", t=tj, z=[1.0, 1.0, 1.0], eps=1e-12),
        rec("IntersectionFrames.lean:317-322", "normal_unit", t=tj, i=2, eps=1e-12),
        rec("IntersectionFrames.lean:329-339", "normals_reflect", t=perp, eps=1e-12),
        rec("IntersectionFrames.lean:343-350", "widths_equal", t=trij, l=[1.0, 1.0, 1.0], eps=1e-12),
        rec("IntersectionFrames.lean:354-368", "frame_homogeneous", t=X1, n=[0.0, 0.0, 1.0], l=1.0, s=2.0,
            eps=1e-12),
    ]
    first = [0.0, 0.0, 1.0, 1.0, 0.0, 0.0, -1.0, 1.0]
    last = [1.0, 0.0, 0.0, 5.0, -1.0, 0.0, 0.0, 3.0]
    out += [
        rec("CurveInterp.lean:86-95", "interp", first=first, last=last, n=2,
            entries=[[0, 3, 1.0], [0, 2, 1.0], [1, 3, 5.0], [1, 0, 1.0], [0, 6, -1.0], [1, 4, -1.0]], eps=1e-12),
        rec("CurveInterp.lean:98-110", "interp", first=first, last=last, n=3,
            entries=[[1, 0, 0.5], [1, 1, 0.0], [1, 2, 0.5], [1, 3, 3.0], [1, 4, -0.5], [1, 6, -0.5], [1, 7, 2.0]],
            eps=1e-12),
        rec("CurveInterp.lean:112-120", "interp", first=first, last=last, n=5,
            entries=[[1, 3, 2.0], [2, 3, 3.0]], eps=1e-12),
        rec("CurveInterp.lean:122-125", "interp_size", first=first, last=last, n=1, size=1),
        rec("CurveInterp.lean:127-130", "interp_size", first=first, last=last, n=0, size=0),
    ]
    # ---------------------------------------------------------------- Direct Delta Mush
    ident = [1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0]

    def trans(tx, ty, tz):
        return [1.0, 0.0, 0.0, tx, 0.0, 1.0, 0.0, ty, 0.0, 0.0, 1.0, tz, 0.0, 0.0, 0.0, 1.0]
    out += [
        rec("DirectDeltaMush.lean:115-120", "lbs", T=[ident], infl=[[0, 1.0]], rest=[1.5, -2.0, 0.75],
            expected=[1.5, -2.0, 0.75], eps=1e-12),
        rec("DirectDeltaMush.lean:122-127", "lbs", T=[trans(2.0, -3.0, 1.0)], infl=[[0, 1.0]], rest=[1.0, 1.0, 1.0],
            expected=[3.0, -2.0, 2.0], eps=1e-12),
        rec("DirectDeltaMush.lean:129-134", "lbs", T=[ident, ident], infl=[[0, 0.5], [1, 0.5]], rest=[4.0, -1.0, 2.0],
            expected=[4.0, -1.0, 2.0], eps=1e-12),
        rec("DirectDeltaMush.lean:136-145", "lbs", T=[trans(1.0, 0.0, 0.0), trans(-1.0, 0.0, 0.0)],
            infl=[[0, 0.7], [1, 0.3]], rest=[0.0, 0.0, 0.0], expected=[0.4, 0.0, 0.0], eps=1e-12),
        rec("DirectDeltaMush.lean:147-155", "lbs", T=[ident], infl=[], rest=[1.0, 1.0, 1.0],
            expected=[0.0, 0.0, 0.0], eps=1e-12),
        rec("DirectDeltaMush.lean:157-165", "lbs", T=[ident] * 4, infl=[[0, 0.25], [1, 0.25], [2, 0.25], [3, 0.25]],
            rest=[7.0, 8.0, 9.0], expected=[7.0, 8.0, 9.0], eps=1e-12),
    ]
    path4 = [[1], [0, 2], [1, 3], [2]]
    idW = [[1.0 if i == v else 0.0 for i in range(4)] for v in range(4)]
    halfW = [[0.5, 0.5, 0.0, 0.0] for _ in range(4)]
    out += [
        rec("DirectDeltaMushBind.lean:169", "pou", W=idW, eps=1e-12),
        rec("DirectDeltaMushBind.lean:171-175", "smooth_entries", W=idW, adj=path4, nu=0, omega=0.5,
            entries=[[0, 0, 1.0], [1, 1, 1.0]], eps=1e-12),
        rec("DirectDeltaMushBind.lean:188", "pou", W=halfW, eps=1e-12),
        rec("DirectDeltaMushBind.lean:190-192", "smooth_pou", W=halfW, adj=path4, nu=5, omega=0.5, eps=1e-12),
        rec("DirectDeltaMushBind.lean:194-197", "smooth_entries", W=halfW, adj=path4, nu=5, omega=0.5,
            entries=[[0, 0, 0.5], [2, 1, 0.5]], eps=1e-12),
        rec("DirectDeltaMushBind.lean:205-207", "topk_size", W=[[0.4, 0.3, 0.2, 0.1]], K=2, size=2),
        rec("DirectDeltaMushBind.lean:209-211", "topk_rowsum", W=[[0.4, 0.3, 0.2, 0.1]], K=2, eps=1e-12),
        rec("DirectDeltaMushBind.lean:213-216", "topk_values", W=[[0.4, 0.3, 0.2, 0.1]], K=2,
            values=[4.0 / 7.0, 3.0 / 7.0], eps=1e-12),
        rec("DirectDeltaMushBind.lean:218-224", "topk_rowsum", W=idW[:1], K=4, eps=1e-12),
        rec("DirectDeltaMushBind.lean:240-245", "smooth_topk_pou", W=idW, adj=path4, nu=2, omega=0.5, K=2, eps=1e-9),
        rec("DirectDeltaMushBind.lean:248-253", "smooth_topk_pou", W=idW, adj=path4, nu=2, omega=0.5, K=4, eps=1e-9),
        rec("DirectDeltaMushBind.lean:257-262", "smooth_topk_pou", W=halfW, adj=path4, nu=1,
            omega=0.3, K=1, eps=1e-9),
    ]
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "known_answers.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(out)} fixtures to {path}")


if __name__ == "__main__":
    main()
