"""Parity of the batched, cluster-per-mesh persistent solve with the oracle:
every mesh of a mixed batch (cylinders and tori of uneven size, 1-4 seams,
8 poses x 3 coordinates) against the oracle's FP64 solve of the same mesh,
for several cluster shapes (including fewer clusters than meshes, so the
per-cluster scratch is reused mesh after mesh)."""
import functools

import numpy as np
import pytest

from tests.helpers import rel_err
from tool_godot_curvenet_b200 import BatchSolver, cut_mesh, synth

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-9
MIXED_TOL = 1e-6


@functools.lru_cache(maxsize=None)
def small_batch(n=10, poses=8, seed=40):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        if i % 2:
            U, V = int(rng.integers(24, 64)), int(rng.integers(12, 40))
            ns = int(rng.integers(1, 5))
            m = synth.torus(U, V, cut_u=tuple(sorted({(k * U) // ns for k in range(ns)})), seed=seed + i)
        else:
            a, l = int(rng.integers(10, 40)), int(rng.integers(10, 60))
            ns = int(rng.integers(1, 4))
            rows = tuple(sorted({1 + (k + 1) * (l - 2) // (ns + 1) for k in range(ns)}))
            m = synth.cylinder(a, l, cut_rows=rows, seed=seed + i)
        h = synth.pick_handles(m, 0.03, seed + 100 + i)
        t = synth.normal_targets(m.positions, h, 0.1, seed + 200 + i, poses=poses)
        tris, parent = cut_mesh(m.positions.shape[0], m.tris, m.loops)
        out.append((np.ascontiguousarray(m.positions[parent]), tris, h, t))
    return tuple(out)


@functools.lru_cache(maxsize=None)
def oracle_solutions(poses=8):
    from oracle import oracle as O
    sols = []
    for pos, tris, h, t in small_batch(poses=poses):
        st, x, _, _ = O.System(pos, tris, h).solve(t, mode=1, tol=1e-13)
        assert st == 0
        sols.append(x)
    return sols


@pytest.mark.parametrize("csize,nclusters", [(4, 0), (1, 3), (2, 2), (8, 0), (16, 0)])
def test_batch_matches_oracle_fp64_and_mixed(csize, nclusters):
    meshes = small_batch()
    ref = oracle_solutions()
    with BatchSolver([(p, t, h) for p, t, h, _ in meshes], k=24, cluster_size=csize, n_clusters=nclusters) as B:
        xs, st = B.solve([m[3] for m in meshes], precision="fp64", tol=1e-13)
        assert st.status == 0 and st.n_failed == 0
        assert st.max_rel_residual <= 1e-13
        for x, xo in zip(xs, ref):
            assert rel_err(x, xo) <= FP64_TOL
        xs, st = B.solve([m[3] for m in meshes], precision="mixed", tol=1e-8)
        assert st.status == 0 and st.max_rel_residual <= 1e-8
        for x, xo in zip(xs, ref):
            assert rel_err(x, xo) <= MIXED_TOL
        sts, its, rel = B.mesh_stats()
        assert np.all(sts == 0) and np.all(rel <= 1e-8) and np.all(its > 0)


def test_batch_three_rhs_and_repeated_graph_launch():
    meshes = small_batch(poses=1)
    ref = oracle_solutions(poses=1)
    with BatchSolver([(p, t, h) for p, t, h, _ in meshes], k=3) as B:
        for _ in range(3):  # the captured graph is reused
            xs, st = B.solve([m[3] for m in meshes], precision="mixed", tol=1e-8)
            assert st.status == 0
            for x, xo in zip(xs, ref):
                assert rel_err(x, xo) <= MIXED_TOL


def test_batch_matches_single_mesh_solver():
    from tool_godot_curvenet_b200 import CutMeshSolver
    meshes = small_batch()
    with BatchSolver([(p, t, h) for p, t, h, _ in meshes], k=24) as B:
        xs, _ = B.solve([m[3] for m in meshes], precision="fp64", tol=1e-12)
    for (pos, tris, h, t), xb in zip(meshes[:3], xs[:3]):
        with CutMeshSolver(pos, tris, h) as s:
            for p in range(8):
                r = s.solve(t[:, 3 * p:3 * p + 3], precision="fp64", tol=1e-12)
                assert rel_err(xb[:, 3 * p:3 * p + 3], r.x) <= 1e-9


@pytest.mark.parametrize("precond", ["jacobi", "ic0"])
def test_batch_preconditioners_converge_to_oracle(precond):
    """Both batch preconditioners (the inner dot (r, M^-1 r) is taken as
    ||L^-1 r||^2 from the forward sweep; A p by the recurrence A z + beta A p';
    x += alpha p one pass late) reach the oracle's solution in FP64 and mixed
    precision, including a run with too few iterations that must report
    max_iter rather than a wrong answer."""
    meshes = small_batch()
    ref = oracle_solutions()
    with BatchSolver([(p, t, h) for p, t, h, _ in meshes], k=24, precond=precond) as B:
        for precision, tol, bar in [("fp64", 1e-13, FP64_TOL), ("mixed", 1e-8, MIXED_TOL)]:
            xs, st = B.solve([m[3] for m in meshes], precision=precision, tol=tol, max_iter=20000)
            assert st.status == 0 and st.max_rel_residual <= tol
            for x, xo in zip(xs, ref):
                assert rel_err(x, xo) <= bar
        xs, st = B.solve([m[3] for m in meshes], precision="fp64", tol=1e-13, max_iter=3, check=False)
        assert st.n_failed > 0


@pytest.mark.parametrize("nclusters", [0, 1])
def test_batch_lanes_per_size_class_match_oracle(nclusters):
    """Rows per warp per size class (cn_batch_set_lanes): the small meshes at
    4 lanes per row, the large ones at 8, in one graph launch (two kernels
    side by side, or one after the other with a single cluster), FP64 and
    mixed against the oracle."""
    meshes = small_batch()
    ref = oracle_solutions()
    with BatchSolver([(p, t, h) for p, t, h, _ in meshes], k=24, n_clusters=nclusters) as B:
        B.set_lanes([600, 1 << 30], [4, 8])
        lanes = B.lanes()
        assert set(lanes.tolist()) == {4, 8}
        for precision, tol, bar in [("fp64", 1e-13, FP64_TOL), ("mixed", 1e-8, MIXED_TOL)]:
            xs, st = B.solve([m[3] for m in meshes], precision=precision, tol=tol, max_iter=20000)
            assert st.status == 0 and st.n_failed == 0 and st.max_rel_residual <= tol
            for x, xo in zip(xs, ref):
                assert rel_err(x, xo) <= bar
        B.set_lanes([1 << 30], [4])  # every mesh at 4 lanes per row
        xs, st = B.solve([m[3] for m in meshes], precision="mixed", tol=1e-8)
        assert st.status == 0
        for x, xo in zip(xs, ref):
            assert rel_err(x, xo) <= MIXED_TOL
