"""IC(0) in mixed precision on a multi-block grid: the triangular sweeps
without grid barriers (every published value carries the number of the
preconditioner application it belongs to; cn_icsf.cu) under the
single-reduction CG.

Reference semantics: SparseLinAlg.lean:104-163 (PCG) with the IC(0) apply of
IncompleteCholesky.lean:83-101.  Checked against the oracle's FP64 IC(0)-PCG
to 1e-13 and against the level-scheduled kernel on the same handle
(algo="classic").  Bars: FP64 to 1e-13 within 1e-9 of the oracle; mixed
precision stopped at 1e-8 within 1e-6 (the mixed bar of the other parity
tests); mixed precision driven to 1e-11 by the FP64 refinement within 1e-8;
the iteration count within 10 % (or 8) of the level-scheduled kernel's (same
preconditioner, same stopping rule, a different CG recurrence)."""
import numpy as np
import pytest

from tests.helpers import rel_err, workload
from tool_godot_curvenet_b200 import CnError, CutMeshSolver
from tool_godot_curvenet_b200 import _lib as L

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-9
MIXED_TOL = 1e-6
TIGHT_TOL = 1e-8

# (mesh, launch): small meshes on forced multi-block grids (one thread per
# row or fewer; several blocks per SM), the 18k-vertex torus on the default
# launch (one block per SM)
CASES = [
    ("torus_small", {"grid": 8, "block": 256}),
    ("torus_small", {"grid": 148, "block": 512}),
    ("torus_small", {"grid": 296, "block": 256}),
    ("c1", {"grid": 4, "block": 128}),
    ("c3_0", {"grid": 16, "block": 512}),
    ("torus_mid", {}),
]


@pytest.mark.parametrize("name,kw", CASES)
@pytest.mark.parametrize("k", [1, 3, 9])
def test_sync_free_ic0_matches_oracle_and_level_scheduled(name, kw, k, oracle):
    pos, tris, h, _ = workload(name)
    rng = np.random.default_rng(100 + k)
    t = rng.normal(size=(h.size, k))
    st, xo, _, _ = oracle.System(pos, tris, h).solve(t, mode=0, tol=1e-13)
    assert st == 0
    with CutMeshSolver(pos, tris, h, max_rhs=k, precond="ic0", **kw) as s:
        assert s.info()["grid"] > 1
        rf = s.solve(t, mode="harmonic", precision="mixed", tol=1e-8, max_iter=20000)
        rs = s.solve(t, mode="harmonic", precision="mixed", tol=1e-8, max_iter=20000, algo="single")
        rt = s.solve(t, mode="harmonic", precision="mixed", tol=1e-11, max_iter=20000)
        rc = s.solve(t, mode="harmonic", precision="mixed", tol=1e-8, max_iter=20000, algo="classic")
        # FP64 takes the sweeps without grid barriers by default from 50,000
        # to 500,000 rows; SINGLE asks for them on any size
        r64 = s.solve(t, mode="harmonic", precision="fp64", tol=1e-13, max_iter=20000, algo="single")
    for r in (rf, rs, rt, rc, r64):
        assert r.status == L.CN_OK
    assert np.all(r64.rel_residual <= 1e-13)
    assert rel_err(r64.x, xo) <= FP64_TOL
    assert np.all(rf.rel_residual <= 1e-8) and np.all(rt.rel_residual <= 1e-11)
    assert rel_err(rf.x, xo) <= MIXED_TOL
    assert rel_err(rt.x, xo) <= TIGHT_TOL
    # FUSED and SINGLE run the same kernel; its runs are deterministic up to
    # the order in which the sweeps' waits end, which changes no value
    assert np.array_equal(rf.x, rs.x) and rf.iterations == rs.iterations
    if k == 9:
        # k = 9 stays on the level-scheduled kernel (one launch for the nine
        # columns): the same solve as CLASSIC
        assert np.array_equal(rf.x, rc.x) and rf.iterations == rc.iterations
    else:
        assert abs(rf.iterations - rc.iterations) <= max(8, 0.1 * rc.iterations)


def test_sync_free_ic0_deform_mode_repeatable(oracle):
    """Deform mode on the 18k-vertex torus, solved three times on one handle:
    every solve restarts the application numbers, so stale words of the
    previous solve are never taken for current ones."""
    pos, tris, h, t = workload("torus_mid")
    t = t[:, :3]
    st, xo, _, _ = oracle.System(pos, tris, h).solve(t, mode=1, tol=1e-13)
    with CutMeshSolver(pos, tris, h, precond="ic0") as s:
        rs = [s.solve(t, mode="deform", precision="mixed", tol=1e-8) for _ in range(3)]
    for r in rs:
        assert r.status == L.CN_OK and np.all(r.rel_residual <= 1e-8)
        assert rel_err(r.x, xo) <= MIXED_TOL
        assert np.array_equal(r.x, rs[0].x)


def test_sync_free_ic0_fp64_matches_level_scheduled(oracle):
    """FP64 (two words a value: the high and the low half, each with the
    application number; SINGLE asks for it below the 50,000 rows where FP64
    takes it by default) against the level-scheduled FP64 kernel and the
    oracle, deform mode on the 18k-vertex torus, twice (bit for bit)."""
    pos, tris, h, t = workload("torus_mid")
    t = t[:, :3]
    st, xo, _, _ = oracle.System(pos, tris, h).solve(t, mode=1, tol=1e-13)
    with CutMeshSolver(pos, tris, h, precond="ic0") as s:
        rs = s.solve(t, mode="deform", precision="fp64", tol=1e-13, max_iter=20000, algo="single")
        rs2 = s.solve(t, mode="deform", precision="fp64", tol=1e-13, max_iter=20000, algo="single")
        rc = s.solve(t, mode="deform", precision="fp64", tol=1e-13, max_iter=20000, algo="classic")
    for r in (rs, rs2, rc):
        assert r.status == L.CN_OK and np.all(r.rel_residual <= 1e-13)
        assert rel_err(r.x, xo) <= FP64_TOL
    assert np.array_equal(rs.x, rs2.x)
    assert abs(rs.iterations - rc.iterations) <= max(8, 0.1 * rc.iterations)


@pytest.mark.parametrize("kw", [{"grid": 8, "block": 256}, {"grid": 148, "block": 512}, {}])
def test_sync_free_ic0_repeats_bit_for_bit(kw):
    """Twenty solves of one system on one handle give the same bits and the
    same iteration count every time: every value a sweep reads is the one of
    the current application (a stale or torn read would change the result of
    some solve), and the reductions sum in a fixed order."""
    pos, tris, h, t = workload("torus_small")
    t = t[:, :3]
    with CutMeshSolver(pos, tris, h, precond="ic0", **kw) as s:
        r0 = s.solve(t, mode="deform", precision="mixed", tol=1e-8)
        for _ in range(19):
            r = s.solve(t, mode="deform", precision="mixed", tol=1e-8)
            assert r.iterations == r0.iterations and r.refinements == r0.refinements
            assert np.array_equal(r.x, r0.x)
