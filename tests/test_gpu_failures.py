"""Failure paths of the solve, made without a GPU fault (SparseLinAlg.lean:89-97,118
are the reference's degenerate cases; here they are status codes):

* a bounded device-side wait that runs out: a multi-block solve given a
  wait limit far below one grid barrier's duration ends with CN_TIMEOUT (no
  hang: every block leaves at its next barrier once one block has raised
  the abort flag), and the same handle then solves cleanly with the default
  limit;
* an IC(0) factor whose pivots stay non-positive through the diagonal-shift
  retries (A + s diag(A), s in {1e-3, 1e-2, 1e-1}) makes cn_build return
  CN_NONPOS_PIVOT, while a Jacobi build of the same mesh solves;
* too few iterations report CN_MAX_ITER with the residual reached."""
import numpy as np
import pytest

from tests.helpers import pivot_breakdown_mesh, rel_err, workload
from tool_godot_curvenet_b200 import CnError, CutMeshSolver
from tool_godot_curvenet_b200 import _lib as L

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precond,precision", [("bssor", "mixed"), ("jacobi", "fp64"), ("jacobi", "mixed"),
                                               ("ic0", "mixed"), ("ic0", "fp64")])
def test_wait_limit_ends_solve_with_timeout_then_handle_recovers(precond, precision, oracle):
    pos, tris, h, t = workload("torus_mid")
    t = t[:, :3]
    with CutMeshSolver(pos, tris, h, precond=precond) as s:
        assert s.info()["grid"] > 1  # a cooperative multi-block launch with grid barriers
        r = s.solve(t, mode="deform", precision=precision, tol=1e-8, wait_limit_ms=1e-6, check=False)
        assert r.status == L.CN_TIMEOUT
        with pytest.raises(CnError) as e:
            s.solve(t, mode="deform", precision=precision, tol=1e-8, wait_limit_ms=1e-6)
        assert e.value.status == L.CN_TIMEOUT
        r = s.solve(t, mode="deform", precision=precision, tol=1e-8)
        assert r.status == L.CN_OK and np.all(r.rel_residual <= 1e-8)
    st, xo, _, _ = oracle.System(pos, tris, h).solve(t, mode=1, tol=1e-13)
    assert st == 0
    assert rel_err(r.x, xo) <= 2e-6


def test_nonpositive_pivot_after_shift_retries(oracle):
    pos, tris, h = pivot_breakdown_mesh()
    ref = oracle.System(pos, tris, h, ordering=1)
    assert ref.status == L.CN_NONPOS_PIVOT
    with pytest.raises(CnError) as e:
        CutMeshSolver(pos, tris, h, precond="ic0")
    assert e.value.status == L.CN_NONPOS_PIVOT
    targets = pos[h] + 0.1
    with CutMeshSolver(pos, tris, h, precond="jacobi") as s:
        r = s.solve(targets, mode="deform", precision="fp64", tol=1e-12, max_iter=20000)
    refj = oracle.System(pos, tris, h, precond=0)
    st, xo, _, _ = refj.solve(targets, mode=1, tol=1e-13)
    assert st == 0 and rel_err(r.x, xo) <= 1e-8


def test_max_iter_is_reported_not_a_wrong_answer():
    pos, tris, h, t = workload("torus_mid")
    with CutMeshSolver(pos, tris, h, precond="bssor") as s:
        r = s.solve(t[:, :3], mode="deform", precision="fp64", tol=1e-13, max_iter=5, max_refine=1, check=False)
        assert r.status == L.CN_MAX_ITER
        assert r.rel_residual.max() > 1e-13
