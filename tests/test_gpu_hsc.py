"""The HSC preconditioner (hierarchy from the elimination primitive of
HierarchicalSparsifyCompensate.lean:97-125, V-cycle inside the persistent
solve) against the numpy/scipy restatement in oracle/hsc.py: the level-0
elimination set bit for bit, the hierarchy's shape, the solution against the
oracle's FP64 solve, and the iteration count against the oracle's HSC-PCG."""
import numpy as np
import pytest
import scipy.sparse as sp

from tests.helpers import rel_err, workload
from tool_godot_curvenet_b200 import CutMeshSolver

pytestmark = pytest.mark.gpu


def _oracle_hsc(oracle, pos, tris, h):
    from oracle import hsc as H
    ref = oracle.System(pos, tris, h, ordering=0, precond=0)
    e = ref.export()
    Ap, Ac, Av = e["A"]
    n = Ap.size - 1
    A = sp.csr_matrix((Av, Ac, Ap), shape=(n, n))
    # the product builds the hierarchy on A with the free vertices in
    # ascending vertex order; the oracle's solve order is level-sorted
    perm = np.argsort(e["free_of"], kind="stable")
    A = sp.csr_matrix(A[perm][:, perm])
    A.sort_indices()
    ref.nat_perm = perm
    return ref, A, H.build(A, theta=0.01), H


@pytest.mark.parametrize("name", ["c1", "torus_small", "torus_mid", "c2"])
def test_hsc_solve_matches_oracle(name, oracle):
    pos, tris, h, t = workload(name)
    t = t[:, :3]
    ref, A, hh, H = _oracle_hsc(oracle, pos, tris, h)
    st, xo, _, _ = oracle.System(pos, tris, h).solve(t, mode=1, tol=1e-13)
    with CutMeshSolver(pos, tris, h, precond="hsc") as s:
        nl, tail, nc, off, order = s.hsc_info()
        # level 0 is determined by A's pattern alone: bit-exact
        o0 = hh["levels"][0]["nf"] if hh["levels"] else 0
        assert off[1 if nl else 0] == o0 or nl == 0
        assert np.array_equal(order[:o0], hh["order"][:o0])
        assert abs(nl - len(hh["levels"])) <= 1
        r64 = s.solve(t, mode="deform", precision="fp64", tol=1e-13, max_iter=20000)
        rmx = s.solve(t, mode="deform", precision="mixed", tol=1e-8)
        r8 = s.solve(t, mode="deform", precision="fp64", tol=1e-8)
    assert r64.status == 0 and rmx.status == 0
    assert rel_err(r64.x, xo) <= 1e-9
    assert rel_err(rmx.x, xo) <= 1e-6
    # iteration count against the oracle's FP64 HSC-PCG on the first column
    b = ref.rhs(t, 1)[ref.nat_perm, 0]
    _, it_o = H.pcg(A, b, hh, tol=1e-8)
    assert r8.iterations <= 1.25 * it_o + 3


def test_hsc_apply_is_symmetric_positive_definite(oracle):
    pos, tris, h, _ = workload("torus_small")
    _, A, hh, H = _oracle_hsc(oracle, pos, tris, h)
    rng = np.random.default_rng(3)
    u, v = rng.normal(size=A.shape[0]), rng.normal(size=A.shape[0])
    Mu, Mv = H.apply(hh, u), H.apply(hh, v)
    assert abs(u @ Mv - v @ Mu) <= 1e-10 * abs(u @ Mv)
    assert u @ Mu > 0
