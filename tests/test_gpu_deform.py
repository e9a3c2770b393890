"""Parity of the two-stage DeGoes22 solve (cn_solve_deformation,
DeformSolve.lean:110-135) with the oracle.

* the reference's own known answers (DeformSolve.lean:167-253 and the curve
  examples of EndToEndExample.lean:144-211) on triangleWithSample;
* the dense oracle restatement (orc_solve_deformation: Stage 1, computeFh,
  averageOverFaces, computeYh, Stage 2) on a cut cylinder;
* on larger cut meshes, a composition of oracle pieces: the oracle's k = 9
  harmonic solve, the bridge written out in numpy from the oracle's per-face
  cot Laplacian, and a sparse direct solve of Stage 2 on the oracle's A.
Bars: 1e-9 relative in FP64 (1e-13 residual), 1e-6 in the mixed form."""
import json
import os

import numpy as np
import pytest

from tests.helpers import composed_deformation, random_gradients, rel_err, sample_col, workload
from tool_godot_curvenet_b200 import CnError, CutMeshSolver
from tool_godot_curvenet_b200 import _lib as L

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-9
MIXED_TOL = 1e-6
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")


def _fixtures(kinds):
    with open(GOLDEN) as f:
        return [g for g in json.load(f) if g["kind"] in kinds]


def _segment_gradient(oracle, f):
    O = oracle

    def bez(P, t):
        out = np.empty(3)
        O.lib().orc_bezier3(O.dp(O.f64(P)), t, O.dp(out))
        return out

    rp, rq = bez(f["P_rest"], f["t"]), bez(f["P_rest"], f["t_fwd"])
    pp, pq = bez(f["P_posed"], f["t"]), bez(f["P_posed"], f["t_fwd"])
    F = np.empty(9)
    O.lib().orc_isolated_segment_gradient(O.dp(rp), O.dp(rq), O.dp(pp), O.dp(pq), O.dp(F))
    return F, pp


@pytest.mark.parametrize("fx", _fixtures(("deform", "curve_deform")), ids=lambda f: f["src"])
def test_known_answers(fx, oracle):
    if fx["kind"] == "deform":
        Fc, Xc = np.array(fx["Fc"]), np.array(fx["Xc"])
    else:
        Fc, Xc = _segment_gradient(oracle, fx)
    pos = np.array(fx["pos"])
    with CutMeshSolver(pos, np.array(fx["tris"], np.int32), np.array(fx["handles"], np.int32), max_rhs=9) as s:
        r = s.solve_deformation(Fc.reshape(1, 9), Xc.reshape(1, 3), precision="fp64", tol=1e-13)
    for row, want in fx["rows"].items():
        assert np.all(np.abs(r.x[int(row)] - np.array(want)) < fx["eps"])


def test_dense_oracle_cylinder(oracle):
    pos, tris, h, t = workload("cyl_tiny")
    Fc = random_gradients(h.size, 3)
    he = oracle.halfedges_from_triangles(pos.shape[0], tris)
    want = oracle.solve_deformation(pos.shape[0], tris.shape[0], he, sample_col(pos.shape[0], h), pos, Fc, t)
    want[h] = t  # the spec leaves the promoted slots 0; the product overlays X_c
    with CutMeshSolver(pos, tris, h, max_rhs=9) as s:
        r = s.solve_deformation(Fc, t, precision="fp64", tol=1e-13, max_iter=20000)
        rm = s.solve_deformation(Fc, t, precision="mixed", tol=1e-8)
    assert r.status == 0 and np.all(r.rel_residual <= 1e-13)
    assert rel_err(r.x, want) <= FP64_TOL
    assert rel_err(rm.x, want) <= MIXED_TOL
    assert np.array_equal(r.x[h], t)  # DeformSolve.lean:108-109 overlay


@pytest.mark.parametrize("name", ["c1", "torus_small"])
@pytest.mark.parametrize("precond", ["ic0", "jacobi"])
def test_composed_oracle(name, precond, oracle):
    pos, tris, h, t = workload(name)
    t = t[:, :3]
    Fc = random_gradients(h.size, 7)
    want = composed_deformation(oracle, pos, tris, h, Fc, t)
    with CutMeshSolver(pos, tris, h, max_rhs=9, precond=precond) as s:
        r = s.solve_deformation(Fc, t, precision="fp64", tol=1e-13, max_iter=50000)
        rm = s.solve_deformation(Fc, t, precision="mixed", tol=1e-8, max_iter=50000)
    assert r.status == 0
    assert rel_err(r.x, want) <= FP64_TOL
    assert rel_err(rm.x, want) <= MIXED_TOL


def test_identity_gradient_and_rest_handles_reproduce_rest():
    pos, tris, h, _ = workload("torus_small")
    Fc = np.tile(np.eye(3).ravel(), (h.size, 1))
    with CutMeshSolver(pos, tris, h, max_rhs=9) as s:
        r = s.solve_deformation(Fc, pos[h], precision="fp64", tol=1e-13)
    assert np.abs(r.x - pos).max() < 1e-9


def test_rigid_motion_is_reproduced():
    """F_c = R everywhere and X_c = R rest + t: the solve returns R rest + t."""
    pos, tris, h, _ = workload("c1")
    th = 0.7
    R = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
    tr = np.array([0.3, -1.2, 2.0])
    with CutMeshSolver(pos, tris, h, max_rhs=9) as s:
        r = s.solve_deformation(np.tile(R.ravel(), (h.size, 1)), pos[h] @ R.T + tr, precision="fp64", tol=1e-13)
    assert np.abs(r.x - (pos @ R.T + tr)).max() < 1e-8


def test_needs_nine_rhs_build():
    pos, tris, h, t = workload("cyl_tiny")
    with CutMeshSolver(pos, tris, h) as s:
        with pytest.raises(CnError) as e:
            s.solve_deformation(np.tile(np.eye(3).ravel(), (h.size, 1)), t)
    assert e.value.status == L.CN_BAD_INPUT


def test_nan_gradient_reported():
    pos, tris, h, t = workload("cyl_tiny")
    Fc = np.tile(np.eye(3).ravel(), (h.size, 1))
    Fc[2, 4] = np.nan
    with CutMeshSolver(pos, tris, h, max_rhs=9) as s:
        with pytest.raises(CnError) as e:
            s.solve_deformation(Fc, t)
    assert e.value.status == L.CN_NAN
