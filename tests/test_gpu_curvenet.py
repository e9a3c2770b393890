"""The curve side on the GPU (cn_bind_curvenet, cn_curvenet_constraints,
cn_deform_curvenet): per-handle F_c and X_c from posed profile curves
(ScaledFrames.lean, SegmentGradient.lean, IntersectionFrames.lean,
CurveInterp.lean, EndToEndExample.lean:52-60), then the two-stage solve
(DeformSolve.lean:110-135).

Bars: F_c and X_c equal the oracle's restatement bit for bit (the kernels keep
the reference's operation order without FMA contraction); the reference's own
known answers (isolated rotation R_z(90), scaling, identity pose of an
intersection net) to 1e-12; the deformed positions of cn_deform_curvenet
equal cn_solve_deformation fed with the same F_c / X_c bit for bit and lie
within 1e-9 relative of the oracle composition (FP64 solves to 1e-13)."""
import numpy as np
import pytest

from tests.helpers import composed_deformation, line_curve, loop_curvenet, rel_err, star_curvenet, workload
from tool_godot_curvenet_b200 import CnError, CutMeshSolver

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-9


def _bind(s, net):
    s.bind_curvenet(net["rest_cp"], net["sample_tau"], net["handle_curve"], net["handle_sample"],
                    net["handle_side"], closed=net["closed"], node_ptr=net["node_ptr"], node_ends=net["node_ends"])


def test_intersection_net_bit_exact_with_oracle(oracle):
    pos, tris, h, _ = workload("torus_small")
    net, rest_cp = star_curvenet(h.size, seed=3)
    rng = np.random.default_rng(8)
    posed = rest_cp[None] + rng.normal(0.0, 0.08, (5,) + rest_cp.shape)
    posed[0] = rest_cp
    with CutMeshSolver(pos, tris, h, precond="jacobi", max_rhs=9) as s:
        _bind(s, net)
        F, X = s.curvenet_constraints(posed)
        F2, X2 = s.curvenet_constraints(posed[1:3])  # a second call with fewer poses reuses the scratch
    Fo, Xo = oracle.curvenet_constraints(net, pos, h, posed)
    assert np.array_equal(F.view(np.uint64), Fo.view(np.uint64))
    assert np.array_equal(X.view(np.uint64), Xo.view(np.uint64))
    assert np.array_equal(F2, Fo[1:3]) and np.array_equal(X2, Xo[1:3])
    # SegmentGradient.lean:104-113: rest = posed gives F = I on both sides
    assert np.abs(F[0] - np.eye(3)).max() < 1e-12
    unbound = net["handle_curve"] < 0
    assert np.array_equal(F[:, unbound], np.broadcast_to(np.eye(3), F[:, unbound].shape))
    assert np.array_equal(X[:, unbound], np.broadcast_to(pos[h[unbound]], X[:, unbound].shape))


def test_isolated_known_answers_on_gpu():
    """ScaledFrames.lean:168-171 and :182-185 through the GPU path: a straight
    rest curve along +x posed along +y gives R_z(90); stretched to twice its
    length along +x, 2 I.  X_c is the posed sample (EndToEndExample.lean)."""
    pos, tris, h, _ = workload("cyl_tiny")
    rest = line_curve([0, 0, 0], [1, 0, 0], 1)[None]
    rot = line_curve([0, 0, 0], [0, 1, 0], 1)[None]
    stretch = line_curve([0, 0, 0], [2, 0, 0], 1)[None]
    nh = h.size
    net = dict(rest_cp=rest, sample_tau=np.array([[0.0, 0.25, 0.5, 0.75]]), closed=np.zeros(1, np.int32),
               node_ptr=np.zeros(1, np.int32), node_ends=np.zeros(0, np.int32),
               handle_curve=np.zeros(nh, np.int32), handle_sample=(np.arange(nh) % 4).astype(np.int32),
               handle_side=np.zeros(nh, np.int32))
    RZ = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    with CutMeshSolver(pos, tris, h, max_rhs=9) as s:
        _bind(s, net)
        F, X = s.curvenet_constraints(np.stack([rot, stretch]))
    assert np.abs(F[0] - RZ).max() < 1e-12
    assert np.abs(F[1] - 2.0 * np.eye(3)).max() < 1e-12
    tau = net["sample_tau"][0][net["handle_sample"]]
    assert np.abs(X[0] - np.stack([0 * tau, tau, 0 * tau], 1)).max() < 1e-12
    assert np.abs(X[1] - np.stack([2 * tau, 0 * tau, 0 * tau], 1)).max() < 1e-12


@pytest.mark.parametrize("precond", ["ic0", "jacobi"])
def test_deform_curvenet_matches_two_stage_and_oracle(precond, oracle):
    """Closed seam curves of the torus 128 x 64 workload (isolated curves;
    seam vertex on the plus side, its copy on the minus side)."""
    pos, tris, h, net = loop_curvenet()
    rng = np.random.default_rng(12)
    posed = net["rest_cp"] + rng.normal(0.0, 0.03, net["rest_cp"].shape)
    with CutMeshSolver(pos, tris, h, precond=precond, max_rhs=9) as s:
        _bind(s, net)
        F, X = s.curvenet_constraints(posed[None])
        r = s.deform_curvenet(posed, precision="fp64", tol=1e-13, max_iter=20000)
        r2 = s.solve_deformation(F[0].reshape(-1, 9), X[0], precision="fp64", tol=1e-13, max_iter=20000)
        rm = s.deform_curvenet(posed, precision="mixed", tol=1e-10, max_refine=20)
    Fo, Xo = oracle.curvenet_constraints(net, pos, h, posed[None])
    assert np.array_equal(F, Fo) and np.array_equal(X, Xo)
    assert np.array_equal(r.x, r2.x)
    assert np.array_equal(r.x[h], X[0])
    want = composed_deformation(oracle, pos, tris, h, Fo[0].reshape(-1, 9), Xo[0])
    assert rel_err(r.x, want) <= FP64_TOL
    assert rel_err(rm.x, want) <= 1e-7


def test_bind_rejects_malformed_nets():
    pos, tris, h, _ = workload("cyl_tiny")
    net, rest_cp = star_curvenet(h.size)
    with CutMeshSolver(pos, tris, h, max_rhs=9) as s:
        bad = dict(net)
        bad["node_ends"] = net["node_ends"].copy()
        bad["node_ends"][1] = bad["node_ends"][0]  # one curve end used twice
        with pytest.raises(CnError):
            _bind(s, bad)
        bad = dict(net)
        bad["sample_tau"] = net["sample_tau"][:, ::-1].copy()  # parameters must rise
        with pytest.raises(CnError):
            _bind(s, bad)
        with pytest.raises(CnError):
            s.deform_curvenet(rest_cp)  # nothing bound yet
