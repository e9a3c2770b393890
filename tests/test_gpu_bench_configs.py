"""Parity on the workloads the benchmark figures are quoted on, through the
exact handles and calls bench.py times.

* torus 512 x 256 (131,072 vertices, 8 seams, 2% handles, 3 RHS): the block
  SSOR handle with the default launch (one block per SM, automatic block
  size), mixed precision to 1e-8 through the device-pointer call and through
  cn_solve with host buffers; the FP64 solve of the same handle; the Jacobi
  handle in mixed precision (two-reduction form), FP64 (pipelined form) and
  the plain one-kernel-per-primitive FP64 PCG; the level-scheduled IC(0)
  solve.
* the batch workload: 20 of the 512 meshes of the batch (the 8 largest, near
  60k vertices, the 4 smallest, 4 from the middle of the size order and
  meshes 0-3), 8 poses x 3 coordinates, in one graph launch, FP64 and mixed.
* torus 1024 x 1024 (1.05M vertices, 16 seams, 1% handles; marked slow):
  IC(0), HSC and block SSOR in mixed precision, FP64 IC(0).

Reference semantics: SparseLinAlg.lean:104-163 (PCG), DeformSolve.lean:123-135
(Stage 2 with F_f = I, handles overlaid).  The oracle solves every case in
FP64 IC(0)-PCG to 1e-13 relative residual.  Bars:

* FP64 solves to 1e-13: within 1e-9 relative of the oracle;
* mixed-precision solves driven to 1e-11 by the FP64 refinement: within 1e-8
  (this isolates the FP32 arithmetic from the stopping rule);
* solves stopped at 1e-8 relative residual (the benchmark's tolerance):
  within 5x the error of the oracle's own FP64 solve stopped at 1e-8, which
  lies 4.1e-7 (131k-vertex torus) and 1.9e-6 (1.05M-vertex torus) from its
  1e-13 solution: 2e-6 and 1e-5."""
import ctypes as C
import functools

import numpy as np
import pytest

from tests.helpers import rel_err, workload
from tool_godot_curvenet_b200 import BatchSolver, CutMeshSolver, cut_mesh, synth
from tool_godot_curvenet_b200 import _lib as L

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-9
TIGHT_TOL = 1e-8  # mixed precision refined to 1e-11
STOP_TOL = 2e-6  # solves stopped at 1e-8 relative residual, meshes up to 131k vertices
STOP_TOL_C5 = 1e-5  # the same on the 1.05M-vertex torus

# indices of the batch workload's meshes checked here (sizes from synth.config3_mesh)
C3_LARGEST = (486, 186, 180, 256, 464, 272, 172, 428)  # 57k-60k vertices
C3_SMALLEST = (211, 475, 317, 204)  # ~2k vertices
C3_MIDDLE = (307, 300, 436, 384)  # ~10k vertices
C3_INDICES = C3_LARGEST + C3_SMALLEST + C3_MIDDLE + (0, 1, 2, 3)


@functools.lru_cache(maxsize=None)
def oracle_solution(name, tol=1e-13):
    from oracle import oracle as O
    pos, tris, h, t = workload(name)
    t = t[:, :3] if name in ("c2", "c5") else t
    st, x, _, rel = O.System(pos, tris, h).solve(t, mode=1, tol=tol, threads=3)
    assert st == 0 and np.all(rel <= 2 * tol)  # the oracle stops on its recursive residual
    return x


def _check(r, tol):
    assert r.status == 0
    assert np.all(r.rel_residual <= tol)


def test_c2_headline_handle_matches_oracle():
    """The headline: block SSOR handle, default launch, mixed to 1e-8 through
    cn_solve_device (the timed call) and cn_solve (the end-to-end call)."""
    import torch
    pos, tris, h, t = workload("c2")
    xo = oracle_solution("c2")
    with CutMeshSolver(pos, tris, h, precond="bssor") as s:
        info = s.info()
        assert info["grid"] > 1  # the cooperative row-cached launch, not the one-block path
        d_t = torch.from_numpy(t).cuda()
        d_x = torch.empty((pos.shape[0], 3), dtype=torch.float64, device="cuda")
        st = s.solve_device(3, d_t.data_ptr(), d_x.data_ptr(), stats=True, mode="deform",
                            precision="mixed", algo="fused", tol=1e-8)
        assert st.status == 0 and st.max_rel_residual <= 1e-8
        assert rel_err(d_x.cpu().numpy(), xo) <= STOP_TOL
        # the same solve through cn_solve with pinned host buffers (bench e2e leg)
        h_t = torch.from_numpy(t.copy()).pin_memory()
        h_x = torch.empty((pos.shape[0], 3), dtype=torch.float64).pin_memory()
        o = CutMeshSolver.make_opts(mode="deform", precision="mixed", tol=1e-8)
        stt = L.SolveStats()
        DP = C.POINTER(C.c_double)
        rc = L.lib().cn_solve(s._h, 3, C.cast(h_t.data_ptr(), DP), None, C.cast(h_x.data_ptr(), DP),
                              C.byref(o), C.byref(stt))
        assert rc == 0 and stt.max_rel_residual <= 1e-8
        x = h_x.numpy()
        assert rel_err(x, xo) <= STOP_TOL
        assert np.array_equal(x[h], t)  # handles overlaid (DeformSolve.lean:108-109)
        # FP64 on the same handle (block SSOR lists in global memory at this size)
        r = s.solve(t, mode="deform", precision="fp64", tol=1e-13, max_iter=20000)
        _check(r, 1e-13)
        assert rel_err(r.x, xo) <= FP64_TOL
        r = s.solve(t, mode="deform", precision="mixed", tol=1e-11, max_refine=30)
        _check(r, 1e-11)
        assert rel_err(r.x, xo) <= TIGHT_TOL


@pytest.mark.parametrize("precision,algo", [("mixed", "fused"), ("fp64", "fused"), ("mixed", "pipelined"),
                                            ("fp64", "plain")])
def test_c2_jacobi_variants_match_oracle(precision, algo):
    pos, tris, h, t = workload("c2")
    xo = oracle_solution("c2")
    with CutMeshSolver(pos, tris, h, precond="jacobi") as s:
        r = s.solve(t, mode="deform", precision=precision, algo=algo, tol=1e-8, max_iter=100000)
        _check(r, 1e-8)
        assert rel_err(r.x, xo) <= STOP_TOL
        if algo == "fused" and precision == "fp64":
            r = s.solve(t, mode="deform", precision="fp64", tol=1e-13, max_iter=20000)
            _check(r, 1e-13)
            assert rel_err(r.x, xo) <= FP64_TOL


def test_c2_ic0_matches_oracle():
    """IC(0): mixed precision through the default call (the sweeps without
    grid barriers) and the level-scheduled kernel (classic), FP64."""
    pos, tris, h, t = workload("c2")
    xo = oracle_solution("c2")
    with CutMeshSolver(pos, tris, h, precond="ic0") as s:
        for algo in ("fused", "classic"):
            r = s.solve(t, mode="deform", precision="mixed", tol=1e-8, algo=algo)
            _check(r, 1e-8)
            assert rel_err(r.x, xo) <= STOP_TOL
            r = s.solve(t, mode="deform", precision="mixed", tol=1e-11, max_refine=30, algo=algo)
            _check(r, 1e-11)
            assert rel_err(r.x, xo) <= TIGHT_TOL
        r = s.solve(t, mode="deform", precision="fp64", tol=1e-13, max_iter=20000)
        _check(r, 1e-13)
        assert rel_err(r.x, xo) <= FP64_TOL


@functools.lru_cache(maxsize=None)
def c3_meshes():
    out = []
    for i in C3_INDICES:
        m, h, t = synth.config3_mesh(i)
        tris, parent = cut_mesh(m.positions.shape[0], m.tris, m.loops)
        out.append((np.ascontiguousarray(m.positions[parent]), tris, h, t))
    return out


@functools.lru_cache(maxsize=None)
def c3_oracle():
    from oracle import oracle as O
    sols = []
    for pos, tris, h, t in c3_meshes():
        st, x, _, rel = O.System(pos, tris, h).solve(t, mode=1, tol=1e-13, threads=8)
        assert st == 0
        sols.append(x)
    return sols


def test_c3_batch_meshes_match_oracle():
    """The batch handle as bench.py builds it (IC(0), default cluster shape,
    k = 24) on real meshes of the batch workload, up to 60k vertices."""
    meshes = c3_meshes()
    assert max(p.shape[0] for p, _, _, _ in meshes) > 57000
    ref = c3_oracle()
    with BatchSolver([(p, t, h) for p, t, h, _ in meshes], k=24) as B:
        xs, st = B.solve([m[3] for m in meshes], precision="fp64", tol=1e-13, max_iter=20000)
        assert st.status == 0 and st.n_failed == 0 and st.max_rel_residual <= 1e-13
        for x, xo in zip(xs, ref):
            assert rel_err(x, xo) <= FP64_TOL
        xs, st = B.solve([m[3] for m in meshes], precision="mixed", tol=1e-8)
        assert st.status == 0 and st.n_failed == 0 and st.max_rel_residual <= 1e-8
        for (pos, tris, h, t), x, xo in zip(meshes, xs, ref):
            assert rel_err(x, xo) <= STOP_TOL
            assert np.array_equal(x[h], t)
        xs, st = B.solve([m[3] for m in meshes], precision="mixed", tol=1e-11, max_refine=30)
        assert st.status == 0 and st.n_failed == 0 and st.max_rel_residual <= 1e-11
        for x, xo in zip(xs, ref):
            assert rel_err(x, xo) <= TIGHT_TOL


@pytest.mark.slow
def test_c5_solvers_match_oracle():
    """torus 1024 x 1024: IC(0), HSC and block SSOR in mixed precision and
    FP64 IC(0), each against the oracle's FP64 IC(0) solve to 1e-13."""
    pos, tris, h, t = workload("c5")
    xo = oracle_solution("c5")
    for precond in ("ic0", "hsc", "bssor"):
        with CutMeshSolver(pos, tris, h, precond=precond) as s:
            r = s.solve(t, mode="deform", precision="mixed", tol=1e-8, max_iter=20000)
            _check(r, 1e-8)
            assert rel_err(r.x, xo) <= STOP_TOL_C5, precond
            if precond == "ic0":
                r = s.solve(t, mode="deform", precision="mixed", tol=1e-11, max_iter=3000, max_refine=30)
                _check(r, 1e-11)
                assert rel_err(r.x, xo) <= TIGHT_TOL
                r = s.solve(t, mode="deform", precision="fp64", tol=1e-13, max_iter=40000)
                _check(r, 1e-13)
                assert rel_err(r.x, xo) <= FP64_TOL


@pytest.mark.parametrize("precond", ["bssor", "jacobi"])
def test_c2_single_reduction_form_matches_oracle(precond):
    pos, tris, h, t = workload("c2")
    xo = oracle_solution("c2")
    with CutMeshSolver(pos, tris, h, precond=precond) as s:
        r = s.solve(t, mode="deform", precision="mixed", algo="single", tol=1e-8)
        _check(r, 1e-8)
        assert rel_err(r.x, xo) <= STOP_TOL
        r = s.solve(t, mode="deform", precision="mixed", algo="single", tol=1e-11, max_refine=30)
        _check(r, 1e-11)
        assert rel_err(r.x, xo) <= TIGHT_TOL
        r = s.solve(t, mode="deform", precision="fp64", algo="single", tol=1e-13, max_iter=20000)
        _check(r, 1e-13)
        assert rel_err(r.x, xo) <= FP64_TOL
