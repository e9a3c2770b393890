"""Parity of the CUDA path (through the C ABI) with the CPU FP64 oracle.

Bars: sparsity pattern, cut topology, elimination order and assembled FP64
values bit-exact; the FP64 IC(0) factor bit-exact (same order, no FMA
contraction on either side); deformed positions within 1e-9 relative of the
oracle in FP64 (both sides solved to 1e-13 relative residual) and within
1e-6 relative in the mixed FP32/FP64-refinement form at 1e-8 residual."""
import numpy as np
import pytest

from tests.helpers import rel_err, workload
from tool_godot_curvenet_b200 import CnError, CutMeshSolver
from tool_godot_curvenet_b200 import _lib as L

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-9
MIXED_TOL = 1e-6


def _dense_from(ptr, col, val, n):
    D = np.zeros((n, n))
    for i in range(n):
        D[i, col[ptr[i]:ptr[i + 1]]] = val[ptr[i]:ptr[i + 1]]
    return D


@pytest.mark.parametrize("name", ["cyl_tiny", "c1", "torus_small"])
@pytest.mark.parametrize("lap", ["cot", "robust"])
def test_assembly_bit_exact(name, lap, oracle):
    pos, tris, h, _ = workload(name)
    kind = 1 if lap == "robust" else 0
    with CutMeshSolver(pos, tris, h, laplacian=lap, mollify_delta=1e-3) as s:
        p, c, v = s.export_k()
    po, co, vo = oracle.assemble_csr(pos.shape[0], tris, pos, kind, 1e-3)
    assert np.array_equal(p, po) and np.array_equal(c, co)
    assert np.array_equal(v.view(np.uint64), vo.view(np.uint64))


@pytest.mark.parametrize("name", ["cyl_tiny", "c1", "torus_small"])
@pytest.mark.parametrize("ordering", ["color", "natural"])
def test_reduction_order_and_factor_bit_exact(name, ordering, oracle):
    pos, tris, h, _ = workload(name)
    with CutMeshSolver(pos, tris, h, ordering=ordering) as s:
        free_of, Ap, Ac, Av = s.export_csr()
        Lp, Lc, Lv = s.export_factor()
        info = s.info()
    ref = oracle.System(pos, tris, h, ordering=1 if ordering == "color" else 0)
    assert ref.status == 0
    e = ref.export()
    assert np.array_equal(free_of, e["free_of"])
    assert np.array_equal(Ap, e["A"][0]) and np.array_equal(Ac, e["A"][1])
    assert np.array_equal(Av.view(np.uint64), e["A"][2].view(np.uint64))
    assert np.array_equal(Lp, e["L"][0]) and np.array_equal(Lc, e["L"][1])
    assert np.array_equal(Lv.view(np.uint64), e["L"][2].view(np.uint64))
    assert info["n_levels"] == ref.n_levels


@pytest.mark.parametrize("name", ["cyl_tiny", "c1", "torus_small", "c3_0"])
@pytest.mark.parametrize("precond", ["ic0", "jacobi"])
def test_deform_solve_fp64_matches_oracle(name, precond, oracle):
    pos, tris, h, t = workload(name)
    t = t[:, :3]
    ref = oracle.System(pos, tris, h, precond=1)
    st, xo, _, _ = ref.solve(t, mode=1, tol=1e-13)
    assert st == 0
    with CutMeshSolver(pos, tris, h, precond=precond) as s:
        r = s.solve(t, mode="deform", precision="fp64", tol=1e-13, max_iter=20000)
    assert r.status == 0
    assert np.all(r.rel_residual <= 1e-13)
    assert rel_err(r.x, xo) <= FP64_TOL


@pytest.mark.parametrize("name", ["cyl_tiny", "c1", "torus_small", "c3_0"])
def test_deform_solve_mixed_matches_oracle(name, oracle):
    pos, tris, h, t = workload(name)
    t = t[:, :3]
    ref = oracle.System(pos, tris, h)
    st, xo, _, _ = ref.solve(t, mode=1, tol=1e-13)
    with CutMeshSolver(pos, tris, h) as s:
        r = s.solve(t, mode="deform", precision="mixed", tol=1e-8)
    assert r.status == 0
    assert np.all(r.rel_residual <= 1e-8)
    assert rel_err(r.x, xo) <= MIXED_TOL


@pytest.mark.parametrize("name", ["c1", "torus_small"])
def test_harmonic_mode_matches_oracle(name, oracle):
    pos, tris, h, t = workload(name)
    t = t[:, :3]
    ref = oracle.System(pos, tris, h)
    st, xo, _, _ = ref.solve(t, mode=0, tol=1e-13)
    with CutMeshSolver(pos, tris, h) as s:
        r = s.solve(t, mode="harmonic", precision="fp64", tol=1e-13)
    assert rel_err(r.x, xo) <= FP64_TOL


def test_rhs_matches_oracle_and_handles_overlaid(oracle):
    pos, tris, h, t = workload("c1")
    with CutMeshSolver(pos, tris, h) as s:
        r = s.solve(t, mode="deform", precision="fp64", tol=1e-12)
    assert np.array_equal(r.x[h], t)  # DeformSolve.lean:108-109 overlay


def test_identity_pose_reproduces_rest():
    pos, tris, h, _ = workload("torus_small")
    with CutMeshSolver(pos, tris, h) as s:
        r = s.solve(pos[h], mode="deform", precision="fp64", tol=1e-12)
    assert np.abs(r.x - pos).max() < 1e-9


def test_plain_fp64_path_matches(oracle):
    pos, tris, h, t = workload("c1")
    ref = oracle.System(pos, tris, h)
    st, xo, _, _ = ref.solve(t, mode=1, tol=1e-13)
    with CutMeshSolver(pos, tris, h) as s:
        r = s.solve(t, mode="deform", precision="fp64", algo="plain", tol=1e-11, max_iter=100000)
    assert r.status == 0
    assert rel_err(r.x, xo) <= 1e-7


def test_warm_start_converges_faster_to_same_answer():
    pos, tris, h, t = workload("torus_small")
    with CutMeshSolver(pos, tris, h) as s:
        a = s.solve(t, mode="deform", precision="fp64", tol=1e-10)
        b = s.solve(t * 1.0, mode="deform", precision="fp64", tol=1e-10, warm_start=True)
    assert b.iterations < a.iterations
    assert rel_err(b.x, a.x) < 1e-8


def test_x0_initial_guess():
    pos, tris, h, t = workload("c1")
    with CutMeshSolver(pos, tris, h) as s:
        a = s.solve(t, mode="deform", precision="fp64", tol=1e-12)
        b = s.solve(t, x0=a.x, mode="deform", precision="fp64", tol=1e-10)
    assert b.iterations == 0
    assert rel_err(b.x, a.x) < 1e-12


@pytest.mark.parametrize("k", [1, 9])
def test_other_rhs_counts(k, oracle):
    pos, tris, h, _ = workload("torus_small")
    rng = np.random.default_rng(5)
    t = rng.normal(size=(h.size, k))
    ref = oracle.System(pos, tris, h)
    st, xo, _, _ = ref.solve(t, mode=0, tol=1e-13)
    with CutMeshSolver(pos, tris, h, max_rhs=k) as s:
        r = s.solve(t, mode="harmonic", precision="fp64", tol=1e-13)
        rm = s.solve(t, mode="harmonic", precision="mixed", tol=1e-8)
    assert rel_err(r.x, xo) <= FP64_TOL
    assert rel_err(rm.x, xo) <= MIXED_TOL


@pytest.mark.parametrize("grid,block,lanes", [(1, 256, 1), (1, 1024, 8), (8, 256, 2), (148, 512, 4), (296, 256, 16)])
def test_launch_shapes_agree(grid, block, lanes, oracle):
    pos, tris, h, t = workload("torus_small")
    ref = oracle.System(pos, tris, h)
    st, xo, _, _ = ref.solve(t, mode=1, tol=1e-13)
    with CutMeshSolver(pos, tris, h, grid=grid, block=block, lanes=lanes) as s:
        r = s.solve(t, mode="deform", precision="fp64", tol=1e-13)
        rm = s.solve(t, mode="deform", precision="mixed", tol=1e-8)
    assert rel_err(r.x, xo) <= FP64_TOL
    assert rel_err(rm.x, xo) <= MIXED_TOL


# ----------------------------------------------------------------- errors
def test_singular_component_reported():
    pos, tris, h, _ = workload("c1")
    top_only = h[h >= 64]  # the bottom band keeps no handle
    with pytest.raises(CnError) as e:
        CutMeshSolver(pos, tris, top_only)
    assert e.value.status == L.CN_SINGULAR_COMPONENT


def test_nan_positions_reported():
    pos, tris, h, _ = workload("cyl_tiny")
    pos = pos.copy()
    pos[5, 1] = np.nan
    with pytest.raises(CnError) as e:
        CutMeshSolver(pos, tris, h)
    assert e.value.status == L.CN_NAN


def test_bad_triangles_reported():
    pos, tris, h, _ = workload("cyl_tiny")
    bad = tris.copy()
    bad[3, 1] = pos.shape[0] + 5
    with pytest.raises(CnError) as e:
        CutMeshSolver(pos, bad, h)
    assert e.value.status == L.CN_BAD_INPUT
    dup = np.concatenate([h, h[:1]])
    with pytest.raises(CnError) as e:
        CutMeshSolver(pos, tris, dup)
    assert e.value.status == L.CN_BAD_INPUT


def test_nan_targets_reported():
    pos, tris, h, t = workload("cyl_tiny")
    t = t.copy()
    t[0, 0] = np.inf
    with CutMeshSolver(pos, tris, h) as s:
        with pytest.raises(CnError) as e:
            s.solve(t)
    assert e.value.status == L.CN_NAN


def test_max_iter_reported():
    pos, tris, h, t = workload("c1")
    with CutMeshSolver(pos, tris, h) as s:
        r = s.solve(t, precision="fp64", tol=1e-12, max_iter=3, max_refine=1, check=False)
    assert r.status == L.CN_MAX_ITER


@pytest.mark.parametrize("precond", ["ic0", "jacobi", "bssor"])
def test_autotuner_picks_a_shape_that_solves(precond, oracle, tmp_path):
    import torch

    from tool_godot_curvenet_b200 import tune
    pos, tris, h, t = workload("torus_mid")
    ref = oracle.System(pos, tris, h)
    st, xo, _, _ = ref.solve(t, mode=1, tol=1e-13)
    with CutMeshSolver(pos, tris, h, precond=precond) as s:
        d_t = torch.from_numpy(np.ascontiguousarray(t)).cuda()
        best, table = tune.autotune(s, d_t.data_ptr(), 3, precond, reps=1, cache=str(tmp_path / "c.json"),
                                    mode="deform", precision="mixed", tol=1e-8)
        assert len(table) >= 12 and best["ms"] == min(r["ms"] for r in table)
        i = s.info()
        assert (i["lanes"], i["block"]) == (best["lanes"], best["block"])
        r = s.solve(t, mode="deform", precision="fp64", tol=1e-13, max_iter=20000)
        assert rel_err(r.x, xo) <= FP64_TOL
        with CutMeshSolver(pos, tris, h, precond=precond) as s2:
            assert tune.apply_cached(s2, precond=precond, cache=str(tmp_path / "c.json")) == best


@pytest.mark.parametrize("k", [1, 3, 9])
@pytest.mark.parametrize("grid,block", [(1, 1024), (8, 256), (2, 128), (148, 1024)])
def test_jacobi_pipelined_matches_oracle_and_classic(k, grid, block, oracle):
    """The row-cached Jacobi kernel (shared-memory row cache with one or
    several row slices per thread, or global rows when a block holds more
    slices than the cache does): pipelined in FP64 and on request in mixed
    precision, two-reduction in mixed precision by default; against the
    oracle and the level-scheduled classic kernel."""
    pos, tris, h, _ = workload("torus_small")
    rng = np.random.default_rng(11 + k)
    t = rng.normal(size=(h.size, k))
    ref = oracle.System(pos, tris, h)
    st, xo, _, _ = ref.solve(t, mode=0, tol=1e-13)
    with CutMeshSolver(pos, tris, h, max_rhs=k, precond="jacobi", grid=grid, block=block) as s:
        r = s.solve(t, mode="harmonic", precision="fp64", tol=1e-13, max_iter=20000)
        rm = s.solve(t, mode="harmonic", precision="mixed", tol=1e-8, max_iter=20000)
        rc = s.solve(t, mode="harmonic", precision="fp64", tol=1e-13, max_iter=20000, algo="classic")
        rp = s.solve(t, mode="harmonic", precision="mixed", tol=1e-8, max_iter=20000, algo="pipelined")
    assert r.status == 0 and rm.status == 0 and rc.status == 0 and rp.status == 0
    assert rel_err(rp.x, xo) <= MIXED_TOL
    assert np.all(r.rel_residual <= 1e-13) and np.all(rm.rel_residual <= 1e-8)
    assert rel_err(r.x, xo) <= FP64_TOL
    assert rel_err(rm.x, xo) <= MIXED_TOL
    assert rel_err(rc.x, xo) <= FP64_TOL
    # pipelined and classic take about the same number of iterations
    assert r.iterations <= 1.5 * rc.iterations + 20


def test_bad_algo_rejected():
    pos, tris, h, t = workload("cyl_tiny")
    with CutMeshSolver(pos, tris, h) as s:
        o = s.make_opts()
        o.algo = 7
        st = L.lib().cn_solve(s._h, 3, t.ctypes.data_as(L.C.POINTER(L.C.c_double)), None,
                              np.empty((pos.shape[0], 3)).ctypes.data_as(L.C.POINTER(L.C.c_double)),
                              L.C.byref(o), None)
    assert st == L.CN_BAD_INPUT


@pytest.mark.parametrize("mesh", [39, 143])
def test_jacobi_mixed_converges_where_fp32_pipelining_drifts(mesh, oracle):
    """Meshes of the batch workload (about 40k free rows) on which the FP32
    pipelined recurrences lose track of the residual: the default mixed path
    (two-reduction form) and the FP64 pipelined path converge and match the
    oracle."""
    from tool_godot_curvenet_b200 import cut_mesh, synth
    m, h, t = synth.config3_mesh(mesh)
    tris, parent = cut_mesh(m.positions.shape[0], m.tris, m.loops)
    pos = np.ascontiguousarray(m.positions[parent])
    t = np.ascontiguousarray(t.reshape(t.shape[0], -1)[:, :3])
    ref = oracle.System(pos, tris, h)
    st, xo, _, _ = ref.solve(t, mode=1, tol=1e-12)
    with CutMeshSolver(pos, tris, h, precond="jacobi") as s:
        rm = s.solve(t, mode="deform", precision="mixed", tol=1e-8)
        rd = s.solve(t, mode="deform", precision="fp64", tol=1e-12, max_iter=20000)
    assert rm.status == 0 and rd.status == 0
    assert rel_err(rm.x, xo) <= MIXED_TOL
    assert rel_err(rd.x, xo) <= 1e-8


@pytest.mark.parametrize("name", ["torus_small", "c2"])
@pytest.mark.parametrize("k", [1, 3, 9, 24])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_spmv_matches_csr(name, k, precision):
    """cn_spmv_device against the exported matrix applied on the host, in
    both kernels: FP32 with k = 1 or 3 runs the staged kernel (row tiles
    copied to shared memory with bulk copies), the rest the grid-stride
    kernel."""
    import scipy.sparse as sp
    import torch
    pos, tris, h, _ = workload(name)
    with CutMeshSolver(pos, tris, h, precond="jacobi") as s:
        free_of, ptr, col, val = s.export_csr()
        n = ptr.size - 1
        A = sp.csr_matrix((val, col, ptr), shape=(n, n))
        x = np.random.default_rng(k).normal(size=(n, k))
        dt = torch.float32 if precision == "mixed" else torch.float64
        d_x = torch.from_numpy(x).to(dt).cuda()
        d_y = torch.empty((n, k), dtype=dt, device="cuda")
        s.spmv_device(k, d_x.data_ptr(), d_y.data_ptr(), precision=precision)
        torch.cuda.synchronize()
        y = d_y.double().cpu().numpy()
    want = A @ x.astype(np.float32).astype(np.float64) if precision == "mixed" else A @ x
    assert rel_err(y, want) <= (2e-6 if precision == "mixed" else 1e-14)


@pytest.mark.slow
@pytest.mark.parametrize("k", [1, 3])
def test_spmv_staged_ring_wraps(k):
    """The staged kernel on the 1.05M-row torus: about 4,100 tiles over the
    resident blocks, so every block reuses each of its shared-memory stages
    several times (the mbarrier phases alternate); bit-exact against the
    grid-stride kernel's summation order is not asked, the host product in
    FP64 of the FP32 inputs is."""
    import scipy.sparse as sp
    import torch
    pos, tris, h, _ = workload("c5")
    with CutMeshSolver(pos, tris, h, precond="jacobi") as s:
        free_of, ptr, col, val = s.export_csr()
        n = ptr.size - 1
        A = sp.csr_matrix((val.astype(np.float32).astype(np.float64), col, ptr), shape=(n, n))
        x = np.random.default_rng(7 + k).normal(size=(n, k)).astype(np.float32)
        d_x = torch.from_numpy(x).cuda()
        d_y = torch.full((n, k), float("nan"), dtype=torch.float32, device="cuda")
        for _ in range(2):  # a second call on the same handle and buffers
            s.spmv_device(k, d_x.data_ptr(), d_y.data_ptr(), precision="mixed")
        torch.cuda.synchronize()
        y = d_y.double().cpu().numpy()
    want = A @ x.astype(np.float64)
    assert np.isfinite(y).all()
    assert rel_err(y, want) <= 2e-6


def test_spmv_rejects_bad_arguments():
    pos, tris, h, _ = workload("cyl_tiny")
    with CutMeshSolver(pos, tris, h) as s:
        with pytest.raises(CnError) as e:
            s.spmv_device(5, 256, 256)
        assert e.value.status == L.CN_BAD_INPUT
        with pytest.raises(CnError) as e:
            s.spmv_device(3, 260, 256)  # misaligned
        assert e.value.status == L.CN_BAD_INPUT


@pytest.mark.parametrize("name", ["cyl_tiny", "c1", "torus_small", "c3_0"])
@pytest.mark.parametrize("grid,block", [(0, 0), (1, 512), (6, 256)])
@pytest.mark.parametrize("k", [1, 3, 9])
def test_block_ssor_matches_oracle(name, grid, block, k, oracle):
    """Block SSOR on the row-cached kernel: colour lists in shared memory
    (several blocks), the own rows in global memory (one block, no row
    cache); FP64 and mixed precision against the oracle's answer."""
    pos, tris, h, _ = workload(name)
    rng = np.random.default_rng(5 + k)
    t = rng.normal(size=(h.size, k))
    ref = oracle.System(pos, tris, h)
    st, xo, _, _ = ref.solve(t, mode=0, tol=1e-13)
    assert st == 0
    kw = {} if grid == 0 else {"grid": grid, "block": block}
    with CutMeshSolver(pos, tris, h, max_rhs=k, precond="bssor", **kw) as s:
        r = s.solve(t, mode="harmonic", precision="fp64", tol=1e-13, max_iter=20000)
        rm = s.solve(t, mode="harmonic", precision="mixed", tol=1e-8, max_iter=20000)
    assert r.status == 0 and rm.status == 0
    assert np.all(r.rel_residual <= 1e-13) and np.all(rm.rel_residual <= 1e-8)
    assert rel_err(r.x, xo) <= FP64_TOL
    assert rel_err(rm.x, xo) <= MIXED_TOL


def test_block_ssor_takes_fewer_iterations_than_jacobi():
    pos, tris, h, t = workload("torus_small")
    t = t[:, :3]
    its = {}
    for precond in ["jacobi", "bssor"]:
        with CutMeshSolver(pos, tris, h, precond=precond) as s:
            r = s.solve(t, mode="deform", precision="fp64", tol=1e-10, max_iter=20000, algo="classic")
            assert r.status == 0
            its[precond] = r.iterations
    assert its["bssor"] < 0.8 * its["jacobi"], its


@pytest.mark.parametrize("name", ["cyl_tiny", "torus_small", "torus_mid"])
@pytest.mark.parametrize("algo", ["fused", "pipelined", "classic"])
def test_block_ssor_cg_forms_match_oracle(name, algo, oracle):
    """Block SSOR in mixed precision in its three CG forms: the default
    (pipelined, u = M^-1 r and q = M^-1 s by recurrence, falling back to the
    two-reduction form if an inner solve stalls), the pipelined form alone
    and the two-reduction form, each to the oracle's answer; the pipelined
    form is FP32 only."""
    pos, tris, h, t = workload(name)
    t = t[:, :3]
    ref = oracle.System(pos, tris, h)
    st, xo, _, _ = ref.solve(t, mode=1, tol=1e-13)
    assert st == 0
    with CutMeshSolver(pos, tris, h, precond="bssor") as s:
        r = s.solve(t, mode="deform", precision="mixed", tol=1e-8, algo=algo, max_iter=20000)
        assert r.status == 0 and np.all(r.rel_residual <= 1e-8)
        assert rel_err(r.x, xo) <= MIXED_TOL
        if algo == "pipelined":
            with pytest.raises(CnError) as e:
                s.solve(t, mode="deform", precision="fp64", algo="pipelined")
            assert e.value.status == L.CN_BAD_INPUT


@pytest.mark.parametrize("name", ["cyl_tiny", "c1", "torus_small", "torus_mid", "c3_0"])
@pytest.mark.parametrize("precond", ["bssor", "jacobi"])
@pytest.mark.parametrize("k", [1, 3, 9])
def test_single_reduction_form_matches_oracle(name, precond, k, oracle):
    """The single-reduction CG (one grid barrier per iteration, z exchanged
    with the neighbour blocks by release / acquire flags) on the row-cached
    kernel: FP64 and mixed precision against the oracle, default launch and
    a one-block launch."""
    pos, tris, h, _ = workload(name)
    rng = np.random.default_rng(11 + k)
    t = rng.normal(size=(h.size, k))
    ref = oracle.System(pos, tris, h)
    st, xo, _, _ = ref.solve(t, mode=0, tol=1e-13)
    assert st == 0
    for kw in ({}, {"grid": 1, "block": 512}):
        with CutMeshSolver(pos, tris, h, max_rhs=k, precond=precond, **kw) as s:
            r = s.solve(t, mode="harmonic", precision="fp64", tol=1e-13, max_iter=20000, algo="single")
            rm = s.solve(t, mode="harmonic", precision="mixed", tol=1e-8, max_iter=20000, algo="single")
            rc = s.solve(t, mode="harmonic", precision="mixed", tol=1e-8, max_iter=20000, algo="classic")
        assert r.status == 0 and rm.status == 0
        assert np.all(r.rel_residual <= 1e-13) and np.all(rm.rel_residual <= 1e-8)
        assert rel_err(r.x, xo) <= FP64_TOL
        assert rel_err(rm.x, xo) <= MIXED_TOL
        # the same iteration count as the two-reduction form, within rounding drift
        assert abs(rm.iterations - rc.iterations) <= max(8, 0.1 * rc.iterations)


def test_single_reduction_rejected_on_level_scheduled_handles():
    pos, tris, h, t = workload("c1")
    with CutMeshSolver(pos, tris, h, precond="hsc") as s:
        with pytest.raises(CnError):
            s.solve(t, mode="deform", precision="mixed", algo="single")
