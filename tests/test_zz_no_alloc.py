"""GPU test of cn_pcg_csr_noalloc, the entry point for callers that cannot
allocate GPU memory while they run (a frame loop with a fixed memory budget,
code recording a CUDA stream).  It must give the solution of the
handle-based entry point (cn_solve with CN_MODE_RHS on a Jacobi-preconditioned
handle of the same matrix) and of the oracle's FP64 Jacobi-PCG
(SparseLinAlg.lean:104-163) call after call, for 1, 3 and 9 right-hand sides,
both through the one-block path (up to 12,288 rows) and the cooperative grid
path; the asynchronous form (no statistics pointer, a non-default stream)
must give the same solution, its statistics read afterwards with
cn_pcg_csr_noalloc_last_stats; and it must refuse systems larger than its
fixed scratch with a clear error.

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C
import functools

import numpy as np
import pytest

from tests.helpers import rel_err, workload
from tool_godot_curvenet_b200 import CutMeshSolver
from tool_godot_curvenet_b200 import _lib as L

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-9  # the FP64 parity tolerance of the GPU tests


def _noalloc(n, d_ptr, d_col, d_val, k, d_b, d_x, tol=1e-13, max_iter=20000, stats=True, stream=None):
    st = L.SolveStats()
    rc = L.lib().cn_pcg_csr_noalloc(n, d_ptr, d_col, d_val, k, d_b, d_x, tol, max_iter, stream,
                                    C.byref(st) if stats else None)
    return rc, st


@functools.lru_cache(maxsize=None)
def exported(name):
    pos, tris, h, _ = workload(name)
    with CutMeshSolver(pos, tris, h, precond="jacobi", max_rhs=9) as s:
        return s.export_csr()


def oracle_solve(ptr, col, val, b):
    """The oracle's FP64 Jacobi-PCG per column, to an absolute residual of
    1e-14 ||b|| (the spec's absolute test, scaled)."""
    from oracle import oracle as O
    x = np.empty_like(b)
    for c in range(b.shape[1]):
        x[:, c], _ = O.cg_ref(ptr, col, val, b[:, c], 200000, 1e-14 * np.linalg.norm(b[:, c]))
    return x


@pytest.mark.parametrize("name,k", [("c1", 3), ("torus_small", 1), ("torus_mid", 1), ("torus_mid", 3),
                                    ("torus_mid", 9)])
def test_noalloc_matches_handle_and_oracle_on_two_calls(name, k):
    import torch
    pos, tris, h, _ = workload(name)
    free_of, ptr, col, val = exported(name)
    n = ptr.size - 1
    rng = np.random.default_rng(17 + k)
    d_ptr = torch.from_numpy(ptr).cuda()
    d_col = torch.from_numpy(col).cuda()
    d_val = torch.from_numpy(val).cuda()
    with CutMeshSolver(pos, tris, h, precond="jacobi", max_rhs=9) as s:
        for _ in range(2):  # two calls in a row share the static scratch
            b = rng.normal(size=(n, k))
            ref = s.solve(b, mode="rhs", precision="fp64", tol=1e-13, max_iter=20000).x[free_of]
            d_b = torch.from_numpy(b).cuda()
            d_x = torch.zeros((n, k), dtype=torch.float64, device="cuda")
            rc, st = _noalloc(n, d_ptr.data_ptr(), d_col.data_ptr(), d_val.data_ptr(), k, d_b.data_ptr(),
                              d_x.data_ptr())
            assert rc == L.CN_OK, L.last_error()
            assert st.k == k and st.max_rel_residual <= 1e-13
            x = d_x.cpu().numpy()
            assert rel_err(x, ref) <= FP64_TOL
            assert rel_err(x, oracle_solve(ptr, col, val, b)) <= FP64_TOL


def test_noalloc_asynchronous_on_a_stream_then_last_stats():
    """The capture-friendly form: no statistics pointer, a non-default
    stream; the result and then the statistics are read after a sync."""
    import torch
    name = "torus_mid"
    pos, tris, h, _ = workload(name)
    free_of, ptr, col, val = exported(name)
    n = ptr.size - 1
    b = np.random.default_rng(5).normal(size=(n, 3))
    d_ptr = torch.from_numpy(ptr).cuda()
    d_col = torch.from_numpy(col).cuda()
    d_val = torch.from_numpy(val).cuda()
    d_b = torch.from_numpy(b).cuda()
    d_x = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    rc, _ = _noalloc(n, d_ptr.data_ptr(), d_col.data_ptr(), d_val.data_ptr(), 3, d_b.data_ptr(), d_x.data_ptr(),
                     stats=False, stream=stream.cuda_stream)
    assert rc == L.CN_OK, L.last_error()
    stream.synchronize()
    st = L.SolveStats()
    rc = L.lib().cn_pcg_csr_noalloc_last_stats(C.byref(st))
    assert rc == L.CN_OK and st.status == L.CN_OK, L.last_error()
    assert st.k == 3 and st.iterations > 0 and st.max_rel_residual <= 1e-13
    assert rel_err(d_x.cpu().numpy(), oracle_solve(ptr, col, val, b)) <= FP64_TOL


def test_noalloc_rejects_sizes_beyond_its_scratch():
    rc, _ = _noalloc(65537, 1, 1, 1, 1, 1, 1)
    assert rc == L.CN_BAD_INPUT
    assert "limit" in L.last_error()
    rc, _ = _noalloc(65536, 1, 1, 1, 9, 1, 1)
    assert rc == L.CN_BAD_INPUT
    assert "limit" in L.last_error()
