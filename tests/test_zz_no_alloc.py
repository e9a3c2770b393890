"""GPU test of cn_pcg_csr_noalloc, the entry point for callers that cannot
allocate GPU memory while they run (a frame loop with a fixed memory budget,
code recording a CUDA stream).  It must give the same solution as the
handle-based entry point (cn_solve with CN_MODE_RHS on a Jacobi-preconditioned
handle of the same matrix), call after call, and it must refuse systems larger
than its fixed scratch with a clear error.

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

from tests.helpers import rel_err, workload
from tool_godot_curvenet_b200 import CutMeshSolver
from tool_godot_curvenet_b200 import _lib as L

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-9  # the FP64 parity tolerance of the GPU tests


def _noalloc(n, d_ptr, d_col, d_val, k, d_b, d_x, tol=1e-13, max_iter=20000, stats=True):
    st = L.SolveStats()
    rc = L.lib().cn_pcg_csr_noalloc(n, d_ptr, d_col, d_val, k, d_b, d_x, tol, max_iter, None,
                                    C.byref(st) if stats else None)
    return rc, st


@pytest.mark.parametrize("name", ["c1", "torus_small", "torus_mid"])
def test_noalloc_matches_handle_solve_on_two_calls(name):
    import torch
    pos, tris, h, _ = workload(name)
    rng = np.random.default_rng(17)
    with CutMeshSolver(pos, tris, h, precond="jacobi") as s:
        free_of, ptr, col, val = s.export_csr()
        n = ptr.size - 1
        d_ptr = torch.from_numpy(ptr).cuda()
        d_col = torch.from_numpy(col).cuda()
        d_val = torch.from_numpy(val).cuda()
        for _ in range(2):  # two calls in a row share the static scratch
            b = rng.normal(size=(n, 3))
            ref = s.solve(b, mode="rhs", precision="fp64", tol=1e-13, max_iter=20000).x[free_of]
            d_b = torch.from_numpy(b).cuda()
            d_x = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
            rc, st = _noalloc(n, d_ptr.data_ptr(), d_col.data_ptr(), d_val.data_ptr(), 3, d_b.data_ptr(),
                              d_x.data_ptr())
            assert rc == L.CN_OK, L.last_error()
            assert st.max_rel_residual <= 1e-13
            x = d_x.cpu().numpy()
            assert rel_err(x, ref) <= FP64_TOL


def test_noalloc_rejects_sizes_beyond_its_scratch():
    rc, _ = _noalloc(65537, 1, 1, 1, 1, 1, 1)
    assert rc == L.CN_BAD_INPUT
    assert "limit" in L.last_error()
    rc, _ = _noalloc(65536, 1, 1, 1, 9, 1, 1)
    assert rc == L.CN_BAD_INPUT
    assert "limit" in L.last_error()
