"""Direct Delta Mush on the GPU against the oracle.

* runtime (cn_lbs_matvec_device): the reference's known answers
  (DirectDeltaMush.lean:115-165) and random influences against the oracle's
  lbsMatvec, FP64 to 1e-13 and FP32 to 1e-5 relative;
* bind (cn_ddm_bind): against the oracle pipeline on the same mesh — the
  oracle's harmonic solve with unit targets, smoothWeights over the cut-mesh
  adjacency (K's off-diagonal pattern, ascending) and sparsifyTopK — compared
  as dense rows (ties among equal |w| may keep different zero columns), to
  1e-8 with both solves at 1e-12; rows sum to 1; a rigid motion of all
  handles moves every vertex rigidly."""
import json
import os

import numpy as np
import pytest
import torch

from tests.helpers import workload
from tool_godot_curvenet_b200 import CnError, CutMeshSolver, lbs_matvec_device
from tool_godot_curvenet_b200 import _lib as L

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")


def _gpu_lbs(rest, T, start, idx, w, precision):
    dt = torch.float32 if precision == "mixed" else torch.float64
    d_rest = torch.as_tensor(np.asarray(rest, np.float64).reshape(-1, 3), dtype=dt).cuda()
    d_T = torch.as_tensor(np.asarray(T, np.float64).reshape(-1, 16), dtype=dt).cuda()
    d_start = torch.as_tensor(np.asarray(start, np.int32)).cuda()
    d_idx = torch.as_tensor(np.asarray(idx, np.int32) if len(idx) else np.zeros(1, np.int32)).cuda()
    d_w = torch.as_tensor(np.asarray(w, np.float64) if len(w) else np.zeros(1), dtype=dt).cuda()
    d_out = torch.empty_like(d_rest)
    lbs_matvec_device(d_rest.shape[0], d_rest.data_ptr(), d_T.data_ptr(), d_start.data_ptr(), d_idx.data_ptr(),
                      d_w.data_ptr(), d_out.data_ptr(), precision=precision)
    torch.cuda.synchronize()
    return d_out.double().cpu().numpy()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_lbs_known_answers(precision):
    with open(GOLDEN) as f:
        fx = [g for g in json.load(f) if g["kind"] == "lbs"]
    assert len(fx) == 6
    for g in fx:
        infl = g["infl"]
        out = _gpu_lbs([g["rest"]], g["T"], [0, len(infl)], [i for i, _ in infl], [x for _, x in infl], precision)
        eps = g["eps"] if precision == "fp64" else 1e-6
        assert np.all(np.abs(out[0] - g["expected"]) < eps), g["src"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_lbs_random_matches_oracle(precision, oracle):
    rng = np.random.default_rng(4)
    nv, nh, K = 5000, 40, 6
    rest = rng.normal(size=(nv, 3))
    T = np.tile(np.eye(4), (nh, 1, 1))
    T[:, :3, :] += 0.2 * rng.normal(size=(nh, 3, 4))
    lens = rng.integers(0, K + 1, nv)
    start = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    idx = rng.integers(0, nh, start[-1]).astype(np.int32)
    w = rng.uniform(0.0, 1.0, start[-1])
    want = oracle.lbs_matvec_csr(rest, T.reshape(nh, 16), start, idx, w)
    got = _gpu_lbs(rest, T.reshape(nh, 16), start, idx, w, precision)
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= (1e-13 if precision == "fp64" else 1e-5) * scale


def _oracle_bind(oracle, s, pos, tris, h, nu, omega, K):
    ref = oracle.System(pos, tris, h)
    st, W, _, _ = ref.solve(np.eye(h.size), mode=0, tol=1e-13)
    assert st == 0
    W[h] = np.eye(h.size)
    ptr, col, _ = s.export_k()
    adj = [[int(u) for u in col[ptr[v]:ptr[v + 1]] if u != v] for v in range(pos.shape[0])]
    Ws = oracle.smooth_weights(W, adj, nu, omega)
    idx, w = oracle.sparsify_topk(Ws, K)
    dense = np.zeros_like(Ws)
    np.put_along_axis(dense, idx, w, axis=1)
    return dense


@pytest.mark.parametrize("name,nu,omega,K", [("cyl_tiny", 2, 0.5, 4), ("cyl_tiny", 0, 0.5, 3),
                                             ("torus_small", 3, 0.3, 8)])
def test_bind_matches_oracle(name, nu, omega, K, oracle):
    pos, tris, h, _ = workload(name)
    with CutMeshSolver(pos, tris, h, max_rhs=9, precond="jacobi") as s:
        idx, w = s.ddm_bind(nu=nu, omega=omega, top_k=K, precision="fp64", tol=1e-12, max_iter=20000)
        want = _oracle_bind(oracle, s, pos, tris, h, nu, omega, K)
    assert idx.shape == (pos.shape[0], min(K, h.size))
    got = np.zeros_like(want)
    np.put_along_axis(got, idx, w, axis=1)
    assert np.abs(got - want).max() <= 1e-8
    assert np.abs(w.sum(axis=1) - 1.0).max() <= 1e-12
    # largest |w| first
    assert np.all(np.abs(w[:, :-1]) >= np.abs(w[:, 1:]))


def test_bind_then_runtime_moves_rigidly():
    pos, tris, h, _ = workload("torus_small")
    with CutMeshSolver(pos, tris, h, max_rhs=9) as s:
        idx, w = s.ddm_bind(nu=2, omega=0.5, top_k=6, precision="fp64", tol=1e-12)
    nv, take = idx.shape
    th = 0.4
    M = np.eye(4)
    M[:3, :3] = [[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]]
    M[:3, 3] = [0.5, -1.0, 2.0]
    T = np.tile(M.reshape(16), (h.size, 1))
    start = np.arange(nv + 1, dtype=np.int32) * take
    out = _gpu_lbs(pos, T, start, idx.reshape(-1), w.reshape(-1), "fp64")
    assert np.abs(out - (pos @ M[:3, :3].T + M[:3, 3])).max() <= 1e-10


def test_bind_rejects_bad_arguments():
    pos, tris, h, _ = workload("cyl_tiny")
    with CutMeshSolver(pos, tris, h) as s:  # max_rhs = 3
        with pytest.raises(CnError) as e:
            s.ddm_bind()
        assert e.value.status == L.CN_BAD_INPUT
    with CutMeshSolver(pos, tris, h, max_rhs=9) as s:
        with pytest.raises(CnError) as e:
            s.ddm_bind(top_k=0)
        assert e.value.status == L.CN_BAD_INPUT
