"""The hand-written adjoint (cn_deform / cn_adjoint) on the profile-curve
workload (torus 128 x 64, 4 seams = 4 profile curves of 16 cubic control
points, per-curve weights): gradient of L = 1/2 ||x - x_target||^2 with
respect to the posed control points and the weights, against the oracle's
FP64 CPU adjoint, against central finite differences (h = 1e-6, FP64, the
scope's 1e-5 relative bar), and through torch.autograd.gradcheck."""
import functools

import numpy as np
import pytest

from tool_godot_curvenet_b200 import synth

pytestmark = pytest.mark.gpu

TOL = 1e-13
FD_H = 1e-6
FD_REL = 1e-5


@functools.lru_cache(maxsize=None)
def problem():
    return synth.config4()


@functools.lru_cache(maxsize=None)
def deformer():
    from tool_godot_curvenet_b200.autograd import CurveDeformer
    pos, tris, h, cof, tau, rest_cp, _, _, _, _ = problem()
    return CurveDeformer(pos, tris, h, cof, tau, rest_cp)


def target():
    d = deformer()
    *_, tcp, tw = problem()
    return d.deform(tcp, tw, tol=TOL)


def loss_and_grad(P, w):
    d = deformer()
    xt = target()
    x = d.deform(P, w, tol=TOL)
    g = x - xt
    dP, dw = d.adjoint(g, tol=TOL)
    return 0.5 * float((g * g).sum()), dP, dw


def test_adjoint_matches_oracle_adjoint(oracle):
    pos, tris, h, cof, tau, rest_cp, P, w, tcp, tw = problem()
    loss, dP, dw = loss_and_grad(P, w)
    ref = oracle.System(pos, tris, h)
    e = ref.export()
    Kp, Kc, Kv = oracle.assemble_csr(pos.shape[0], tris, pos)
    xt = target()
    S = rest_cp.shape[1] // 3
    x = np.empty((pos.shape[0], 3))
    dPo = np.empty_like(rest_cp)
    dwo = np.empty(rest_cp.shape[0])
    O = oracle
    lo = O.lib().orc_deform_adjoint(ref._h, pos.shape[0], O.ip(Kp), O.ip(Kc), O.dp(Kv), ref.n,
                                    O.ip(e["free_of"]), rest_cp.shape[0], S, O.dp(O.f64(rest_cp)),
                                    O.dp(O.f64(P)), O.dp(O.f64(w)), h.size, O.ip(O.i32(h)), O.ip(O.i32(cof)),
                                    O.dp(O.f64(tau)), O.dp(O.f64(pos)), O.dp(O.f64(xt)), 1e-13, 100000,
                                    O.dp(x), O.dp(dPo), O.dp(dwo))
    assert abs(lo - loss) <= 1e-9 * abs(lo)
    g = np.concatenate([dP.ravel(), dw])
    go = np.concatenate([dPo.ravel(), dwo])
    assert np.linalg.norm(g - go) <= 1e-8 * np.linalg.norm(go)


def test_adjoint_matches_central_differences():
    _, _, _, _, _, rest_cp, P, w, _, _ = problem()
    loss, dP, dw = loss_and_grad(P, w)
    d = deformer()
    xt = target()

    def L(Pv, wv):
        x = d.deform(Pv, wv, tol=TOL)
        return 0.5 * float(((x - xt) ** 2).sum())

    fd = np.zeros(P.size + w.size)
    Pf = P.ravel()
    for i in range(Pf.size):
        a, b = Pf.copy(), Pf.copy()
        a[i] += FD_H
        b[i] -= FD_H
        fd[i] = (L(a.reshape(P.shape), w) - L(b.reshape(P.shape), w)) / (2 * FD_H)
    for i in range(w.size):
        a, b = w.copy(), w.copy()
        a[i] += FD_H
        b[i] -= FD_H
        fd[P.size + i] = (L(P, a) - L(P, b)) / (2 * FD_H)
    g = np.concatenate([dP.ravel(), dw])
    rel = np.linalg.norm(g - fd) / np.linalg.norm(fd)
    assert rel <= FD_REL, rel


def test_torch_gradcheck():
    import torch

    from tool_godot_curvenet_b200.autograd import deform
    _, _, _, _, _, _, P, w, _, _ = problem()
    d = deformer()
    xt = torch.from_numpy(target())
    Pt = torch.tensor(P, dtype=torch.float64, requires_grad=True)
    wt = torch.tensor(w, dtype=torch.float64, requires_grad=True)

    def f(Pv, wv):
        x = deform(Pv, wv, d, TOL)
        return 0.5 * ((x - xt) ** 2).sum()

    assert torch.autograd.gradcheck(f, (Pt, wt), eps=FD_H, atol=1e-5, rtol=1e-4, nondet_tol=1e-7)
    loss = f(Pt, wt)
    loss.backward()
    _, dP, dw = loss_and_grad(P, w)
    assert np.allclose(Pt.grad.numpy(), dP, rtol=1e-9, atol=1e-12)
    assert np.allclose(wt.grad.numpy(), dw, rtol=1e-9, atol=1e-12)


def test_identity_curves_give_rest_pose():
    pos, _, _, _, _, rest_cp, _, _, _, _ = problem()
    d = deformer()
    x = d.deform(rest_cp, np.ones(rest_cp.shape[0]), tol=TOL)
    assert np.abs(x - pos).max() < 1e-9


def test_adjoint_with_block_ssor_matches_default():
    """The adjoint solve of a block-SSOR handle (a different preconditioner,
    the same A) gives the gradient of the default handle."""
    from tool_godot_curvenet_b200.autograd import CurveDeformer
    pos, tris, h, cof, tau, rest_cp, P, w, _, _ = problem()
    loss, dP, dw = loss_and_grad(P, w)
    d2 = CurveDeformer(pos, tris, h, cof, tau, rest_cp, precond="bssor")
    xt = target()
    x = d2.deform(P, w, tol=TOL)
    g = x - xt
    dP2, dw2 = d2.adjoint(g, tol=TOL)
    a = np.concatenate([dP.ravel(), dw])
    b = np.concatenate([dP2.ravel(), dw2])
    assert np.linalg.norm(a - b) <= 1e-8 * np.linalg.norm(a)
