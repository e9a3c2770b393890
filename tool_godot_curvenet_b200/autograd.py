"""torch.autograd bridge of the deform solve: forward = cn_deform (profile
curves -> handle targets -> deform solve), backward = cn_adjoint (one solve
with the same IC(0) factor, A = A^T, then the chain to the curve control
points and weights).  Float64 CPU tensors in and out; the solves run on the
handle's GPU."""
import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .solver import CnError, CutMeshSolver, _dp, _f64, _i32


class CurveDeformer:
    """A CutMeshSolver with its handles bound to profile curves."""

    def __init__(self, positions, tris, handles, curve_of, tau, rest_cp, **build):
        self.solver = CutMeshSolver(positions, tris, handles, **build)
        self.rest_cp = _f64(rest_cp)
        self.ncurves, npts, _ = self.rest_cp.shape
        self.nseg = (npts - 1) // 3
        st = L.lib().cn_bind_curves(self.solver._h, self.ncurves, self.nseg, _dp(self.rest_cp),
                                    _i32(curve_of).ctypes.data_as(C.POINTER(C.c_int32)), _dp(_f64(tau)))
        if st != L.CN_OK:
            raise CnError(st, "cn_bind_curves")
        self.n_verts = self.solver.n_verts

    def close(self):
        self.solver.close()

    def deform(self, posed_cp, weights, tol=1e-13, precision="fp64"):
        p = _f64(posed_cp)
        w = _f64(weights)
        x = np.empty((self.n_verts, 3))
        o = CutMeshSolver.make_opts(mode="deform", precision=precision, tol=tol, max_iter=20000)
        stats = L.SolveStats()
        st = L.lib().cn_deform(self.solver._h, _dp(p), _dp(w), _dp(x), C.byref(o), C.byref(stats))
        if st != L.CN_OK:
            raise CnError(st, "cn_deform")
        return x

    def adjoint(self, dL_dx, tol=1e-13, precision="fp64"):
        g = _f64(dL_dx)
        dP = np.empty_like(self.rest_cp)
        dw = np.empty(self.ncurves)
        o = CutMeshSolver.make_opts(mode="rhs", precision=precision, tol=tol, max_iter=20000)
        stats = L.SolveStats()
        st = L.lib().cn_adjoint(self.solver._h, _dp(g), _dp(dP), _dp(dw), C.byref(o), C.byref(stats))
        if st != L.CN_OK:
            raise CnError(st, "cn_adjoint")
        return dP, dw


class DeformFunction(torch.autograd.Function):
    """x = deform(posed_cp, weights); backward through the hand-written adjoint."""

    @staticmethod
    def forward(ctx, posed_cp, weights, deformer, tol):
        x = deformer.deform(posed_cp.detach().cpu().numpy(), weights.detach().cpu().numpy(), tol=tol)
        ctx.deformer = deformer
        ctx.tol = tol
        ctx.save_for_backward(posed_cp, weights)
        return torch.from_numpy(x)

    @staticmethod
    def backward(ctx, grad_x):
        posed_cp, weights = ctx.saved_tensors
        d = ctx.deformer
        # the adjoint linearises at the last forward; re-run it at these inputs
        d.deform(posed_cp.detach().cpu().numpy(), weights.detach().cpu().numpy(), tol=ctx.tol)
        dP, dw = d.adjoint(grad_x.detach().cpu().numpy(), tol=ctx.tol)
        return torch.from_numpy(dP), torch.from_numpy(dw), None, None


def deform(posed_cp, weights, deformer, tol=1e-13):
    return DeformFunction.apply(posed_cp, weights, deformer, tol)
