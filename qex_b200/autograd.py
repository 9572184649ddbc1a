"""torch.autograd wrapper of the staggered fermion action, as a test harness
for the hand-written adjoint (the library's force solve and fermForce outer
products); the HMC itself calls the library directly.

StaggeredAction.apply(W, phi, stag, m) returns S = phi_e^dagger A^-1 phi_e,
A = stagD2ee(m^2), for the phased link list W (complex128, device layout
(nlinks, 3, 3, V), the links the operator `stag` was built from) and an
even-site source phi (device layout (3, V)).  Its gradient with respect to W
follows from dS = Re sum conj(f) dW / 8, f = fermForce's outer products of
QEX's psi = (4y, (2D)_oe 4y) (hmcAction.nim:669-771), so torch's gradient
(d/dRe W + i d/dIm W) is f / 8.
"""
from __future__ import annotations

import torch

from . import stag as S


class StaggeredAction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, W, phi, stag, m, r2req=1e-24):
        stag.update_links(W.detach().contiguous())
        y = torch.zeros_like(phi)
        stag.solveEE(y, phi, m, S.SolverParams(r2req=r2req))
        ctx.stag, ctx.m, ctx.r2req = stag, m, r2req
        ctx.save_for_backward(phi)
        V = phi.shape[1]
        return torch.vdot(phi[:, : V // 2].reshape(-1), y[:, : V // 2].reshape(-1)).real

    @staticmethod
    def backward(ctx, grad_out):
        (phi,) = ctx.saved_tensors
        stag = ctx.stag
        psi = torch.zeros_like(phi)
        stag.force_solve(psi, phi, ctx.m, S.SolverParams(r2req=ctx.r2req))
        f = torch.zeros((stag.nlinks, 3, 3, phi.shape[1]), dtype=torch.complex128, device=phi.device)
        stag.ferm_outer(f, psi)
        return grad_out * f / 8.0, None, None, None, None
