"""Adjoint of one implicit step (new; StiffGIPC has no differentiation).

For the implicit step x* = argmin E(x; E_t, v0) the optimality condition g(x*) = 0 gives,
by the implicit function theorem,

    dL/dtheta = -lambda^T dg/dtheta,      A lambda = dL/dx*,

with A the projected Hessian the Newton solve assembles (same BSR, same MAS-PCG).  The
batched solve handles several losses (right-hand sides) per read of A and of the MAS
inverses; ``sgipc_adjoint_param_grads`` contracts lambda with the per-tet Young's-modulus
and per-vertex initial-velocity derivatives, recomputing element quantities from x*.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import torch

from . import _native as N
from .system import GIPC, MASPreconditioner, PCGSolver, PCGSolverConfig, _p, _stream, params_struct


def adjoint(g: GIPC, dLdx: torch.Tensor, precision: str = "fp64", tol: float = 1e-8,
            criterion: int = N.CRIT_TRUE, rebuild_mas: bool = True, max_iter_ratio: float = 1.0):
    """dL/dE (nrhs, T) and dL/dv0 (nrhs, 3V) for adjoint right-hand sides dLdx (nrhs, 3V).

    ``g`` must hold the system assembled at the converged step x*.  Rows of Dirichlet
    vertices are zeroed in the right-hand side, as the assembled gradient zeroes them.
    """
    if dLdx.dim() == 1:
        dLdx = dLdx[None]
    nrhs = dLdx.shape[0]
    b = dLdx.to(torch.float64).clone()
    free = (g.tet.BoundaryType == 0).to(torch.float64).repeat_interleave(3)
    b *= free[None]
    if rebuild_mas:
        MASPreconditioner(g).setPreconditioner(precision)
    cfg = PCGSolverConfig(precision=precision, global_tol_rate=tol, criterion=criterion,
                          max_iter_ratio=max_iter_ratio)
    lam, stats = PCGSolver(g, cfg).solve_batched(b)
    nt = g.scene.nt
    dLdE = torch.empty((nrhs, nt), dtype=torch.float64, device=b.device)
    dLdv0 = torch.empty_like(b)
    f = g.tet.fem_struct()
    prm = params_struct(g.params)
    N.check(N.lib().sgipc_adjoint_param_grads(g.ctx, C.byref(f), C.byref(prm), float(g.scene.poisson), nrhs,
                                              _p(lam), _p(dLdE), _p(dLdv0), _stream()), g.ctx)
    return dLdE, dLdv0, lam, stats
