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


# ------------------------------------------------------------------------------------------
# implicit step as a differentiable function
# ------------------------------------------------------------------------------------------
GRAVITY = (0.0, -9.8, 0.0)


def set_parameters(g: GIPC, E: Optional[torch.Tensor] = None, v0: Optional[torch.Tensor] = None) -> None:
    """Write per-tet Young's moduli E (T,) and initial velocities v0 (V,3) into the device
    state: lengthRate / volumeRate of the stable Neo-Hookean model (StiffGIPC/gl_main.cu:
    609-617) and the inertial target xTilta = x_prev + dt v0 (+ dt^2 g on free vertices,
    StiffGIPC/GIPC.cu:8073-8097)."""
    tet, nu = g.tet, float(g.scene.poisson)
    if E is not None:
        E = E.to(torch.float64).reshape(-1)
        mu = E / (2.0 * (1.0 + nu))
        lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
        tet.lengthRate.copy_(4.0 * mu / 3.0)
        tet.volumeRate.copy_(lam + 5.0 * mu / 6.0)
    if v0 is not None:
        dt = float(g.params["dt"])
        grav = torch.tensor(GRAVITY, dtype=torch.float64, device=tet.xTilta.device)
        free = (tet.BoundaryType == 0).to(torch.float64)[:, None]
        tet.xTilta.copy_(tet.o_vertexes + dt * v0.to(torch.float64).reshape(-1, 3) + dt * dt * free * grav[None])


def newton_solve(g: GIPC, tol: float = 1e-11, max_newton: int = 30, precision: str = "fp64",
                 contacts: bool = False, max_move: Optional[float] = None) -> torch.Tensor:
    """Minimise the incremental potential for the current parameters: Newton steps
    x <- x - alpha dx with A dx = g(x) solved by the MAS-PCG.  alpha is first bounded as the
    reference bounds it before its line search (GIPC.cu:10895-10901): by the ground plane's
    largest feasible step over every surface vertex and, with ``contacts``, by the additive
    CCD's over the candidate pairs of the step, both at slackness 0.8; then it is halved until
    ||g|| decreases.  Stops when ||g(x)|| <= tol * ||g(x_start)||, or when no step length
    reduces ||g|| any more (round-off level), keeping the best iterate.  Returns x* (V,3),
    left in ``g.tet.vertexes``, with the system assembled at x*.

    contacts=False keeps the contact pairs and ground pairs of ``g.tet`` fixed.  contacts=True
    finds them again at every trial iterate with the GPU pair search (``GIPC.buildCP``), as the
    reference's line search does, so that x* minimises the energy with the contacts of x*.  A
    step then moves no vertex further than ``max_move`` (default 2 d-hat), and its CCD
    candidates are the pairs within d-hat + 2 max_move of the current iterate: every pair that
    the step can bring into contact.  The lagged friction sets stay those of the frame start,
    as in the reference (buildFrictionSets once per frame, GIPC.cu:11119).

    The reference's Newton loop (energy line search, kappa updates, GIPC.cu:10830-10976) is not
    part of this path; this driver exists so that the adjoint can be checked against finite
    differences of a converged step."""
    cfg = PCGSolverConfig(precision=precision, global_tol_rate=1e-13, criterion=N.CRIT_TRUE, max_iter_ratio=1.0)
    x = g.tet.vertexes
    dhat = float(g.params["dHat"]) ** 0.5
    max_move = 2.0 * dhat if max_move is None else max_move
    if contacts:
        g.buildCP()
    g.computeGradientAndHessian()
    r = g.rhs().norm().item()
    r0 = max(r, 1e-300)
    g._surface()
    surf = g._surf_arrays[0]
    for _ in range(max_newton):
        if r <= tol * r0:
            break
        g.calculateMovingDirection(cfg)
        dx = g.moveDir.view(-1, 3).clone()
        x_prev = x.clone()
        alpha = 1.0
        if surf.numel():
            alpha = min(alpha, g.ground_largestFeasibleStepSize(0.8, g.moveDir, surf))
        if contacts:
            far = dx.norm(dim=1).max().item()
            if far * alpha > max_move:
                alpha = max_move / far
            reach = dhat + 2.0 * alpha * far
            cand = g.buildCP(update=False, dHat=reach * reach)["ccd_pairs"]
            if cand.shape[0]:
                alpha = min(alpha, g.self_largestFeasibleStepSize(0.8, g.moveDir, cand.contiguous()))
        while True:
            x.copy_(x_prev - alpha * dx)
            if contacts:
                g.buildCP()
            g.computeGradientAndHessian()
            rn = g.rhs().norm().item()
            if rn < r or alpha < 1e-3:
                break
            alpha *= 0.5
        if not rn < r:  # no decrease: x_prev is converged to round-off
            x.copy_(x_prev)
            if contacts:
                g.buildCP()
            g.computeGradientAndHessian()
            break
        r = rn
    return x


class ImplicitStep(torch.autograd.Function):
    """x* = argmin_x E(x; E_t, v0) as a differentiable function of the per-tet Young's
    moduli and the initial velocities.  Forward runs :func:`newton_solve`; backward solves
    the adjoint system A lambda = dL/dx* with the same matrix and MAS-PCG and contracts it
    with dg/dE_t and dg/dv0 (``sgipc_adjoint_param_grads``)."""

    @staticmethod
    def forward(ctx, E: torch.Tensor, v0: torch.Tensor, g: GIPC, tol: float = 1e-11,
                contacts: bool = False):
        set_parameters(g, E, v0)
        x = newton_solve(g, tol=tol, contacts=contacts)
        ctx.g = g
        ctx.v0_shape = v0.shape
        return x.clone()

    @staticmethod
    def backward(ctx, dLdx: torch.Tensor):
        g = ctx.g
        g.computeGradientAndHessian()  # A and dg/dtheta at x* (the state forward left)
        dLdE, dLdv0, _, _ = adjoint(g, dLdx.reshape(1, -1).contiguous(), precision="fp64", tol=1e-12,
                                    criterion=N.CRIT_TRUE)
        return dLdE[0], dLdv0[0].reshape(ctx.v0_shape), None, None, None
