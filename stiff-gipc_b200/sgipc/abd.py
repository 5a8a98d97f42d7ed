"""Affine bodies over the C ABI: ``ABDSystem`` and ``ABDPreconditioner``.

Mirrors StiffGIPC's ``ABDSystem::setup_abd_system_gradient_hessian``
(abd_system/abd_system_function/setup_abd_system_gradient_and_hessian.cu:162-610) and
``ABDPreconditioner::assemble / apply`` (linear_system/preconditioner/abd_preconditioner.cu:
15-38): per-body gradients and 12x12 Hessians (dyadic-mass kinetic term + projected
orthogonality potential), point barrier gradients and point-space contact blocks mapped to
body space with the affine Jacobians, and the 12x12 block-Jacobi preconditioner.  Body b
owns block rows 4b..4b+3; FEM rows follow at 4 * body_num.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np
import torch

from . import _native as N
from .system import _dev, _p, _stream


def _hp(keep, a, dt):
    a = np.ascontiguousarray(a, dt)
    keep.append(a)
    return None if a.size == 0 else a.ctypes.data_as(C.c_void_p)


class ABDSystem:
    """Body-space gradient / Hessian assembly for ``body_num`` affine bodies.

    ``bodies`` holds host arrays: ``point_body`` (P,), ``x_bar`` (P,3), ``dyadic_mass``
    (B,13), ``volume`` (B,), ``boundary_type`` (B,)."""

    def __init__(self, bodies: dict, max_abd_blocks: int, max_fem_blocks: int, device: Optional[int] = None):
        dev = torch.cuda.current_device() if device is None else device
        keep = []
        t = N.SgipcAbdTopology()
        t.body_num = int(len(bodies["volume"]))
        t.point_num = int(len(bodies["point_body"]))
        t.point_body = _hp(keep, bodies["point_body"], np.int32)
        t.x_bar = _hp(keep, bodies["x_bar"], np.float64)
        t.dyadic_mass = _hp(keep, bodies["dyadic_mass"], np.float64)
        t.volume = _hp(keep, bodies["volume"], np.float64)
        t.boundary_type = _hp(keep, bodies["boundary_type"], np.int32)
        t.max_abd_blocks, t.max_fem_blocks = int(max_abd_blocks), int(max_fem_blocks)
        h = C.c_void_p()
        st = N.lib().sgipc_abd_create(C.byref(t), dev, C.byref(h))
        if st != N.OK:
            raise N.SgipcError(st, "sgipc_abd_create")
        self.ctx = h
        self.body_num = t.body_num
        self.point_num = t.point_num
        self.body_grad = torch.zeros(12 * self.body_num, dtype=torch.float64, device=_dev())

    def close(self):
        if getattr(self, "ctx", None):
            N.lib().sgipc_abd_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != N.OK:
            raise N.SgipcError(st, N.lib().sgipc_abd_last_error(self.ctx).decode())

    def setup_abd_system_gradient_hessian(self, q: torch.Tensor, q_tilde: torch.Tensor, kappa: float, dt: float,
                                          point_grad: Optional[torch.Tensor] = None,
                                          abd_blocks: Optional[Tuple[torch.Tensor, torch.Tensor, torch.Tensor]] = None,
                                          fem_blocks: Optional[Tuple[torch.Tensor, torch.Tensor, torch.Tensor]] = None,
                                          fem_boundary: Optional[torch.Tensor] = None) -> torch.Tensor:
        """Body gradient (12 * body_num,); the body-space matrix stays in the context.
        ``abd_blocks`` / ``fem_blocks``: (rows int32, cols int32, vals (n,3,3) float64) device
        tensors of point-space contact blocks (ABD-ABD with row <= col; ABD point x FEM vertex)."""
        a = abd_blocks or (None, None, None)
        f = fem_blocks or (None, None, None)
        na = 0 if abd_blocks is None else int(a[0].numel())
        nf = 0 if fem_blocks is None else int(f[0].numel())
        self._check(N.lib().sgipc_abd_grad_hess(self.ctx, _p(q), _p(q_tilde), float(kappa), float(dt), _p(point_grad),
                                                na, _p(a[0]), _p(a[1]), _p(a[2]), nf, _p(f[0]), _p(f[1]), _p(f[2]),
                                                _p(fem_boundary), _p(self.body_grad), _stream()))
        return self.body_grad

    def export_bcoo(self):
        cnt = C.c_int32()
        self._check(N.lib().sgipc_abd_export_bcoo(self.ctx, 0, None, None, None, C.byref(cnt)))
        n = cnt.value
        rows, cols = np.zeros(n, np.int32), np.zeros(n, np.int32)
        vals = np.zeros((n, 3, 3))
        self._check(N.lib().sgipc_abd_export_bcoo(self.ctx, n, rows.ctypes.data_as(C.c_void_p),
                                                  cols.ctypes.data_as(C.c_void_p), vals.ctypes.data_as(C.c_void_p),
                                                  C.byref(cnt)))
        return rows, cols, vals


class ABDPreconditioner:
    """12x12 block-Jacobi preconditioner of the affine bodies (``ABDPreconditioner``)."""

    def __init__(self, abd: ABDSystem):
        self.abd = abd

    def assemble(self):
        self.abd._check(N.lib().sgipc_abd_precond_build(self.abd.ctx, _stream()))

    def apply(self, r: torch.Tensor, z: Optional[torch.Tensor] = None) -> torch.Tensor:
        z = torch.empty_like(r) if z is None else z
        self.abd._check(N.lib().sgipc_abd_precond_apply(self.abd.ctx, _p(r), _p(z), _stream()))
        return z


class GlobalLinearSystem:
    """The global FEM + ABD system (``GlobalLinearSystem`` with ``ABDLinearSubsystem`` first
    and ``FEMLinearSubsystem`` after it, StiffGIPC/gipc/gipc.cu:42-70): one PCG
    (``PCGSolver::pcg``) over [12 * body_num ABD DOFs | 3 n FEM DOFs] with the ABD block
    Jacobi on the body rows and the MAS on the FEM rows
    (``GlobalLinearSystem::apply_preconditioner``, global_linear_system.cu:152-166).

    ``gipc`` is a :class:`sgipc.system.GIPC` whose system is assembled and whose MAS is built;
    ``abd`` an :class:`ABDSystem` after ``setup_abd_system_gradient_hessian`` and
    :meth:`ABDPreconditioner.assemble`."""

    def __init__(self, gipc, abd: ABDSystem):
        self.gipc = gipc
        self.abd = abd
        self.nb = 4 * abd.body_num
        self.dof = 3 * (self.nb + gipc.n)

    def right_hand_side(self, fem_rhs: Optional[torch.Tensor] = None) -> torch.Tensor:
        """b = [body gradient | FEM right-hand side] (``build_linear_system``'s rhs assembly)."""
        fem = self.gipc.rhs() if fem_rhs is None else fem_rhs
        return torch.cat([self.abd.body_grad, fem.reshape(-1).to(torch.float64)])

    def solve_linear_system(self, b: torch.Tensor, tol: float = 1e-4, criterion: int = N.CRIT_RZ,
                            max_iter_ratio: float = 0.3):
        """x (dof,), the ABD points' dx (P, 3) = J(x_bar) dq, and the solve stats."""
        b = b.reshape(-1).to(torch.float64).contiguous()
        if b.numel() != self.dof:
            raise ValueError("global right-hand side has %d entries, expected %d" % (b.numel(), self.dof))
        x = torch.empty_like(b)
        P = int(self.abd.point_num)
        pdx = torch.empty((max(P, 1), 3), dtype=torch.float64, device=b.device)
        st = N.SgipcSolveStats()
        s = N.lib().sgipc_global_pcg_solve(self.gipc.ctx, self.abd.ctx, int(criterion), float(tol),
                                           int(max_iter_ratio * self.dof), _p(b), _p(x), _p(pdx) if P else None,
                                           C.byref(st), _stream())
        N.check(s, self.gipc.ctx, allow=(N.OK, N.NOT_CONVERGED))
        return x, pdx[:P], st

    def distribute_solution(self, x: torch.Tensor):
        """(body dq (B, 12), FEM move direction (n, 3)) of a global solution."""
        return x[:3 * self.nb].reshape(-1, 12), x[3 * self.nb:].reshape(-1, 3)
