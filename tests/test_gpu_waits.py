"""Bounded device waits, made to run out on purpose (no fault, no hang).

The persistent PCG solve and the one-launch MAS hierarchy build separate their phases with
grid barriers whose waits are bounded: past the limit a CTA raises the kernel's abort word,
every CTA leaves at its next barrier, and the call returns SGIPC_CUDA_ERROR with a message.
``sgipc_set_wait_limit(ctx, 1)`` shortens every wait to a couple of polls, so that the first
CTA to arrive gives up before the grid has gathered; limit 0 restores the default (about
2 s).  After such a call the context must solve normally: with the same preconditioner the
same iterations and the same solution, bit for bit (the persistent solve is deterministic); with
a rebuilt one the solution to 1e-10 (the domain matrices are summed with atomics).
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sgipc import scenes, system  # noqa: E402
from sgipc import _native as N  # noqa: E402


@pytest.fixture(scope="module")
def g():
    sc = scenes.scene_two_cubes(7, seed=5)
    gg = system.GIPC(sc)
    yield gg
    gg.close()


def _solve(g, prec):
    g.computeGradientAndHessian()
    system.MASPreconditioner(g).setPreconditioner(prec)
    x, st = system.PCGSolver(g, system.PCGSolverConfig(precision=prec)).solve(g.rhs())
    return x.cpu().numpy(), st


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_pcg_barrier_wait_runs_out_and_the_context_recovers(g, prec):
    L = N.lib()
    g.computeGradientAndHessian()
    system.MASPreconditioner(g).setPreconditioner(prec)
    solver = system.PCGSolver(g, system.PCGSolverConfig(precision=prec))
    x0, st0 = solver.solve(g.rhs())
    x0 = x0.cpu().numpy()
    assert st0.status == N.OK
    b = g.rhs()
    x = torch.empty_like(b)
    N.check(L.sgipc_set_wait_limit(g.ctx, 1), g.ctx)
    try:
        st = N.SgipcSolveStats()
        s = L.sgipc_pcg_solve(g.ctx, N.PRECISION[prec], N.CRIT_RZ, 1e-4, 0, ctypes.c_void_p(b.data_ptr()),
                              ctypes.c_void_p(x.data_ptr()), ctypes.byref(st), None)
        assert s == N.CUDA_ERROR, s
        assert b"wait limit" in L.sgipc_last_error(g.ctx)
    finally:
        N.check(L.sgipc_set_wait_limit(g.ctx, 0), g.ctx)
    torch.cuda.synchronize()  # the device is healthy: nothing is pending or faulted
    # the same preconditioner: the persistent solve is deterministic, bit for bit
    x1, st1 = solver.solve(g.rhs())
    assert st1.status == N.OK and st1.iterations == st0.iterations
    assert np.array_equal(x1.cpu().numpy(), x0)


def test_hierarchy_barrier_wait_runs_out_and_the_context_recovers(g):
    L = N.lib()
    x0, st0 = _solve(g, "fp64")
    N.check(L.sgipc_set_wait_limit(g.ctx, 1), g.ctx)
    try:
        g.computeGradientAndHessian()  # starts the one-launch hierarchy build beside the assembly
        con = g.tet.contact_struct_cached()
        s = L.sgipc_mas_build(g.ctx, ctypes.byref(con), N.PRECISION["fp64"], None)
        assert s == N.CUDA_ERROR, s
        assert b"hierarchy" in L.sgipc_last_error(g.ctx)
    finally:
        N.check(L.sgipc_set_wait_limit(g.ctx, 0), g.ctx)
    torch.cuda.synchronize()
    # a new hierarchy and domain matrices (accumulated with atomics: equal to rounding)
    x1, st1 = _solve(g, "fp64")
    assert st1.status == N.OK and st1.iterations == st0.iterations
    assert np.abs(x1 - x0).max() <= 1e-10 * np.abs(x0).max()


def test_wait_limit_rejects_negative_values(g):
    assert N.lib().sgipc_set_wait_limit(g.ctx, -1) == N.BAD_INPUT
