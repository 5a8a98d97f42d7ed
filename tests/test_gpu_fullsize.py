"""The bench workload at full size (two stacked 21^3 cubes, 18 522 vertices, 80 000 tets,
contacts) through size-independent properties; the oracle covers the same code paths on the
smaller parity scenes.

Tolerances: SpMV and FP64 MAS symmetry 1e-12 / 1e-10 relative to |u||A v|; reported relative
residual within 1e-6 of one recomputed with the library's FP64 SpMV; persistent vs graph
FP64 solves 1e-9; tight (1e-10 true residual) mixed vs FP64 solutions 1e-7; every column of
a 4-RHS batch within its tolerance and 1e-8 of the single-RHS solve.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sgipc import scenes, system  # noqa: E402
from sgipc import _native as N  # noqa: E402


@pytest.fixture(scope="module")
def c2():
    sc = scenes.scene_two_cubes(21, seed=1)
    g = system.GIPC(sc, max_rhs=4)
    g.computeGradientAndHessian()
    yield sc, g
    g.close()


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-300))


def _residual(g, b, x):
    return float((b - g.spmv(x)).norm() / b.norm())


def test_fullsize_operators_are_symmetric_and_positive(c2):
    sc, g = c2
    gen = torch.Generator(device="cuda").manual_seed(3)
    u = torch.randn(3 * sc.nv, dtype=torch.float64, device="cuda", generator=gen)
    v = torch.randn(3 * sc.nv, dtype=torch.float64, device="cuda", generator=gen)
    Au, Av = g.spmv(u), g.spmv(v)
    assert float((u @ Av - v @ Au).abs()) <= 1e-12 * float(u.norm() * Av.norm())
    assert float(u @ Au) > 0
    mas = system.MASPreconditioner(g)
    mas.setPreconditioner("fp64")
    Mu, Mv = mas.preconditioning(u), mas.preconditioning(v)
    assert float((u @ Mv - v @ Mu).abs()) <= 1e-10 * float(u.norm() * Mv.norm())
    assert float(u @ Mu) > 0


@pytest.mark.parametrize("prec", ["fp64", "mixed", "ref"])
def test_fullsize_solve_meets_its_criterion(c2, prec):
    sc, g = c2
    system.MASPreconditioner(g).setPreconditioner(prec)
    b = g.rhs()
    x, st = system.PCGSolver(g, system.PCGSolverConfig(precision=prec)).solve(b)
    assert st.status == N.OK and 0 < st.iterations < 0.3 * 3 * sc.nv
    assert st.rel_residual == pytest.approx(_residual(g, b, x), rel=1e-6)
    assert abs(st.rz) <= 1e-4 * st.rz0 * (1 + 1e-9)


def test_fullsize_persistent_and_graph_agree(c2, monkeypatch):
    sc, g = c2
    system.MASPreconditioner(g).setPreconditioner("fp64")
    solver = system.PCGSolver(g, system.PCGSolverConfig(precision="fp64"))
    xa, sa = solver.solve(g.rhs())
    monkeypatch.setenv("SGIPC_PCG_GRAPH", "1")
    xb, sb = solver.solve(g.rhs())
    monkeypatch.delenv("SGIPC_PCG_GRAPH")
    assert abs(sa.iterations - sb.iterations) <= 1
    if sa.iterations == sb.iterations:
        assert _rel(xa, xb) < 1e-9


def test_fullsize_tight_mixed_matches_fp64(c2):
    sc, g = c2
    xs = {}
    for prec in ("fp64", "mixed"):
        system.MASPreconditioner(g).setPreconditioner(prec)
        cfg = system.PCGSolverConfig(precision=prec, global_tol_rate=1e-10, criterion=N.CRIT_TRUE, max_iter_ratio=1.0)
        xs[prec], st = system.PCGSolver(g, cfg).solve(g.rhs())
        assert st.status == N.OK, prec
        assert _residual(g, g.rhs(), xs[prec]) < 1e-9, prec
    assert _rel(xs["mixed"], xs["fp64"]) < 1e-7


def test_fullsize_four_rhs_batch_matches_single_solves(c2):
    sc, g = c2
    system.MASPreconditioner(g).setPreconditioner("fp64")
    gen = torch.Generator(device="cuda").manual_seed(5)
    B = torch.randn(4, 3 * sc.nv, dtype=torch.float64, device="cuda", generator=gen)
    cfg = system.PCGSolverConfig(precision="fp64", global_tol_rate=1e-10, criterion=N.CRIT_TRUE, max_iter_ratio=1.0)
    solver = system.PCGSolver(g, cfg)
    X, sts = solver.solve_batched(B)
    for r in range(4):
        assert sts[r].status == N.OK
        assert _residual(g, B[r], X[r]) < 1e-9
        x1, _ = solver.solve(B[r].contiguous())
        assert _rel(X[r], x1) < 1e-8
