"""The bench workload at full size (two stacked 21^3 cubes, 18 522 vertices, 80 000 tets,
contacts): against the oracle (the CPU restatement finishes this size in about a second:
assembled blocks and right-hand side 1e-9 of the largest entry, MAS tables identical and
domain inverses 1e-9, the FP64 solve's iteration count within one of the oracle's and its
solution 1e-6), and through size-independent properties.

Tolerances: SpMV and FP64 MAS symmetry 1e-12 / 1e-10 relative to |u||A v|; reported relative
residual within 1e-6 of one recomputed with the library's FP64 SpMV; persistent vs graph
FP64 solves 1e-9; tight (1e-10 true residual) mixed vs FP64 solutions 1e-7; every column of
a 4-RHS batch within its tolerance and 1e-8 of the single-RHS solve.
"""
import numpy as np
import pytest

import oracle

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


@pytest.fixture(scope="module")
def c2_oracle(c2):
    sc, _ = c2
    ob, orow, ocol, oval, _ = oracle.assemble(sc)
    return ob, orow, ocol, oval


def test_fullsize_assembly_matches_oracle(c2, c2_oracle):
    sc, g = c2
    ob, orow, ocol, oval = c2_oracle
    rows, cols, vals = g.export_bcoo()
    assert np.array_equal(rows, orow) and np.array_equal(cols, ocol)
    assert np.abs(vals - oval).max() < 1e-9 * np.abs(oval).max()
    b = g.rhs().cpu().numpy()
    assert np.abs(b - ob).max() < 1e-9 * np.abs(ob).max()


def test_fullsize_mas_and_fp64_solve_match_oracle(c2, c2_oracle):
    sc, g = c2
    ob, orow, ocol, oval = c2_oracle
    g.computeGradientAndHessian()
    mas = system.MASPreconditioner(g)
    mas.setPreconditioner("fp64")
    om = oracle.Mas(sc, orow, ocol, oval)
    L, _, counts, total = om.info()
    gl, gcounts, gtotal = mas.info()
    assert gl == L and gtotal == total and np.array_equal(gcounts, counts)
    assert np.array_equal(mas.tables(), om.table())
    gd, od = mas.domains(), om.domains()
    assert np.abs(gd - od).max(axis=(1, 2)).max() < 1e-9 * np.abs(od).max()
    ox, oit, orz0, _ = oracle.pcg(orow, ocol, oval, sc.nv, om, ob, 1e-4)
    x, st = system.PCGSolver(g, system.PCGSolverConfig(precision="fp64")).solve(g.rhs())
    assert st.status == N.OK and abs(st.iterations - oit) <= 1, (st.iterations, oit)
    assert abs(st.rz0 - orz0) <= 1e-9 * abs(orz0)
    if st.iterations == oit:
        x = x.cpu().numpy()
        assert np.linalg.norm(x - ox) / np.linalg.norm(ox) < 1e-6


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
