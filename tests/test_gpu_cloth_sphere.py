"""The cloth-on-sphere workload at full size: a 256 x 256 cloth (66 049 vertices, 130 050
triangles, 195 585 bending hinges) rolled into layers 0.4 mm apart over a 20 000-tet sphere
resting on the ground, with d-hat 0.5 mm.  Its contacts come from the GPU pair search
(``sgipc_build_cp``, about a million pairs, mostly cloth self-contact) and its lagged friction
sets from ``sgipc_friction_setup``; the Newton system is then checked against the oracle's
assembly of the same inputs and solved in FP64 and mixed precision.

Tolerances: integer outputs exact; assembled blocks and right-hand side 1e-9 of the largest
entry; MAS tables identical, domain inverses 1e-8 (Gauss-Jordan without pivoting on
ill-conditioned cloth domains); SpMV symmetry 1e-12 relative to
|u||A v|; reported relative residual within 1e-6 of one recomputed with the FP64 SpMV; tight
(1e-10 true residual) mixed vs FP64 solutions 1e-6 (this matrix is far less well conditioned
than the two-cube one: membrane and bending stiffness against millimetre layers).
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
def c3():
    sc = scenes.scene_cloth_on_sphere(256, 4000, contacts=False)
    g = system.GIPC(sc, max_rhs=1, pair_capacity=2_000_000)
    out = g.buildCP()
    g.buildFrictionSets()
    g.computeGradientAndHessian()
    torch.cuda.synchronize()
    yield sc, g, out
    g.close()


@pytest.fixture(scope="module")
def c3_host(c3):
    """The scene with the GPU's contact and friction arrays, for the oracle."""
    sc, g, _ = c3
    t = g.tet
    s = scenes.Scene(**{**sc.__dict__})
    s.pairs, s.ground_pairs = t.pairs.cpu().numpy(), t.ground_pairs.cpu().numpy()
    s.fric_pairs, s.fric_lambda = t.fric_pairs.cpu().numpy(), t.fric_lambda.cpu().numpy()
    s.fric_coord, s.fric_basis = t.fric_coord.cpu().numpy(), t.fric_basis.cpu().numpy().reshape(-1, 3, 2)
    s.fric_gd_pairs, s.fric_gd_lambda = t.fric_gd_pairs.cpu().numpy(), t.fric_gd_lambda.cpu().numpy()
    ob, orow, ocol, oval, _ = oracle.assemble(s)
    return s, (ob, orow, ocol, oval)


def _residual(g, b, x):
    return float((b - g.spmv(x)).norm() / b.norm())


def test_contact_sets_are_dense_ranked_and_repeatable(c3):
    sc, g, out = c3
    cp = out["cp_num"]
    assert cp[0] > 500_000 and cp[0] == cp[2] + cp[3] + cp[4]
    assert out["gp_num"] > 0 and len(g.tet.fric_pairs) > 0
    p, mi = out["pairs"].cpu().numpy(), out["mat_index"].cpu().numpy()
    size = np.where(p[:, 0] >= 0, 4, np.where(p[:, 2] < 0, 2, np.where(p[:, 3] < 0, 3, 4)))
    for k, nv in ((2, 2), (3, 3), (4, 4)):
        assert np.array_equal(mi[size == nv], np.arange(cp[k]))
    again = g.buildCP(update=False)
    for k in ("pairs", "ccd_pairs", "mat_index", "ground_pairs"):
        assert torch.equal(again[k], out[k]), k


def test_assembly_matches_oracle(c3, c3_host):
    sc, g, _ = c3
    _, (ob, orow, ocol, oval) = c3_host
    rows, cols, vals = g.export_bcoo()
    assert np.array_equal(rows, orow) and np.array_equal(cols, ocol)
    assert np.abs(vals - oval).max() < 1e-9 * np.abs(oval).max()
    b = g.rhs().cpu().numpy()
    assert np.abs(b - ob).max() < 1e-9 * np.abs(ob).max()


def test_mas_matches_oracle(c3, c3_host):
    sc, g, _ = c3
    s, (ob, orow, ocol, oval) = c3_host
    g.computeGradientAndHessian()
    mas = system.MASPreconditioner(g)
    mas.setPreconditioner("fp64")
    om = oracle.Mas(s, orow, ocol, oval)
    L, _, counts, total = om.info()
    gl, gcounts, gtotal = mas.info()
    assert gl == L and gtotal == total and np.array_equal(gcounts, counts)
    assert np.array_equal(mas.tables(), om.table())
    gd, od = mas.domains(), om.domains()
    # Gauss-Jordan without pivoting on both sides: the cloth's worst domains amplify the
    # assembly's 1e-12 rounding differences to a few 1e-9 of the largest entry
    assert np.abs(gd - od).max(axis=(1, 2)).max() < 1e-8 * np.abs(od).max()


def test_matrix_is_symmetric_and_positive(c3):
    sc, g, _ = c3
    gen = torch.Generator(device="cuda").manual_seed(5)
    u = torch.randn(3 * sc.nv, dtype=torch.float64, device="cuda", generator=gen)
    v = torch.randn(3 * sc.nv, dtype=torch.float64, device="cuda", generator=gen)
    Au, Av = g.spmv(u), g.spmv(v)
    assert float((u @ Av - v @ Au).abs()) <= 1e-12 * float(u.norm() * Av.norm())
    assert float(u @ Au) > 0


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_solve_meets_its_criterion(c3, prec):
    sc, g, _ = c3
    system.MASPreconditioner(g).setPreconditioner(prec)
    b = g.rhs()
    x, st = system.PCGSolver(g, system.PCGSolverConfig(precision=prec)).solve(b)
    assert st.status == N.OK and 0 < st.iterations
    assert st.rel_residual == pytest.approx(_residual(g, b, x), rel=1e-6)
    assert abs(st.rz) <= 1e-4 * st.rz0 * (1 + 1e-9)


def test_tight_mixed_matches_fp64(c3):
    sc, g, _ = c3
    xs = {}
    for prec in ("fp64", "mixed"):
        system.MASPreconditioner(g).setPreconditioner(prec)
        cfg = system.PCGSolverConfig(precision=prec, global_tol_rate=1e-10, criterion=N.CRIT_TRUE, max_iter_ratio=1.0)
        xs[prec], st = system.PCGSolver(g, cfg).solve(g.rhs())
        assert st.status == N.OK, prec
        assert _residual(g, g.rhs(), xs[prec]) < 1e-9, prec
    d = (xs["mixed"] - xs["fp64"]).abs().max() / xs["fp64"].abs().max()
    assert float(d) < 1e-6
