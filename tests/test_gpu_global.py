"""The global FEM + ABD solve (``sgipc_global_pcg_solve``, ``sgipc.abd.GlobalLinearSystem``)
on the GPU against the oracle's global PCG, through the C ABI.

Tolerances: iteration counts within 1; r0.z0 within 1e-9 (FP64 MAS) / 1e-5 (FP32 MAS
inverses); the solution within 1e-6 (FP64 MAS) / 1e-4 (FP32 MAS) of the oracle's when the
counts agree; a tight solve within 1e-8 of numpy's direct solution; the ABD points'
dx = J(x_bar) dq within 1e-12 of numpy's.
"""
import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sgipc import abd, scenes, system  # noqa: E402
from sgipc import _native as N  # noqa: E402
from test_oracle import global_system  # noqa: E402

NB = 12  # bodies


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _dev(a, dtype):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _abd_system(bodies, c, precond=True):
    sysm = abd.ABDSystem(bodies, max_abd_blocks=len(c["abd"][0]), max_fem_blocks=len(c["fem"][0]))
    i32, f64 = torch.int32, torch.float64
    sysm.setup_abd_system_gradient_hessian(
        _dev(bodies["q"], f64), _dev(bodies["q_tilde"], f64), bodies["kappa"], bodies["dt"],
        point_grad=_dev(c["point_grad"], f64),
        abd_blocks=tuple(_dev(a, t) for a, t in zip(c["abd"], (i32, i32, f64))),
        fem_blocks=tuple(_dev(a, t) for a, t in zip(c["fem"], (i32, i32, f64))),
        fem_boundary=_dev(c["fem_boundary"], i32))
    if precond:
        abd.ABDPreconditioner(sysm).assemble()
    return sysm


@pytest.fixture(scope="module")
def coupled():
    sc = scenes.scene_cube(5, touching=True, seed=3)
    bodies = scenes.scene_abd_boxes(NB, seed=7)
    A, fem, c, _ = global_system(sc, bodies, seed=4)
    g = system.GIPC(sc)
    g.computeGradientAndHessian()
    sysm = _abd_system(bodies, c)
    yield sc, bodies, A, fem, c, g, sysm
    sysm.close()
    g.close()


def _point_dx(bodies, x):
    dq = x[:12 * NB].reshape(NB, 12)[bodies["point_body"]]
    xb = bodies["x_bar"]
    return dq[:, :3] + np.einsum("pc,prc->pr", xb, dq[:, 3:].reshape(-1, 3, 3))


@pytest.mark.parametrize("prec", ["fp64", "ref"])
def test_global_solve_matches_oracle(coupled, prec):
    sc, bodies, A, (frow, fcol, fval), c, g, sysm = coupled
    assert np.linalg.eigvalsh(A).min() > 0
    system.MASPreconditioner(g).setPreconditioner(prec)
    om = oracle.Mas(sc, frow, fcol, fval)
    b = np.random.default_rng(11).normal(size=A.shape[0])
    gls = abd.GlobalLinearSystem(g, sysm)
    x, pdx, st = gls.solve_linear_system(torch.tensor(b, device="cuda"), tol=1e-4)
    x, pdx = x.cpu().numpy(), pdx.cpu().numpy()
    ox, oit, orz0, orz = oracle.global_pcg(A, NB, om, b, 1e-4, single=(prec == "ref"))
    assert st.status == N.OK
    assert abs(st.iterations - oit) <= 1
    assert st.rz0 == pytest.approx(orz0, rel=1e-9 if prec == "fp64" else 1e-5)
    if st.iterations == oit:
        assert _rel(x, ox) < (1e-6 if prec == "fp64" else 1e-4)
    res = np.linalg.norm(b - A @ x) / np.linalg.norm(b)
    assert st.rel_residual == pytest.approx(res, rel=1e-6)
    assert _rel(pdx, _point_dx(bodies, x)) < 1e-12
    dq, dx_fem = gls.distribute_solution(torch.tensor(x, device="cuda"))
    assert dq.shape == (NB, 12) and dx_fem.shape == (sc.nv, 3)


def test_global_solve_converges_to_direct_solution(coupled):
    sc, bodies, A, fem, c, g, sysm = coupled
    system.MASPreconditioner(g).setPreconditioner("fp64")
    b = np.random.default_rng(12).normal(size=A.shape[0])
    x, _, st = abd.GlobalLinearSystem(g, sysm).solve_linear_system(torch.tensor(b, device="cuda"), tol=1e-13,
                                                                  criterion=N.CRIT_TRUE, max_iter_ratio=2.0)
    assert st.status == N.OK
    ex = np.linalg.solve(A, b)
    assert _rel(x.cpu().numpy(), ex) < 1e-8


def test_global_solve_needs_both_preconditioners(coupled):
    sc, bodies, A, fem, c, g, _ = coupled
    system.MASPreconditioner(g).setPreconditioner("fp64")
    sysm = _abd_system(bodies, c, precond=False)
    try:
        b = torch.zeros(A.shape[0], dtype=torch.float64, device="cuda")
        with pytest.raises(N.SgipcError) as e:
            abd.GlobalLinearSystem(g, sysm).solve_linear_system(b)
        assert e.value.status == N.NOT_READY
    finally:
        sysm.close()


def test_global_solve_stops_at_cap_and_on_zero_rhs(coupled):
    """The loop's state lives on the device: at the iteration cap the solve reports
    NOT_CONVERGED after max_iter - 1 updates, at the iterate of the oracle's loop with the same
    cap (1e-9); a zero right-hand side stops before the first update (status OK, x = 0)."""
    sc, bodies, A, (frow, fcol, fval), c, g, sysm = coupled
    system.MASPreconditioner(g).setPreconditioner("fp64")
    om = oracle.Mas(sc, frow, fcol, fval)
    gls = abd.GlobalLinearSystem(g, sysm)
    b = np.random.default_rng(13).normal(size=A.shape[0])
    cap = 4
    x, _, st = gls.solve_linear_system(torch.tensor(b, device="cuda"), tol=1e-14, max_iter_ratio=(cap + 0.5) / gls.dof)
    ox, oit, orz0, _ = oracle.global_pcg(A, NB, om, b, 1e-14, max_iter=cap)
    assert st.status == N.NOT_CONVERGED
    assert st.iterations == cap - 1 and oit == cap  # the oracle counts as or_pcg does
    assert _rel(x.cpu().numpy(), ox) < 1e-9
    z, _, st0 = gls.solve_linear_system(torch.zeros(A.shape[0], dtype=torch.float64, device="cuda"))
    assert st0.status == N.OK and st0.iterations == 0
    assert float(z.abs().max()) == 0.0
