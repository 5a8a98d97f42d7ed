"""The implicit-step adjoint on the GPU (no counterpart in the reference).

For the implicit step x*(theta) with g(x*; theta) = 0 and a loss L(x*):
    A lambda = dL/dx*,   dL/dtheta = -lambda^T dg/dtheta
(theta = per-tet Young's modulus E_t, per-vertex initial velocity v0).  Checked against
  * an FP64 dense solve of the oracle's assembled matrix and the oracle's gradient
    differentiated along random parameter directions (g is linear in E and in v0, so a
    finite step is exact up to rounding): 1e-8 relative;
  * 4 right-hand sides in one batched solve vs four single solves: 1e-8;
  * ``ImplicitStep`` (torch.autograd.Function: Newton forward, adjoint backward) against
    the dense FP64 adjoint of the same projected Hessian (1e-7), and central finite
    differences (h = 1e-6 along random directions in E and v0) of the converged step's
    loss against the adjoint with the exact Hessian (1e-4).
"""
import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sgipc import adjoint, scenes, system  # noqa: E402
from sgipc import _native as N  # noqa: E402


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def touching_cube():
    sc = scenes.scene_cube(5, touching=True, seed=7)
    g = system.GIPC(sc, max_rhs=4)
    g.computeGradientAndHessian()
    yield sc, g
    g.close()


def test_adjoint_matches_dense_fp64(touching_cube):
    sc, g = touching_cube
    rng = np.random.default_rng(11)
    dLdx = rng.normal(size=(4, 3 * sc.nv))
    dLdE, dLdv0, lam, stats = adjoint.adjoint(g, torch.tensor(dLdx, device="cuda"), precision="fp64", tol=1e-12,
                                              criterion=N.CRIT_TRUE)
    dLdE, dLdv0, lam = dLdE.cpu().numpy(), dLdv0.cpu().numpy(), lam.cpu().numpy()
    assert all(s.status == N.OK for s in stats)
    b0, rows, cols, vals, _ = oracle.assemble(sc)
    A = oracle.dense(rows, cols, vals, sc.nv)
    lam_ref = np.linalg.solve(A, dLdx.T).T
    assert _rel(lam, lam_ref) < 1e-8
    # dg/dE along random directions dE: g(E + dE) - g(E), exact because g is linear in E
    for k in range(3):
        dE = rng.uniform(-0.5, 0.5, sc.nt) * sc.youngs
        sc2 = scenes.Scene(**{**sc.__dict__})
        sc2.length_rate, sc2.volume_rate = scenes.snk_rates(sc.youngs + dE, sc.poisson)
        db = oracle.assemble(sc2)[0] - b0
        assert (dLdE @ dE) == pytest.approx(-(lam_ref @ db), rel=1e-8)
    # dg/dv0 = -dt M on free rows
    dt = sc.params["dt"]
    free = np.repeat(sc.boundary_type == 0, 3)
    ref_v0 = dt * np.repeat(sc.masses, 3)[None] * lam_ref * free[None]
    assert _rel(dLdv0, ref_v0) < 1e-8


def test_batched_adjoint_matches_single(touching_cube):
    sc, g = touching_cube
    rng = np.random.default_rng(12)
    dLdx = torch.tensor(rng.normal(size=(4, 3 * sc.nv)), device="cuda")
    E4, v4, l4, _ = adjoint.adjoint(g, dLdx, precision="fp64", tol=1e-12, criterion=N.CRIT_TRUE)
    for r in range(4):
        E1, v1, l1, _ = adjoint.adjoint(g, dLdx[r:r + 1].contiguous(), precision="fp64", tol=1e-12,
                                        criterion=N.CRIT_TRUE)
        assert _rel(l4[r].cpu().numpy(), l1[0].cpu().numpy()) < 1e-8
        assert _rel(E4[r].cpu().numpy(), E1[0].cpu().numpy()) < 1e-8


@pytest.fixture(scope="module")
def clamped_cube():
    """A soft cube whose bottom layer is held (Dirichlet), sagging under gravity: the step
    strains the solid, so the loss depends on every tet's modulus."""
    sc = scenes.scene_cube(4, touching=False, seed=8)
    y = sc.rest_vertexes[:, 1]
    sc.boundary_type = (y < y.min() + 1e-9).astype(np.int32)
    sc.xTilta = sc.o_vertexes + sc.params["dt"] ** 2 * np.where(sc.boundary_type[:, None] == 0,
                                                                np.array([[0.0, -9.8, 0.0]]), 0.0)
    sc.params["dt"] = 0.05   # a longer step sags the cube further
    g = system.GIPC(sc, max_rhs=4)
    yield sc, g
    g.close()


def _loss(x, target, w):
    return (w * (x - target) ** 2).sum()


def test_implicit_step_gradient_matches_finite_differences(clamped_cube):
    """``ImplicitStep`` (forward: Newton to convergence; backward: the adjoint) against
    (a) the dense FP64 adjoint with the same projected Hessian the path solves with, and
    (b) central finite differences of the converged step's loss along random directions in
    E and v0, compared with the adjoint built on the exact (unprojected) Hessian: the
    projection of the stable Neo-Hookean Hessian (active even near rest) is the only
    difference between (a) and the true derivative."""
    sc, g = clamped_cube
    rng = np.random.default_rng(13)
    x_start = g.tet.vertexes.clone()
    E0 = torch.tensor(sc.youngs, device="cuda")
    v00 = torch.tensor(rng.normal(scale=0.1, size=(sc.nv, 3)), device="cuda")
    target = torch.tensor(sc.vertexes + rng.normal(scale=1e-3, size=(sc.nv, 3)), device="cuda")
    w = torch.tensor(rng.uniform(0.5, 1.5, size=(sc.nv, 1)), device="cuda")

    def run(E, v0):
        g.tet.vertexes.copy_(x_start)
        return adjoint.ImplicitStep.apply(E, v0, g)

    E = E0.clone().requires_grad_(True)
    v0 = v00.clone().requires_grad_(True)
    x = run(E, v0)
    assert g.rhs().norm().item() < 1e-10
    L = _loss(x, target, w)
    L.backward()
    gE, gv = E.grad.cpu().numpy(), v0.grad.cpu().numpy().ravel()
    xs = x.detach().cpu().numpy()
    dLdx = (2.0 * w * (x.detach() - target)).cpu().numpy().ravel() * np.repeat(sc.boundary_type == 0, 3)

    # the converged state on the host, with the parameters ImplicitStep wrote
    st = scenes.Scene(**{**sc.__dict__})
    st.vertexes = xs
    st.xTilta = g.tet.xTilta.cpu().numpy()
    st.length_rate, st.volume_rate = scenes.snk_rates(sc.youngs, sc.poisson)
    b0, rows, cols, vals, _ = oracle.assemble(st)
    lam = np.linalg.solve(oracle.dense(rows, cols, vals, sc.nv), dLdx)
    with oracle.exact_snk_hessian():
        _, rows2, cols2, vals2, _ = oracle.assemble(st)
    lam_exact = np.linalg.solve(oracle.dense(rows2, cols2, vals2, sc.nv), dLdx)

    dt = sc.params["dt"]
    free = np.repeat(sc.boundary_type == 0, 3)
    for k in range(2):
        dE = rng.uniform(-0.5, 0.5, sc.nt) * sc.youngs
        s2 = scenes.Scene(**{**st.__dict__})
        s2.length_rate, s2.volume_rate = scenes.snk_rates(sc.youngs + dE, sc.poisson)
        db = oracle.assemble(s2)[0] - b0       # exact: g is linear in E
        assert gE @ dE == pytest.approx(-(lam @ db), rel=1e-7)
        h = 1e-6
        with torch.no_grad():
            dEt = torch.tensor(dE, device="cuda")
            fd = (_loss(run(E0 + h * dEt, v00), target, w) - _loss(run(E0 - h * dEt, v00), target, w)).item() / (2 * h)
        assert fd == pytest.approx(-(lam_exact @ db), rel=1e-4)
        dv = rng.normal(size=3 * sc.nv)
        dbv = -dt * np.repeat(sc.masses, 3) * dv * free  # dg/dv0 . dv
        assert gv @ dv == pytest.approx(-(lam @ dbv), rel=1e-7)
        with torch.no_grad():
            dvt = torch.tensor(dv.reshape(-1, 3), device="cuda")
            fd = (_loss(run(E0, v00 + h * dvt), target, w) - _loss(run(E0, v00 - h * dvt), target, w)).item() / (2 * h)
        assert fd == pytest.approx(-(lam_exact @ dbv), rel=1e-4)
