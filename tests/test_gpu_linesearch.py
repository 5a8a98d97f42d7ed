"""The line-search entry points together, through the C ABI: trial positions
(``sgipc_step_forward``) against numpy, and one backtracking line search as the reference's
``GIPC::lineSearch`` runs it (GIPC.cu:10676): the step bounded by the ground and CCD bounds,
halved until the energy falls below the start; the accepted energy equals the oracle's at
the same positions.

Tolerances: trial positions bit for bit (product and difference rounded separately, as
the reference evaluates them); energies 1e-10.
"""
import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sgipc import scenes, system  # noqa: E402


@pytest.fixture(scope="module")
def g():
    sc = scenes.scene_two_cubes(7, seed=5)
    gg = system.GIPC(sc)
    yield sc, gg
    gg.close()


def _ccd_candidates(pairs):
    """Point-triangle and edge-edge candidates out of the barrier pair list."""
    enc = np.asarray(pairs, np.int32).reshape(-1, 4)
    keep = ((enc[:, 0] < 0) & (enc[:, 2] >= 0) & (enc[:, 3] >= 0)) | (enc[:, 0] >= 0)
    cand = enc[keep].copy()
    ee = cand[:, 0] >= 0
    cand[ee, 3] = np.where(cand[ee, 3] < 0, -cand[ee, 3] - 1, cand[ee, 3])
    return cand


def test_step_forward_matches_numpy(g):
    sc, gg = g
    rng = np.random.default_rng(2)
    xb = sc.vertexes + 1e-3 * rng.standard_normal(sc.vertexes.shape)
    d = rng.standard_normal(sc.vertexes.shape)
    # a few fixed vertices, so that move_boundary=False has rows to keep
    btype = sc.boundary_type.copy()
    sc.boundary_type = btype.copy()
    sc.boundary_type[::7] = 1
    try:
        tet = system.DeviceTetraData(sc)
    finally:
        sc.boundary_type, fixed_type = btype, sc.boundary_type
    for move_boundary in (False, True):
        tet.vertexes.copy_(torch.tensor(sc.vertexes, device="cuda"))
        gg.step_forward(0.37, torch.tensor(xb, device="cuda"), torch.tensor(d, device="cuda"), tet=tet,
                        move_boundary=move_boundary)
        want = xb - 0.37 * d
        if not move_boundary:
            fixed = fixed_type != 0
            assert fixed.any()
            want[fixed] = sc.vertexes[fixed]
        got = tet.vertexes.cpu().numpy()
        assert np.array_equal(got, want)


def test_backtracking_line_search_decreases_the_energy(g):
    sc, gg = g
    gg.computeGradientAndHessian()
    st = gg.calculateMovingDirection(system.PCGSolverConfig(precision="fp64"))
    assert st.iterations > 0
    x0 = gg.tet.vertexes.clone()
    e0 = gg.computeEnergy()
    verts = torch.arange(sc.nv, dtype=torch.int32, device="cuda")
    cand = torch.tensor(_ccd_candidates(sc.pairs), device="cuda")
    alpha = min(1.0, gg.ground_largestFeasibleStepSize(0.8, gg.moveDir, verts),
                gg.self_largestFeasibleStepSize(0.8, gg.moveDir, cand))
    assert 0.0 < alpha <= 1.0
    try:
        for _ in range(9):
            gg.step_forward(alpha, x0)
            e = gg.computeEnergy()
            if e < e0:
                break
            alpha /= 2
        assert e < e0, (e, e0, alpha)
        x = gg.tet.vertexes.cpu().numpy()
        assert e == pytest.approx(oracle.energy(sc, x=x), rel=1e-10, abs=0.0)
    finally:
        gg.tet.vertexes.copy_(x0)
