"""The line-search energy (``sgipc_compute_energy``, ``GIPC.computeEnergy``) against the
oracle's objective on the parity scenes, at the assembled positions and at perturbed ones,
through the C ABI.

Tolerances: 1e-10 relative to the oracle's total (the same per-element formulas, summed in
another order); the nine terms add up to the total to 1e-13; two calls agree bit for bit.
"""
import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sgipc import scenes, system  # noqa: E402

TERMS = ("kinetic", "tets", "triangles", "hinges", "soft", "barrier", "ground", "friction", "ground_friction")


def _soft_cube():
    sc = scenes.scene_cube(5, touching=True, seed=4)
    idx = np.arange(0, sc.nv, 11, dtype=np.int32)
    sc.soft_index = idx
    sc.soft_target = sc.vertexes[idx] + np.array([1e-3, 2e-3, -1e-3])
    sc.params["motionRate"] = 1.0
    sc.params["softRate"] = 1.0
    return sc


SCENES = {
    "c1_cube": lambda: scenes.scene_cube(11, touching=False, seed=0),
    "cube_touch": lambda: scenes.scene_cube(6, touching=True, seed=3),
    "two_cubes": lambda: scenes.scene_two_cubes(7, seed=5),
    "cloth_on_cube": lambda: scenes.scene_cloth_on_cube(10, 5, seed=6),
    "cube_soft": _soft_cube,
}


@pytest.fixture(scope="module", params=list(SCENES))
def case(request):
    sc = SCENES[request.param]()
    g = system.GIPC(sc)
    yield request.param, sc, g
    g.close()


def test_energy_matches_oracle(case):
    name, sc, g = case
    e, parts = g.computeEnergy(terms=True)
    eo = oracle.energy(sc)
    assert e == pytest.approx(eo, rel=1e-10, abs=0.0)
    assert abs(parts.sum() - e) <= 1e-13 * abs(e)
    assert parts[0] > 0  # the positions differ from x_tilde
    if name in ("cube_touch", "two_cubes", "cloth_on_cube", "cube_soft"):  # pair or ground contacts
        assert parts[5] + parts[6] > 0, dict(zip(TERMS, parts))
    if name == "cloth_on_cube":
        assert parts[2] > 0 and parts[3] != 0
    if name == "cube_soft":
        assert parts[4] > 0


def test_energy_at_perturbed_positions(case):
    name, sc, g = case
    rng = np.random.default_rng(21)
    x = sc.vertexes + 1e-7 * rng.standard_normal(sc.vertexes.shape)
    tet = system.DeviceTetraData(sc)
    tet.vertexes = torch.tensor(x, dtype=torch.float64, device="cuda")
    e = g.computeEnergy(tet)
    assert e == pytest.approx(oracle.energy(sc, x=x), rel=1e-10, abs=0.0)
    assert e != g.computeEnergy()


def test_energy_is_deterministic(case):
    _, _, g = case
    a, pa = g.computeEnergy(terms=True)
    b, pb = g.computeEnergy(terms=True)
    assert a == b and np.array_equal(pa, pb)


def test_energy_full_size():
    """Two stacked 21^3 cubes (80 000 tets, 21 628 barrier and friction pairs)."""
    sc = scenes.scene_two_cubes(21, seed=1)
    g = system.GIPC(sc)
    try:
        e, parts = g.computeEnergy(terms=True)
        assert e == pytest.approx(oracle.energy(sc), rel=1e-10, abs=0.0)
        assert parts[5] > 0 and parts[7] > 0
    finally:
        g.close()
