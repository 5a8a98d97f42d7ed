"""Line-search step bounds on the GPU (``sgipc_self_step_size``, ``sgipc_ground_step_size``)
against the oracle, through the C ABI: the known-answer cases, and random point-triangle and
edge-edge candidates over the vertices of a scene with random step directions.

Tolerances: known answers 1e-12; random candidates: each time of impact within 1e-9 of the
oracle's (the same arithmetic up to FMA contraction; a comparison that flips on the last bit
could change one candidate by one additive step, so at most 0.1 % of them may differ, by
less than 5 %); the step of the set within 1e-9.
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
from test_oracle_ccd import EDGES, EE, PT, TRI, _dir  # noqa: E402


def _dev(a, dtype=torch.float64):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


@pytest.fixture(scope="module")
def g():
    sc = scenes.scene_two_cubes(7, seed=5)
    gg = system.GIPC(sc)
    yield sc, gg
    gg.close()


def _candidates(nv, n, rng):
    """n random candidates over distinct vertices, half point-triangle (x < 0)."""
    q = np.array([rng.choice(nv, 4, replace=False) for _ in range(n)], np.int32)
    pt = rng.random(n) < 0.5
    q[pt, 0] = -q[pt, 0] - 1
    return q


def test_known_answers(g):
    sc, gg = g
    x = np.zeros((sc.nv, 3))
    cases = [(TRI, _dir(4, [0], [0, 0, -2.0]), PT), (EDGES, _dir(4, [0, 1], [0, 0, -2.0]), EE)]
    for pos, d, pairs in cases:
        x[:4] = pos
        dd = np.zeros((sc.nv, 3))
        dd[:4] = d
        a = gg.self_largestFeasibleStepSize(0.8, _dev(dd), _dev(pairs, torch.int32), x=_dev(x))
        assert a == pytest.approx(0.4, rel=1e-12)
    x[:4] = TRI
    assert gg.self_largestFeasibleStepSize(0.8, _dev(np.zeros((sc.nv, 3))), _dev(PT, torch.int32), x=_dev(x)) == 1.0


@pytest.mark.parametrize("scale", [0.02, 0.2])
def test_random_candidates_match_oracle(g, scale):
    sc, gg = g
    rng = np.random.default_rng(int(scale * 100))
    x = sc.vertexes + 1e-3 * rng.standard_normal((sc.nv, 3))  # no exactly collinear lattice triples
    d = scale * rng.standard_normal((sc.nv, 3))
    pairs = _candidates(sc.nv, 4000, rng)
    toi = torch.zeros(len(pairs), dtype=torch.float64, device="cuda")
    a = gg.self_largestFeasibleStepSize(0.8, _dev(d), _dev(pairs, torch.int32), x=_dev(x), toi=toi)
    ao, to = oracle.self_step(x, d, pairs, 0.8)
    tg = toi.cpu().numpy()
    rel = np.abs(tg - to) / np.maximum(np.abs(to), 1e-300)
    assert (rel > 1e-9).mean() <= 1e-3 and rel.max() < 0.05
    assert a == pytest.approx(ao, rel=1e-9)
    assert 0.0 < a <= 1.0 and np.all(tg > 0) and np.all(tg <= 1.0)


def test_ground_bound_matches_oracle(g):
    sc, gg = g
    rng = np.random.default_rng(3)
    d = 0.05 * rng.standard_normal((sc.nv, 3))
    verts = np.arange(sc.nv, dtype=np.int32)
    a = gg.ground_largestFeasibleStepSize(0.8, _dev(d), _dev(verts, torch.int32))
    ao = oracle.ground_step(sc.vertexes, d, verts.astype(np.uint32), sc.params.get("ground_offset", 0.0), 0.8)
    assert a == pytest.approx(ao, rel=1e-12)


def test_cfl_speed_matches_oracle(g):
    sc, gg = g
    d = np.random.default_rng(4).standard_normal((sc.nv, 3))
    verts = np.arange(0, sc.nv, 3, dtype=np.int32)
    v = gg.cfl_largestSpeed(_dev(d), _dev(verts, torch.int32))
    assert v == pytest.approx(oracle.cfl_speed(d, verts.astype(np.uint32)), rel=1e-14)
    assert gg.cfl_largestSpeed(_dev(d), torch.zeros(0, dtype=torch.int32, device="cuda")) == 0.0


def test_empty_sets_and_bad_indices(g):
    sc, gg = g
    z = _dev(np.zeros((sc.nv, 3)))
    assert gg.self_largestFeasibleStepSize(0.8, z, torch.zeros((0, 4), dtype=torch.int32, device="cuda")) == 1.0
    assert gg.ground_largestFeasibleStepSize(0.8, z, torch.zeros(0, dtype=torch.int32, device="cuda")) == 1.0
    with pytest.raises(N.SgipcError) as e:
        gg.self_largestFeasibleStepSize(0.8, z, _dev([[0, 1, 2, sc.nv]], torch.int32))
    assert e.value.status == N.BAD_INPUT
