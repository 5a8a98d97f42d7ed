"""Host side of the end-to-end path: ``HostNewtonState`` packs the step's inputs into one
buffer, each array at a 256-byte boundary, and its views hold the scene's values exactly.
(The buffer is page-locked on a GPU machine; here pinning is replaced by the plain buffer.)"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from sgipc import scenes, system  # noqa: E402


@pytest.fixture
def host(monkeypatch):
    monkeypatch.setattr(torch.Tensor, "pin_memory", lambda self: self)
    sc = scenes.scene_two_cubes(7, seed=5)
    return sc, system.HostNewtonState(sc)


def test_layout_is_aligned_and_disjoint(host):
    sc, h = host
    ends = []
    for name, off, dt, shape in h._layout:
        assert off % 256 == 0
        nb = int(np.prod(shape)) * torch.tensor([], dtype=dt).element_size()
        ends.append((off, off + nb))
    for (a0, a1), (b0, b1) in zip(ends, ends[1:]):
        assert a1 <= b0
    assert ends[-1][1] <= h._bytes


def test_views_hold_the_scene(host):
    sc, h = host
    src = {"vertexes": sc.vertexes, "pairs": sc.pairs.reshape(-1, 4), "ground_pairs": sc.ground_pairs,
           "fric_pairs": sc.fric_pairs.reshape(-1, 4), "fric_lambda": sc.fric_lambda,
           "fric_coord": sc.fric_coord.reshape(-1, 2), "fric_basis": sc.fric_basis.reshape(-1, 6),
           "fric_gd_pairs": sc.fric_gd_pairs, "fric_gd_lambda": sc.fric_gd_lambda}
    for name in system.HostNewtonState.NAMES:
        v = getattr(h, name)
        assert v.data_ptr() - h._host.data_ptr() == dict((n, o) for n, o, _, _ in h._layout)[name]
        assert np.array_equal(v.numpy(), np.asarray(src[name]).astype(v.numpy().dtype))
    assert h.h2d_bytes() == sum(getattr(h, n).numel() * getattr(h, n).element_size() for n in h.NAMES)
