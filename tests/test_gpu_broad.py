"""The GPU contact-pair search (``sgipc_build_cp``) and lagged friction set-up
(``sgipc_friction_setup``) through the C ABI.

* Against the reference's own pair checks and friction set-up, host-compiled from a reference
  checkout (``tests/golden/ref_golden.npz``, on the two scenes stored beside it): the same
  multiset of (pair, CCD candidate) rows, every pair size's MatIndex ranks 0 .. count - 1
  once, the same counters _cpNum[5] and ground pairs; the friction arrays pair for pair.
* Against the host generator (``sgipc.contacts``, itself pinned to the same goldens on the
  CPU) at the bench's size (two 21^3 cubes), on a cloth over a cube and on a rolled cloth over
  a sphere.
* Deterministic: two calls give the same arrays in the same order; the order is point-triangle
  pairs by surface point, then edge-edge pairs by edge.
* The Newton system assembled from the GPU's pairs and friction sets equals the oracle's
  assembly of the same inputs (1e-9).

Integer outputs are compared exactly; the friction forces 1e-12 relative, coordinates and
bases 1e-12 absolute (the same formulas; log and sqrt may round differently by an ulp).
"""
import os

import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sgipc import contacts, scenes, system  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "ref_golden.npz"))
FILES = {"cubes": "scene_two_cubes4.npz", "cloth": "scene_cloth6_cube4.npz"}


def _rows_sorted(*arrays):
    return np.array(sorted(map(tuple, np.concatenate([np.asarray(a).reshape(len(a), -1) for a in arrays], 1))))


def _sizes(p):
    return np.where(p[:, 0] >= 0, 4, np.where(p[:, 2] < 0, 2, np.where(p[:, 3] < 0, 3, 4)))


def _check_mat_index(p, mi, cp):
    """MatIndex = rank in output order among the pairs of the same size."""
    size = _sizes(p)
    for g, nv in ((2, 2), (3, 3), (4, 4)):
        assert np.array_equal(mi[size == nv], np.arange(cp[g])), nv
    assert cp[0] == len(p) and cp[1] == 0


@pytest.fixture(scope="module", params=["cubes", "cloth"])
def golden(request):
    sc = scenes.Scene.load(os.path.join(HERE, "golden", FILES[request.param]))
    g = system.GIPC(sc, pair_capacity=4096)
    yield request.param, sc, g
    g.close()


@pytest.mark.parametrize("variant", ["self", "bodies"])
def test_pairs_match_reference(golden, variant):
    tag, sc, g = golden
    q = "%s_cp_%s_" % (tag, variant)
    body = torch.tensor(G[q + "body"], device="cuda")
    out = g.buildCP(body=body, update=False)
    p, c, mi = out["pairs"].cpu().numpy(), out["ccd_pairs"].cpu().numpy(), out["mat_index"].cpu().numpy()
    assert np.array_equal(_rows_sorted(p, c), _rows_sorted(G[q + "pairs"], G[q + "ccd"]))
    assert list(out["cp_num"]) == list(G[q + "cpnum"])
    _check_mat_index(p, mi, out["cp_num"])
    assert np.array_equal(out["cp_num_dev"].cpu().numpy(), G[q + "cpnum"].astype(np.int32))
    gp = out["ground_pairs"].cpu().numpy()
    assert np.array_equal(np.sort(gp), np.sort(G[tag + "_cp_ground"])) and out["gp_num"] == len(gp)


def test_friction_sets_match_reference(golden):
    tag, sc, g = golden
    tet = system.DeviceTetraData(sc)
    cp = g.buildFrictionSets(tet)
    assert np.array_equal(tet.fric_pairs.cpu().numpy(), sc.fric_pairs)
    assert list(cp) == list(G[tag + "_lag_cpnum"])
    lam = tet.fric_lambda.cpu().numpy()
    assert np.abs(lam - sc.fric_lambda).max() <= 1e-12 * np.abs(sc.fric_lambda).max()
    assert np.abs(tet.fric_coord.cpu().numpy() - sc.fric_coord).max() <= 1e-12
    assert np.abs(tet.fric_basis.cpu().numpy().reshape(-1, 3, 2) - sc.fric_basis).max() <= 1e-12
    assert np.array_equal(tet.fric_gd_pairs.cpu().numpy(), sc.fric_gd_pairs)
    gl = tet.fric_gd_lambda.cpu().numpy()
    assert np.abs(gl - sc.fric_gd_lambda).max() <= 1e-12 * np.abs(sc.fric_gd_lambda).max()


@pytest.fixture(scope="module", params=["two_cubes21", "cloth24_cube6", "cloth_roll64_sphere"])
def large(request):
    if request.param == "two_cubes21":
        sc = scenes.scene_two_cubes(21, seed=1)
    elif request.param == "cloth24_cube6":
        sc = scenes.scene_cloth_on_cube(24, 6, seed=2)
    else:  # rolled cloth layers 0.4 mm apart: dense self-contact, about 50 000 pairs
        sc = scenes.scene_cloth_on_sphere(64, 500)
    g = system.GIPC(sc, pair_capacity=max(4 * len(sc.pairs), 4096))
    yield request.param, sc, g
    g.close()


def test_pairs_match_host_generator_and_repeat(large):
    name, sc, g = large
    pairs, ccd = contacts.find_pairs(sc.vertexes, sc.rest_vertexes, sc.surf_tris, sc.surf_edges, sc.surf_verts,
                                     sc.params["dHat"], sc.body_of_vertex, with_ccd=True)
    out = g.buildCP(update=False)
    p, c, mi = out["pairs"].cpu().numpy(), out["ccd_pairs"].cpu().numpy(), out["mat_index"].cpu().numpy()
    assert len(p) == len(pairs) > 0
    assert np.array_equal(_rows_sorted(p, c), _rows_sorted(pairs, ccd))
    _check_mat_index(p, mi, out["cp_num"])
    # the documented order: point-triangle pairs by surface point (their CCD candidates start
    # with -point - 1), then edge-edge pairs by (edge, other edge)
    pt = c[:, 0] < 0
    npt = int(pt.sum())
    assert pt[:npt].all() and not pt[npt:].any()
    pos = {int(v): i for i, v in enumerate(sc.surf_verts)}
    order = np.array([pos[-int(v) - 1] for v in c[:npt, 0]])
    assert (np.diff(order) >= 0).all()
    gp = contacts.ground_pairs(sc.vertexes, sc.surf_verts, sc.params["dHat"], sc.params["ground_offset"])
    assert np.array_equal(out["ground_pairs"].cpu().numpy(), gp)
    again = g.buildCP(update=False)
    for k in ("pairs", "ccd_pairs", "mat_index", "ground_pairs"):
        assert torch.equal(again[k], out[k]), k


def test_friction_sets_match_host_generator(large):
    name, sc, g = large
    tet = system.DeviceTetraData(sc)
    g.buildFrictionSets(tet)
    lp, lam, coord, basis, gpairs, glam = contacts.lag_friction(sc.o_vertexes, sc.pairs, sc.ground_pairs,
                                                                sc.params["dHat"], sc.params["kappa"],
                                                                sc.params["ground_offset"])
    assert np.array_equal(tet.fric_pairs.cpu().numpy(), lp)
    assert np.abs(tet.fric_lambda.cpu().numpy() - lam).max() <= 1e-12 * np.abs(lam).max()
    assert np.abs(tet.fric_coord.cpu().numpy() - coord).max() <= 1e-10
    assert np.abs(tet.fric_basis.cpu().numpy().reshape(-1, 3, 2) - basis).max() <= 1e-12
    assert np.array_equal(tet.fric_gd_pairs.cpu().numpy(), gpairs)


def test_newton_system_from_gpu_contacts_matches_oracle():
    """One Newton system whose contacts come from the GPU: the pair search at x, the friction
    sets at the start-of-step positions, then the assembly; against the oracle given the
    same pairs and friction arrays."""
    sc = scenes.scene_two_cubes(7, seed=5)
    g = system.GIPC(sc, pair_capacity=4 * len(sc.pairs))
    try:
        g.buildCP()
        g.buildFrictionSets()
        g.computeGradientAndHessian()
        rows, cols, vals = g.export_bcoo()
        b = g.rhs().cpu().numpy()
        s2 = scenes.Scene(**{**sc.__dict__})
        t = g.tet
        s2.pairs, s2.ground_pairs = t.pairs.cpu().numpy(), t.ground_pairs.cpu().numpy()
        s2.fric_pairs, s2.fric_lambda = t.fric_pairs.cpu().numpy(), t.fric_lambda.cpu().numpy()
        s2.fric_coord, s2.fric_basis = t.fric_coord.cpu().numpy(), t.fric_basis.cpu().numpy().reshape(-1, 3, 2)
        s2.fric_gd_pairs, s2.fric_gd_lambda = t.fric_gd_pairs.cpu().numpy(), t.fric_gd_lambda.cpu().numpy()
        ob, orow, ocol, oval, _ = oracle.assemble(s2)
        assert np.array_equal(rows, orow) and np.array_equal(cols, ocol)
        assert np.abs(vals - oval).max() < 1e-9 * np.abs(oval).max()
        assert np.abs(b - ob).max() < 1e-9 * np.abs(ob).max()
        assert len(s2.pairs) == len(sc.pairs)
    finally:
        g.close()


def test_capacity_is_reported():
    sc = scenes.scene_two_cubes(7, seed=5)
    g = system.GIPC(sc)
    try:
        from sgipc import _native as N

        with pytest.raises(N.SgipcError) as e:
            g.buildCP(capacity=8, update=False)
        assert e.value.status == N.CAPACITY
        assert b"capacity" in N.lib().sgipc_last_error(g.ctx)
        out = g.buildCP(update=False)  # the context stays usable
        assert out["cp_num"][0] == len(sc.pairs)
    finally:
        g.close()
