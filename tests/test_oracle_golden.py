"""The oracle against the reference's own code (``tests/golden/ref_golden.npz``).

The fixture holds per-element results of the reference's functions and kernels, compiled
for the host from a reference checkout by ``oracle/ref_build.py`` and run by
``tests/golden/make_golden.py`` on two small seeded scenes (stored beside it) and on
synthetic pairs of every barrier kind.  Each test restates one reference item:

* barrier energy and gradient per pair, all seven pair kinds
  (__cal_Barrier_energy GIPC.cu:701-944, _calBarrierGradient GIPC.cu:5272-6337);
* friction energy and gradient per lagged pair and per ground vertex
  (__cal_Friction_energy / _gd_energy GIPC.cu:1252-1300, _calFrictionGradient(_gd)
  GIPC.cu:5047-5269);
* the lagged friction set-up of the host generator ``sgipc.contacts.lag_friction``
  (_calFrictionLastH_DistAndTan / _gd GIPC.cu:8362-8499);
* the ground barrier gradient, the kinetic and soft-constraint gradients, the SNK and
  membrane gradients summed over a scene, against the oracle's assembled gradient
  (_computeGroundGradient GIPC.cu:6516, _calKineticGradient :6339,
  _computeSoftConstraintGradient :6409, _calculate_fem_gradient femEnergy.cu:2264,
  _calculate_triangle_fem_gradient femEnergy.cu:2217), Dirichlet rows zeroed as
  FEMLinearSubsystem::assemble does;
* stable Neo-Hookean energy and PK1 at large deformations, inverted tets included
  (femEnergy.cu:432-459, 1031-1050);
* the line-search step bounds per candidate / per vertex (_reduct_min_selfTimeStep_to_double
  GIPC.cu:7052, _reduct_min_groundTimeStep_to_double :6902, point_triangle_ccd /
  edge_edge_ccd ACCD.cu:373-535);
* the inertial target (_computeXTilta GIPC.cu:8073) of the scene builder.

Tolerances: 1e-10 relative for energies and gradients (same formulas, other evaluation
order: dual numbers and hand derivations in the oracle, MATLAB-generated code in the
reference); the CCD times of impact 1e-9 relative (iterated conservative advances).
"""
import os

import numpy as np
import pytest

import oracle
from sgipc import contacts, scenes

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "ref_golden.npz"))
SCENES = {"cubes": os.path.join(HERE, "golden", "scene_two_cubes4.npz"),
          "cloth": os.path.join(HERE, "golden", "scene_cloth6_cube4.npz")}


def _scene(tag):
    return scenes.Scene.load(SCENES[tag])


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


def _rows(vid, grad):
    """vertex -> gradient row of one pair"""
    return {int(v): np.asarray(grad[k]) for k, v in enumerate(vid) if v >= 0}


@pytest.mark.parametrize("tag", ["syn", "cubes", "cloth"])
def test_barrier_energy_and_gradient_per_pair(tag):
    if tag == "syn":
        x, rest, pairs = G["syn_x"], G["syn_rest"], G["syn_pairs"]
        dhat, kappa = float(G["syn_dhat"]), float(G["syn_kappa"])
    else:
        sc = _scene(tag)
        x, rest, pairs = sc.vertexes, sc.rest_vertexes, sc.pairs
        dhat, kappa = sc.params["dHat"], sc.params["kappa"]
    e_ref, vid_ref, g_ref = G[tag + "_bar_energy"], G[tag + "_bar_vid"], G[tag + "_bar_grad"]
    assert len(pairs) == len(e_ref) > 0
    scale = np.abs(g_ref).max()
    for k, enc in enumerate(pairs):
        vid, e, g, _ = oracle.barrier_pair(enc, x, rest, dhat, kappa)
        assert abs(e - e_ref[k]) <= 1e-10 * max(abs(e_ref[k]), 1e-300), (tag, k, enc, e, e_ref[k])
        mine, ref = _rows(vid, g.reshape(-1, 3)), _rows(vid_ref[k], g_ref[k])
        assert set(mine) <= set(ref), (tag, k, enc)
        for v, row in ref.items():
            got = mine.get(v, np.zeros(3))
            assert np.abs(got - row).max() <= 1e-10 * max(np.abs(g_ref[k]).max(), 1e-12 * scale), (tag, k, enc, v)


def test_synthetic_pairs_cover_every_kind():
    enc = G["syn_pairs"]
    kinds = set()
    for x, y, z, w in enc:
        if x >= 0:
            kinds.add("EE" if w >= 0 else "mEE")
        elif z < 0:
            kinds.add("PP" if y >= 0 else "mPP")
        elif w < 0:
            kinds.add("PE" if y >= 0 else "mPE")
        else:
            kinds.add("PT")
    assert kinds == {"PP", "PE", "PT", "EE", "mEE", "mPP", "mPE"}
    # the mollified ones carry energy (the mollifier is active)
    assert (G["syn_bar_energy"] > 0).all()


@pytest.mark.parametrize("tag", ["syn", "cubes", "cloth"])
def test_lagged_friction_setup_matches_reference(tag):
    if tag == "syn":
        x, pairs = G["syn_x"], G["syn_pairs"]
        dhat, kappa, gp, off = float(G["syn_dhat"]), float(G["syn_kappa"]), np.zeros(0, np.int32), -1.0
        ref_pairs, ref_lam = G["syn_lag_pairs"], G["syn_lag_lambda"]
        ref_coord, ref_basis = G["syn_lag_coord"], G["syn_lag_basis"]
    else:
        sc = _scene(tag)
        x, pairs = sc.o_vertexes, sc.pairs
        dhat, kappa, gp, off = sc.params["dHat"], sc.params["kappa"], sc.ground_pairs, sc.params["ground_offset"]
        ref_pairs, ref_lam, ref_coord, ref_basis = sc.fric_pairs, sc.fric_lambda, sc.fric_coord, sc.fric_basis
    lp, lam, coord, basis, gpairs, glam = contacts.lag_friction(x, pairs, gp, dhat, kappa, off)
    assert np.array_equal(lp, ref_pairs)
    assert _rel(lam, ref_lam) < 1e-12
    assert np.abs(coord - ref_coord).max() < 1e-10
    assert np.abs(basis - ref_basis).max() < 1e-12
    if tag != "syn":
        assert np.array_equal(gpairs, sc.fric_gd_pairs)
        assert _rel(glam, sc.fric_gd_lambda) < 1e-12
        cp = G[tag + "_lag_cpnum"]
        assert cp[0] == len(lp) == cp[2] + cp[3] + cp[4]


@pytest.mark.parametrize("tag", ["cubes", "cloth"])
def test_friction_energy_and_gradient_per_pair(tag):
    sc = _scene(tag)
    eps2 = sc.params["fDhat"] * sc.params["dt"] ** 2
    e_ref, vid_ref, g_ref = G[tag + "_fric_energy"], G[tag + "_fric_vid"], G[tag + "_fric_grad"]
    assert len(sc.fric_pairs) == len(e_ref) > 0
    assert (np.abs(g_ref) > 0).any()
    for k, enc in enumerate(sc.fric_pairs):
        vid, e, g, _ = oracle.friction_pair(enc, sc.vertexes, sc.o_vertexes, sc.fric_coord[k], sc.fric_basis[k],
                                         sc.fric_lambda[k], 1.0, eps2)
        assert abs(e - e_ref[k]) <= 1e-10 * abs(e_ref[k]) + 1e-300, (k, e, e_ref[k])
        mine, ref = _rows(vid, g.reshape(-1, 3)), _rows(vid_ref[k], g_ref[k])
        for v, row in ref.items():
            assert np.abs(mine[v] - row).max() <= 1e-10 * np.abs(g_ref[k]).max() + 1e-300, (k, v)


@pytest.mark.parametrize("tag", ["cubes", "cloth"])
def test_ground_friction_per_vertex(tag):
    sc = _scene(tag)
    eps2 = sc.params["fDhat"] * sc.params["dt"] ** 2
    for k, v in enumerate(sc.fric_gd_pairs):
        e, g, _ = oracle_ground_friction(sc.vertexes[v], sc.o_vertexes[v], sc.fric_gd_lambda[k], eps2)
        assert abs(e - G[tag + "_gfric_energy"][k]) <= 1e-10 * abs(G[tag + "_gfric_energy"][k]) + 1e-300
        assert np.abs(g - G[tag + "_gfric_grad"][k]).max() <= 1e-10 * np.abs(G[tag + "_gfric_grad"][k]).max() + 1e-300


def oracle_ground_friction(x, x0, lam, eps2):
    import ctypes

    e, g, H = np.zeros(1), np.zeros(3), np.zeros(9)
    x, x0 = np.ascontiguousarray(x, np.float64), np.ascontiguousarray(x0, np.float64)
    p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    oracle.lib().or_friction_ground(p(x), p(x0), lam, 1.0, eps2, p(e), p(g), p(H))
    return e[0], g, H


def test_scene_gradient_is_the_sum_of_the_reference_kernels():
    """The oracle's assembled right-hand side of the two-cube scene (with Dirichlet
    vertices and soft constraints) equals the sum of the reference kernels' gradients."""
    sc = _scene("cubes")
    p = sc.params
    tag = "cubes_"
    total = G[tag + "kin_grad"] + G[tag + "fem_grad"] + G[tag + "soft_grad"]
    for k, vid in enumerate(G[tag + "bar_vid"]):
        for a, v in enumerate(vid):
            if v >= 0:
                total[v] += G[tag + "bar_grad"][k, a]
    for k, vid in enumerate(G[tag + "fric_vid"]):
        for a, v in enumerate(vid):
            if v >= 0:
                total[v] += p["frictionRate"] * G[tag + "fric_grad"][k, a]
    for k, v in enumerate(sc.ground_pairs):
        total[v] += G[tag + "ground_grad"][k]
    for k, v in enumerate(sc.fric_gd_pairs):
        total[v] += p["gd_frictionRate"] * G[tag + "gfric_grad"][k]
    # FEMLinearSubsystem::assemble zeroes the Dirichlet rows of the right-hand side
    fixed = sc.boundary_type != 0
    assert fixed.any() and len(sc.soft_index) and len(sc.fric_pairs) and len(sc.ground_pairs)
    total[fixed] = 0.0
    b = oracle.assemble(sc)[0].reshape(-1, 3)
    assert _rel(b, total) < 1e-10


def test_membrane_gradient_and_energy():
    sc = _scene("cloth")
    p = sc.params
    dt2 = p["dt"] ** 2
    g = np.zeros_like(sc.vertexes)
    for k, t in enumerate(sc.tris):
        e, gk, _ = oracle.tri_bw(sc.vertexes[t], sc.tri_dm_inv[k], sc.area[k], p["stretchStiff"], p["shearStiff"],
                                 p["strainRate"], 1.0)
        assert abs(e - G["cloth_tri_energy"][k]) <= 1e-10 * abs(G["cloth_tri_energy"][k]) + 1e-300, k
        _, gk, _ = oracle.tri_bw(sc.vertexes[t], sc.tri_dm_inv[k], sc.area[k], p["stretchStiff"], p["shearStiff"],
                                 p["strainRate"], dt2)
        for a, v in enumerate(t):
            g[v] += gk[3 * a:3 * a + 3]
    assert _rel(g, G["cloth_tri_grad"]) < 1e-10


@pytest.mark.parametrize("tag", ["cubes", "cloth"])
def test_snk_scene_energy_and_gradient(tag):
    sc = _scene(tag)
    dt2 = sc.params["dt"] ** 2
    g = np.zeros_like(sc.vertexes)
    for k, t in enumerate(sc.tets):
        e, _, _ = oracle.snk_tet(sc.vertexes[t], sc.dm_inv[k], sc.volum[k], sc.length_rate[k], sc.volume_rate[k], 1.0)
        assert abs(e - G[tag + "_snk_energy"][k]) <= 1e-10 * abs(G[tag + "_snk_energy"][k]) + 1e-18, k
        _, gk, _ = oracle.snk_tet(sc.vertexes[t], sc.dm_inv[k], sc.volum[k], sc.length_rate[k], sc.volume_rate[k],
                                  dt2)
        for a, v in enumerate(t):
            g[v] += gk[3 * a:3 * a + 3]
    assert _rel(g, G[tag + "_fem_grad"]) < 1e-10


def test_snk_energy_and_stress_at_large_deformations():
    """Energy and PK1 at seeded large deformations (a seventh of the tets inverted): the
    oracle's gradient is vol * P Dm^-T on vertices 1..3 and minus their sum on vertex 0."""
    X, Dm, lr, vr = G["el_tet_x"], G["el_tet_dminv"], G["el_tet_lr"], G["el_tet_vr"]
    vol = float(G["el_tet_vol"])
    assert (np.linalg.det(np.einsum("kij,kjl->kil", np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0],
                                                              X[:, 3] - X[:, 0]], 2), Dm)) < 0).any()
    for k in range(len(X)):
        e, g, _ = oracle.snk_tet(X[k], Dm[k], vol, lr[k], vr[k], 1.0)
        assert abs(e - G["el_tet_energy"][k]) <= 1e-10 * abs(G["el_tet_energy"][k]), k
        H = vol * G["el_tet_pk1"][k] @ Dm[k].T
        want = np.concatenate([-H.sum(1), H[:, 0], H[:, 1], H[:, 2]])
        assert _rel(g, want) < 1e-10, k


@pytest.mark.parametrize("tag", ["cubes", "cloth"])
def test_step_bounds_per_candidate(tag):
    sc = _scene(tag)
    cand, inv = G[tag + "_ccd_cand"], G[tag + "_ccd_inv"]
    _, toi = oracle.self_step(sc.vertexes, G[tag + "_move"], cand, 0.8)
    assert len(cand) > 0 and (inv > 1.0).any()
    assert _rel(1.0 / toi, inv) < 1e-9
    for k, v in enumerate(sc.ground_pairs):
        a = oracle.ground_step(sc.vertexes, G[tag + "_gmove"], [v], sc.params["ground_offset"], 0.8)
        assert abs(a - 1.0 / max(1.0, G[tag + "_ground_step_inv"][k])) <= 1e-14, k


def test_accd_straight_calls():
    x, d, eta = G["ccd_x"], G["ccd_d"], G["ccd_eta"]
    assert (G["ccd_thickness"] == 0).all()
    assert (G["ccd_pt"] < 1).any() and (G["ccd_ee"] < 1).any()
    for k in range(len(x)):
        assert abs(oracle.accd(False, x[k], d[k], eta[k]) - G["ccd_pt"][k]) <= 1e-9 * G["ccd_pt"][k], k
        assert abs(oracle.accd(True, x[k], d[k], eta[k]) - G["ccd_ee"][k]) <= 1e-9 * G["ccd_ee"][k], k


@pytest.mark.parametrize("tag", ["cubes", "cloth"])
def test_inertial_target(tag):
    sc = _scene(tag)
    xt = scenes.inertial_target(sc.o_vertexes, sc.velocities, sc.boundary_type, sc.params["dt"],
                                G[tag + "_xtilta_gravity"])
    assert np.abs(xt - G[tag + "_xtilta"]).max() <= 1e-15


def _rows_sorted(*arrays):
    return np.array(sorted(map(tuple, np.concatenate([np.asarray(a).reshape(len(a), -1) for a in arrays], 1))))


@pytest.mark.parametrize("tag", ["cubes", "cloth"])
@pytest.mark.parametrize("variant", ["self", "bodies"])
def test_host_pair_generator_matches_reference_build_cp(tag, variant):
    """sgipc.contacts.find_pairs against the reference's pair checks (_checkPTintersection /
    _checkEEintersection with the BVH queries' filters, mlbvh.cu:534-1059, 1306-1742): the same
    multiset of (pair, CCD candidate) rows, nearly parallel edge pairs with w = -other - 2
    included; and the ground pairs of _GroundCollisionDetect."""
    sc = _scene(tag)
    q = "%s_cp_%s_" % (tag, variant)
    pairs, ccd = contacts.find_pairs(sc.vertexes, sc.rest_vertexes, sc.surf_tris, sc.surf_edges, sc.surf_verts,
                                     sc.params["dHat"], sc.body_of_vertex, inter_body_only=(variant == "bodies"),
                                     with_ccd=True)
    assert np.array_equal(_rows_sorted(pairs, ccd), _rows_sorted(G[q + "pairs"], G[q + "ccd"]))
    cp = G[q + "cpnum"]
    assert cp[0] == len(pairs) == cp[2] + cp[3] + cp[4] and cp[1] == 0
    # MatIndex: each pair's rank among the pairs of its size (the reference's order is that of
    # its atomics; any order gives every size the ranks 0 .. count-1 once)
    mi, p = G[q + "matindex"], G[q + "pairs"]
    size = np.where(p[:, 0] >= 0, 4, np.where(p[:, 2] < 0, 2, np.where(p[:, 3] < 0, 3, 4)))
    for g, nv in ((2, 2), (3, 3), (4, 4)):
        assert np.array_equal(np.sort(mi[size == nv]), np.arange(cp[g]))
    gp = contacts.ground_pairs(sc.vertexes, sc.surf_verts, sc.params["dHat"], sc.params["ground_offset"])
    assert np.array_equal(np.sort(gp), np.sort(G[tag + "_cp_ground"]))
