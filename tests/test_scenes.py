"""Scene generators of the workloads (CPU): placement, contact density and the Newton system
they give, at parity-test sizes.

* The cloth-on-sphere workload: the sphere's lowest vertex 0.5 d-hat above the ground (before
  the seeded 1e-6 m perturbation), the rolled cloth's lowest vertex less than d-hat above the
  sphere's top, layers 0.4 mm apart (below d-hat, so every layer is in contact with the next
  and none crosses another), every contact pair within d-hat, and an SPD assembled matrix.  contacts=False leaves the contact arrays
  empty (the GPU pair search fills them).
"""
import numpy as np

import oracle
from sgipc import contacts, scenes


def _pair_d2(x, pairs):
    out = []
    for a, b, c, d in np.asarray(pairs, np.int64):
        if a >= 0:
            out.append(contacts.d_ee(x[a][None], x[b][None], x[c][None], x[d if d >= 0 else -d - 1][None])[0])
        elif c < 0:
            out.append(contacts.d_pp(x[-a - 1][None], x[b][None])[0])
        elif d < 0:
            out.append(contacts.d_pe(x[-a - 1][None], x[b][None], x[c][None])[0])
        else:
            out.append(contacts.d_pt(x[-a - 1][None], x[b][None], x[c][None], x[d][None])[0])
    return np.array(out)


def test_cloth_on_sphere_placement_and_contacts():
    sc = scenes.scene_cloth_on_sphere(24, 200)
    dhat = sc.params["dHat"] ** 0.5
    ground = sc.params["ground_offset"]
    tet_verts = np.unique(np.asarray(sc.tets).ravel())
    cloth = np.setdiff1d(np.arange(sc.nv), tet_verts)
    y = sc.vertexes[:, 1]
    # placed exactly, then every vertex perturbed by at most 1e-6 m per axis
    assert abs(y[tet_verts].min() - (ground + 0.5 * dhat)) <= 1e-6
    # the roll's outer turn touches the sphere's top within d-hat (its vertices sit near, not
    # at, the spiral's lowest point)
    assert 0.0 < y[cloth].min() - y[tet_verts].max() < dhat
    assert len(sc.ground_pairs) > 0 and np.isin(sc.ground_pairs, tet_verts).all()
    d2 = _pair_d2(sc.vertexes, sc.pairs)
    assert len(d2) > 5 * len(cloth)  # dense self-contact: several pairs per cloth vertex
    assert (d2 < sc.params["dHat"]).all() and (d2 > 0).all()
    b, rows, cols, vals, _ = oracle.assemble(sc)
    A = oracle.dense(rows, cols, vals, sc.nv)
    assert np.allclose(A, A.T, rtol=0, atol=1e-12 * np.abs(A).max())
    assert np.linalg.eigvalsh(A).min() > 0
    bare = scenes.scene_cloth_on_sphere(24, 200, contacts=False)
    assert len(bare.pairs) == 0 and len(bare.ground_pairs) == 0 and len(bare.fric_pairs) == 0
    assert np.array_equal(bare.vertexes, sc.vertexes)


def test_abd_on_bed_layout_and_system():
    """The affine-bodies-on-a-bed workload: the bed's vertices first, the boxes' points after
    them (Dirichlet, unit mass), every point at J(x_bar) q of its body; resting boxes 0.5 d-hat
    above the bed, no two boxes closer than 2 d-hat; the bed 0.5 d-hat above the ground; the
    FEM system SPD with the points' rows decoupled; contact pairs between boxes and bed."""
    sc, bodies = scenes.scene_abd_on_bed(12, (6, 2, 6), seed=1, resting=0.7)
    af = bodies["abd_first"]
    dhat = sc.params["dHat"] ** 0.5
    assert (sc.boundary_type[:af] == 0).all() and (sc.boundary_type[af:] == 1).all()
    assert np.allclose(sc.masses[af:], 1.0)
    q = bodies["q"]
    A = q[:, 3:].reshape(-1, 3, 3)
    pb = bodies["point_body"]
    J = np.einsum("pij,pj->pi", A[pb], bodies["x_bar"]) + q[pb, :3]
    assert np.abs(J - sc.vertexes[af:]).max() == 0.0
    bed_y = sc.vertexes[:af, 1]
    assert abs(bed_y.min() - (sc.params["ground_offset"] + 0.5 * dhat)) < 1e-12
    top = bed_y.max()
    for b in np.nonzero(bodies["resting"])[0]:
        assert abs(sc.vertexes[af:][pb == b, 1].min() - (top + 0.5 * dhat)) < 1e-12
    lo = np.array([sc.vertexes[af:][pb == b].min(0) for b in range(len(q))])
    hi = np.array([sc.vertexes[af:][pb == b].max(0) for b in range(len(q))])
    for i in range(len(q)):
        for j in range(i + 1, len(q)):
            sep = np.maximum(lo[j] - hi[i], lo[i] - hi[j])
            assert sep.max() >= 2 * dhat - 1e-9
    b, rows, cols, vals, _ = oracle.assemble(sc)
    Af = oracle.dense(rows, cols, vals, sc.nv)
    assert np.linalg.eigvalsh(Af).min() > 0
    assert np.abs(Af[3 * af:, :3 * af]).max() == 0.0 and np.allclose(Af[3 * af:, 3 * af:], np.eye(3 * (sc.nv - af)))
    assert (b[3 * af:] == 0).all()
    pairs = np.asarray(sc.pairs)
    touches = [(np.abs(np.where(p < 0, -p - 1, p)) >= af).any() for p in pairs]
    assert any(touches) and len(sc.ground_pairs) > 0
