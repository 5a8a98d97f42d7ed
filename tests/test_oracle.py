"""CPU tests of the oracle: pinned to the reference's generated Jacobians (golden vectors),
its closed-form scalar expressions, and finite-difference identities of its energies."""
import math
import os

import numpy as np
import pytest

import oracle
from sgipc import contacts, scenes

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "pfpx_golden.npz"))


# ------------------------------------------------------------------------------------------
# barrier derivatives vs the reference's generated pFpx_* code (tests/golden/make_golden.py)
# ------------------------------------------------------------------------------------------
CASES = {  # function -> (pair encoding over vertices 0..3, column of d(d/sqrt dhat)/dx, column of dc/dx)
    "pFpx_pp2": ((-1, 1, -1, -1), None, None),
    "pFpx_pe2": ((-1, 1, 2, -1), 3, None),
    "pFpx_pt2": ((-1, 1, 2, 3), 8, None),
    "pFpx_ee2": ((0, 1, 2, 3), 8, None),
    "pFpx_peeV0V1": ((0, 1, 2, -4), 8, 4),
    "pFpx_ppeV0V1": ((-1, -2, 2, -4), 8, 4),
    "pFpx_pppV0V1": ((-1, -2, -3, -4), 8, 4),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_distance_jacobians_match_reference_generated_code(name):
    enc, fcol, ccol = CASES[name]
    X, D, OUT = GOLD[name + "_x"], GOLD[name + "_d"], GOLD[name + "_out"]
    for x, d, out in zip(X, D, OUT):
        nv, f, gf, c, gc = oracle.pair_geom(np.array(enc), x, d * d)
        ref_gf = out if fcol is None else out[:3 * nv, fcol]
        assert np.allclose(gf, ref_gf, rtol=1e-9, atol=1e-9 * np.abs(ref_gf).max())
        if ccol is not None:
            ref_gc = out[:, ccol]
            assert np.allclose(gc, ref_gc, rtol=1e-9, atol=1e-9 * np.abs(ref_gc).max())


# ------------------------------------------------------------------------------------------
# barrier scalars: the reference's closed forms (GIPC.cu, RANK 2 branches) restated
# ------------------------------------------------------------------------------------------
def ref_pk1_scale(I, k, dh):       # GIPC.cu:3191-3194: flatten_pk1 = f * this
    L = math.log(I)
    return 2 * (2 * k * dh * dh * L * (I - 1) * (I + I * L - 1)) / I


def ref_lambda0(I, k, dh):         # GIPC.cu:3233-3236
    L = math.log(I)
    return -(4 * k * dh * dh * (4 * I + L - 3 * I * I * L * L + 6 * I * L - 2 * I * I + I * L * L
                                 - 7 * I * I * L - 2)) / I


@pytest.mark.parametrize("I", [0.01, 0.1, 0.25, 0.5, 0.9, 0.999])
def test_barrier_scalars_match_reference_closed_forms(I):
    k, dh = 3.7, 1e-6
    x = np.array([0.0, 0.0, 0.0, math.sqrt(I * dh), 0.0, 0.0])
    vid, e, g, H = oracle.barrier_pair(np.array([-1, 1, -1, -1]), x, x, dh, k)
    f = math.sqrt(I)
    gradf = np.array([-1.0, 0, 0, 1.0, 0, 0]) / math.sqrt(dh)
    assert np.allclose(g, ref_pk1_scale(I, k, dh) * f * gradf, rtol=1e-10)
    assert np.allclose(H, ref_lambda0(I, k, dh) * np.outer(gradf, gradf), rtol=1e-9,
                       atol=1e-12 * abs(ref_lambda0(I, k, dh)) / dh)
    assert e == pytest.approx(k * (I * dh - dh) ** 2 * math.log(I) ** 2, rel=1e-12)


def test_barrier_lambda0_clamp_below_gauss_threshold():
    # d^2 < 1e-6 dhat uses the Hessian scale at I = 1e-6 (GIPC.cu:3258-3272)
    k, dh = 1.0, 1e-6
    I = 1e-8
    x = np.array([0.0, 0.0, 0.0, math.sqrt(I * dh), 0.0, 0.0])
    _, _, _, H = oracle.barrier_pair(np.array([-1, 1, -1, -1]), x, x, dh, k)
    gradf = np.array([-1.0, 0, 0, 1.0, 0, 0]) / math.sqrt(dh)
    assert np.allclose(H, ref_lambda0(1e-6, k, dh) * np.outer(gradf, gradf), rtol=1e-9)


def _fd_grad(fun, x, h):
    g = np.zeros_like(x)
    for i in range(len(x)):
        xp, xm = x.copy(), x.copy()
        xp[i] += h
        xm[i] -= h
        g[i] = (fun(xp) - fun(xm)) / (2 * h)
    return g


def _pair_config(enc, rng, parallel=False):
    X = rng.uniform(-1e-3, 1e-3, (4, 3))
    X[0] = [0, 0, 0]
    if parallel:
        e = np.array([1.0, 0.2, 0.1])
        e /= np.linalg.norm(e)
        X[1] = X[0] + 4e-3 * e + rng.uniform(-2e-6, 2e-6, 3)
        X[2] = np.array([0.0, 5e-4, 0.0]) + rng.uniform(-1e-4, 1e-4, 3)
        X[3] = X[2] + 4e-3 * e + rng.uniform(-2e-6, 2e-6, 3)
    return X


@pytest.mark.parametrize("enc", [(-1, 1, -1, -1), (-1, 1, 2, -1), (-1, 1, 2, 3), (0, 1, 2, 3),
                                 (0, 1, 2, -4), (-1, -2, 2, -4), (-1, -2, -3, -4)])
def test_barrier_gradient_is_energy_derivative(enc):
    rng = np.random.default_rng(abs(hash(enc)) % 2 ** 32)
    moll = enc[0] >= 0 and enc[3] < 0 or enc[1] < 0
    dh, k = 4e-6, 2.0
    for _ in range(5):
        if moll:
            X = _pair_config(enc, rng, parallel=True)
            R = X.copy()
            R[1] = R[0] + 4e-3 * np.array([0.0, 0.0, 1.0])   # rest edges not parallel: large eps
        else:
            X = rng.normal(size=(4, 3)) * 1e-3
            R = X.copy()
        nv, f, *_ = oracle.pair_geom(np.array(enc), X, dh)
        if not (0.05 < f < 0.95):
            continue
        _, e, g, H = oracle.barrier_pair(np.array(enc), X, R, dh, k)
        fd = _fd_grad(lambda x: oracle.barrier_pair(np.array(enc), x.reshape(4, 3), R, dh, k)[1],
                      X.reshape(-1), 1e-9)
        assert np.allclose(g, fd[:3 * nv], rtol=1e-5, atol=1e-6 * np.abs(g).max())
        assert np.allclose(H, H.T, atol=1e-12 * np.abs(H).max())
        if moll:
            assert np.linalg.eigvalsh(H).min() >= -1e-9 * np.abs(H).max()


# ------------------------------------------------------------------------------------------
# stable Neo-Hookean
# ------------------------------------------------------------------------------------------
def _tet(rng, strain=0.05):
    R = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]]) * 0.01
    Dm = np.stack([R[1] - R[0], R[2] - R[0], R[3] - R[0]], 1)
    X = R + rng.uniform(-strain, strain, R.shape) * 0.01
    return X, np.linalg.inv(Dm), abs(np.linalg.det(Dm)) / 6


def test_snk_rest_state_has_zero_gradient():
    lr, vr = scenes.snk_rates(1e5, 0.4)
    X, Di, vol = _tet(np.random.default_rng(0), strain=0.0)
    e, g, H = oracle.snk_tet(X, Di, vol, float(lr), float(vr))
    assert np.abs(g).max() < 1e-12 * float(lr) * vol / 0.01
    assert e == pytest.approx(0.5 * vol * vr * (lr / vr) ** 2, rel=1e-12)


def test_snk_gradient_and_projected_hessian():
    lr, vr = [float(v) for v in scenes.snk_rates(1e5, 0.45)]
    rng = np.random.default_rng(1)
    for _ in range(5):
        X, Di, vol = _tet(rng, 0.1)
        e, g, H = oracle.snk_tet(X, Di, vol, lr, vr, 1e-4)
        fd = _fd_grad(lambda x: oracle.snk_tet(x, Di, vol, lr, vr, 1e-4)[0], X.reshape(-1), 1e-8)
        assert np.allclose(g, fd, rtol=1e-6, atol=1e-8 * np.abs(g).max())
        w = np.linalg.eigvalsh(H)
        assert w.min() > -1e-10 * w.max()
        # where the exact Hessian is already PSD, the projection leaves it unchanged
        Hfd = np.stack([_fd_grad(lambda x: oracle.snk_tet(x, Di, vol, lr, vr, 1e-4)[1][i], X.reshape(-1), 1e-8)
                        for i in range(12)])
        if np.linalg.eigvalsh(0.5 * (Hfd + Hfd.T)).min() > 1e-6 * w.max():
            assert np.allclose(H, Hfd, rtol=1e-4, atol=1e-5 * w.max())


# ------------------------------------------------------------------------------------------
# friction
# ------------------------------------------------------------------------------------------
@pytest.mark.parametrize("enc", [(-1, 1, -1, -1), (-1, 1, 2, -1), (-1, 1, 2, 3), (0, 1, 2, 3)])
@pytest.mark.parametrize("scale", [0.1, 10.0])   # static (|u| < eps) and sliding regimes
def test_friction_gradient_and_hessian(enc, scale):
    rng = np.random.default_rng(7)
    X0 = rng.normal(size=(4, 3)) * 1e-2
    eps2 = 1e-8
    dX = rng.normal(size=(4, 3))
    dX *= scale * math.sqrt(eps2) / np.abs(dX).max()
    X = X0 + dX
    basis = np.linalg.qr(rng.normal(size=(3, 2)))[0]
    coord = rng.uniform(0.2, 0.4, 2)
    args = (coord, basis, 0.7, 0.2, eps2)
    vid, e, g, H = oracle.friction_pair(np.array(enc), X, X0, *args)
    n = len(vid)
    fd = _fd_grad(lambda x: oracle.friction_pair(np.array(enc), x.reshape(4, 3), X0, *args)[1], X.reshape(-1),
                  1e-4 * math.sqrt(eps2))
    assert np.allclose(g, fd[:3 * n], rtol=1e-5, atol=1e-7 * np.abs(g).max())
    Hfd = np.stack([_fd_grad(lambda x: oracle.friction_pair(np.array(enc), x.reshape(4, 3), X0, *args)[2][i],
                             X.reshape(-1), 1e-4 * math.sqrt(eps2))[:3 * n] for i in range(3 * n)])
    assert np.allclose(H, Hfd, rtol=1e-4, atol=1e-5 * np.abs(H).max())


# ------------------------------------------------------------------------------------------
# system level
# ------------------------------------------------------------------------------------------
@pytest.fixture(scope="module")
def small_two_cubes():
    return scenes.scene_two_cubes(5, seed=3)


def test_assembled_gradient_is_total_energy_derivative(small_two_cubes):
    sc = small_two_cubes
    b, rows, cols, vals, e0 = oracle.assemble(sc)
    rng = np.random.default_rng(0)
    for _ in range(3):
        d = rng.normal(size=3 * sc.nv) * 1e-7
        ep = oracle.energy(sc, sc.vertexes + d.reshape(-1, 3))
        em = oracle.energy(sc, sc.vertexes - d.reshape(-1, 3))
        assert (ep - em) / 2 == pytest.approx(b @ d, rel=1e-4)


def test_assembled_matrix_symmetric_positive_definite(small_two_cubes):
    sc = small_two_cubes
    b, rows, cols, vals, _ = oracle.assemble(sc)
    assert (rows <= cols).all()
    A = oracle.dense(rows, cols, vals, sc.nv)
    assert np.allclose(A, A.T)
    assert np.linalg.eigvalsh(A).min() > 0


def test_mas_levels_match_reference_rule():
    # computeNumLevels (MASPreconditioner.cu:1724-1743)
    assert oracle.lib().or_mas_num_levels(1344) == 4
    assert oracle.lib().or_mas_num_levels(18528) == 5
    assert oracle.lib().or_mas_num_levels(16) == 2
    assert oracle.lib().or_mas_num_levels(10 ** 7) == 6


def test_mas_symmetric_positive_and_hierarchy_connected(small_two_cubes):
    sc = small_two_cubes
    b, rows, cols, vals, _ = oracle.assemble(sc)
    M = oracle.Mas(sc, rows, cols, vals)
    rng = np.random.default_rng(2)
    r, s = rng.normal(size=3 * sc.nv), rng.normal(size=3 * sc.nv)
    assert r @ M.apply(s) == pytest.approx(s @ M.apply(r), rel=1e-10)
    assert r @ M.apply(r) > 0
    L, starts, counts, total = M.info()
    tab = M.table()
    assert (tab[:, 0] == sc.real_map_part).all()
    # every coarse node's vertices form a connected set of the mesh + contact graph
    adj = [set() for _ in range(sc.nv)]
    for v in range(sc.nv):
        adj[v].update(sc.nbr_list[sc.nbr_start[v]:sc.nbr_start[v + 1]])
    for p in sc.pairs:
        vs = [(-v - 1 if v < 0 else v) for v in p]
        vs = [v for v in vs if 0 <= v < sc.nv]
        for a in vs:
            adj[a].update(vs)
    for lvl in range(1, L):
        for node in np.unique(tab[:, lvl]):
            members = set(np.nonzero(tab[:, lvl] == node)[0].tolist())
            seen, stack = set(), [next(iter(members))]
            while stack:
                u = stack.pop()
                if u in seen:
                    continue
                seen.add(u)
                stack.extend(w for w in adj[u] if w in members and w not in seen)
            assert seen == members


def test_pcg_converges_to_direct_solution(small_two_cubes):
    sc = small_two_cubes
    b, rows, cols, vals, _ = oracle.assemble(sc)
    A = oracle.dense(rows, cols, vals, sc.nv)
    M = oracle.Mas(sc, rows, cols, vals)
    x, it, rz0, rz = oracle.pcg(rows, cols, vals, sc.nv, M, b, 1e-20, max_iter=10 * sc.nv)
    ex = np.linalg.solve(A, b)
    assert np.linalg.norm(x - ex) / np.linalg.norm(ex) < 1e-8
    x4, it4, rz04, rz4 = oracle.pcg(rows, cols, vals, sc.nv, M, b, 1e-4)
    assert it4 < it and abs(rz4) <= 1e-4 * rz04 * 1.0000001


def test_contact_generator_encoding(small_two_cubes):
    sc = small_two_cubes
    p = sc.pairs
    assert len(p) > 0
    # every pair is within d-hat under its own distance type
    for enc in p[:200]:
        nv, f, *_ = oracle.pair_geom(enc, sc.vertexes, sc.params["dHat"])
        assert 0.0 < f < 1.0


# ------------------------------------------------------------------------------------------
# cloth: Baraff-Witkin membrane and quadratic bending
# ------------------------------------------------------------------------------------------
def _cloth_tri():
    v, t = scenes.cloth_grid(3, 0.1)
    dm, area = scenes.tri_rest_data(v, t, 1e-3)
    return v[t[0]], dm[0], area[0]


def _bw_fd_grad(X, dm, area, k, h=1e-7):
    g = np.zeros(9)
    for i in range(9):
        d = np.zeros(9)
        d[i] = h
        g[i] = (oracle.tri_bw(X.ravel() + d, dm, area, *k)[0] - oracle.tri_bw(X.ravel() - d, dm, area, *k)[0]) / (2 * h)
    return g


@pytest.mark.parametrize("scale", [0.9, 1.0, 1.15])
def test_cloth_membrane_gradient_is_energy_derivative(scale):
    X0, dm, area = _cloth_tri()
    rng = np.random.default_rng(int(scale * 100))
    k = (3.3e5, 1.0e6, 100.0, 1e-4)
    for _ in range(3):
        X = X0 * scale + rng.normal(scale=3e-3, size=(3, 3))
        e, g, H = oracle.tri_bw(X, dm, area, *k)
        assert np.allclose(g, _bw_fd_grad(X, dm, area, k), rtol=1e-5, atol=1e-6 * np.abs(g).max())
        assert np.allclose(H, H.T) and np.linalg.eigvalsh(H).min() >= -1e-9 * np.abs(H).max()


def test_cloth_membrane_rest_state_and_exact_hessian_under_pure_stretch():
    X0, dm, area = _cloth_tri()
    k = (3.3e5, 1.0e6, 100.0, 1e-4)
    e, g, H = oracle.tri_bw(X0, dm, area, *k)
    assert e == pytest.approx(0.0, abs=1e-18) and np.abs(g).max() < 1e-12
    # stretch both material directions (|f0|, |f1| > 1, f0 . f1 = 0): every term is convex
    # there, so the projected Hessian equals the exact one (finite differences of the gradient)
    Dm = np.linalg.inv(dm)
    F = np.array([[1.1, 0.0], [0.0, 1.2], [0.0, 0.0]])
    Ds = F @ Dm
    X = np.stack([np.zeros(3), Ds[:, 0], Ds[:, 1]])
    e, g, H = oracle.tri_bw(X, dm, area, *k)
    h = 1e-7
    Hfd = np.zeros((9, 9))
    for i in range(9):
        d = np.zeros(9)
        d[i] = h
        Hfd[:, i] = (oracle.tri_bw(X.ravel() + d, dm, area, *k)[1] - oracle.tri_bw(X.ravel() - d, dm, area, *k)[1]) / (2 * h)
    assert np.allclose(H, Hfd, rtol=1e-5, atol=1e-6 * np.abs(H).max())


def test_quadratic_bending_matrix_properties():
    v, t = scenes.cloth_grid(5, 0.2)
    e, adj = scenes.hinge_topology(t)
    Q = scenes.quad_bending_q(v, e, adj)
    inner = adj[:, 1] >= 0
    assert inner.sum() > 0 and np.abs(Q[~inner]).max() == 0.0
    # symmetric, rank one, annihilates rigid translations and the flat rest shape
    assert np.allclose(Q, np.transpose(Q, (0, 2, 1)))
    assert np.allclose(Q[inner].sum(2), 0.0, atol=1e-9 * np.abs(Q).max())
    X = np.stack([v[e[inner, 0]], v[e[inner, 1]], v[adj[inner, 0]], v[adj[inner, 1]]], 1)
    assert np.abs(np.einsum("hij,hjk->hik", Q[inner], X)).max() < 1e-9 * np.abs(Q).max()


@pytest.fixture(scope="module")
def small_cloth():
    return scenes.scene_cloth_on_cube(8, 4, seed=4)


def test_cloth_scene_gradient_is_total_energy_derivative(small_cloth):
    sc = small_cloth
    assert len(sc.tris) and len(sc.hinges) and len(sc.pairs)
    b, rows, cols, vals, e0 = oracle.assemble(sc)
    rng = np.random.default_rng(5)
    for _ in range(3):
        d = rng.normal(size=3 * sc.nv) * 1e-8
        ep = oracle.energy(sc, sc.vertexes + d.reshape(-1, 3))
        em = oracle.energy(sc, sc.vertexes - d.reshape(-1, 3))
        assert (ep - em) / 2 == pytest.approx(b @ d, rel=1e-4)


def test_cloth_scene_matrix_symmetric_positive_definite(small_cloth):
    sc = small_cloth
    b, rows, cols, vals, _ = oracle.assemble(sc)
    A = oracle.dense(rows, cols, vals, sc.nv)
    assert np.allclose(A, A.T) and np.linalg.eigvalsh(A).min() > 0


# ------------------------------------------------------------------------------------------
# affine bodies
# ------------------------------------------------------------------------------------------
def _abd_J(x):
    J = np.zeros((3, 12))
    J[:, :3] = np.eye(3)
    for r in range(3):
        J[r, 3 + 3 * r:6 + 3 * r] = x
    return J


def abd_contacts(bodies, n_fem=40, seed=0):
    """Seeded point-space contact blocks: ABD-ABD (different bodies, row < col, and some
    diagonal blocks), ABD-FEM, point gradients and a FEM Dirichlet mask."""
    rng = np.random.default_rng(seed)
    pb = bodies["point_body"]
    P = len(pb)
    pairs = []
    while len(pairs) < 60:
        i, j = sorted(rng.integers(0, P, 2))
        if pb[i] != pb[j]:
            pairs.append((i, j))
    diag = rng.choice(P, 10, replace=False)
    rows = np.array([p[0] for p in pairs] + list(diag), np.int32)
    cols = np.array([p[1] for p in pairs] + list(diag), np.int32)

    def spd(n):
        M = rng.normal(size=(n, 3, 3))
        return np.einsum("nij,nkj->nik", M, M) * 1e3

    vals = spd(len(rows))
    frows = rng.integers(0, P, 25).astype(np.int32)
    fcols = rng.integers(0, n_fem, 25).astype(np.int32)
    fvals = rng.normal(size=(25, 3, 3)) * 1e3
    fbt = (rng.uniform(size=n_fem) < 0.2).astype(np.int32)
    grad = rng.normal(size=(P, 3))
    return dict(abd=(rows, cols, vals), fem=(frows, fcols, fvals), fem_boundary=fbt, point_grad=grad, n_fem=n_fem)


def test_abd_orthogonality_potential():
    rng = np.random.default_rng(1)
    R, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    b = scenes.scene_abd_boxes(2, seed=1)
    q = b["q"].copy()
    q[0, 3:] = R.ravel()
    g, rows, cols, vals = oracle.abd_assemble(b, q, q, b["kappa"], b["dt"])
    assert np.abs(g[:12]).max() < 1e-6 * b["kappa"] * b["volume"][0] * b["dt"] ** 2
    # away from a rotation: the body gradient is the derivative of the body energy
    bodies = dict(b, boundary_type=np.zeros(2, np.int32))
    q = b["q"] + rng.normal(scale=1e-2, size=b["q"].shape)
    g, *_ = oracle.abd_assemble(bodies, q, b["q_tilde"], b["kappa"], b["dt"])

    def energy(qq):
        E = 0.0
        for k in range(2):
            d = qq[k] - b["q_tilde"][k]
            dm = b["dyadic_mass"][k]
            M = np.zeros((12, 12))
            for r in range(3):
                M[r, r] = dm[0]
                M[r, 3 + 3 * r:6 + 3 * r] = M[3 + 3 * r:6 + 3 * r, r] = dm[1:4]
                M[3 + 3 * r:6 + 3 * r, 3 + 3 * r:6 + 3 * r] = dm[4:].reshape(3, 3)
            A = qq[k, 3:].reshape(3, 3)
            C = A @ A.T - np.eye(3)
            E += 0.5 * d @ M @ d + b["kappa"] * b["volume"][k] * b["dt"] ** 2 * (C ** 2).sum()
        return E

    h = 1e-7
    for k in rng.choice(24, 6, replace=False):
        qp, qm = q.copy(), q.copy()
        qp.flat[k] += h
        qm.flat[k] -= h
        assert (energy(qp) - energy(qm)) / (2 * h) == pytest.approx(g[k], rel=1e-5, abs=1e-9 * np.abs(g).max())


def test_abd_contact_mapping_is_the_point_space_quadratic_form():
    b = scenes.scene_abd_boxes(12, seed=4)
    c = abd_contacts(b, seed=5)
    B, F = 12, c["n_fem"]
    g0, r0, c0, v0 = oracle.abd_assemble(b, b["q"], b["q_tilde"], b["kappa"], b["dt"])
    g1, r1, c1, v1 = oracle.abd_assemble(b, b["q"], b["q_tilde"], b["kappa"], b["dt"], point_grad=c["point_grad"],
                                         abd_blocks=c["abd"], fem_blocks=c["fem"], fem_boundary=c["fem_boundary"])
    n = 4 * B + F

    def quad(rows, cols, vals, y):
        A = oracle.dense(rows, cols, vals, n)
        return y @ A @ y

    rng = np.random.default_rng(6)
    y = rng.normal(size=3 * n)
    d = np.stack([_abd_J(b["x_bar"][p]) @ y[12 * b["point_body"][p]:12 * b["point_body"][p] + 12]
                  for p in range(len(b["point_body"]))])
    yf = y[12 * B:].reshape(F, 3)
    expect = 0.0
    for i, j, H in zip(*c["abd"]):
        expect += d[i] @ H @ d[j] * (1 if i == j else 2)
    for i, f, H in zip(*c["fem"]):
        if c["fem_boundary"][f] == 0:
            expect += 2 * d[i] @ H @ yf[f]
    assert quad(r1, c1, v1, y) - quad(r0, c0, v0, y) == pytest.approx(expect, rel=1e-10)
    # point gradients: J^T g summed per body
    ref = np.zeros(12 * B)
    for p in range(len(b["point_body"])):
        k = b["point_body"][p]
        ref[12 * k:12 * k + 12] += _abd_J(b["x_bar"][p]).T @ c["point_grad"][p]
    assert np.allclose(g1 - g0, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def global_system(sc, bodies, seed=0, coupling=0.05):
    """A coupled FEM + ABD test system: the oracle's FEM matrix of ``sc``, the body-space
    matrix of ``bodies`` with seeded ABD-ABD contact blocks, and ABD-FEM coupling blocks
    scaled to ``coupling`` x the smallest FEM / body diagonal so that A stays SPD.  Returns
    (A dense, FEM rows/cols/vals, ABD contact inputs, the body-space bcoo)."""
    fb, frow, fcol, fval, _ = oracle.assemble(sc)
    Aff = oracle.dense(frow, fcol, fval, sc.nv)
    rng = np.random.default_rng(seed)
    c = abd_contacts(bodies, n_fem=sc.nv, seed=seed)
    # ABD-ABD contacts as PSD pair Hessians: H on both diagonal blocks, -H between
    pb = bodies["point_body"]
    pairs = []
    while len(pairs) < 40:
        i, j = sorted(rng.integers(0, len(pb), 2))
        if pb[i] != pb[j]:
            pairs.append((i, j))
    M = rng.normal(size=(len(pairs), 3, 3))
    H = np.einsum("nij,nkj->nik", M, M) * 1e2
    pi = np.array([p[0] for p in pairs], np.int32)
    pj = np.array([p[1] for p in pairs], np.int32)
    c["abd"] = (np.concatenate([pi, pj, pi]), np.concatenate([pi, pj, pj]), np.concatenate([H, H, -H]))
    g0, r0, c0, v0 = oracle.abd_assemble(bodies, bodies["q"], bodies["q_tilde"], bodies["kappa"], bodies["dt"],
                                         abd_blocks=c["abd"])
    Aaa = oracle.dense(r0, c0, v0, 4 * len(bodies["volume"]))
    scale = coupling * np.sqrt(np.linalg.eigvalsh(Aff).min() * np.linalg.eigvalsh(Aaa).min())
    frows, fcols, fvals = c["fem"]
    fvals = rng.normal(size=fvals.shape)
    fvals *= scale / np.abs(fvals).max()
    c["fem"] = (frows, fcols, fvals)
    c["fem_boundary"] = (sc.boundary_type != 0).astype(np.int32)
    g, rows, cols, vals = oracle.abd_assemble(bodies, bodies["q"], bodies["q_tilde"], bodies["kappa"],
                                              bodies["dt"], point_grad=c["point_grad"], abd_blocks=c["abd"],
                                              fem_blocks=c["fem"], fem_boundary=c["fem_boundary"])
    nb = 4 * len(bodies["volume"])
    A = oracle.dense(np.concatenate([rows, frow + nb]), np.concatenate([cols, fcol + nb]),
                     np.concatenate([vals, fval]), nb + sc.nv)
    return A, (frow, fcol, fval), c, g


def test_global_pcg_without_bodies_is_the_fem_pcg(small_two_cubes):
    """The oracle's global PCG with no ABD rows runs or_pcg's loop on the FEM system."""
    sc = small_two_cubes
    b, rows, cols, vals, _ = oracle.assemble(sc)
    A = oracle.dense(rows, cols, vals, sc.nv)
    M = oracle.Mas(sc, rows, cols, vals)
    x, it, rz0, rz = oracle.pcg(rows, cols, vals, sc.nv, M, b, 1e-4)
    xg, itg, rz0g, rzg = oracle.global_pcg(A, 0, M, b, 1e-4)
    assert itg == it
    assert rz0g == pytest.approx(rz0, rel=1e-12)
    # numpy's dense products and dots round differently from the C loop's sparse ones
    assert np.abs(xg - x).max() <= 1e-7 * np.abs(x).max()


def test_global_pcg_solves_the_coupled_system():
    sc = scenes.scene_cube(4, touching=True, seed=3)
    bodies = scenes.scene_abd_boxes(6, seed=7)
    A, (frow, fcol, fval), c, g = global_system(sc, bodies, seed=4)
    assert np.linalg.eigvalsh(A).min() > 0
    M = oracle.Mas(sc, frow, fcol, fval)
    b = np.random.default_rng(5).normal(size=A.shape[0])
    x, it, rz0, rz = oracle.global_pcg(A, 6, M, b, 1e-20, max_iter=10 * A.shape[0])
    ex = np.linalg.solve(A, b)
    assert np.linalg.norm(x - ex) / np.linalg.norm(ex) < 1e-8
