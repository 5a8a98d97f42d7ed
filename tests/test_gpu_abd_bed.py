"""Affine bodies on a soft bed: the contact class partition (``sgipc_contact_partition``,
GIPC::partitionContactHessian GIPC.cu:9932-10108) and the coupled FEM + ABD Newton system.

The scene (``scenes.scene_abd_on_bed``) holds the bed's vertices first and the boxes' points
after them, Dirichlet in the FEM context: ``sgipc_assemble`` keeps the FEM-FEM parts of the
contact terms, and the partition returns the blocks that touch a box point, ABD-ABD and
ABD-FEM, with the contact gradient at the points, for ``sgipc_abd_grad_hess``.

* Small scene (12 boxes, 6 x 2 x 6 bed cells), contacts from the host generator: the
  partition's blocks summed per (row, col) equal the oracle's barrier and ground Hessians of
  the same pairs (1e-9 of the largest block), its point gradient the oracle's (1e-9), the
  counts exact; the coupled solve (``GlobalLinearSystem``) matches the oracle's global PCG on
  the dense system built from the oracle's FEM assembly and ``or_abd_assemble`` of the
  partition's blocks (iterations within one, x 1e-6).
* The workload at full size (500 boxes, 100 000-tet bed), contacts from the GPU pair search:
  boxes resting on the bed give ABD-FEM blocks, every ABD-ABD block has row <= col and every
  ABD-FEM column is a bed vertex, the points' dx equal J(x_bar) dq, and the coupled solve meets
  its criterion in FP64 and with FP32 MAS inverses, the two within 1e-3 of each other.
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


def _dev(a, dtype):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _coupled(sc, bodies, g, prec="fp64"):
    """Assembly, partition, body terms and both preconditioners of the Newton system."""
    g.computeGradientAndHessian()
    part = g.contactPartition(bodies["abd_first"])
    ar, ac, av = part["abd_blocks"]
    fr, fc, fv = part["fem_blocks"]
    sysm = abd.ABDSystem(bodies, max_abd_blocks=max(1, ar.numel()), max_fem_blocks=max(1, fr.numel()))
    f64 = torch.float64
    sysm.setup_abd_system_gradient_hessian(_dev(bodies["q"], f64), _dev(bodies["q_tilde"], f64), bodies["kappa"],
                                           bodies["dt"], point_grad=part["point_grad"], abd_blocks=(ar, ac, av),
                                           fem_blocks=(fr, fc, fv), fem_boundary=g.tet.BoundaryType)
    abd.ABDPreconditioner(sysm).assemble()
    system.MASPreconditioner(g).setPreconditioner(prec)
    return part, sysm


@pytest.fixture(scope="module")
def small():
    sc, bodies = scenes.scene_abd_on_bed(12, (6, 2, 6), seed=1, resting=0.7)
    g = system.GIPC(sc)
    part, sysm = _coupled(sc, bodies, g)
    yield sc, bodies, g, part, sysm
    sysm.close()
    g.close()


def _oracle_partition(sc, af):
    """Per (row, col) sums of the oracle's contact Hessian blocks that touch a point >= af
    (upper orientation, as the partition keys them) and the contact gradient at the points."""
    p = sc.params
    X, R = sc.vertexes.reshape(-1), sc.rest_vertexes.reshape(-1)
    blocks, grad = {}, np.zeros((sc.nv, 3))
    for enc in np.asarray(sc.pairs):
        vid, _, gr, H = oracle.barrier_pair(enc, X, R, p["dHat"], p["kappa"])
        for a, va in enumerate(vid):
            grad[va] += gr[3 * a:3 * a + 3]
            for b, vb in enumerate(vid):
                if b < a or max(va, vb) < af:
                    continue
                r, c = (va, vb) if va <= vb else (vb, va)
                blk = H[3 * a:3 * a + 3, 3 * b:3 * b + 3]
                if va > vb:
                    blk = blk.T
                blocks[(int(r), int(c))] = blocks.get((int(r), int(c)), 0.0) + blk
    dh, kap, off = p["dHat"], p["kappa"], p["ground_offset"]
    for v in np.asarray(sc.ground_pairs):
        if v < af:
            continue
        d = sc.vertexes[v, 1] - off
        d2, t = d * d, d * d - dh
        gb = t * np.log(d2 / dh) * -2.0 - t * t / d2
        hb = (np.log(d2 / dh) * -2.0 - t * 4.0 / d2) + t * t / (d2 * d2)
        grad[v, 1] += kap * gb * 2.0 * d
        H = np.zeros((3, 3))
        H[1, 1] = kap * (4.0 * hb * d2 + 2.0 * gb)
        blocks[(int(v), int(v))] = blocks.get((int(v), int(v)), 0.0) + H
    return blocks, grad[af:]


def test_partition_matches_oracle(small):
    sc, bodies, g, part, _ = small
    af = bodies["abd_first"]
    ref, ref_grad = _oracle_partition(sc, af)
    got = {}
    for (r, c, v), fem in ((part["abd_blocks"], False), (part["fem_blocks"], True)):
        for rr, cc, vv in zip(r.cpu().numpy(), c.cpu().numpy(), v.cpu().numpy()):
            # back to upper orientation in scene indices: ABD-FEM blocks are (point, FEM vertex)
            key = (int(cc), int(rr) + af) if fem else (int(rr) + af, int(cc) + af)
            got[key] = got.get(key, 0.0) + (vv.T if fem else vv)
    assert len(ref) > 0 and set(got) == set(ref)
    scale = max(np.abs(b).max() for b in ref.values())
    for k, b in ref.items():
        assert np.abs(got[k] - b).max() <= 1e-9 * scale, k
    pg = part["point_grad"].cpu().numpy()
    assert np.abs(pg - ref_grad).max() <= 1e-9 * max(np.abs(ref_grad).max(), 1e-300)


def test_coupled_solve_matches_oracle(small):
    sc, bodies, g, part, sysm = small
    B = len(bodies["volume"])
    # the dense global system: body space from or_abd_assemble of the partition's blocks, FEM
    # rows from the oracle's assembly (the box points Dirichlet: decoupled unit rows)
    ar, ac, av = (t.cpu().numpy() for t in part["abd_blocks"])
    fr, fc, fv = (t.cpu().numpy() for t in part["fem_blocks"])
    gb, rows, cols, vals = oracle.abd_assemble(bodies, bodies["q"], bodies["q_tilde"], bodies["kappa"], bodies["dt"],
                                               point_grad=part["point_grad"].cpu().numpy(), abd_blocks=(ar, ac, av),
                                               fem_blocks=(fr, fc, fv), fem_boundary=sc.boundary_type)
    fb, frow, fcol, fval, _ = oracle.assemble(sc)
    nb = 4 * B
    A = oracle.dense(np.concatenate([rows, frow + nb]), np.concatenate([cols, fcol + nb]),
                     np.concatenate([vals, fval.reshape(-1, 3, 3)]), nb + sc.nv)
    assert np.linalg.eigvalsh(A).min() > 0
    gls = abd.GlobalLinearSystem(g, sysm)
    b = gls.right_hand_side()
    assert np.abs(b.cpu().numpy()[:12 * B] - gb).max() <= 1e-9 * max(np.abs(gb).max(), 1e-300)
    assert np.abs(b.cpu().numpy()[12 * B:] - fb).max() <= 1e-9 * max(np.abs(fb).max(), 1e-300)
    x, pdx, st = gls.solve_linear_system(b, tol=1e-4)
    om = oracle.Mas(sc, frow, fcol, fval)
    ox, oit, orz0, _ = oracle.global_pcg(A, B, om, b.cpu().numpy(), 1e-4)
    assert st.status == N.OK and abs(st.iterations - oit) <= 1
    assert st.rz0 == pytest.approx(orz0, rel=1e-9)
    if st.iterations == oit:
        x = x.cpu().numpy()
        assert np.linalg.norm(x - ox) / np.linalg.norm(ox) < 1e-6


@pytest.fixture(scope="module")
def full():
    sc, bodies = scenes.scene_abd_on_bed(500, contacts=False)
    g = system.GIPC(sc, pair_capacity=400_000)
    g.buildCP(body=torch.tensor(sc.body_of_vertex, dtype=torch.int32, device="cuda"))
    yield sc, bodies, g
    g.close()


def test_fullsize_coupled_solve_meets_its_criterion(full):
    sc, bodies, g = full
    af = bodies["abd_first"]
    p = g.tet.pairs.cpu().numpy()
    assert len(p) > 0
    xs = {}
    for prec in ("fp64", "ref"):
        part, sysm = _coupled(sc, bodies, g, prec)
        try:
            na, nf = part["abd_blocks"][0].numel(), part["fem_blocks"][0].numel()
            assert nf > 0  # boxes rest on the bed
            assert (part["abd_blocks"][0] <= part["abd_blocks"][1]).all()
            assert int(part["fem_blocks"][1].max()) < af
            gls = abd.GlobalLinearSystem(g, sysm)
            b = gls.right_hand_side()
            x, pdx, st = gls.solve_linear_system(b, tol=1e-4)
            assert st.status == N.OK and 0 < st.iterations
            assert abs(st.rz) <= 1e-4 * st.rz0 * (1 + 1e-9)
            xs[prec] = x
            # the points' dx = J(x_bar) dq
            dq = x[:12 * sysm.body_num].reshape(-1, 12)[torch.tensor(bodies["point_body"], device="cuda").long()]
            xb = torch.tensor(bodies["x_bar"], device="cuda")
            J = dq[:, :3] + torch.einsum("pc,prc->pr", xb, dq[:, 3:].reshape(-1, 3, 3))
            assert (J - pdx).abs().max() <= 1e-12 * max(float(J.abs().max()), 1e-300)
        finally:
            sysm.close()
    d = (xs["ref"] - xs["fp64"]).norm() / xs["fp64"].norm()
    assert float(d) < 1e-3
