"""GPU parity: every CUDA path through the C ABI against the CPU oracle.

Tolerances (FP64 unless stated):
  * assembled blocks and right-hand side: 1e-9 of the largest entry (same formulas,
    different evaluation order: analytic SNK eigensystem vs numeric projection, hand
    derivatives vs dual numbers);
  * SpMV: 1e-12 relative;
  * MAS hierarchy: identical integer tables; MAS apply: 1e-9 (FP64), 2e-5 (FP32 inverses);
  * PCG: same iteration count within 1, solution within 1e-6 relative of the oracle's.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sgipc import scenes, system  # noqa: E402
from sgipc import _native as N  # noqa: E402


def _soft_cube():
    """A touching cube with soft constraints pulling a few vertices toward offset targets."""
    sc = scenes.scene_cube(5, touching=True, seed=4)
    idx = np.arange(0, sc.nv, 11, dtype=np.int32)
    sc.soft_index = idx
    sc.soft_target = sc.vertexes[idx] + np.array([1e-3, 2e-3, -1e-3])
    sc.params["motionRate"] = 1.0
    sc.params["softRate"] = 1.0
    return sc


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module", params=["c1_cube", "cube_touch", "two_cubes", "cloth_on_cube", "cube_soft",
                                        "cubes_dirichlet", "cloth_roll_sphere"])
def case(request):
    if request.param == "cubes_dirichlet":
        # two 4^3 cubes with Dirichlet vertices (every ninth), soft constraints, ground and
        # pair friction at a moved iterate (the scene of the reference golden vectors):
        # Dirichlet rows and columns zeroed, mass diagonal kept (GIPC.cu:10295-10336)
        sc = scenes.Scene.load(os.path.join(GOLDEN, "scene_two_cubes4.npz"))
        assert (sc.boundary_type != 0).any()
    elif request.param == "cube_soft":
        sc = _soft_cube()
    elif request.param == "c1_cube":
        # the smallest workload: an 11^3 cube 0.05 m above the ground, no contact yet
        sc = scenes.scene_cube(11, touching=False, seed=0)
    elif request.param == "cube_touch":
        sc = scenes.scene_cube(6, touching=True, seed=3)
    elif request.param == "cloth_roll_sphere":
        # the cloth-on-sphere workload at parity size: a 32 x 32 cloth rolled into layers
        # 0.4 mm apart over a 300-cell tet sphere resting on the ground (dense self-contact,
        # bending hinges, membrane strain limiting)
        sc = scenes.scene_cloth_on_sphere(32, 300)
    elif request.param == "two_cubes":
        sc = scenes.scene_two_cubes(7, seed=5)
    else:
        sc = scenes.scene_cloth_on_cube(10, 5, seed=6)
    g = system.GIPC(sc)
    g.computeGradientAndHessian()
    torch.cuda.synchronize()
    ob, orow, ocol, oval, _ = oracle.assemble(sc)
    yield sc, g, (ob, orow, ocol, oval)
    g.close()


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_assembly_blocks(case):
    sc, g, (ob, orow, ocol, oval) = case
    rows, cols, vals = g.export_bcoo()
    assert np.array_equal(rows, orow) and np.array_equal(cols, ocol)
    assert _rel(vals, oval) < 1e-9


def test_rhs(case):
    sc, g, (ob, *_r) = case
    b = g.rhs().cpu().numpy()
    assert _rel(b, ob) < 1e-9


def test_spmv(case):
    sc, g, (ob, orow, ocol, oval) = case
    x = np.random.default_rng(0).normal(size=3 * sc.nv)
    y = g.spmv(torch.tensor(x, device="cuda")).cpu().numpy()
    assert _rel(y, oracle.spmv(orow, ocol, oval, sc.nv, x)) < 1e-12


def test_mas_hierarchy_and_apply(case):
    sc, g, (ob, orow, ocol, oval) = case
    mas = system.MASPreconditioner(g)
    mas.setPreconditioner("fp64")
    om = oracle.Mas(sc, orow, ocol, oval)
    L, starts, counts, total = om.info()
    gl, gcounts, gtotal = mas.info()
    assert gl == L and gtotal == total and np.array_equal(gcounts, counts)
    assert np.array_equal(mas.tables(), om.table())
    gd, od = mas.domains(), om.domains()
    for d in range(len(od)):
        assert _rel(gd[d], od[d]) < 1e-9, d
    r = np.random.default_rng(1).normal(size=3 * sc.nv)
    # restriction operator: R[g] = sum of r over the vertices of cluster g, every level
    R = np.zeros(3 * total)
    rt = torch.tensor(r, device="cuda")
    N.check(N.lib().sgipc_mas_restrict(g.ctx, ctypes.c_void_p(rt.data_ptr()), R.ctypes.data_as(ctypes.c_void_p)))
    Rd = np.zeros((total, 3))
    tab = om.table()
    for lvl in range(L):
        np.add.at(Rd, tab[:, lvl], r.reshape(-1, 3))
    assert _rel(R.reshape(-1, 3), Rd) < 1e-12
    z = mas.preconditioning(torch.tensor(r, device="cuda")).cpu().numpy()
    assert _rel(z, om.apply(r)) < 1e-9
    mas.setPreconditioner("ref")
    z32 = mas.preconditioning(torch.tensor(r, device="cuda")).cpu().numpy()
    assert _rel(z32, om.apply(r, single=True)) < 2e-5


def test_pcg_fp64_matches_oracle(case):
    sc, g, (ob, orow, ocol, oval) = case
    mas = system.MASPreconditioner(g)
    mas.setPreconditioner("fp64")
    om = oracle.Mas(sc, orow, ocol, oval)
    ox, oit, orz0, orz = oracle.pcg(orow, ocol, oval, sc.nv, om, ob, 1e-4)
    solver = system.PCGSolver(g, system.PCGSolverConfig(precision="fp64"))
    x, st = solver.solve(g.rhs())
    x = x.cpu().numpy()
    assert st.status == N.OK
    assert abs(st.iterations - oit) <= 1
    assert abs(st.rz0 - orz0) <= 1e-9 * abs(orz0)
    if st.iterations == oit:
        assert _rel(x, ox) < 1e-6


def test_mixed_and_ref_meet_criterion(case):
    sc, g, (ob, orow, ocol, oval) = case
    A = oracle.dense(orow, ocol, oval, sc.nv)
    exact = np.linalg.solve(A, ob)
    for prec in ("mixed", "ref"):
        mas = system.MASPreconditioner(g)
        mas.setPreconditioner(prec)
        solver = system.PCGSolver(g, system.PCGSolverConfig(precision=prec))
        x, st = solver.solve(g.rhs())
        x = x.cpu().numpy()
        assert st.status == N.OK, prec
        assert abs(st.rz) <= 1e-4 * st.rz0 * 1.0001, prec
        res = np.linalg.norm(ob - A @ x) / np.linalg.norm(ob)
        assert abs(res - st.rel_residual) < 1e-6 * max(1.0, res)
        # the 1e-4 r.z criterion leaves about a 1e-2 relative error in x; the rolled cloth's
        # matrix (condition number about 9e6: 3 mg cloth vertices against membrane and
        # barrier stiffness) keeps about half of it at that stop
        bound = 0.6 if sc.name.startswith("cloth") and "sphere" in sc.name else 0.1
        assert np.linalg.norm(x - exact) / np.linalg.norm(exact) < bound
        assert x @ ob > 0  # a PCG iterate of an SPD system is a descent direction


def test_tight_mixed_matches_fp64(case):
    sc, g, (ob, orow, ocol, oval) = case
    A = oracle.dense(orow, ocol, oval, sc.nv)
    exact = np.linalg.solve(A, ob)
    for prec in ("fp64", "mixed"):
        mas = system.MASPreconditioner(g)
        mas.setPreconditioner(prec)
        # up to 4 x 3n iterations: the rolled cloth needs about 3 000 for 1e-9 (4 566 dofs)
        cfg = system.PCGSolverConfig(precision=prec, global_tol_rate=1e-9, criterion=N.CRIT_TRUE, max_iter_ratio=4.0)
        x, st = system.PCGSolver(g, cfg).solve(g.rhs())
        err = np.linalg.norm(x.cpu().numpy() - exact) / np.linalg.norm(exact)
        assert st.status == N.OK and err < 1e-6, (prec, err, st.iterations, st.refinements)


def test_solve_entry_point(case):
    sc, g, (ob, orow, ocol, oval) = case
    st = g.calculateMovingDirection(system.PCGSolverConfig(precision="fp64"))
    assert st.status == N.OK and st.iterations > 0
    A = oracle.dense(orow, ocol, oval, sc.nv)
    dx = g.moveDir.cpu().numpy()
    assert np.linalg.norm(ob - A @ dx) / np.linalg.norm(ob) == pytest.approx(st.rel_residual, rel=1e-6, abs=1e-12)


def test_batched_four_rhs(case):
    sc, g, (ob, orow, ocol, oval) = case
    rng = np.random.default_rng(7)
    B = rng.normal(size=(4, 3 * sc.nv)) * np.abs(ob).max()
    for prec in ("fp64", "mixed", "ref"):
        mas = system.MASPreconditioner(g)
        mas.setPreconditioner(prec)
        cfg = system.PCGSolverConfig(precision=prec, global_tol_rate=1e-10, criterion=N.CRIT_TRUE,
                                     max_iter_ratio=4.0)
        X, sts = system.PCGSolver(g, cfg).solve_batched(torch.tensor(B, device="cuda"))
        A = oracle.dense(orow, ocol, oval, sc.nv)
        # the batched mixed solve runs FP32 end to end (no FP64 refinement): its attainable
        # residual is about cond(A) x 6e-8, 0.06 on the rolled cloth (cond about 9e6)
        ill = sc.name.startswith("cloth") and "sphere" in sc.name
        tol = 1e-8 if prec != "mixed" else (0.1 if ill else 1e-4)
        for r in range(4):
            res = np.linalg.norm(B[r] - A @ X[r].cpu().numpy()) / np.linalg.norm(B[r])
            assert res < max(tol, 1e-9), (prec, r, res, sts[r].iterations)


@pytest.mark.parametrize("prec", ["fp64", "mixed", "ref"])
def test_persistent_and_graph_solves_agree(case, prec, monkeypatch):
    """The one-kernel persistent solve and the graph of per-phase kernels run the same
    algorithm up to rounding: the summation order of the dot products differs, and the fused
    persistent iteration forms A p and p.Ap by recurrences."""
    sc, g, _ = case
    mas = system.MASPreconditioner(g)
    mas.setPreconditioner(prec)
    solver = system.PCGSolver(g, system.PCGSolverConfig(precision=prec))
    xa, sa = solver.solve(g.rhs())
    xa = xa.cpu().numpy()
    monkeypatch.setenv("SGIPC_PCG_GRAPH", "1")
    xb, sb = solver.solve(g.rhs())
    xb = xb.cpu().numpy()
    monkeypatch.delenv("SGIPC_PCG_GRAPH")
    assert sa.status == N.OK and sb.status == N.OK
    assert abs(sa.iterations - sb.iterations) <= 1
    assert abs(sa.rz0 - sb.rz0) <= 1e-9 * abs(sb.rz0)
    if sa.iterations == sb.iterations:
        assert _rel(xa, xb) < (1e-9 if prec == "fp64" else 1e-4)


def test_mas_build_with_other_contacts_rebuilds_the_hierarchy(case):
    """sgipc_assemble prebuilds the hierarchy for its contacts; a build given other contacts
    (here none) must build its own, equal to the oracle's for those contacts."""
    sc, g, (ob, orow, ocol, oval) = case
    g.computeGradientAndHessian()
    N.check(N.lib().sgipc_mas_build(g.ctx, None, N.PRECISION["fp64"], None), g.ctx)
    om = oracle.Mas(sc, orow, ocol, oval, pairs=np.zeros((0, 4), np.int32))
    mas = system.MASPreconditioner(g)
    assert np.array_equal(mas.tables(), om.table())
    mas.setPreconditioner("fp64")  # back to the assembled contacts
    assert np.array_equal(mas.tables(), oracle.Mas(sc, orow, ocol, oval).table())


def test_mas_build_after_a_new_static_matrix_uses_it(case):
    """sgipc_assemble scatters its static blocks into the prebuilt hierarchy's domains ahead of
    the build; a static matrix rewritten in between (sgipc_fem_grad_hess at other positions)
    must replace them: the build equals one that scatters everything itself."""
    sc, g, _ = case
    mas = system.MASPreconditioner(g)
    g.computeGradientAndHessian()
    mas.setPreconditioner("fp64")
    d0 = mas.domains()
    tet2 = system.DeviceTetraData(sc)
    gen = torch.Generator(device="cuda").manual_seed(8)
    tet2.vertexes = tet2.vertexes + 1e-3 * torch.randn(tet2.vertexes.shape, dtype=torch.float64, device="cuda",
                                                       generator=gen)
    grad = torch.zeros(3 * sc.nv, dtype=torch.float64, device="cuda")
    try:
        g.computeGradientAndHessian()
        g.calculate_fem_gradient_hessian(grad, tet2)
        mas.setPreconditioner("fp64")  # the prebuilt hierarchy, its scatter stale
        d1 = mas.domains()
        mas.setPreconditioner("fp64")  # hierarchy rebuilt, everything scattered by the build
        d2 = mas.domains()
    finally:
        g.computeGradientAndHessian()
    assert _rel(d1, d2) < 1e-9
    assert np.abs(d2 - d0).max() > 100 * np.abs(d1 - d2).max()


def test_step_from_host_matches_device_step(case):
    """The host-state path (inputs packed in one pinned buffer, one copy per step) solves the
    same system as the device path; twice, the second time through the bound buffers."""
    sc, g, _ = case
    cfg = system.PCGSolverConfig(precision="fp64")
    g.computeGradientAndHessian()
    st0 = g.calculateMovingDirection(cfg)
    x0 = g.moveDir.cpu().numpy()
    host = system.HostNewtonState(sc)
    for _ in range(2):
        host.move_dir.zero_()
        st = system.step_from_host(g, host, cfg)
        assert st.status == N.OK and abs(st.iterations - st0.iterations) <= 1
        assert _rel(host.move_dir.numpy(), x0) < 1e-9
    g.computeGradientAndHessian()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_zero_rhs_gives_zero_solution(case, prec):
    sc, g, _ = case
    system.MASPreconditioner(g).setPreconditioner(prec)
    b = torch.zeros(3 * sc.nv, dtype=torch.float64, device="cuda")
    x, st = system.PCGSolver(g, system.PCGSolverConfig(precision=prec)).solve(b)
    assert st.status == N.OK and st.iterations == 0
    assert float(x.abs().max()) == 0.0


def test_iteration_cap_reports_not_converged(case):
    sc, g, _ = case
    mas = system.MASPreconditioner(g)
    mas.setPreconditioner("fp64")
    L = N.lib()
    b = g.rhs()
    x = torch.empty_like(b)
    for graph in (False, True):
        if graph:
            import os
            os.environ["SGIPC_PCG_GRAPH"] = "1"
        try:
            st = N.SgipcSolveStats()
            s = L.sgipc_pcg_solve(g.ctx, N.FP64, N.CRIT_RZ, 1e-12, 4, ctypes.c_void_p(b.data_ptr()),
                                  ctypes.c_void_p(x.data_ptr()), ctypes.byref(st), None)
        finally:
            if graph:
                del os.environ["SGIPC_PCG_GRAPH"]
        assert s == N.NOT_CONVERGED and st.status == N.NOT_CONVERGED, graph
        assert st.iterations == 3, graph   # max_iter 4: SpMVs k = 1 .. max_iter-1


def test_bad_inputs_are_reported(case):
    sc, g, _ = case
    L = N.lib()
    prm = system.params_struct(g.params)
    f = g.tet.fem_struct()
    assert L.sgipc_assemble(g.ctx, None, None, None, None) == N.BAD_INPUT
    bad = dict(g.params)
    bad["dHat"] = -1.0
    pb = system.params_struct(bad)
    assert L.sgipc_assemble(g.ctx, f, None, pb, None) == N.BAD_INPUT
    k = g.tet.contact_struct()
    k.pair_num = 10 ** 7
    assert L.sgipc_assemble(g.ctx, f, k, prm, None) == N.CAPACITY
    # a pair naming a vertex outside the mesh: skipped by the assembly, reported by the solve
    if len(sc.pairs):
        pairs = g.tet.pairs.clone()
        pairs[0, 1] = 10 ** 6
        k = g.tet.contact_struct()
        k.pairs = system._p(pairs)
        assert L.sgipc_assemble(g.ctx, f, k, prm, None) == N.OK
        st = N.SgipcSolveStats()
        dx = torch.empty(3 * sc.nv, dtype=torch.float64, device="cuda")
        assert L.sgipc_solve(g.ctx, k, N.FP64, N.CRIT_RZ, 1e-4, 0, system._p(dx), ctypes.byref(st), None) \
            == N.BAD_INPUT
        assert b"outside" in L.sgipc_last_error(g.ctx)
    # the context stays usable
    g.computeGradientAndHessian()
    st = g.calculateMovingDirection(system.PCGSolverConfig(precision="fp64"))
    assert st.status == N.OK
    torch.cuda.synchronize()


def test_phase_profile_of_the_persistent_solve(case):
    """sgipc_profile_pcg: every CTA stamps every barrier of one solve in order (arrival
    before departure, departure before the next arrival), the phases follow the solve's
    structure, and the profiled solve takes the iterations of an ordinary one."""
    sc, g, _ = case
    mas = system.MASPreconditioner(g)
    mas.setPreconditioner("fp64")
    _, st = system.PCGSolver(g, system.PCGSolverConfig(precision="fp64")).solve(g.rhs())
    stamps, phases = g.profile_pcg("pcg64")
    grid, epochs = stamps.shape[0], stamps.shape[1]
    assert grid >= 1 and epochs >= 3
    assert (stamps[:, :, 1] >= stamps[:, :, 0]).all()
    assert (stamps[:, 1:, 0] >= stamps[:, :-1, 1]).all()
    assert phases[0] == "start" and phases[1] == "init" and "?" not in phases
    # one SpMV phase per iteration: the four-phase iteration's or the fused one's
    assert phases.count("spmv") + phases.count("fused_spmv") == st.iterations
    mas.setPreconditioner("mixed")
    stamps4, phases4 = g.profile_pcg("pcg32x4")
    assert phases4.count("spmv") + phases4.count("fused_spmv") >= 1
    assert (stamps4[:, :, 1] >= stamps4[:, :, 0]).all()


@pytest.mark.parametrize("prec", ["fp64", "mixed", "ref"])
def test_fused_and_four_phase_persistent_solves_agree(case, prec, monkeypatch):
    """With three MAS levels or more the persistent solve runs the fused iteration (three
    barriers: z prolonged into the SpMV, the level-0/1 domains solved in the update, p.Ap from
    the recurrence z.w + 2 beta z.Ap_old + beta^2 p_old.Ap_old); SGIPC_PCG_FUSED=0 runs the
    four-phase one.  Same iteration counts within one, r0.z0 to 1e-12, solutions to 1e-9
    (FP64) / 1e-4 (FP32 vectors)."""
    sc, g, _ = case
    mas = system.MASPreconditioner(g)
    mas.setPreconditioner(prec)
    solver = system.PCGSolver(g, system.PCGSolverConfig(precision=prec))
    xa, sa = solver.solve(g.rhs())
    monkeypatch.setenv("SGIPC_PCG_FUSED", "0")
    xb, sb = solver.solve(g.rhs())
    monkeypatch.delenv("SGIPC_PCG_FUSED")
    assert sa.status == N.OK and sb.status == N.OK
    assert abs(sa.iterations - sb.iterations) <= 1
    assert abs(sa.rz0 - sb.rz0) <= 1e-12 * abs(sb.rz0)
    if sa.iterations == sb.iterations:
        assert _rel(xa.cpu().numpy(), xb.cpu().numpy()) < (1e-9 if prec == "fp64" else 1e-4)
