"""The CUDA path against the reference's own code, through the C ABI.

``tests/golden/ref_golden.npz`` holds results of the reference's functions and kernels
compiled for the host from a reference checkout (``oracle/ref_build.py``,
``tests/golden/make_golden.py``) on the two scenes stored beside it: two 4^3 cubes in
contact with friction, ground contact, soft constraints and Dirichlet vertices, and a cloth
on a cube.  Here the GPU computes the same quantities for those scenes and is compared
with the reference directly, not through the oracle:

* the assembled right-hand side against the sum of the reference's gradient kernels
  (kinetic, SNK, barrier, friction, ground barrier, ground friction, soft constraints),
  Dirichlet rows zeroed as FEMLinearSubsystem::assemble does;
* the line-search energy's terms against the reference's per-element energies (SNK,
  membrane, barrier, friction, ground friction), weighted as GIPC::computeEnergy weights
  them (GIPC.cu:10520-10580);
* every CCD candidate's time of impact and every ground vertex's step bound against the
  reference's step-size kernels (GIPC.cu:6902, 7052; ACCD.cu:373-535);
* the trial step of GIPC::step_forward (_stepForward GIPC.cu:7937) with fixed vertices.

Tolerances: right-hand side and energies 1e-10 relative (FP64, other summation order);
times of impact 1e-9 relative; the trial step bit for bit.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sgipc import scenes, system  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "ref_golden.npz"))
FILES = {"cubes": "scene_two_cubes4.npz", "cloth": "scene_cloth6_cube4.npz"}


@pytest.fixture(scope="module", params=["cubes", "cloth"])
def case(request):
    sc = scenes.Scene.load(os.path.join(HERE, "golden", FILES[request.param]))
    g = system.GIPC(sc)
    yield request.param, sc, g
    g.close()


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


def _scatter(total, vid, grad, w=1.0):
    for k in range(len(vid)):
        for a, v in enumerate(vid[k]):
            if v >= 0:
                total[v] += w * grad[k, a]


def test_rhs_is_the_sum_of_the_reference_gradient_kernels(case):
    tag, sc, g = case
    if tag != "cubes":
        pytest.skip("the cloth scene's quadratic bending gradient has no host-compiled reference")
    p = sc.params
    t = tag + "_"
    total = G[t + "kin_grad"] + G[t + "fem_grad"] + G[t + "soft_grad"]
    _scatter(total, G[t + "bar_vid"], G[t + "bar_grad"])
    _scatter(total, G[t + "fric_vid"], G[t + "fric_grad"], p["frictionRate"])
    for k, v in enumerate(sc.ground_pairs):
        total[v] += G[t + "ground_grad"][k]
    for k, v in enumerate(sc.fric_gd_pairs):
        total[v] += p["gd_frictionRate"] * G[t + "gfric_grad"][k]
    fixed = sc.boundary_type != 0
    assert fixed.any()
    total[fixed] = 0.0
    g.computeGradientAndHessian()
    b = g.rhs().cpu().numpy().reshape(-1, 3)
    assert _rel(b, total) < 1e-10


def test_energy_terms_match_the_reference_elements(case):
    tag, sc, g = case
    p = sc.params
    dt2 = p["dt"] ** 2
    t = tag + "_"
    _, parts = g.computeEnergy(terms=True)
    want = {1: dt2 * G[t + "snk_energy"].sum(), 5: G[t + "bar_energy"].sum(),
            7: p["frictionRate"] * G[t + "fric_energy"].sum(), 8: p["gd_frictionRate"] * G[t + "gfric_energy"].sum()}
    if tag == "cloth":
        want[2] = dt2 * G[t + "tri_energy"].sum()
    for k, w in want.items():
        assert w > 0.0, k
        assert parts[k] == pytest.approx(w, rel=1e-10, abs=0.0), k


def test_step_bounds_match_the_reference(case):
    tag, sc, g = case
    t = tag + "_"
    cand = torch.tensor(G[t + "ccd_cand"], device="cuda")
    move = torch.tensor(G[t + "move"], device="cuda")
    toi = torch.empty(len(cand), dtype=torch.float64, device="cuda")
    alpha = g.self_largestFeasibleStepSize(0.8, move, cand, toi=toi)
    inv = G[t + "ccd_inv"]
    assert _rel(1.0 / toi.cpu().numpy(), inv) < 1e-9
    assert alpha == pytest.approx(1.0 / max(1.0, inv.max()), rel=1e-9)
    gmove = torch.tensor(G[t + "gmove"], device="cuda")
    for k, v in enumerate(sc.ground_pairs):
        a = g.ground_largestFeasibleStepSize(0.8, gmove, torch.tensor([v], dtype=torch.int32, device="cuda"))
        assert a == pytest.approx(1.0 / max(1.0, G[t + "ground_step_inv"][k]), rel=1e-14), k


def test_step_forward_matches_the_reference(case):
    tag, sc, g = case
    assert (sc.boundary_type != 0).any() or tag == "cloth"
    tet = system.DeviceTetraData(sc)
    xb = torch.tensor(sc.vertexes, device="cuda")
    move = torch.tensor(G[tag + "_move"], device="cuda")
    for mb in (0, 1):
        tet.vertexes.zero_()  # the reference kernel leaves a fixed vertex's current position
        g.step_forward(0.37, xb, move, tet=tet, move_boundary=bool(mb))
        assert np.array_equal(tet.vertexes.cpu().numpy(), G[tag + "_step_forward_%d" % mb]), mb
