"""ABDSystem / ABDPreconditioner on the GPU against the oracle, through the C ABI.

Tolerances: body-space blocks identical in pattern, values within 1e-9 of the largest
entry (the 9x9 projection is a Jacobi eigen-decomposition on both sides, in different
orders); body gradients 1e-9; preconditioner apply 1e-9 against numpy inverses of the
oracle's diagonal body groups.
"""
import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sgipc import abd, scenes  # noqa: E402
from sgipc import _native as N  # noqa: E402
from test_oracle import abd_contacts  # noqa: E402


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _dev(a, dtype):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


@pytest.mark.parametrize("fixed", [False, True])
def test_abd_system_matches_oracle(fixed):
    b = scenes.scene_abd_boxes(40, seed=7)
    if fixed:
        b["boundary_type"][::5] = 1
    c = abd_contacts(b, seed=8)
    sysm = abd.ABDSystem(b, max_abd_blocks=len(c["abd"][0]), max_fem_blocks=len(c["fem"][0]))
    try:
        i32, f64 = torch.int32, torch.float64
        g = sysm.setup_abd_system_gradient_hessian(
            _dev(b["q"], f64), _dev(b["q_tilde"], f64), b["kappa"], b["dt"], point_grad=_dev(c["point_grad"], f64),
            abd_blocks=tuple(_dev(a, t) for a, t in zip(c["abd"], (i32, i32, f64))),
            fem_blocks=tuple(_dev(a, t) for a, t in zip(c["fem"], (i32, i32, f64))),
            fem_boundary=_dev(c["fem_boundary"], i32))
        g = g.cpu().numpy()
        rows, cols, vals = sysm.export_bcoo()
        og, orow, ocol, oval = oracle.abd_assemble(b, b["q"], b["q_tilde"], b["kappa"], b["dt"],
                                                   point_grad=c["point_grad"], abd_blocks=c["abd"],
                                                   fem_blocks=c["fem"], fem_boundary=c["fem_boundary"])
        assert np.array_equal(rows, orow) and np.array_equal(cols, ocol)
        assert _rel(vals, oval) < 1e-9
        assert _rel(g, og) < 1e-9
        # block-Jacobi preconditioner: inverse of each body's 12x12 diagonal group
        pre = abd.ABDPreconditioner(sysm)
        pre.assemble()
        rng = np.random.default_rng(9)
        r = rng.normal(size=12 * 40)
        z = pre.apply(_dev(r, f64)).cpu().numpy()
        zr = np.zeros_like(r)
        A = oracle.dense(orow, ocol, oval, 4 * 40 + c["n_fem"])
        for k in range(40):
            blk = A[12 * k:12 * k + 12, 12 * k:12 * k + 12]
            zr[12 * k:12 * k + 12] = np.linalg.solve(blk, r[12 * k:12 * k + 12])
        assert _rel(z, zr) < 1e-9
    finally:
        sysm.close()


def test_abd_bad_point_index_is_reported():
    b = scenes.scene_abd_boxes(4, seed=2)
    sysm = abd.ABDSystem(b, max_abd_blocks=2, max_fem_blocks=0)
    try:
        f64 = torch.float64
        rows = torch.tensor([0, 1], dtype=torch.int32, device="cuda")
        cols = torch.tensor([9, 10 ** 6], dtype=torch.int32, device="cuda")
        vals = torch.zeros((2, 3, 3), dtype=f64, device="cuda")
        with pytest.raises(N.SgipcError) as e:
            sysm.setup_abd_system_gradient_hessian(_dev(b["q"], f64), _dev(b["q_tilde"], f64), b["kappa"], b["dt"],
                                                   abd_blocks=(rows, cols, vals))
        assert e.value.status == N.BAD_INPUT
        with pytest.raises(N.SgipcError) as e:  # more blocks than the context holds
            sysm.setup_abd_system_gradient_hessian(_dev(b["q"], f64), _dev(b["q_tilde"], f64), b["kappa"], b["dt"],
                                                   abd_blocks=(rows.repeat(2), cols.repeat(2), vals.repeat(2, 1, 1)))
        assert e.value.status == N.CAPACITY
    finally:
        sysm.close()
