"""sgipc_mas_apply_noalloc against sgipc_mas_apply, through the C ABI.

The no-allocation entry point serves hosts that may not allocate device memory while a
solver call runs (their pool owns every allocation, or an allocation's implicit
synchronisation is not allowed in their loop).  It runs the same preconditioner apply with
its work vectors in a fixed array inside the library, so its result must equal the regular
entry point's.  Two calls in a row check that what the first call leaves in the shared
array does not leak into the second.  Tolerance: 1e-12 relative, as the SpMV parity test
(the kernels and their summation order are the same, so the results are in fact equal).

This file is named to be collected last, so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sgipc import scenes, system  # noqa: E402
from sgipc import _native as N  # noqa: E402


def _apply(fn, g, r):
    z = torch.full_like(r, float("nan"))
    st = fn(g.ctx, ctypes.c_void_p(r.data_ptr()), ctypes.c_void_p(z.data_ptr()), None)
    torch.cuda.synchronize()
    return st, z.cpu().numpy()


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("precision", ["fp64", "ref"])
def test_noalloc_apply_matches_regular(precision):
    sc = scenes.scene_two_cubes(7, seed=5)
    g = system.GIPC(sc)
    try:
        g.computeGradientAndHessian()
        mas = system.MASPreconditioner(g)
        mas.setPreconditioner(precision)
        assert mas.info()[2] <= 65536
        rng = np.random.default_rng(7)
        lib = N.lib()
        for call in range(2):
            r = torch.tensor(rng.normal(size=3 * sc.nv), device="cuda")
            st0, z_ref = _apply(lib.sgipc_mas_apply, g, r)
            st1, z = _apply(lib.sgipc_mas_apply_noalloc, g, r)
            assert st0 == 0 and st1 == 0, (st0, st1, N.lib().sgipc_last_error(g.ctx))
            assert np.isfinite(z).all()
            assert _rel(z, z_ref) < 1e-12, (precision, call)
    finally:
        g.close()


def test_noalloc_apply_rejects_large_hierarchy():
    # 42^3 = 74088 vertices: more level-0 positions than the fixed array serves
    sc = scenes.scene_cube(42, touching=False, seed=0)
    g = system.GIPC(sc)
    try:
        g.computeGradientAndHessian()
        mas = system.MASPreconditioner(g)
        mas.setPreconditioner("fp64")
        assert mas.info()[2] > 65536
        r = torch.zeros(3 * sc.nv, dtype=torch.float64, device="cuda")
        st, _ = _apply(N.lib().sgipc_mas_apply_noalloc, g, r)
        assert st == N.CAPACITY
        msg = N.lib().sgipc_last_error(g.ctx)
        assert b"static scratch" in msg
    finally:
        g.close()
