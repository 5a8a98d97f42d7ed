"""Barrier stiffness adaptation on the GPU (GIPC::initKappa / suggestKappa / upperBoundKappa,
GIPC.cu:9850-9929; the close-constraint checks of GIPC::postLineSearch, GIPC.cu:10777-10806).

* ``sgipc_init_kappa`` against a numpy restatement built from the oracle's element and pair
  gradients: g_E = kinetic + stable Neo-Hookean tets (the reference leaves the cloth terms
  out) + soft constraints, g_c = barrier + ground at kappa = 1, kappa = -(g_c.g_E)/(g_c.g_c)
  raised to the suggestion and bounded by 100 times it (1e-9 relative), on the reference
  golden scene (two 4^3 cubes with Dirichlet vertices, soft constraints and contacts).
* ``sgipc_close_record`` / ``sgipc_close_check``: the recorded counts are the ground vertices
  and pairs below the tolerance, the check is false at the recorded positions and true once a
  recorded ground vertex comes closer; ``GIPC.postLineSearch`` then doubles kappa.
"""
import ctypes as C
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

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _ground_grad(x, verts, offset, dhat, kappa):
    g = np.zeros_like(x)
    for v in verts:
        d = x[v, 1] - offset
        d2, t = d * d, d * d - dhat
        gb = t * np.log(d2 / dhat) * -2.0 - t * t / d2
        g[v, 1] += kappa * gb * 2.0 * d
    return g


def test_init_kappa_matches_restatement():
    sc = scenes.Scene.load(os.path.join(GOLDEN, "scene_two_cubes4.npz"))
    assert len(sc.pairs) > 0
    p = sc.params
    g = system.GIPC(sc)
    try:
        x = sc.vertexes
        GE = sc.masses[:, None] * (x - sc.xTilta)
        for t, dm, vol, mu, lam in zip(sc.tets, sc.dm_inv, sc.volum, sc.length_rate, sc.volume_rate):
            _, gr, _ = oracle.snk_tet(x[t], dm, vol, mu, lam, p["dt"] ** 2)
            GE[t] += gr.reshape(4, 3)
        ks = p["motionRate"] * p["softRate"] ** 2
        for i, v in enumerate(sc.soft_index):
            GE[v] += ks * (x[v] - sc.soft_target[i])
        gc = _ground_grad(x, sc.ground_pairs, p["ground_offset"], p["dHat"], 1.0)
        X, R = x.reshape(-1), sc.rest_vertexes.reshape(-1)
        for enc in sc.pairs:
            vid, _, gr, _ = oracle.barrier_pair(enc, X, R, p["dHat"], 1.0)
            gc[vid] += gr.reshape(-1, 3)
        K = p["kappa"]
        minK = -(gc * GE).sum() / (gc * gc).sum()
        if minK > 0:
            K = minK
        sug = scenes.suggest_kappa(p["bboxDiag2"], p["dHat"], p["meanMass"])
        K = min(max(K, sug), 100.0 * sug)
        got = g.initKappa()
        assert got == pytest.approx(K, rel=1e-9)
        assert g.params["kappa"] == got
    finally:
        g.close()


def test_close_constraints_and_kappa_doubling():
    sc = scenes.scene_two_cubes(4, seed=3)
    g = system.GIPC(sc)
    try:
        L = N.lib()
        k = g.tet.contact_struct_cached()
        dhat, off = sc.params["dHat"], sc.params["ground_offset"]
        cnt = (C.c_int32 * 2)()
        N.check(L.sgipc_close_record(g.ctx, C.c_void_p(g.tet.vertexes.data_ptr()), C.byref(k), dhat, off, cnt, None),
                g.ctx)
        x = sc.vertexes
        ng = int(((x[sc.ground_pairs, 1] - off) ** 2 < dhat).sum())
        assert cnt[0] == ng > 0
        assert cnt[1] == len(sc.pairs) > 0  # every listed pair lies within d-hat
        changed = C.c_int32()
        N.check(L.sgipc_close_check(g.ctx, C.c_void_p(g.tet.vertexes.data_ptr()), off, C.byref(changed), None), g.ctx)
        assert changed.value == 0
        moved = g.tet.vertexes.clone()
        v = int(sc.ground_pairs[0])
        moved[v, 1] -= 0.1 * (x[v, 1] - off)
        N.check(L.sgipc_close_check(g.ctx, C.c_void_p(moved.data_ptr()), off, C.byref(changed), None), g.ctx)
        assert changed.value == 1
        # postLineSearch: the positions of tet come closer -> kappa doubles (below its bound)
        k0 = g.params["kappa"] = 1.0
        g.tet.vertexes.copy_(moved)
        assert g.postLineSearch() == pytest.approx(2.0 * k0)
    finally:
        g.close()
