"""A context created from device-resident topology arrays (the reference keeps its
connectivity in device_TetraData) equals one created from host arrays: the same static
pattern and assembled matrix, bit for bit, and the same right-hand side to rounding.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from sgipc import scenes, system  # noqa: E402
from sgipc import _native as N  # noqa: E402


def test_device_topology_matches_host_topology():
    sc = scenes.scene_cloth_on_cube(10, 5, seed=6)
    host = system.GIPC(sc)
    keep = []

    def dev(a, dt):
        t = torch.tensor(np.ascontiguousarray(a, dt).reshape(-1), device="cuda")
        keep.append(t)
        return C.c_void_p(t.data_ptr()) if t.numel() else None

    t = N.SgipcTopology()
    t.vertex_num, t.tet_num = sc.nv, sc.nt
    t.tri_num, t.tri_edge_num, t.soft_num = len(sc.tris), len(sc.hinges), len(sc.soft_index)
    t.tetrahedras = dev(sc.tets, np.int32)
    t.triangles = dev(sc.tris, np.int32)
    t.tri_edges = dev(sc.hinges, np.int32)
    t.tri_edge_adj_vertex = dev(sc.hinge_adj, np.int32)
    t.targetIndex = dev(sc.soft_index, np.int32)
    t.part_map_size = len(sc.part_map_real)
    t.partId_map_real = dev(sc.part_map_real, np.int32)
    t.real_map_partId = dev(sc.real_map_part, np.int32)
    t.neighborStart = dev(sc.nbr_start, np.int32)
    t.neighborList = dev(sc.nbr_list, np.int32)
    t.max_pairs = max(len(sc.pairs), 1)
    t.max_ground = max(len(sc.ground_pairs), len(sc.surf_verts))
    t.max_fric_pairs = max(len(sc.fric_pairs), 1)
    t.max_fric_ground = max(len(sc.fric_gd_pairs), len(sc.surf_verts))
    t.max_rhs = 1
    h = C.c_void_p()
    N.check(N.lib().sgipc_create(C.byref(t), torch.cuda.current_device(), C.byref(h)))
    try:
        devctx = system.GIPC.__new__(system.GIPC)
        devctx.__dict__.update({k: v for k, v in host.__dict__.items() if k != "ctx"})
        devctx.ctx = h
        host.computeGradientAndHessian()
        a = host.export_bcoo()
        devctx.computeGradientAndHessian()
        b = devctx.export_bcoo()
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
        # the right-hand side takes the contact gradients through atomics: equal to rounding
        ra, rb = host.rhs(), devctx.rhs()
        assert float((ra - rb).abs().max()) <= 1e-12 * float(ra.abs().max())
    finally:
        N.lib().sgipc_destroy(h)
        devctx.ctx = None
        host.close()
