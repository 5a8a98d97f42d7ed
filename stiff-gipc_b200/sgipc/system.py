"""Host-side mirror of StiffGIPC's Newton-system interfaces over the C ABI.

Names follow the reference so that a caller of the reference finds the same entry
points:

* :class:`DeviceTetraData` — the SoA device arrays of ``device_TetraData``
  (StiffGIPC/device_fem_data.cuh:17-78), held in torch CUDA tensors;
* :class:`GIPC` — ``computeGradientAndHessian`` (GIPC.cu:10110),
  ``calBarrierGradientAndHessian`` (GIPC.cu:9112), ``calFrictionGradientAndHessian``
  (GIPC.cu:9164-9217) and ``calculateMovingDirection`` (GIPC.cu:10581);
* :class:`MASPreconditioner` — ``setPreconditioner_bcoo`` / ``preconditioning``
  (MASPreconditioner.cu:2180-2262);
* :class:`PCGSolver` with :class:`PCGSolverConfig` (linear_system/solver/pcg_solver.h).

Torch only provides device memory and the current stream; every computation is a call
into ``libsgipc.so``.  Errors surface as :class:`sgipc._native.SgipcError`.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional

import numpy as np
import torch

from . import _native as N


def _dev():
    if not torch.cuda.is_available():
        raise RuntimeError("sgipc needs a CUDA device; there is no CPU path")
    return torch.device("cuda", torch.cuda.current_device())


def _t(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=_dev()).contiguous()


def _p(t: Optional[torch.Tensor]):
    return None if t is None or t.numel() == 0 else C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class DeviceTetraData:
    """Device copies of a :class:`sgipc.scenes.Scene`'s per-Newton arrays."""

    def __init__(self, sc):
        f64, i32 = torch.float64, torch.int32
        self.vertexes = _t(sc.vertexes, f64)
        self.o_vertexes = _t(sc.o_vertexes, f64)
        self.rest_vertexes = _t(sc.rest_vertexes, f64)
        self.xTilta = _t(sc.xTilta, f64)
        self.masses = _t(sc.masses, f64)
        self.BoundaryType = _t(sc.boundary_type, i32)
        self.DmInverses = _t(sc.dm_inv.reshape(-1, 9), f64)
        self.volum = _t(sc.volum, f64)
        self.lengthRate = _t(sc.length_rate, f64)
        self.volumeRate = _t(sc.volume_rate, f64)
        self.triDmInverses = _t(sc.tri_dm_inv.reshape(-1, 4), f64)
        self.area = _t(sc.area, f64)
        self.quad_bending_Q = _t(np.transpose(sc.hinge_q, (0, 2, 1)).reshape(-1, 16), f64)
        self.targetVert = _t(sc.soft_target.reshape(-1, 3), f64)
        self.pairs = _t(sc.pairs.reshape(-1, 4), i32)
        self.ground_pairs = _t(sc.ground_pairs, i32)
        self.fric_pairs = _t(sc.fric_pairs.reshape(-1, 4), i32)
        self.fric_lambda = _t(sc.fric_lambda, f64)
        self.fric_coord = _t(sc.fric_coord.reshape(-1, 2), f64)
        self.fric_basis = _t(sc.fric_basis.reshape(-1, 6), f64)
        self.fric_gd_pairs = _t(sc.fric_gd_pairs, i32)
        self.fric_gd_lambda = _t(sc.fric_gd_lambda, f64)

    # The C structs hold raw device pointers; they are rebuilt only after an attribute of
    # this object is (re)assigned -- in-place updates (copy_) keep the pointers valid.
    def __setattr__(self, name, value):
        object.__setattr__(self, name, value)
        if not name.startswith("_"):
            object.__setattr__(self, "_structs", {})

    def _cached(self, key, build):
        cache = self.__dict__.setdefault("_structs", {})
        if key not in cache:
            cache[key] = build()
        return cache[key]

    def fem_struct(self) -> N.SgipcFemData:
        return self._fem_struct()

    def contact_struct(self) -> N.SgipcContacts:
        return self._contact_struct()

    def fem_struct_cached(self) -> N.SgipcFemData:
        """Shared struct for the library's own calls (never modify it)."""
        return self._cached("fem", self._fem_struct)

    def contact_struct_cached(self) -> N.SgipcContacts:
        """Shared struct for the library's own calls (never modify it)."""
        return self._cached("con", self._contact_struct)

    def _fem_struct(self) -> N.SgipcFemData:
        f = N.SgipcFemData()
        for name in ("vertexes", "o_vertexes", "rest_vertexes", "xTilta", "masses", "BoundaryType", "DmInverses",
                     "volum", "lengthRate", "volumeRate", "triDmInverses", "area", "quad_bending_Q", "targetVert"):
            setattr(f, name, _p(getattr(self, name)))
        return f

    def _contact_struct(self) -> N.SgipcContacts:
        k = N.SgipcContacts()
        k.pairs, k.pair_num = _p(self.pairs), self.pairs.shape[0]
        k.ground_pairs, k.ground_num = _p(self.ground_pairs), self.ground_pairs.shape[0]
        k.fric_pairs, k.fric_num = _p(self.fric_pairs), self.fric_pairs.shape[0]
        k.fric_lambda, k.fric_coord, k.fric_basis = _p(self.fric_lambda), _p(self.fric_coord), _p(self.fric_basis)
        k.fric_gd_pairs, k.fric_gd_num = _p(self.fric_gd_pairs), self.fric_gd_pairs.shape[0]
        k.fric_gd_lambda = _p(self.fric_gd_lambda)
        return k


@dataclasses.dataclass
class PCGSolverConfig:
    """``PCGSolverConfig`` (linear_system/solver/pcg_solver.h:8-18)."""

    max_iter_ratio: float = 0.3
    global_tol_rate: float = 1e-4
    precision: str = "fp64"       # "fp64" | "mixed" | "ref"
    criterion: int = N.CRIT_RZ


def params_struct(p: dict) -> N.SgipcParams:
    s = N.SgipcParams()
    for name, _ in N.SgipcParams._fields_:
        setattr(s, name, float(p.get(name, 0.0)))
    return s


class GIPC:
    """One Newton system on the GPU (context = static BSR pattern + MAS + PCG workspaces)."""

    def __init__(self, sc, device: Optional[int] = None, max_rhs: int = 4, pair_capacity: Optional[int] = None):
        self.scene = sc
        dev = torch.cuda.current_device() if device is None else device
        torch.cuda.set_device(dev)
        L = N.lib()
        self._host = []
        t = N.SgipcTopology()
        t.vertex_num, t.tet_num = sc.nv, sc.nt
        t.tri_num, t.tri_edge_num, t.soft_num = len(sc.tris), len(sc.hinges), len(sc.soft_index)
        t.tetrahedras = self._hp(sc.tets, np.uint32)
        t.triangles = self._hp(sc.tris, np.uint32)
        t.tri_edges = self._hp(sc.hinges, np.uint32)
        t.tri_edge_adj_vertex = self._hp(sc.hinge_adj, np.int32)
        t.targetIndex = self._hp(sc.soft_index, np.uint32)
        t.part_map_size = len(sc.part_map_real)
        t.partId_map_real = self._hp(sc.part_map_real, np.int32)
        t.real_map_partId = self._hp(sc.real_map_part, np.int32)
        t.neighborStart = self._hp(sc.nbr_start, np.uint32)
        t.neighborList = self._hp(sc.nbr_list, np.uint32)
        cap = pair_capacity if pair_capacity is not None else max(len(sc.pairs), 1)
        t.max_pairs = cap
        self.pair_capacity = cap
        t.max_ground = max(len(sc.ground_pairs), len(sc.surf_verts))
        t.max_fric_pairs = max(len(sc.fric_pairs), cap)
        t.max_fric_ground = max(len(sc.fric_gd_pairs), len(sc.surf_verts))
        t.max_rhs = max_rhs
        h = C.c_void_p()
        N.check(L.sgipc_create(C.byref(t), dev, C.byref(h)))
        self.ctx = h
        self._host = None
        self.tet = DeviceTetraData(sc)
        self.params = dict(sc.params)
        self.n = sc.nv
        self.moveDir = torch.zeros(3 * sc.nv, dtype=torch.float64, device=_dev())

    def _hp(self, a, dt):
        a = np.ascontiguousarray(a, dt)
        self._host.append(a)
        return None if a.size == 0 else a.ctypes.data_as(C.c_void_p)

    def close(self):
        if getattr(self, "ctx", None):
            N.lib().sgipc_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- assembly -------------------------------------------------------------------
    def _params(self):
        key = tuple(sorted(self.params.items()))
        if getattr(self, "_prm_key", None) != key:
            self._prm_key, self._prm_cached = key, params_struct(self.params)
        return self._prm_cached

    def computeGradientAndHessian(self, tet: Optional[DeviceTetraData] = None):
        tet = tet or self.tet
        self._fem, self._con, self._prm = tet.fem_struct_cached(), tet.contact_struct_cached(), self._params()
        N.check(N.lib().sgipc_assemble(self.ctx, C.byref(self._fem), C.byref(self._con), C.byref(self._prm),
                                       _stream()), self.ctx)

    def calBarrierGradientAndHessian(self, grad: torch.Tensor, tet: Optional[DeviceTetraData] = None):
        tet = tet or self.tet
        f, k, p = tet.fem_struct(), tet.contact_struct(), params_struct(self.params)
        N.check(N.lib().sgipc_barrier_grad_hess(self.ctx, C.byref(f), C.byref(k), C.byref(p), _p(grad), _stream()),
                self.ctx)

    def calFrictionGradientAndHessian(self, grad: torch.Tensor, tet: Optional[DeviceTetraData] = None):
        tet = tet or self.tet
        f, k, p = tet.fem_struct(), tet.contact_struct(), params_struct(self.params)
        N.check(N.lib().sgipc_friction_grad_hess(self.ctx, C.byref(f), C.byref(k), C.byref(p), _p(grad), _stream()),
                self.ctx)

    def calculate_fem_gradient_hessian(self, grad: torch.Tensor, tet: Optional[DeviceTetraData] = None):
        tet = tet or self.tet
        f, p = tet.fem_struct(), params_struct(self.params)
        N.check(N.lib().sgipc_fem_grad_hess(self.ctx, C.byref(f), C.byref(p), _p(grad), _stream()), self.ctx)

    def computeEnergy(self, tet: Optional[DeviceTetraData] = None, terms: bool = False):
        """GIPC::computeEnergy (GIPC.cu:10520): the line-search objective at tet's vertexes.
        With terms=True also the nine parts (kinetic, tets, triangles, hinges, soft, barrier,
        ground, friction, ground friction) as a numpy array."""
        tet = tet or self.tet
        f, k, p = tet.fem_struct_cached(), tet.contact_struct_cached(), self._params()
        e = C.c_double(0.0)
        parts = np.zeros(9)
        N.check(N.lib().sgipc_compute_energy(self.ctx, C.byref(f), C.byref(k), C.byref(p), C.byref(e),
                                             parts.ctypes.data_as(C.c_void_p), _stream()), self.ctx)
        return (e.value, parts) if terms else e.value

    def self_largestFeasibleStepSize(self, slackness: float, move_dir: torch.Tensor, pairs: torch.Tensor,
                                     x: Optional[torch.Tensor] = None, toi: Optional[torch.Tensor] = None):
        """GIPC::self_largestFeasibleStepSize (GIPC.cu:8880): the step along -move_dir that keeps
        every CCD candidate (int32 [n, 4] on the device: x < 0 point -x-1 vs triangle, else edge
        vs edge) apart; toi (optional, float64 [n]) receives each candidate's time of impact."""
        x = self.tet.vertexes if x is None else x
        pairs = pairs.contiguous()
        a = C.c_double(0.0)
        N.check(N.lib().sgipc_self_step_size(self.ctx, _p(x), _p(move_dir), _p(pairs), pairs.shape[0], slackness,
                                             C.byref(a), _p(toi) if toi is not None else None, _stream()),
                self.ctx)
        return a.value

    def ground_largestFeasibleStepSize(self, slackness: float, move_dir: torch.Tensor, verts: torch.Tensor,
                                       x: Optional[torch.Tensor] = None):
        """GIPC::ground_largestFeasibleStepSize (GIPC.cu:8986) for the vertices verts (uint32 /
        int32 on the device) against the plane y = ground_offset."""
        x = self.tet.vertexes if x is None else x
        verts = verts.contiguous()
        a = C.c_double(0.0)
        N.check(N.lib().sgipc_ground_step_size(self.ctx, _p(x), _p(move_dir), _p(verts), verts.shape[0],
                                               self.params.get("ground_offset", 0.0), slackness, C.byref(a),
                                               _stream()), self.ctx)
        return a.value

    def cfl_largestSpeed(self, move_dir: torch.Tensor, verts: torch.Tensor):
        """GIPC::cfl_largestSpeed (GIPC.cu:8916): the largest |move_dir| over the vertices."""
        verts = verts.contiguous()
        v = C.c_double(0.0)
        N.check(N.lib().sgipc_cfl_largest_speed(self.ctx, _p(move_dir), _p(verts), verts.shape[0], C.byref(v),
                                                _stream()), self.ctx)
        return v.value

    def step_forward(self, alpha: float, x_base: torch.Tensor, move_dir: Optional[torch.Tensor] = None,
                     tet: Optional[DeviceTetraData] = None, move_boundary: bool = False):
        """GIPC::step_forward (GIPC.cu:9637): tet.vertexes = x_base - alpha move_dir (default
        ``self.moveDir``) for the free vertices, in place (the cached structs stay valid)."""
        tet = tet or self.tet
        d = self.moveDir if move_dir is None else move_dir
        N.check(N.lib().sgipc_step_forward(self.ctx, _p(tet.vertexes), _p(x_base), _p(d), _p(tet.BoundaryType),
                                           alpha, int(move_boundary), _stream()), self.ctx)

    def rhs(self) -> torch.Tensor:
        b = torch.empty(3 * self.n, dtype=torch.float64, device=_dev())
        N.check(N.lib().sgipc_get_rhs(self.ctx, _p(b), _stream()), self.ctx)
        return b

    def export_bcoo(self):
        cnt = C.c_int32()
        N.check(N.lib().sgipc_export_bcoo(self.ctx, 0, None, None, None, C.byref(cnt)), self.ctx)
        n = cnt.value
        rows, cols = np.zeros(n, np.int32), np.zeros(n, np.int32)
        vals = np.zeros((n, 3, 3))
        N.check(N.lib().sgipc_export_bcoo(self.ctx, n, rows.ctypes.data_as(C.c_void_p),
                                          cols.ctypes.data_as(C.c_void_p), vals.ctypes.data_as(C.c_void_p),
                                          C.byref(cnt)), self.ctx)
        return rows, cols, vals

    def launch_count(self) -> int:
        n = C.c_int64()
        N.check(N.lib().sgipc_launch_count(self.ctx, C.byref(n)), self.ctx)
        return int(n.value)

    def time_kernel(self, name: str, reps: int = 20):
        """(avg ms, algorithmic bytes per launch) of one hot kernel, CUDA events on the
        current stream."""
        ms, by = C.c_float(), C.c_double()
        N.check(N.lib().sgipc_time_kernel(self.ctx, name.encode(), reps, _stream(), C.byref(ms), C.byref(by)),
                self.ctx)
        return float(ms.value), float(by.value)

    PHASES = {1: "init", 2: "mas", 3: "mas_coarse", 4: "prolong", 5: "spmv", 6: "update", 7: "acc64",
              8: "res64", 9: "restrict64", 10: "prolong64", 11: "fused_spmv", 12: "fused_update"}

    def profile_pcg(self, name: str = "pcg32", max_epochs: int = 1024):
        """Barrier stamps of one persistent PCG solve (``sgipc_profile_pcg``): (stamps, phases)
        with stamps an int64 array [grid, epochs, 2] of device-clock nanoseconds, arrival at and
        departure from every grid barrier per CTA (epoch 0: kernel start, end of its
        shared-memory loads), and phases[e] the name of the phase that ends at barrier e."""
        nsm = torch.cuda.get_device_properties(_dev()).multi_processor_count
        cap = 2 * nsm
        buf = np.zeros(cap * max_epochs * 2 + max_epochs, np.uint64)
        grid, ep = C.c_int32(), C.c_int32()
        N.check(N.lib().sgipc_profile_pcg(self.ctx, name.encode(), max_epochs, buf.ctypes.data_as(C.c_void_p),
                                          C.byref(grid), C.byref(ep), _stream()), self.ctx)
        st = buf[:cap * max_epochs * 2].reshape(cap, max_epochs, 2)[:grid.value, :ep.value].astype(np.int64)
        tags = buf[cap * max_epochs * 2:][:ep.value]
        return st, ["start"] + [self.PHASES.get(int(t), "?") for t in tags[1:]]

    # ---- contact pairs of an iterate and the frame's friction sets --------------------------
    def _surface(self):
        if getattr(self, "_surf", None) is None:
            sc = self.scene
            self._surf_arrays = (_t(np.asarray(sc.surf_verts, np.int64).astype(np.int32), torch.int32),
                                 _t(np.asarray(sc.surf_tris, np.int64).astype(np.int32).reshape(-1, 3), torch.int32),
                                 _t(np.asarray(sc.surf_edges, np.int64).astype(np.int32).reshape(-1, 2), torch.int32))
            sv, sf, se = self._surf_arrays
            self._surf = N.SgipcSurface(_p(sv), sv.shape[0], _p(sf), sf.shape[0], _p(se), se.shape[0])
        return self._surf

    def buildCP(self, tet: Optional[DeviceTetraData] = None, body: Optional[torch.Tensor] = None,
                capacity: Optional[int] = None, update: bool = True, dHat: Optional[float] = None):
        """GIPC::buildCP (GIPC.cu:9065): the contact pairs of tet.vertexes on the GPU
        (``sgipc_build_cp``).  body: int32 per vertex (default -1 everywhere: every body also
        collides with itself).  Returns a dict of device tensors (pairs, ccd_pairs, mat_index,
        ground_pairs) and the host counts cp_num (5) and gp_num; with update=True the pairs and
        ground pairs also replace tet's (the Newton system's contact inputs).  dHat (squared
        distance, default the scene's) widens the search, e.g. for CCD candidates of a step."""
        tet = tet or self.tet
        surf = self._surface()
        cap = capacity or self.pair_capacity
        dev = _dev()
        if body is None:
            body = torch.full((self.scene.nv,), -1, dtype=torch.int32, device=dev)
        out = {"pairs": torch.empty((cap, 4), dtype=torch.int32, device=dev),
               "ccd_pairs": torch.empty((cap, 4), dtype=torch.int32, device=dev),
               "mat_index": torch.empty(cap, dtype=torch.int32, device=dev),
               "cp_num_dev": torch.zeros(5, dtype=torch.int32, device=dev),
               "ground_pairs": torch.empty(max(1, surf.surf_vert_num), dtype=torch.int32, device=dev),
               "gp_num_dev": torch.zeros(1, dtype=torch.int32, device=dev)}
        cp = (C.c_uint32 * 5)()
        gp = C.c_uint32()
        N.check(N.lib().sgipc_build_cp(self.ctx, _p(tet.vertexes), _p(tet.rest_vertexes), C.byref(surf), _p(body),
                                       _p(tet.BoundaryType), float(self.params["dHat"] if dHat is None else dHat),
                                       float(self.params.get("ground_offset", 0.0)), cap, _p(out["pairs"]),
                                       _p(out["ccd_pairs"]), _p(out["mat_index"]), _p(out["cp_num_dev"]),
                                       out["ground_pairs"].shape[0], _p(out["ground_pairs"]), _p(out["gp_num_dev"]),
                                       cp, C.byref(gp), _stream()), self.ctx)
        n, ng = int(cp[0]), int(gp.value)
        out.update(pairs=out["pairs"][:n], ccd_pairs=out["ccd_pairs"][:n], mat_index=out["mat_index"][:n],
                   ground_pairs=out["ground_pairs"][:ng], cp_num=list(cp), gp_num=ng)
        if update:
            tet.pairs = out["pairs"]
            tet.ground_pairs = out["ground_pairs"]
        return out

    def buildFrictionSets(self, tet: Optional[DeviceTetraData] = None, x: Optional[torch.Tensor] = None):
        """GIPC::buildFrictionSets (GIPC.cu:8660-8696): the lagged friction arrays of tet's pairs
        and ground pairs at the frame's positions x (default tet.o_vertexes), on the GPU
        (``sgipc_friction_setup``); they replace tet's friction inputs.  Returns cp_num_last."""
        tet = tet or self.tet
        x = tet.o_vertexes if x is None else x
        n, ng = tet.pairs.shape[0], tet.ground_pairs.shape[0]
        dev = _dev()
        fp = torch.empty((max(n, 1), 4), dtype=torch.int32, device=dev)
        fl = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
        fc = torch.empty((max(n, 1), 2), dtype=torch.float64, device=dev)
        fb = torch.empty((max(n, 1), 6), dtype=torch.float64, device=dev)
        gpp = torch.empty(max(ng, 1), dtype=torch.int32, device=dev)
        gl = torch.empty(max(ng, 1), dtype=torch.float64, device=dev)
        cpd = torch.zeros(5, dtype=torch.int32, device=dev)
        cp = (C.c_uint32 * 5)()
        N.check(N.lib().sgipc_friction_setup(self.ctx, _p(x), _p(tet.pairs), n, _p(tet.ground_pairs), ng,
                                             float(self.params["dHat"]), float(self.params["kappa"]),
                                             float(self.params.get("ground_offset", 0.0)), _p(fp), _p(fl), _p(fc),
                                             _p(fb), _p(cpd), _p(gpp), _p(gl), cp, _stream()), self.ctx)
        m = int(cp[0])
        tet.fric_pairs, tet.fric_lambda, tet.fric_coord, tet.fric_basis = fp[:m], fl[:m], fc[:m], fb[:m]
        tet.fric_gd_pairs, tet.fric_gd_lambda = gpp[:ng], gl[:ng]
        return list(cp)

    # ---- barrier stiffness ------------------------------------------------------------
    def initKappa(self, min_kappa_coef: float = 1e11, tet: Optional[DeviceTetraData] = None) -> float:
        """GIPC::initKappa (GIPC.cu:9887-9929, with suggestKappa and upperBoundKappa): the
        barrier stiffness balancing the contact gradient against the kinetic, elastic and
        soft-constraint one at the current positions (``sgipc_init_kappa``); it becomes
        ``params["kappa"]`` and is returned.  Unchanged without contact pairs."""
        tet = tet or self.tet
        f, k, p = tet.fem_struct_cached(), tet.contact_struct_cached(), self._params()
        kap = C.c_double(float(self.params["kappa"]))
        N.check(N.lib().sgipc_init_kappa(self.ctx, C.byref(f), C.byref(k), C.byref(p),
                                         float(self.params.get("meanMass", 0.0)), float(self.params["bboxDiag2"]),
                                         float(min_kappa_coef), C.byref(kap), _stream()), self.ctx)
        self.params["kappa"] = kap.value
        return kap.value

    def closeRecord(self, tet: Optional[DeviceTetraData] = None):
        """computeCloseGroundVal + computeSelfCloseVal (GIPC.cu:8776, 9219) with the
        reference's dTol = 1e-18 bbox^2: (ground vertices, pairs) recorded."""
        tet = tet or self.tet
        k = tet.contact_struct_cached()
        cnt = (C.c_int32 * 2)()
        N.check(N.lib().sgipc_close_record(self.ctx, _p(tet.vertexes), C.byref(k),
                                           1e-18 * float(self.params["bboxDiag2"]),
                                           float(self.params.get("ground_offset", 0.0)), cnt, _stream()), self.ctx)
        return int(cnt[0]), int(cnt[1])

    def postLineSearch(self, min_kappa_coef: float = 1e11, tet: Optional[DeviceTetraData] = None) -> float:
        """GIPC::postLineSearch (GIPC.cu:10777-10806) after a line search to tet.vertexes: with
        kappa 0, initKappa; otherwise kappa doubles (within its upper bound) when a recorded
        close ground vertex or pair came closer, and the close sets are recorded anew."""
        tet = tet or self.tet
        if float(self.params["kappa"]) == 0.0:
            return self.initKappa(min_kappa_coef, tet)
        changed = C.c_int32()
        N.check(N.lib().sgipc_close_check(self.ctx, _p(tet.vertexes), float(self.params.get("ground_offset", 0.0)),
                                          C.byref(changed), _stream()), self.ctx)
        if changed.value:
            from .scenes import suggest_kappa
            kmax = 100.0 * suggest_kappa(float(self.params["bboxDiag2"]), float(self.params["dHat"]),
                                         float(self.params.get("meanMass", 0.0)), min_kappa_coef)
            self.params["kappa"] = min(2.0 * float(self.params["kappa"]), kmax)
        self.closeRecord(tet)
        return float(self.params["kappa"])

    def contactPartition(self, abd_first: int, capacity: Optional[int] = None,
                         tet: Optional[DeviceTetraData] = None):
        """GIPC::partitionContactHessian (GIPC.cu:9932-10108) for a scene whose vertices
        [abd_first, nv) are affine-body points (Dirichlet in BoundaryType): the contact blocks
        that touch them, ABD-ABD as (point, point) and ABD-FEM as (point, FEM vertex), and the
        contact gradient at the points (``sgipc_contact_partition``).  Returns a dict of device
        tensors ``abd_blocks`` / ``fem_blocks`` = (rows, cols, vals (k, 3, 3)) and
        ``point_grad`` (points, 3), the inputs of ``ABDSystem.setup_abd_system_gradient_hessian``."""
        tet = tet or self.tet
        dev = _dev()
        npt = self.n - abd_first
        cap = capacity if capacity is not None else max(1, 10 * (tet.pairs.shape[0] + tet.fric_pairs.shape[0]) +
                                                            tet.ground_pairs.shape[0])
        ar = torch.empty(cap, dtype=torch.int32, device=dev)
        ac = torch.empty(cap, dtype=torch.int32, device=dev)
        av = torch.empty((cap, 3, 3), dtype=torch.float64, device=dev)
        fr = torch.empty(cap, dtype=torch.int32, device=dev)
        fc = torch.empty(cap, dtype=torch.int32, device=dev)
        fv = torch.empty((cap, 3, 3), dtype=torch.float64, device=dev)
        pg = torch.zeros((max(npt, 1), 3), dtype=torch.float64, device=dev)
        na, nf = C.c_int32(), C.c_int32()
        f, k, p = tet.fem_struct_cached(), tet.contact_struct_cached(), self._params()
        N.check(N.lib().sgipc_contact_partition(self.ctx, C.byref(f), C.byref(k), C.byref(p), abd_first, cap,
                                                _p(ar), _p(ac), _p(av), C.byref(na), _p(fr), _p(fc), _p(fv),
                                                C.byref(nf), _p(pg), _stream()), self.ctx)
        a, b = na.value, nf.value
        return {"abd_blocks": (ar[:a], ac[:a], av[:a]), "fem_blocks": (fr[:b], fc[:b], fv[:b]),
                "point_grad": pg[:npt]}

    def spmv(self, x: torch.Tensor) -> torch.Tensor:
        y = torch.empty_like(x)
        N.check(N.lib().sgipc_spmv(self.ctx, _p(x), _p(y), _stream()), self.ctx)
        return y

    # ---- solve ----------------------------------------------------------------------
    def calculateMovingDirection(self, config: Optional[PCGSolverConfig] = None,
                                 tet: Optional[DeviceTetraData] = None):
        """MAS build + PCG; fills ``self.moveDir`` (dx of A dx = b) and returns the stats."""
        config = config or PCGSolverConfig()
        tet = tet or self.tet
        con = tet.contact_struct_cached()
        st = N.SgipcSolveStats()
        prec = N.PRECISION[config.precision]
        max_iter = int(config.max_iter_ratio * 3 * self.n)
        s = N.lib().sgipc_solve(self.ctx, C.byref(con), prec, config.criterion, config.global_tol_rate, max_iter,
                                _p(self.moveDir), C.byref(st), _stream())
        N.check(s, self.ctx, allow=(N.OK, N.NOT_CONVERGED))
        return st


class HostNewtonState:
    """Pinned host copies of the per-Newton inputs (iterate x and the contact arrays),
    for callers that keep their state on the host (``step_from_host``).

    The arrays are packed into one pinned buffer (each at a 256-byte boundary).  The first
    ``step_from_host`` on a GIPC rebinds that GIPC's device arrays to views of one device
    buffer of the same layout, so that every later step moves all inputs with a single
    host-to-device copy instead of one copy per array."""

    NAMES = ("vertexes", "pairs", "ground_pairs", "fric_pairs", "fric_lambda", "fric_coord", "fric_basis",
             "fric_gd_pairs", "fric_gd_lambda")

    def __init__(self, sc):
        f64, i32 = torch.float64, torch.int32
        src = {"vertexes": (sc.vertexes, f64), "pairs": (sc.pairs.reshape(-1, 4), i32),
               "ground_pairs": (sc.ground_pairs, i32), "fric_pairs": (sc.fric_pairs.reshape(-1, 4), i32),
               "fric_lambda": (sc.fric_lambda, f64), "fric_coord": (sc.fric_coord.reshape(-1, 2), f64),
               "fric_basis": (sc.fric_basis.reshape(-1, 6), f64), "fric_gd_pairs": (sc.fric_gd_pairs, i32),
               "fric_gd_lambda": (sc.fric_gd_lambda, f64)}
        self._layout, off = [], 0
        for n in self.NAMES:
            a, dt = src[n]
            t = torch.as_tensor(np.ascontiguousarray(a), dtype=dt)
            self._layout.append((n, off, dt, tuple(t.shape)))
            off += (t.numel() * t.element_size() + 255) // 256 * 256
        self._bytes = max(off, 256)
        self._host = torch.zeros(self._bytes, dtype=torch.uint8).pin_memory()
        for n, o, dt, shape in self._layout:
            v = self._views(self._host, n)
            v.copy_(torch.as_tensor(np.ascontiguousarray(src[n][0]), dtype=dt).reshape(shape))
            setattr(self, n, v)
        self.move_dir = torch.empty(3 * sc.nv, dtype=f64).pin_memory()
        self._dev = None
        self._bound = None

    def _views(self, buf, name):
        for n, o, dt, shape in self._layout:
            if n == name:
                nb = int(np.prod(shape)) * torch.tensor([], dtype=dt).element_size()
                return buf[o:o + nb].view(dt).view(shape)
        raise KeyError(name)

    def bind(self, tet: "DeviceTetraData"):
        """Make tet's input arrays views of one device buffer laid out like the host one."""
        if self._bound is tet:
            return
        self._dev = torch.empty(self._bytes, dtype=torch.uint8, device=_dev())
        self._dev.copy_(self._host)
        for n, _, _, _ in self._layout:
            setattr(tet, n, self._views(self._dev, n))
        self._bound = tet

    def h2d_bytes(self) -> int:
        return int(sum(getattr(self, n).numel() * getattr(self, n).element_size() for n in self.NAMES))

    def d2h_bytes(self) -> int:
        return int(self.move_dir.numel() * self.move_dir.element_size())


def step_from_host(g: "GIPC", host: HostNewtonState, config: Optional[PCGSolverConfig] = None):
    """One Newton system from host inputs: one H2D copy, assembly, MAS + PCG, D2H of dx."""
    tet = g.tet
    host.bind(tet)
    host._dev.copy_(host._host, non_blocking=True)
    g.computeGradientAndHessian(tet)
    st = g.calculateMovingDirection(config, tet)
    host.move_dir.copy_(g.moveDir, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    return st


class MASPreconditioner:
    """``MASPreconditioner`` over a :class:`GIPC` context's assembled matrix."""

    def __init__(self, gipc: GIPC):
        self.g = gipc

    def setPreconditioner(self, precision: str = "fp64", tet: Optional[DeviceTetraData] = None):
        con = (tet or self.g.tet).contact_struct()
        N.check(N.lib().sgipc_mas_build(self.g.ctx, C.byref(con), N.PRECISION[precision], _stream()), self.g.ctx)

    def preconditioning(self, R: torch.Tensor, Z: Optional[torch.Tensor] = None) -> torch.Tensor:
        Z = torch.empty_like(R) if Z is None else Z
        N.check(N.lib().sgipc_mas_apply(self.g.ctx, _p(R), _p(Z), _stream()), self.g.ctx)
        return Z

    def info(self):
        ln, tot = C.c_int32(), C.c_int32()
        counts = (C.c_int32 * 8)()
        N.check(N.lib().sgipc_mas_info(self.g.ctx, C.byref(ln), counts, C.byref(tot)), self.g.ctx)
        return ln.value, np.array(counts[:ln.value]), tot.value

    def domains(self):
        """Dense 48x48 domain inverses, (total_clusters/16, 48, 48) float64."""
        total = self.info()[2]
        d = np.zeros((total // 16, 48, 48))
        N.check(N.lib().sgipc_mas_export_domains(self.g.ctx, d.ctypes.data_as(C.c_void_p)), self.g.ctx)
        return d

    def tables(self):
        L = self.info()[0]
        t = np.zeros(self.g.n * L, np.int32)
        N.check(N.lib().sgipc_mas_export_tables(self.g.ctx, t.ctypes.data_as(C.c_void_p)), self.g.ctx)
        return t.reshape(self.g.n, L)


class PCGSolver:
    """``PCGSolver::solve(x, b)`` on a :class:`GIPC` context (MAS must be set)."""

    def __init__(self, gipc: GIPC, config: Optional[PCGSolverConfig] = None):
        self.g = gipc
        self.config = config or PCGSolverConfig()

    def solve(self, b: torch.Tensor, x: Optional[torch.Tensor] = None):
        x = torch.empty_like(b) if x is None else x
        st = N.SgipcSolveStats()
        cfg = self.config
        max_iter = int(cfg.max_iter_ratio * 3 * self.g.n)
        s = N.lib().sgipc_pcg_solve(self.g.ctx, N.PRECISION[cfg.precision], cfg.criterion, cfg.global_tol_rate,
                                    max_iter, _p(b), _p(x), C.byref(st), _stream())
        N.check(s, self.g.ctx, allow=(N.OK, N.NOT_CONVERGED))
        return x, st

    def solve_batched(self, B: torch.Tensor, X: Optional[torch.Tensor] = None):
        """B: (nrhs, 3n) float64 CUDA tensor; returns X and the per-rhs stats."""
        nrhs = B.shape[0]
        X = torch.empty_like(B) if X is None else X
        st = (N.SgipcSolveStats * nrhs)()
        cfg = self.config
        max_iter = int(cfg.max_iter_ratio * 3 * self.g.n)
        s = N.lib().sgipc_pcg_solve_batched(self.g.ctx, N.PRECISION[cfg.precision], cfg.criterion,
                                            cfg.global_tol_rate, max_iter, nrhs, _p(B), _p(X), st, _stream())
        N.check(s, self.g.ctx, allow=(N.OK, N.NOT_CONVERGED))
        return X, list(st)
