"""ctypes declarations of the C ABI in ``include/sgipc.h`` (``libsgipc.so``).

Loading fails loudly: there is no CPU or Python fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsgipc.so")

OK, CUDA_ERROR, NOT_CONVERGED, BREAKDOWN, BAD_INPUT, CAPACITY, NOT_READY = range(7)
FP64, MIXED, REF = 0, 1, 2
CRIT_RZ, CRIT_TRUE = 0, 1
PRECISION = {"fp64": FP64, "mixed": MIXED, "ref": REF}

_vp = C.c_void_p
_i32 = C.c_int32


class SgipcTopology(C.Structure):
    _fields_ = [("vertex_num", _i32), ("tet_num", _i32), ("tri_num", _i32), ("tri_edge_num", _i32),
                ("soft_num", _i32), ("tetrahedras", _vp), ("triangles", _vp), ("tri_edges", _vp),
                ("tri_edge_adj_vertex", _vp), ("targetIndex", _vp), ("part_map_size", _i32),
                ("partId_map_real", _vp), ("real_map_partId", _vp), ("neighborStart", _vp),
                ("neighborList", _vp), ("max_pairs", _i32), ("max_ground", _i32), ("max_fric_pairs", _i32),
                ("max_fric_ground", _i32), ("max_rhs", _i32)]


class SgipcFemData(C.Structure):
    _fields_ = [(n, _vp) for n in ("vertexes", "o_vertexes", "rest_vertexes", "xTilta", "masses", "BoundaryType",
                                   "DmInverses", "volum", "lengthRate", "volumeRate", "triDmInverses", "area",
                                   "quad_bending_Q", "targetVert")]


class SgipcContacts(C.Structure):
    _fields_ = [("pairs", _vp), ("pair_num", _i32), ("ground_pairs", _vp), ("ground_num", _i32),
                ("fric_pairs", _vp), ("fric_lambda", _vp), ("fric_coord", _vp), ("fric_basis", _vp),
                ("fric_num", _i32), ("fric_gd_pairs", _vp), ("fric_gd_lambda", _vp), ("fric_gd_num", _i32)]


class SgipcParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("dt", "dHat", "kappa", "fDhat", "frictionRate", "gd_frictionRate",
                                          "ground_offset", "stretchStiff", "shearStiff", "strainRate",
                                          "bendStiff", "motionRate", "softRate")]


class SgipcSolveStats(C.Structure):
    _fields_ = [("iterations", _i32), ("refinements", _i32), ("rz0", C.c_double), ("rz", C.c_double),
                ("rel_residual", C.c_double), ("status", _i32)]


class SgipcSurface(C.Structure):
    _fields_ = [("surf_verts", _vp), ("surf_vert_num", _i32), ("faces", _vp), ("face_num", _i32), ("edges", _vp),
                ("edge_num", _i32)]


class SgipcAbdTopology(C.Structure):
    _fields_ = [("body_num", _i32), ("point_num", _i32), ("point_body", _vp), ("x_bar", _vp),
                ("dyadic_mass", _vp), ("volume", _vp), ("boundary_type", _vp), ("max_abd_blocks", _i32),
                ("max_fem_blocks", _i32)]


# every function the header declares, with its argument types
SIGNATURES = {
    "sgipc_create": ([C.POINTER(SgipcTopology), C.c_int, C.POINTER(_vp)], _i32),
    "sgipc_destroy": ([_vp], _i32),
    "sgipc_status_string": ([_i32], C.c_char_p),
    "sgipc_last_error": ([_vp], C.c_char_p),
    "sgipc_assemble": ([_vp, C.POINTER(SgipcFemData), C.POINTER(SgipcContacts), C.POINTER(SgipcParams), _vp], _i32),
    "sgipc_barrier_grad_hess": ([_vp, C.POINTER(SgipcFemData), C.POINTER(SgipcContacts), C.POINTER(SgipcParams),
                                 _vp, _vp], _i32),
    "sgipc_friction_grad_hess": ([_vp, C.POINTER(SgipcFemData), C.POINTER(SgipcContacts), C.POINTER(SgipcParams),
                                  _vp, _vp], _i32),
    "sgipc_fem_grad_hess": ([_vp, C.POINTER(SgipcFemData), C.POINTER(SgipcParams), _vp, _vp], _i32),
    "sgipc_export_bcoo": ([_vp, _i32, _vp, _vp, _vp, C.POINTER(_i32)], _i32),
    "sgipc_get_rhs": ([_vp, _vp, _vp], _i32),
    "sgipc_compute_energy": ([_vp, C.POINTER(SgipcFemData), C.POINTER(SgipcContacts), C.POINTER(SgipcParams),
                              C.POINTER(C.c_double), _vp, _vp], _i32),
    "sgipc_self_step_size": ([_vp, _vp, _vp, _vp, _i32, C.c_double, C.POINTER(C.c_double), _vp, _vp], _i32),
    "sgipc_ground_step_size": ([_vp, _vp, _vp, _vp, _i32, C.c_double, C.c_double, C.POINTER(C.c_double), _vp],
                               _i32),
    "sgipc_cfl_largest_speed": ([_vp, _vp, _vp, _i32, C.POINTER(C.c_double), _vp], _i32),
    "sgipc_step_forward": ([_vp, _vp, _vp, _vp, _vp, C.c_double, _i32, _vp], _i32),
    "sgipc_spmv": ([_vp, _vp, _vp, _vp], _i32),
    "sgipc_mas_build": ([_vp, C.POINTER(SgipcContacts), _i32, _vp], _i32),
    "sgipc_mas_apply": ([_vp, _vp, _vp, _vp], _i32),
    "sgipc_mas_apply_noalloc": ([_vp, _vp, _vp, _vp], _i32),
    "sgipc_mas_info": ([_vp, C.POINTER(_i32), _vp, C.POINTER(_i32)], _i32),
    "sgipc_mas_export_tables": ([_vp, _vp], _i32),
    "sgipc_pcg_solve": ([_vp, _i32, _i32, C.c_double, _i32, _vp, _vp, C.POINTER(SgipcSolveStats), _vp], _i32),
    "sgipc_pcg_solve_batched": ([_vp, _i32, _i32, C.c_double, _i32, _i32, _vp, _vp, C.POINTER(SgipcSolveStats),
                                 _vp], _i32),
    "sgipc_solve": ([_vp, C.POINTER(SgipcContacts), _i32, _i32, C.c_double, _i32, _vp, C.POINTER(SgipcSolveStats),
                     _vp], _i32),
    "sgipc_adjoint_param_grads": ([_vp, C.POINTER(SgipcFemData), C.POINTER(SgipcParams), C.c_double, _i32, _vp,
                                   _vp, _vp, _vp], _i32),
    "sgipc_mas_export_domains": ([_vp, _vp], _i32),
    "sgipc_mas_restrict": ([_vp, _vp, _vp], _i32),
    "sgipc_abd_create": ([C.POINTER(SgipcAbdTopology), C.c_int, C.POINTER(_vp)], _i32),
    "sgipc_abd_destroy": ([_vp], _i32),
    "sgipc_abd_last_error": ([_vp], C.c_char_p),
    "sgipc_abd_grad_hess": ([_vp, _vp, _vp, C.c_double, C.c_double, _vp, _i32, _vp, _vp, _vp, _i32, _vp, _vp, _vp,
                             _vp, _vp, _vp], _i32),
    "sgipc_abd_export_bcoo": ([_vp, _i32, _vp, _vp, _vp, C.POINTER(_i32)], _i32),
    "sgipc_abd_precond_build": ([_vp, _vp], _i32),
    "sgipc_abd_precond_apply": ([_vp, _vp, _vp, _vp], _i32),
    "sgipc_global_pcg_solve": ([_vp, _vp, _i32, C.c_double, _i32, _vp, _vp, _vp, C.POINTER(SgipcSolveStats), _vp],
                               _i32),
    "sgipc_launch_count": ([_vp, C.POINTER(C.c_int64)], _i32),
    "sgipc_time_kernel": ([_vp, C.c_char_p, _i32, _vp, C.POINTER(C.c_float), C.POINTER(C.c_double)], _i32),
    "sgipc_set_wait_limit": ([_vp, C.c_int64], _i32),
    "sgipc_build_cp": ([_vp, _vp, _vp, C.POINTER(SgipcSurface), _vp, _vp, C.c_double, C.c_double, _i32, _vp, _vp,
                        _vp, _vp, _i32, _vp, _vp, _vp, _vp, _vp], _i32),
    "sgipc_friction_setup": ([_vp, _vp, _vp, _i32, _vp, _i32, C.c_double, C.c_double, C.c_double, _vp, _vp, _vp,
                              _vp, _vp, _vp, _vp, _vp, _vp], _i32),
    "sgipc_profile_pcg": ([_vp, C.c_char_p, _i32, _vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), _vp], _i32),
    "sgipc_init_kappa": ([_vp, C.POINTER(SgipcFemData), C.POINTER(SgipcContacts), C.POINTER(SgipcParams),
                          C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double), _vp], _i32),
    "sgipc_close_record": ([_vp, _vp, C.POINTER(SgipcContacts), C.c_double, C.c_double, _vp, _vp], _i32),
    "sgipc_close_check": ([_vp, _vp, C.c_double, C.POINTER(_i32), _vp], _i32),
    "sgipc_contact_partition": ([_vp, C.POINTER(SgipcFemData), C.POINTER(SgipcContacts), C.POINTER(SgipcParams),
                                 _i32, _i32, _vp, _vp, _vp, C.POINTER(_i32), _vp, _vp, _vp, C.POINTER(_i32), _vp,
                                 _vp], _i32),
}

_LIB = None


def lib():
    """Load ``libsgipc.so``; raises if it is missing or lacks a declared symbol."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libsgipc.so not built (%s); run __graft_entry__.build()" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _LIB = L
    return _LIB


class SgipcError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        name = lib().sgipc_status_string(status).decode()
        super().__init__("sgipc status %d (%s)%s" % (status, name, (": " + msg) if msg else ""))


def check(status, ctx=None, allow=(OK,)):
    if status not in allow:
        msg = lib().sgipc_last_error(ctx).decode() if ctx else ""
        raise SgipcError(status, msg)
    return status
