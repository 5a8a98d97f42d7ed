"""ctypes binding of the CPU oracle (``liboracle.so``).

TEST INFRASTRUCTURE ONLY.  The oracle is a CPU FP64 restatement of StiffGIPC's
per-Newton-iteration linear system (see ``sgipc_oracle.cpp`` for the reference
files it follows).  It is imported by ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` — as the checker and the reported CPU baseline — and
never by the ``sgipc`` package.

Parity status: unpinned by the reference's own tests (the reference ships none and
cannot be built here); pinned instead by closed-form and finite-difference identities.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int32)
_u = C.POINTER(C.c_uint32)


def build() -> str:
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "sgipc_oracle.cpp")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return path


def lib():
    global _LIB
    if _LIB is None:
        _LIB = C.CDLL(build())
        L = _LIB
        L.or_snk_tet.argtypes = [_d, _d, C.c_double, C.c_double, C.c_double, C.c_double, _d, _d, _d]
        L.or_barrier_pair.argtypes = [_i, _d, _d, C.c_double, C.c_double, _i, _d, _d, _d]
        L.or_barrier_pair.restype = C.c_int
        L.or_friction_pair.argtypes = [_i, _d, _d, _d, _d, C.c_double, C.c_double, C.c_double, _i, _d, _d, _d]
        L.or_friction_pair.restype = C.c_int
        L.or_friction_ground.argtypes = [_d, _d, C.c_double, C.c_double, C.c_double, _d, _d, _d]
        L.or_make_pd.argtypes = [C.c_int, _d]
        L.or_set_snk_projection.argtypes = [C.c_int]
        L.or_abd_assemble.argtypes = [C.c_int, C.c_int, _i, _d, _d, _d, _i, _d, _d, C.c_double, C.c_double, _d,
                                      C.c_int, _i, _i, _d, C.c_int, _i, _i, _d, _i, _d, C.c_int, _i, _i, _d]
        L.or_abd_assemble.restype = C.c_int
        L.or_tri_bw.argtypes = [_d, _d, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, _d, _d, _d]
        L.or_pair_geom.argtypes = [_i, _d, C.c_double, _d, _d, _d, _d]
        L.or_pair_geom.restype = C.c_int
        L.or_eig.argtypes = [C.c_int, _d, _d, _d]
        L.or_assemble.argtypes = [C.c_void_p, _d, C.c_int, _i, _i, _d, _d]
        L.or_assemble.restype = C.c_int
        L.or_spmv.argtypes = [C.c_int, _i, _i, _d, C.c_int, _d, _d]
        L.or_mas_num_levels.argtypes = [C.c_int]
        L.or_mas_num_levels.restype = C.c_int
        L.or_mas_build.argtypes = [C.c_int, C.c_int, _i, _i, _u, _u, C.c_int, _i, C.c_int, _i, _i, _d]
        L.or_mas_build.restype = C.c_void_p
        L.or_mas_free.argtypes = [C.c_void_p]
        L.or_mas_info.argtypes = [C.c_void_p, _i, _i, _i, _i]
        L.or_mas_table.argtypes = [C.c_void_p, _i]
        L.or_mas_domains.argtypes = [C.c_void_p, _d]
        L.or_mas_apply.argtypes = [C.c_void_p, _d, _d, C.c_int]
        L.or_pcg.argtypes = [C.c_int, _i, _i, _d, C.c_int, C.c_void_p, C.c_int, _d, _d, C.c_double,
                             C.c_int, _d, _d]
        L.or_pcg.restype = C.c_int
        L.or_self_step.argtypes = [_d, _d, _i, C.c_int, C.c_double, _d]
        L.or_self_step.restype = C.c_double
        L.or_ground_step.argtypes = [_d, _d, _u, C.c_int, C.c_double, C.c_double]
        L.or_ground_step.restype = C.c_double
        L.or_accd.argtypes = [C.c_int, _d, _d, C.c_double]
        L.or_accd.restype = C.c_double
        L.or_cfl_speed.argtypes = [_d, _u, C.c_int]
        L.or_cfl_speed.restype = C.c_double
        L.or_num_threads.restype = C.c_int
    return _LIB


def _p(a, t=_d):
    return a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, np.float64)


def _i32(a):
    return np.ascontiguousarray(a, np.int32)


# ------------------------------------------------------------------------------------------
# element level
# ------------------------------------------------------------------------------------------

def snk_tet(X, dminv, vol, mu, lam, dt2=1.0):
    X, dminv = _f64(X).reshape(12), _f64(dminv).reshape(9)
    e = np.zeros(1)
    g = np.zeros(12)
    H = np.zeros(144)
    lib().or_snk_tet(_p(X), _p(dminv), vol, mu, lam, dt2, _p(e), _p(g), _p(H))
    return e[0], g, H.reshape(12, 12)


def barrier_pair(enc, X, R, dhat, kappa):
    enc = _i32(enc).reshape(4)
    X, R = _f64(X).reshape(-1), _f64(R).reshape(-1)
    vid = np.zeros(4, np.int32)
    e = np.zeros(1)
    g = np.zeros(12)
    H = np.zeros(144)
    nv = lib().or_barrier_pair(_p(enc, _i), _p(X), _p(R), dhat, kappa, _p(vid, _i), _p(e), _p(g), _p(H))
    return vid[:nv], e[0], g[:3 * nv], H.reshape(12, 12)[:3 * nv, :3 * nv]


def friction_pair(enc, X, X0, coord, basis, lastH, mu, eps2):
    enc = _i32(enc).reshape(4)
    X, X0 = _f64(X).reshape(-1), _f64(X0).reshape(-1)
    coord, basis = _f64(coord).reshape(2), _f64(basis).reshape(6)
    vid = np.zeros(4, np.int32)
    e = np.zeros(1)
    g = np.zeros(12)
    H = np.zeros(144)
    nv = lib().or_friction_pair(_p(enc, _i), _p(X), _p(X0), _p(coord), _p(basis), lastH, mu, eps2,
                                _p(vid, _i), _p(e), _p(g), _p(H))
    return vid[:nv], e[0], g[:3 * nv], H.reshape(12, 12)[:3 * nv, :3 * nv]


def pair_geom(enc, X, dhat):
    """(nv, f, grad f, c, grad c) of a barrier pair; X holds the scene's positions."""
    enc = _i32(enc).reshape(4)
    X = _f64(X).reshape(-1)
    f, c = np.zeros(1), np.zeros(1)
    gf, gc = np.zeros(12), np.zeros(12)
    nv = lib().or_pair_geom(_p(enc, _i), _p(X), dhat, _p(f), _p(gf), _p(c), _p(gc))
    return nv, f[0], gf[:3 * nv], c[0], gc[:3 * nv]


def tri_bw(X, Dinv, area, kst, ksh, srate, dt2):
    """(energy, grad (9,), H (9,9)) of one Baraff-Witkin cloth triangle."""
    X, Dinv = _f64(X).reshape(9), _f64(Dinv).reshape(4)
    e, g, H = np.zeros(1), np.zeros(9), np.zeros(81)
    lib().or_tri_bw(_p(X), _p(Dinv), area, kst, ksh, srate, dt2, _p(e), _p(g), _p(H))
    return e[0], g, H.reshape(9, 9)


def abd_assemble(bodies, q, q_tilde, kappa, dt, point_grad=None, abd_blocks=None, fem_blocks=None,
                 fem_boundary=None):
    """(body_grad (12B,), rows, cols, vals (n,3,3)): ABD body terms and contact mappings."""
    B, P = len(bodies["volume"]), len(bodies["point_body"])
    pb, xb = _i32(bodies["point_body"]), _f64(bodies["x_bar"]).reshape(-1)
    dm, vol, bt = _f64(bodies["dyadic_mass"]).reshape(-1), _f64(bodies["volume"]), _i32(bodies["boundary_type"])
    q, qt = _f64(q).reshape(-1), _f64(q_tilde).reshape(-1)
    pg = None if point_grad is None else _f64(point_grad).reshape(-1)
    ar, ac, av = (np.zeros(0, np.int32),) * 2 + (np.zeros(0),) if abd_blocks is None else \
        (_i32(abd_blocks[0]), _i32(abd_blocks[1]), _f64(abd_blocks[2]).reshape(-1))
    fr, fc, fv = (np.zeros(0, np.int32),) * 2 + (np.zeros(0),) if fem_blocks is None else \
        (_i32(fem_blocks[0]), _i32(fem_blocks[1]), _f64(fem_blocks[2]).reshape(-1))
    fb = None if fem_boundary is None else _i32(fem_boundary)
    g = np.zeros(12 * B)
    args = [B, P, _p(pb, _i), _p(xb), _p(dm), _p(vol), _p(bt, _i), _p(q), _p(qt), kappa, dt,
            None if pg is None else _p(pg), len(ar), _p(ar, _i), _p(ac, _i), _p(av), len(fr), _p(fr, _i), _p(fc, _i),
            _p(fv), None if fb is None else _p(fb, _i), _p(g)]
    n = lib().or_abd_assemble(*args, 0, None, None, None)
    rows, cols, vals = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros((n, 3, 3))
    lib().or_abd_assemble(*args, n, _p(rows, _i), _p(cols, _i), _p(vals))
    return g, rows, cols, vals


class exact_snk_hessian:
    """Context manager: assemble the stable Neo-Hookean terms with their exact (unprojected)
    Hessian, the true Jacobian of the gradient, instead of the PSD projection."""

    def __enter__(self):
        lib().or_set_snk_projection(0)
        return self

    def __exit__(self, *exc):
        lib().or_set_snk_projection(1)
        return False


def make_pd(A):
    A = _f64(A).copy()
    lib().or_make_pd(A.shape[0], _p(A))
    return A


# ------------------------------------------------------------------------------------------
# system level
# ------------------------------------------------------------------------------------------

class _OrScene(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("nv", "nt", "npairs", "nground", "nfric", "nfric_gd", "nsoft")] + [
        ("x", _d), ("x0", _d), ("rest", _d), ("xt", _d), ("mass", _d), ("btype", _i), ("tets", _i),
        ("dminv", _d), ("vol", _d), ("lr", _d), ("vr", _d), ("pairs", _i), ("gpairs", _i),
        ("fpairs", _i), ("flam", _d), ("fcoord", _d), ("fbasis", _d), ("fgpairs", _i), ("fglam", _d),
        ("soft_idx", _i), ("soft_target", _d)] + [
        (n, C.c_double) for n in ("dt", "dhat", "kappa", "fdhat", "mu", "mu_gd", "ground_offset",
                                   "motion_rate", "soft_rate")] + [
        ("nf", C.c_int), ("nh", C.c_int), ("tris", _i), ("tdminv", _d), ("tarea", _d), ("hinges", _i),
        ("hadj", _i), ("hq", _d)] + [(n, C.c_double) for n in ("stretch", "shear", "strain_rate", "bend")]


def _scene_struct(sc, x=None):
    keep = []

    def f(a):
        a = _f64(a)
        keep.append(a)
        return _p(a)

    def i(a):
        a = _i32(a)
        keep.append(a)
        return _p(a, _i)

    p = sc.params
    s = _OrScene(nv=sc.nv, nt=sc.nt, npairs=len(sc.pairs), nground=len(sc.ground_pairs),
                 nfric=len(sc.fric_pairs), nfric_gd=len(sc.fric_gd_pairs), nsoft=len(sc.soft_index),
                 x=f(sc.vertexes if x is None else x), x0=f(sc.o_vertexes), rest=f(sc.rest_vertexes),
                 xt=f(sc.xTilta), mass=f(sc.masses), btype=i(sc.boundary_type), tets=i(sc.tets),
                 dminv=f(sc.dm_inv), vol=f(sc.volum), lr=f(sc.length_rate), vr=f(sc.volume_rate),
                 pairs=i(sc.pairs.reshape(-1, 4)), gpairs=i(sc.ground_pairs), fpairs=i(sc.fric_pairs.reshape(-1, 4)),
                 flam=f(sc.fric_lambda), fcoord=f(sc.fric_coord.reshape(-1, 2)),
                 fbasis=f(sc.fric_basis.reshape(-1, 6)), fgpairs=i(sc.fric_gd_pairs),
                 fglam=f(sc.fric_gd_lambda), soft_idx=i(sc.soft_index), soft_target=f(sc.soft_target.reshape(-1, 3)),
                 dt=p["dt"], dhat=p["dHat"], kappa=p["kappa"], fdhat=p["fDhat"], mu=p["frictionRate"],
                 mu_gd=p["gd_frictionRate"], ground_offset=p["ground_offset"], motion_rate=p["motionRate"],
                 soft_rate=p["softRate"], nf=len(sc.tris), nh=len(sc.hinges), tris=i(sc.tris.reshape(-1, 3)),
                 tdminv=f(sc.tri_dm_inv.reshape(-1, 4)), tarea=f(sc.area), hinges=i(sc.hinges.reshape(-1, 2)),
                 hadj=i(sc.hinge_adj.reshape(-1, 2)), hq=f(np.transpose(sc.hinge_q, (0, 2, 1)).reshape(-1, 16)),
                 stretch=p.get("stretchStiff", 0.0), shear=p.get("shearStiff", 0.0),
                 strain_rate=p.get("strainRate", 0.0), bend=p.get("bendStiff", 0.0))
    return s, keep


def assemble(sc, x=None):
    """(b, rows, cols, vals, energy): RHS with Dirichlet rows zeroed, merged upper BCOO."""
    s, keep = _scene_struct(sc, x)
    L = lib()
    n = L.or_assemble(C.byref(s), None, 0, None, None, None, None)
    rows = np.zeros(n, np.int32)
    cols = np.zeros(n, np.int32)
    vals = np.zeros((n, 3, 3))
    b = np.zeros(3 * sc.nv)
    e = np.zeros(1)
    L.or_assemble(C.byref(s), _p(b), n, _p(rows, _i), _p(cols, _i), _p(vals), _p(e))
    return b, rows, cols, vals, e[0]


def energy(sc, x=None):
    s, keep = _scene_struct(sc, x)
    e = np.zeros(1)
    b = np.zeros(3 * sc.nv)
    lib().or_assemble(C.byref(s), _p(b), 0, None, None, None, _p(e))
    return e[0]


def self_step(x, move_dir, pairs, slackness):
    """(alpha, toi): GIPC::self_largestFeasibleStepSize (GIPC.cu:8880) over int32[4]
    candidates (x < 0: point -x-1 vs triangle, else edge vs edge) with the additive CCD of
    ACCD.cu:373-535, along -move_dir."""
    x, move_dir, pairs = _f64(x), _f64(move_dir), _i32(np.asarray(pairs).reshape(-1, 4))
    toi = np.zeros(len(pairs))
    a = lib().or_self_step(_p(x), _p(move_dir), _p(pairs, _i), len(pairs), slackness, _p(toi))
    return a, toi


def ground_step(x, move_dir, verts, offset, slackness):
    """GIPC::ground_largestFeasibleStepSize (GIPC.cu:8986), plane y = offset."""
    x, move_dir = _f64(x), _f64(move_dir)
    verts = np.ascontiguousarray(verts, dtype=np.uint32)
    return lib().or_ground_step(_p(x), _p(move_dir), verts.ctypes.data_as(_u), len(verts), offset, slackness)


def accd(edge_edge, x, d, eta):
    """time of impact of one point-triangle (edge_edge False) or edge-edge candidate:
    x, d the four positions and displacements (4, 3), eta the separation ratio kept"""
    x, d = _f64(x).reshape(12), _f64(d).reshape(12)
    return lib().or_accd(int(bool(edge_edge)), _p(x), _p(d), eta)


def cfl_speed(move_dir, verts):
    """GIPC::cfl_largestSpeed (GIPC.cu:8916): the largest |move_dir| over verts."""
    move_dir = _f64(move_dir)
    verts = np.ascontiguousarray(verts, dtype=np.uint32)
    return lib().or_cfl_speed(_p(move_dir), verts.ctypes.data_as(_u), len(verts))


def spmv(rows, cols, vals, n, x):
    rows, cols, vals, x = _i32(rows), _i32(cols), _f64(vals), _f64(x)
    y = np.zeros(3 * n)
    lib().or_spmv(len(rows), _p(rows, _i), _p(cols, _i), _p(vals), n, _p(x), _p(y))
    return y


def dense(rows, cols, vals, n):
    A = np.zeros((3 * n, 3 * n))
    for r, c, v in zip(rows, cols, vals.reshape(-1, 3, 3)):
        A[3 * r:3 * r + 3, 3 * c:3 * c + 3] += v
        if r != c:
            A[3 * c:3 * c + 3, 3 * r:3 * r + 3] += v.T
    return A


class Mas:
    """Oracle MAS hierarchy + dense FP64 domain inverses."""

    def __init__(self, sc, rows, cols, vals, pairs=None):
        self._keep = [_i32(sc.part_map_real), _i32(sc.real_map_part),
                      np.ascontiguousarray(sc.nbr_start, np.uint32), np.ascontiguousarray(sc.nbr_list, np.uint32),
                      _i32(sc.pairs if pairs is None else pairs).reshape(-1), _i32(rows), _i32(cols), _f64(vals)]
        k = self._keep
        self.nv = sc.nv
        self.h = lib().or_mas_build(sc.nv, len(k[0]), _p(k[0], _i), _p(k[1], _i), _p(k[2], _u), _p(k[3], _u),
                                    len(k[4]) // 4, _p(k[4], _i), len(k[5]), _p(k[5], _i), _p(k[6], _i), _p(k[7]))

    def info(self):
        ln = np.zeros(1, np.int32)
        st = np.zeros(8, np.int32)
        ct = np.zeros(8, np.int32)
        tot = np.zeros(1, np.int32)
        lib().or_mas_info(self.h, _p(ln, _i), _p(st, _i), _p(ct, _i), _p(tot, _i))
        L = int(ln[0])
        return L, st[:L].copy(), ct[:L].copy(), int(tot[0])

    def table(self):
        L = self.info()[0]
        t = np.zeros(self.nv * L, np.int32)
        lib().or_mas_table(self.h, _p(t, _i))
        return t.reshape(self.nv, L)

    def domains(self):
        total = self.info()[3]
        d = np.zeros((total // 16, 48, 48))
        lib().or_mas_domains(self.h, _p(d))
        return d

    def apply(self, r, single=False):
        r = _f64(r)
        z = np.zeros_like(r)
        lib().or_mas_apply(self.h, _p(r), _p(z), 1 if single else 0)
        return z

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_mas_free(self.h)
            self.h = None


def pcg(rows, cols, vals, n, mas, b, tol=1e-4, max_iter=None, single=False):
    rows, cols, vals, b = _i32(rows), _i32(cols), _f64(vals), _f64(b)
    x = np.zeros(3 * n)
    if max_iter is None:
        max_iter = int(0.3 * 3 * n)
    rz0 = np.zeros(1)
    rz = np.zeros(1)
    it = lib().or_pcg(len(rows), _p(rows, _i), _p(cols, _i), _p(vals), n, mas.h, 1 if single else 0,
                      _p(b), _p(x), tol, max_iter, _p(rz0), _p(rz))
    return x, it, rz0[0], rz[0]


def global_pcg(A, body_num, mas, b, tol=1e-4, max_iter=None, single=False):
    """PCGSolver::pcg (StiffGIPC/linear_system/solver/pcg_solver.cu:174-267; the loop of
    or_pcg above) on the global FEM + ABD system of GlobalLinearSystem
    (linear_system/linear_system/global_linear_system.cu:8-166, created in gipc/gipc.cu:
    42-70): DOFs [12 body_num ABD | FEM], A (N x N, dense or scipy sparse) symmetric, the
    preconditioner the identity overwritten per subsystem (apply_preconditioner,
    global_linear_system.cu:152-166): ABDPreconditioner's inverse 12x12 diagonal blocks
    (abd_preconditioner.cu:15-38) on the ABD DOFs and the oracle MAS on the FEM DOFs.
    Returns x, the iteration count (or_pcg's convention), r0.z0 and the final r.z."""
    b = _f64(b)
    N = len(b)
    na = 12 * body_num
    dense = A if isinstance(A, np.ndarray) else None
    inv = []
    for k in range(body_num):
        blk = (dense[12 * k:12 * k + 12, 12 * k:12 * k + 12] if dense is not None
               else A[12 * k:12 * k + 12, 12 * k:12 * k + 12].toarray())
        inv.append(np.linalg.inv(blk))

    def prec(r):
        z = r.copy()
        for k in range(body_num):
            z[12 * k:12 * k + 12] = inv[k] @ r[12 * k:12 * k + 12]
        if N > na:
            z[na:] = mas.apply(r[na:], single)
        return z

    if max_iter is None:
        max_iter = int(0.3 * N)
    x = np.zeros(N)
    r = b.copy()
    z = prec(r)
    rz = float(r @ z)
    rz0 = rz
    p = z.copy()
    k = 1
    while k < max_iter:
        Ap = A @ p
        alpha = rz / float(p @ Ap)
        x += alpha * p
        r -= alpha * Ap
        if abs(rz) <= tol * rz0:
            break
        z = prec(r)
        rz_new = float(r @ z)
        p = z + (rz_new / rz) * p
        rz = rz_new
        k += 1
    return x, k, rz0, rz


def num_threads():
    return lib().or_num_threads()
