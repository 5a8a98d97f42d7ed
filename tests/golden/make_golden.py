"""Golden vectors from the reference's own code, for the oracle's parity tests.

Two fixtures, both numbers only (no reference source is stored):

* ``pfpx_golden.npz`` -- the barrier distance Jacobians.  The reference's barrier kernel
  (StiffGIPC/GIPC.cu:3106-4945, NEWF path) takes them from straight-line code emitted by
  MATLAB's Symbolic Math Toolbox in StiffGIPC/GIPC_PDerivative.cuh: pFpx_pp2, pFpx_pe2,
  pFpx_pt2, pFpx_ee2 (the last column is d(d/sqrt(dhat))/dx) and pFpx_pppV0V1,
  pFpx_ppeV0V1, pFpx_peeV0V1 for the mollified pairs (column 4 is dc/dx, c = |e0 x e1|;
  column 8 as above).  Their bodies are read from the checkout and their statements
  evaluated in order at seeded configurations.

* ``ref_golden.npz`` -- per-element results of the reference's functions and kernels
  compiled for the host by ``oracle/ref_build.py`` (barrier energy and gradient of every
  pair kind, friction energy and gradient, the lagged friction set-up, ground barrier and
  ground friction, the line-search step bounds (additive CCD), stable Neo-Hookean PK1,
  energy and gradient, cloth membrane energy and gradient, kinetic and soft-constraint
  gradients, the inertial target, the trial step, and the contact pairs of GIPC::buildCP with
  their MatIndex and counters).  Inputs are two small seeded scenes
  (stored beside it as ``scene_two_cubes4.npz`` and ``scene_cloth6_cube4.npz``) and seeded
  synthetic pairs of every barrier kind, the mollified ones included.

Usage: python tests/golden/make_golden.py path/to/Stiff-GIPC    (the checkout's root)
"""
import ctypes as C
import math
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for _p in (ROOT, os.path.join(ROOT, "stiff-gipc_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

# ------------------------------------------------------------------------------------------
# pfpx_golden.npz: the generated Jacobian code, evaluated statement by statement
# ------------------------------------------------------------------------------------------
FUNCS = {
    "pFpx_pp2": 2,
    "pFpx_pe2": 3,
    "pFpx_pt2": 4,
    "pFpx_ee2": 4,
    "pFpx_pppV0V1": 4,
    "pFpx_ppeV0V1": 4,
    "pFpx_peeV0V1": 4,
}


def extract(src, name):
    m = re.search(r"void\s+%s\s*\(\s*double\s+d\s*," % name, src)
    if not m:
        raise KeyError(name)
    start = src.index("{", m.end())
    depth, i = 0, start
    while True:
        if src[i] == "{":
            depth += 1
        elif src[i] == "}":
            depth -= 1
            if depth == 0:
                return src[start + 1:i]
        i += 1


def evaluate(body, d, x, shape):
    env = {"sqrt": math.sqrt, "pow": math.pow, "fabs": abs, "d": d}
    names = ["x11", "x12", "x13", "x21", "x22", "x23", "x31", "x32", "x33", "x41", "x42", "x43"]
    for n, v in zip(names, x):
        env[n] = v
    out = np.zeros(shape)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    for stmt in body.split(";"):
        s = stmt.strip()
        if not s or s.startswith("double "):
            continue
        lhs, rhs = s.split("=", 1)
        lhs = lhs.strip()
        rhs = " ".join(rhs.split())
        op = lhs[-1] if lhs[-1] in "+-*/" else None   # compound assignment, e.g. `t78 *= t76`
        if op:
            lhs = lhs[:-1].strip()
            rhs = "(%s) %s (%s)" % (lhs, op, rhs)
        val = eval(rhs, {"__builtins__": {}}, env)  # noqa: S307 - arithmetic of a trusted local checkout
        m = re.fullmatch(r"result\[(\d+)\](?:\[(\d+)\])?", lhs)
        if m:
            if m.group(2) is None:
                out[int(m.group(1))] = val
            else:
                out[int(m.group(1)), int(m.group(2))] = val
        else:
            env[lhs] = val
    return out


def make_pfpx(ref_root):
    src = open(os.path.join(ref_root, "StiffGIPC", "GIPC_PDerivative.cuh")).read()
    rng = np.random.default_rng(20240601)
    data = {}
    for name, nv in FUNCS.items():
        body = extract(src, name)
        xs, ds, outs = [], [], []
        for _ in range(8):
            base = rng.uniform(-0.05, 0.05, 3)
            X = base + rng.uniform(-2e-3, 2e-3, (4, 3))
            if name in ("pFpx_pppV0V1", "pFpx_ppeV0V1", "pFpx_peeV0V1"):
                # nearly parallel edges, the regime the mollifier covers
                e = rng.normal(size=3)
                e /= np.linalg.norm(e)
                X[1] = X[0] + 4e-3 * e + rng.uniform(-1e-5, 1e-5, 3)
                X[3] = X[2] + 4e-3 * e + rng.uniform(-1e-5, 1e-5, 3)
            d = math.sqrt(1e-6)
            shape = (6,) if name == "pFpx_pp2" else (3 * nv, 9) if name == "pFpx_pe2" else (12, 9)
            out = evaluate(body, d, X.reshape(-1), shape)
            xs.append(X)
            ds.append(d)
            outs.append(out)
        data[name + "_x"] = np.array(xs)
        data[name + "_d"] = np.array(ds)
        data[name + "_out"] = np.array(outs)
    np.savez(os.path.join(HERE, "pfpx_golden.npz"), **data)
    print("wrote pfpx_golden.npz", len(data), "arrays")


# ------------------------------------------------------------------------------------------
# ref_golden.npz: the reference's functions and kernels compiled for the host
# ------------------------------------------------------------------------------------------
_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int32)
_u = C.POINTER(C.c_uint32)
D, I32, U32 = C.c_double, C.c_int, C.c_uint32


def _p(a, t=_d):
    return a.ctypes.data_as(t)


def load_ref(path):
    L = C.CDLL(path)
    sig = {
        "ref_barrier_energy": (D, [_d, _d, _i, D, D]),
        "ref_barrier_gradient": (None, [_d, _d, _i, I32, D, D, _d]),
        "ref_friction_energy": (D, [_d, _d, _i, D, _d, _d, D, D, D]),
        "ref_friction_gradient": (None, [_d, _d, _i, I32, D, _d, _d, D, _d, D, _d]),
        "ref_friction_gd_energy": (D, [_d, _d, _d, U32, D, D, D]),
        "ref_friction_gd_gradient": (None, [_d, _d, _d, _u, I32, D, D, _d, D, _d]),
        "ref_ground_gradient": (None, [_d, D, _d, _u, I32, D, D, _d]),
        "ref_friction_lasth_gd": (None, [_d, D, _d, _u, I32, D, D, _d, _u]),
        "ref_friction_lasth": (I32, [_d, _i, I32, D, D, _d, _d, _d, _i, _u]),
        "ref_self_step_inv": (D, [_d, _d, _i, D]),
        "ref_ground_step_inv": (D, [_d, U32, D, _d, _d, D]),
        "ref_kinetic_gradient": (None, [_d, _d, _d, I32, _d]),
        "ref_soft_gradient": (None, [_d, _d, _u, I32, D, D, _d]),
        "ref_xtilta": (None, [_i, _d, _d, _i, I32, D, _d]),
        "ref_step_forward": (None, [_d, _d, _d, _i, D, I32, I32]),
        "ref_snk_pk1": (None, [_d, _d, D, D, _d]),
        "ref_snk_energy": (D, [_d, _d, D, D, D]),
        "ref_fem_gradient": (None, [_d, _u, I32, _d, _d, _d, _d, D, _d]),
        "ref_tri_energy": (D, [_d, _d, D, D, D, D]),
        "ref_tri_gradient": (None, [_d, _u, I32, _d, _d, D, D, D, D, _d]),
        "ref_point_triangle_ccd": (D, [_d, _d, D, D]),
        "ref_edge_edge_ccd": (D, [_d, _d, D, D]),
        "ref_find_pairs": (I32, [_d, _d, I32, _u, I32, _u, I32, _u, _i, _i, D, I32, _i, _i, _i, _u]),
        "ref_ground_pairs": (I32, [_d, I32, _u, D, _d, D, _u]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype, f.argtypes = res, args
    return L


def pair_vertices(enc):
    """the distinct vertices a reference-encoded pair touches (StiffGIPC/GIPC.cu:701-944)"""
    x, y, z, w = (int(v) for v in enc)
    if x >= 0:
        return [x, y, z, w if w >= 0 else -w - 1]
    p = -x - 1
    if z < 0:
        return [p, y] if y >= 0 else [p, -y - 1, -z - 1, -w - 1]
    if w < 0:
        return [p, y, z] if y >= 0 else [p, -y - 1, z, -w - 1]
    return [p, y, z, w]


def synthetic_pairs(rng, dhat, per_kind=6):
    """Positions, rest positions and pairs of every barrier kind at distances inside d-hat.

    The mollified kinds use nearly parallel edges (angle 0.003-0.025 rad, so that |e0 x e1|^2
    stays below the reference's eps_x = 1e-3 |r0 - r1|^2 |r2 - r3|^2)."""
    X, P = [], []
    dmax = math.sqrt(dhat)

    def unit(v):
        return v / np.linalg.norm(v)

    def perp(u):
        return unit(np.cross(u, unit(rng.normal(size=3))))

    def rot(u, ang):
        a = perp(u)
        return unit(math.cos(ang) * u + math.sin(ang) * a)

    L = 4e-3
    for kind in ("PP", "PE", "PT", "EE", "mEE", "mPP", "mPE"):
        for _ in range(per_kind):
            b = len(X)
            c = rng.uniform(-0.05, 0.05, 3)
            d = rng.uniform(0.15, 0.95) * dmax
            u = unit(rng.normal(size=3))
            if kind == "PP":
                X += [c, c + d * u]
                P.append([-b - 1, b + 1, -1, -1])
            elif kind == "PE":
                e0, e1 = c, c + L * u
                q = e0 + rng.uniform(0.2, 0.8) * L * u + d * perp(u)
                X += [q, e0, e1]
                P.append([-b - 1, b + 1, b + 2, -1])
            elif kind == "PT":
                t0 = c
                t1 = c + L * u
                t2 = c + L * rot(u, rng.uniform(0.8, 2.2))
                n = unit(np.cross(t1 - t0, t2 - t0))
                w = rng.dirichlet([2, 2, 2])
                q = w[0] * t0 + w[1] * t1 + w[2] * t2 + d * n
                X += [q, t0, t1, t2]
                P.append([-b - 1, b + 1, b + 2, b + 3])
            elif kind == "EE":
                v = rot(u, rng.uniform(0.6, 2.5))
                n = unit(np.cross(u, v))
                a0, a1 = c - 0.5 * L * u, c + 0.5 * L * u
                cb = c + d * n + rng.uniform(-0.2, 0.2) * L * u
                b0, b1 = cb - 0.5 * L * v, cb + 0.5 * L * v
                X += [a0, a1, b0, b1]
                P.append([b, b + 1, b + 2, b + 3])
            else:
                v = rot(u, rng.uniform(0.003, 0.025))
                n = perp(u)
                if kind == "mEE":       # overlapping spans, interior closest points
                    a0, a1 = c, c + L * u
                    b0 = c + d * n + 0.3 * L * u
                    b1 = b0 + L * v
                    X += [a0, a1, b0, b1]
                    P.append([b, b + 1, b + 2, -(b + 3) - 1])
                elif kind == "mPP":     # ends facing each other: point a0 against point b0
                    a0 = c
                    a1 = a0 - L * u
                    b0 = a0 + d * n
                    b1 = b0 - L * v
                    X += [a0, a1, b0, b1]
                    # x = -a0-1, y = -b0-1, z = -a1-1, w = -b1-1: edges (a0, a1) and (b0, b1)
                    P.append([-b - 1, -(b + 2) - 1, -(b + 1) - 1, -(b + 3) - 1])
                else:                   # mPE: point a0 (edge a0-a1) against edge b0-b1
                    a0 = c
                    a1 = a0 - L * u
                    b0 = a0 + d * n - 0.5 * L * v
                    b1 = b0 + L * v
                    X += [a0, a1, b0, b1]
                    # x = -a0-1, y = -b0-1, z = b1, w = -a1-1
                    P.append([-b - 1, -(b + 2) - 1, b + 3, -(b + 1) - 1])
    X = np.asarray(X, np.float64)
    return X, X.copy(), np.asarray(P, np.int32)


def barrier_vectors(L, X, R, pairs, dhat, kappa):
    """per pair: energy, and the gradient rows of its vertices (vid, (4,3), -1 / 0 padded)"""
    n = len(pairs)
    e = np.zeros(n)
    vid = np.full((n, 4), -1, np.int32)
    g = np.zeros((n, 4, 3))
    buf = np.zeros_like(X)
    for k in range(n):
        pk = np.ascontiguousarray(pairs[k])
        e[k] = L.ref_barrier_energy(_p(X), _p(R), _p(pk, _i), dhat, kappa)
        buf[:] = 0.0
        L.ref_barrier_gradient(_p(X), _p(R), _p(pk, _i), 1, dhat, kappa, _p(buf))
        vs = pair_vertices(pk)
        vid[k, :len(vs)] = vs
        g[k, :len(vs)] = buf[vs]
    return e, vid, g


def make_ref(ref_root):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_build
    from sgipc import scenes

    L = load_ref(ref_build.build(ref_root))
    rng = np.random.default_rng(20250301)
    out = {}
    up = np.array([0.0, 1.0, 0.0])

    # ---- synthetic pairs of every kind ----
    dhat, kappa = 1e-6, 1e9
    X, R, P = synthetic_pairs(rng, dhat)
    e, vid, g = barrier_vectors(L, X, R, P, dhat, kappa)
    out.update(syn_x=X, syn_rest=R, syn_pairs=P, syn_dhat=dhat, syn_kappa=kappa, syn_bar_energy=e,
               syn_bar_vid=vid, syn_bar_grad=g)
    lam, crd, bas, plast = np.zeros(len(P)), np.zeros((len(P), 2)), np.zeros((len(P), 3, 2)), np.zeros((len(P), 4), np.int32)
    cp = np.zeros(5, np.uint32)
    nl = L.ref_friction_lasth(_p(X), _p(P, _i), len(P), dhat, kappa, _p(lam), _p(crd), _p(bas), _p(plast, _i), _p(cp, _u))
    out.update(syn_lag_pairs=plast[:nl], syn_lag_lambda=lam[:nl], syn_lag_coord=crd[:nl], syn_lag_basis=bas[:nl],
               syn_lag_cpnum=cp.astype(np.int64))

    # ---- two cubes, 4^3 lattices, with Dirichlet vertices ----
    for tag, sc in (("cubes", scenes.scene_two_cubes(4, seed=5)), ("cloth", scenes.scene_cloth_on_cube(6, 4, seed=6))):
        prm = sc.params
        dt, dh, kap = prm["dt"], prm["dHat"], prm["kappa"]
        eps2 = prm["fDhat"] * dt * dt
        if tag == "cubes":
            sc.boundary_type[np.arange(0, sc.nv, 9)] = 1
            sc.soft_index = np.arange(3, sc.nv, 17, dtype=np.int32)
            sc.soft_target = sc.vertexes[sc.soft_index] + rng.uniform(-2e-3, 2e-3, (len(sc.soft_index), 3))
            sc.params["motionRate"], sc.params["softRate"] = 1.0, 2.0
        # the Newton iterate moves tangentially off the start-of-step positions (friction
        # needs a displacement; sizes around the friction eps, sqrt(fDhat) dt)
        eps = math.sqrt(eps2)
        sc.vertexes = sc.o_vertexes + rng.uniform(-3.0, 3.0, sc.o_vertexes.shape) * eps
        sc.vertexes[sc.boundary_type != 0] = sc.o_vertexes[sc.boundary_type != 0]
        # keep only pairs still inside d-hat at the iterate
        from sgipc import contacts
        x = sc.vertexes
        keep = []
        for k, pr in enumerate(sc.pairs):
            vs = pair_vertices(pr)
            if pr[0] >= 0:
                d2 = contacts.d_ee(*[x[v][None] for v in vs])[0]
            elif len(vs) == 2:
                d2 = contacts.d_pp(x[vs[0]][None], x[vs[1]][None])[0]
            elif len(vs) == 3:
                d2 = contacts.d_pe(*[x[v][None] for v in vs])[0]
            else:
                d2 = contacts.d_pt(*[x[v][None] for v in vs])[0]
            keep.append(d2 < 0.98 * dh)
        sc.pairs = sc.pairs[np.asarray(keep, bool)]
        gd = x[sc.ground_pairs, 1] - prm["ground_offset"]
        sc.ground_pairs = sc.ground_pairs[gd * gd < 0.98 * dh]
        # the lagged friction set from the reference kernels, at the start-of-step positions
        x0 = np.ascontiguousarray(sc.o_vertexes)
        n = len(sc.pairs)
        lam, crd, bas, plast = np.zeros(n), np.zeros((n, 2)), np.zeros((n, 3, 2)), np.zeros((n, 4), np.int32)
        cp = np.zeros(5, np.uint32)
        pr = np.ascontiguousarray(sc.pairs, np.int32)
        nl = L.ref_friction_lasth(_p(x0), _p(pr, _i), n, dh, kap, _p(lam), _p(crd), _p(bas), _p(plast, _i), _p(cp, _u))
        gp = np.ascontiguousarray(sc.ground_pairs, np.uint32)
        glam, gplast = np.zeros(len(gp)), np.zeros(len(gp), np.uint32)
        L.ref_friction_lasth_gd(_p(x0), prm["ground_offset"], _p(up), _p(gp, _u), len(gp), dh, kap, _p(glam),
                                _p(gplast, _u))
        sc.fric_pairs, sc.fric_lambda, sc.fric_coord, sc.fric_basis = plast[:nl], lam[:nl], crd[:nl], bas[:nl]
        sc.fric_gd_pairs, sc.fric_gd_lambda = gplast.astype(np.int32), glam
        sc.save(os.path.join(HERE, "scene_%s.npz" % ("two_cubes4" if tag == "cubes" else "cloth6_cube4")))
        pre = tag + "_"
        out[pre + "lag_cpnum"] = cp.astype(np.int64)
        xs = np.ascontiguousarray(x)
        rest = np.ascontiguousarray(sc.rest_vertexes)
        # barrier
        e, vid, g = barrier_vectors(L, xs, rest, pr, dh, kap)
        out.update({pre + "bar_energy": e, pre + "bar_vid": vid, pre + "bar_grad": g})
        # friction per lagged pair (coef 1): energy and the rows of its vertices
        fe, fvid, fg = np.zeros(nl), np.full((nl, 4), -1, np.int32), np.zeros((nl, 4, 3))
        buf = np.zeros_like(xs)
        for k in range(nl):
            pk = np.ascontiguousarray(plast[k])
            fe[k] = L.ref_friction_energy(_p(xs), _p(x0), _p(pk, _i), dt, _p(np.ascontiguousarray(crd[k])),
                                          _p(np.ascontiguousarray(bas[k])), lam[k], eps2, eps)
            buf[:] = 0.0
            L.ref_friction_gradient(_p(xs), _p(x0), _p(pk, _i), 1, dt, _p(np.ascontiguousarray(crd[k])),
                                    _p(np.ascontiguousarray(bas[k])), eps2, _p(np.ascontiguousarray(lam[k:k + 1])),
                                    1.0, _p(buf))
            vs = pair_vertices(pk)
            fvid[k, :len(vs)] = vs
            fg[k, :len(vs)] = buf[vs]
        out.update({pre + "fric_energy": fe, pre + "fric_vid": fvid, pre + "fric_grad": fg})
        # ground barrier gradient, ground friction energy and gradient (coef 1), per vertex
        ng = len(gp)
        gg, gfe, gfg = np.zeros((ng, 3)), np.zeros(ng), np.zeros((ng, 3))
        for k in range(ng):
            buf[:] = 0.0
            one = gp[k:k + 1].copy()
            L.ref_ground_gradient(_p(xs), prm["ground_offset"], _p(up), _p(one, _u), 1, dh, kap, _p(buf))
            gg[k] = buf[gp[k]]
            gfe[k] = L.ref_friction_gd_energy(_p(xs), _p(x0), _p(up), int(gp[k]), dt, glam[k], eps)
            buf[:] = 0.0
            L.ref_friction_gd_gradient(_p(xs), _p(x0), _p(up), _p(one, _u), 1, dt, eps2,
                                       _p(np.ascontiguousarray(glam[k:k + 1])), 1.0, _p(buf))
            gfg[k] = buf[gp[k]]
        out.update({pre + "ground_grad": gg, pre + "gfric_energy": gfe, pre + "gfric_grad": gfg})
        # elastic terms over the whole mesh (dt scaling inside the kernels)
        nt = sc.nt
        if nt:
            tets = np.ascontiguousarray(sc.tets, np.uint32)
            dm = np.ascontiguousarray(sc.dm_inv)
            vol, lr, vr = (np.ascontiguousarray(a) for a in (sc.volum, sc.length_rate, sc.volume_rate))
            fg_all = np.zeros_like(xs)
            L.ref_fem_gradient(_p(xs), _p(tets, _u), nt, _p(dm), _p(vol), _p(lr), _p(vr), dt, _p(fg_all))
            te = np.array([L.ref_snk_energy(_p(np.ascontiguousarray(xs[t])), _p(np.ascontiguousarray(dm[k])), vol[k],
                                            lr[k], vr[k]) for k, t in enumerate(sc.tets)])
            out.update({pre + "fem_grad": fg_all, pre + "snk_energy": te})
        if len(sc.tris):
            tris = np.ascontiguousarray(sc.tris, np.uint32)
            tdm, area = np.ascontiguousarray(sc.tri_dm_inv), np.ascontiguousarray(sc.area)
            tg = np.zeros_like(xs)
            L.ref_tri_gradient(_p(xs), _p(tris, _u), len(tris), _p(tdm), _p(area), prm["stretchStiff"],
                               prm["shearStiff"], dt, prm["strainRate"], _p(tg))
            tre = np.array([L.ref_tri_energy(_p(np.ascontiguousarray(xs[t])), _p(np.ascontiguousarray(tdm[k])),
                                             area[k], prm["stretchStiff"], prm["shearStiff"], prm["strainRate"])
                            for k, t in enumerate(sc.tris)])
            out.update({pre + "tri_grad": tg, pre + "tri_energy": tre})
        kg = np.zeros_like(xs)
        L.ref_kinetic_gradient(_p(xs), _p(np.ascontiguousarray(sc.xTilta)), _p(np.ascontiguousarray(sc.masses)),
                               sc.nv, _p(kg))
        out[pre + "kin_grad"] = kg
        if len(sc.soft_index):
            sg = np.zeros_like(xs)
            L.ref_soft_gradient(_p(xs), _p(np.ascontiguousarray(sc.soft_target)),
                                _p(np.ascontiguousarray(sc.soft_index, np.uint32), _u), len(sc.soft_index),
                                sc.params["motionRate"], sc.params["softRate"], _p(sg))
            out[pre + "soft_grad"] = sg
        # line-search step bounds along a seeded direction (moveDir; trial x - alpha moveDir)
        move = rng.uniform(-1.0, 1.0, xs.shape) * math.sqrt(dh) * rng.uniform(0.0, 3.0, (sc.nv, 1))
        cand = pr[(pr[:, 0] >= 0) | ((pr[:, 2] >= 0) & (pr[:, 3] >= 0))].copy()
        mol = cand[:, 0] >= 0
        cand[mol, 3] = np.where(cand[mol, 3] < 0, -cand[mol, 3] - 1, cand[mol, 3])
        inv = np.array([L.ref_self_step_inv(_p(xs), _p(move), _p(np.ascontiguousarray(c), _i), 0.8) for c in cand])
        gmove = move.copy()
        gmove[:, 1] = np.abs(gmove[:, 1])  # moving down toward the plane
        ginv = np.array([L.ref_ground_step_inv(_p(xs), int(v), prm["ground_offset"], _p(up), _p(gmove), 0.8)
                         for v in gp])
        out.update({pre + "move": move, pre + "ccd_cand": cand, pre + "ccd_inv": inv, pre + "gmove": gmove,
                    pre + "ground_step_inv": ginv})
        # contact pairs of GIPC::buildCP at the iterate: self-collision everywhere (body -1), and
        # between bodies only (the scene's body ids)
        sv = np.ascontiguousarray(sc.surf_verts, np.uint32)
        sf = np.ascontiguousarray(sc.surf_tris, np.uint32)
        se = np.ascontiguousarray(sc.surf_edges, np.uint32)
        bt = np.ascontiguousarray(sc.boundary_type, np.int32)
        for variant, body in (("self", np.full(sc.nv, -1, np.int32)),
                              ("bodies", np.ascontiguousarray(sc.body_of_vertex, np.int32))):
            cap = 200000
            cpp, ccp, mi = np.zeros((cap, 4), np.int32), np.zeros((cap, 4), np.int32), np.zeros(cap, np.int32)
            cpn = np.zeros(5, np.uint32)
            n = L.ref_find_pairs(_p(xs), _p(rest), len(sv), _p(sv, _u), len(sf), _p(sf, _u), len(se), _p(se, _u),
                                 _p(body, _i), _p(bt, _i), dh, cap, _p(cpp, _i), _p(ccp, _i), _p(mi, _i), _p(cpn, _u))
            assert 0 < n < cap, n
            q = "%scp_%s_" % (pre, variant)
            out.update({q + "pairs": cpp[:n].copy(), q + "ccd": ccp[:n].copy(), q + "matindex": mi[:n].copy(),
                        q + "cpnum": cpn.astype(np.int64), q + "body": body})
        gout = np.zeros(len(sv), np.uint32)
        ng = L.ref_ground_pairs(_p(xs), len(sv), _p(sv, _u), prm["ground_offset"], _p(up), dh, _p(gout, _u))
        out[pre + "cp_ground"] = gout[:ng].astype(np.int32)
        # trial step with mixed boundary types, with and without move_boundary
        for mb in (0, 1):
            xn = np.zeros_like(xs)
            L.ref_step_forward(_p(xn), _p(xs), _p(move), _p(np.ascontiguousarray(sc.boundary_type, np.int32), _i),
                               0.37, mb, sc.nv)
            out[pre + "step_forward_%d" % mb] = xn
        # inertial target: x_prev + dt v + dt^2 g on free vertices with gravity
        agrav = (np.arange(sc.nv) % 5 != 0).astype(np.int32)
        xt = np.zeros_like(xs)
        L.ref_xtilta(_p(np.ascontiguousarray(sc.boundary_type, np.int32), _i), _p(np.ascontiguousarray(sc.velocities)),
                     _p(x0), _p(agrav, _i), sc.nv, dt, _p(xt))
        out.update({pre + "xtilta_gravity": agrav, pre + "xtilta": xt})

    # ---- stable Neo-Hookean and membrane elements at large, seeded deformations ----
    ns = 40
    Xt = rng.uniform(-0.02, 0.02, (ns, 4, 3)) + np.array([[0, 0, 0], [0.03, 0, 0], [0, 0.03, 0], [0, 0, 0.03]])
    Xt[::7, 3, 2] *= -1.0  # a few inverted tets
    Dm = np.linalg.inv(np.stack([np.array([[0.03, 0, 0], [0, 0.03, 0], [0, 0, 0.03]]).T
                                 + rng.uniform(-3e-3, 3e-3, (3, 3)) for _ in range(ns)]))
    lr = rng.uniform(1e4, 1e6, ns)
    vr = lr * rng.uniform(0.8, 30.0, ns)
    P = np.zeros((ns, 3, 3))
    E = np.zeros(ns)
    for k in range(ns):
        xk, dk = np.ascontiguousarray(Xt[k]), np.ascontiguousarray(Dm[k])
        L.ref_snk_pk1(_p(xk), _p(dk), lr[k], vr[k], _p(P[k]))
        E[k] = L.ref_snk_energy(_p(xk), _p(dk), 1.7e-5, lr[k], vr[k])
    out.update(el_tet_x=Xt, el_tet_dminv=Dm, el_tet_lr=lr, el_tet_vr=vr, el_tet_pk1=P, el_tet_energy=E,
               el_tet_vol=1.7e-5)
    # additive CCD at random separation ratios, straight calls (thickness 0, as every caller
    # of the line search passes)
    nc = 24
    cx = rng.uniform(-2e-3, 2e-3, (nc, 4, 3))
    cd = rng.uniform(-3e-3, 3e-3, (nc, 4, 3))
    eta = rng.uniform(0.05, 0.3, nc)
    thick = np.zeros(nc)
    pt = np.array([L.ref_point_triangle_ccd(_p(np.ascontiguousarray(cx[k])), _p(np.ascontiguousarray(cd[k])),
                                            eta[k], thick[k]) for k in range(nc)])
    ee = np.array([L.ref_edge_edge_ccd(_p(np.ascontiguousarray(cx[k])), _p(np.ascontiguousarray(cd[k])),
                                       eta[k], thick[k]) for k in range(nc)])
    out.update(ccd_x=cx, ccd_d=cd, ccd_eta=eta, ccd_thickness=thick, ccd_pt=pt, ccd_ee=ee)
    np.savez_compressed(os.path.join(HERE, "ref_golden.npz"), **out)
    print("wrote ref_golden.npz", len(out), "arrays")


def main():
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    root = sys.argv[1]
    make_pfpx(root)
    make_ref(root)


if __name__ == "__main__":
    main()
