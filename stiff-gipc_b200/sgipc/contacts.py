"""Host-side contact pair generation in StiffGIPC's int4 encoding, and lagged friction data.

The reference finds pairs with an LBVH (StiffGIPC/mlbvh.cu:1306-1742) and encodes each
one by its closest-feature type (StiffGIPC/mlbvh.cu:560-690 for point-triangle,
690-1059 for edge-edge):

* ``( a0,  a1,  b0,  b1)``           edge-edge
* ``(-p-1, t0,  t1,  t2)``           point-triangle
* ``(-p-1, e0,  e1,  w<0)``          point-edge
* ``(-p-1, q,   -1,  w<0)``          point-point
* ``( a0,  a1,  b0, -b1-1)``         mollified (nearly parallel) edge-edge
* ``(-p-1, -q-1, c, -d-1)``          mollified point-edge
* ``(-p-1, -q-1, -c-1, -d-1)``       mollified point-point

The shipping reference generator never emits the three mollified forms (``smooth`` is
false, StiffGIPC/mlbvh.cu:706); the barrier kernels still accept them.  This module is
the harness's input generator (a k-d tree broad phase plus exact type tests) and is not
part of the measured path.  ``lag_friction`` restates the once-per-frame lagged friction
set-up ``_calFrictionLastH_DistAndTan`` / ``_calFrictionLastH_gd``
(StiffGIPC/GIPC.cu:8362-8499).
"""
from __future__ import annotations

import numpy as np
from scipy.spatial import cKDTree

PP, PE, PT, EE = 0, 1, 2, 3


# ----------------------------------------------------------------------------------------
# closest-feature classification (vectorised)
# ----------------------------------------------------------------------------------------

def _det_cols(a, b, c):
    """det[a b c] (columns), term by term in the order of the reference's __Determiant
    (StiffGIPC/gpu_eigen_libs.cu:1193-1201)."""
    return (a[:, 0] * b[:, 1] * c[:, 2] + a[:, 1] * b[:, 2] * c[:, 0] + a[:, 2] * b[:, 0] * c[:, 1]
            - a[:, 2] * b[:, 1] * c[:, 0] - a[:, 0] * c[:, 1] * b[:, 2] - b[:, 0] * a[:, 1] * c[:, 2])


def pt_type(p, t0, t1, t2):
    """Closest feature of triangle (t0,t1,t2) to point p (``_dType_PT``, StiffGIPC/mlbvh.cu:288-447).

    Returns codes matching the reference's switch in ``_checkPTintersection``:
    0/1/2 = point-vertex t0/t1/t2, 3/4/5 = point-edge (t0t1)/(t1t2)/(t2t0), 6 = interior.
    For each edge (a, b) the parameters (s, h) of p - a in the frame [e, e x n, n] come from
    Cramer's rule; the edge is closest when 0 < s < 1 and h >= 0.
    """
    n = np.cross(t1 - t0, t2 - t0)
    s, h = [], []
    for a, b in ((t0, t1), (t1, t2), (t2, t0)):
        e = b - a
        f = np.cross(e, n)
        w = p - a
        D = _det_cols(e, f, n)
        s.append(_det_cols(w, f, n) / D)
        h.append(_det_cols(e, w, n) / D)
    out = np.full(p.shape[0], 6, np.int32)
    # evaluate in reverse priority so that the reference's first match wins
    out[(s[2] <= 0.0) & (s[1] >= 1.0)] = 2
    out[(s[1] <= 0.0) & (s[0] >= 1.0)] = 1
    out[(s[0] <= 0.0) & (s[2] >= 1.0)] = 0
    for i in (2, 1, 0):
        out[(s[i] > 0.0) & (s[i] < 1.0) & (h[i] >= 0.0)] = 3 + i
    return out


def ee_type(a0, a1, b0, b1):
    """Closest features of segments (a0,a1) and (b0,b1) (``_dType_EE``, StiffGIPC/mlbvh.cu:449-530,
    D. Sunday's clamped closest-point parameters s on a, t on b).

    Codes follow the reference's switch: 0 PP(a0,b0), 1 PP(a0,b1), 2 PE(a0; b0b1),
    3 PP(a1,b0), 4 PP(a1,b1), 5 PE(a1; b0b1), 6 PE(b0; a0a1), 7 PE(b1; a0a1), 8 EE.
    Nearly parallel segments whose interior parameters fall inside both take an endpoint
    case (2 or 5) instead of the lines.
    """
    u = a1 - a0
    v = b1 - b0
    w = a0 - b0
    a = (u * u).sum(1)
    b = (u * v).sum(1)
    c = (v * v).sum(1)
    d = (u * w).sum(1)
    e = (v * w).sum(1)
    D = a * c - b * b
    sN = b * e - c * d
    res = np.full(a.shape, 8, np.int32)
    lo = sN <= 0.0
    hi = ~lo & (sN >= D)
    mid = ~lo & ~hi
    tN = np.where(lo, e, np.where(hi, e + b, a * e - b * d))
    tD = np.where(lo | hi, c, D)
    res[lo] = 2
    res[hi] = 5
    uv = np.cross(u, v)
    flat = mid & (tN > 0.0) & (tN < tD) & (((w * uv).sum(1) == 0.0) | ((uv * uv).sum(1) < 1.0e-20 * a * c))
    first = flat & (sN < D / 2)
    second = flat & ~(sN < D / 2)
    tN = np.where(first, e, np.where(second, e + b, tN))
    tD = np.where(flat, c, tD)
    res[first] = 2
    res[second] = 5
    code = res.copy()
    t0 = tN <= 0.0
    code[t0] = np.where(-d[t0] <= 0.0, 0, np.where(-d[t0] >= a[t0], 3, 6))
    t1 = ~t0 & (tN >= tD)
    s1 = -d[t1] + b[t1]
    code[t1] = np.where(s1 <= 0.0, 1, np.where(s1 >= a[t1], 4, 7))
    return code


# squared distances by type (StiffGIPC/mlbvh.cu:229-262)
def d_pp(a, b):
    return ((a - b) ** 2).sum(1)


def d_pe(p, e0, e1):
    c = np.cross(e0 - p, e1 - p)
    return (c * c).sum(1) / ((e1 - e0) ** 2).sum(1)


def d_pt(p, t0, t1, t2):
    n = np.cross(t1 - t0, t2 - t0)
    s = ((p - t0) * n).sum(1)
    return s * s / (n * n).sum(1)


def d_ee(a0, a1, b0, b1):
    n = np.cross(a1 - a0, b1 - b0)
    s = ((b0 - a0) * n).sum(1)
    return s * s / (n * n).sum(1)


def eps_x(r0, r1, r2, r3):
    """Mollifier threshold ``_compute_epx`` (StiffGIPC/mlbvh.cu:264-268)."""
    return 1e-3 * ((r0 - r1) ** 2).sum(1) * ((r2 - r3) ** 2).sum(1)


# ----------------------------------------------------------------------------------------
# pair search
# ----------------------------------------------------------------------------------------

def _size_classes(radius):
    """Index sets of the primitives grouped by size (powers of two of their radius)."""
    r = np.maximum(np.asarray(radius, np.float64), 1e-300)
    key = np.floor(np.log2(r)).astype(np.int64)
    return [np.nonzero(key == k)[0] for k in np.unique(key)]


def find_pairs(x, rest, surf_tris, surf_edges, surf_verts, dhat, body=None,
               inter_body_only=False, with_ccd=False):
    """All barrier pairs with squared distance below ``dhat``, reference-encoded.

    Returns an (P,4) int32 array ordered PT-derived pairs first, then EE-derived pairs; with
    ``with_ccd`` also the CCD candidate of each pair (the point with its whole triangle, or the
    two edges: _ccd_collisionPair, StiffGIPC/mlbvh.cu:534-1059).
    """
    out, ccd = [], []
    gap = np.sqrt(dhat)
    if len(surf_tris) and len(surf_verts):
        tri_c = x[surf_tris].mean(1)
        tri_r = np.sqrt(((x[surf_tris] - tri_c[:, None]) ** 2).sum(2).max(1))
        # candidates class by class of triangle size, so that a few large triangles do not
        # widen the search around every point; then by point, then by triangle
        qpos = np.empty(len(x), np.int64)
        qpos[surf_verts] = np.arange(len(surf_verts))
        cand_p, cand_t = [], []
        for members in _size_classes(tri_r):
            tree = cKDTree(tri_c[members])
            nb = tree.query_ball_point(x[surf_verts], float(tri_r[members].max()) + gap)
            cand_p.append(np.repeat(surf_verts, [len(n) for n in nb]))
            cand_t.append(members[np.concatenate([np.asarray(n, np.int64) for n in nb])] if len(cand_p[-1])
                          else np.zeros(0, np.int64))
        pi = np.concatenate(cand_p).astype(np.int64)
        ti = np.concatenate(cand_t).astype(np.int64)
        order = np.lexsort((ti, qpos[pi]))
        pi, ti = pi[order], ti[order]
        if len(pi):
            t = surf_tris[ti]
            keep = (t != pi[:, None]).all(1)
            if inter_body_only and body is not None:
                keep &= body[pi] != body[t[:, 0]]
            pi, t = pi[keep], t[keep]
            p, a, b, c = x[pi], x[t[:, 0]], x[t[:, 1]], x[t[:, 2]]
            code = pt_type(p, a, b, c)
            d = np.empty(len(pi))
            m = code == 0; d[m] = d_pp(p[m], a[m])
            m = code == 1; d[m] = d_pp(p[m], b[m])
            m = code == 2; d[m] = d_pp(p[m], c[m])
            m = code == 3; d[m] = d_pe(p[m], a[m], b[m])
            m = code == 4; d[m] = d_pe(p[m], b[m], c[m])
            m = code == 5; d[m] = d_pe(p[m], c[m], a[m])
            m = code == 6; d[m] = d_pt(p[m], a[m], b[m], c[m])
            hit = d < dhat
            pi, t, code = pi[hit], t[hit], code[hit]
            enc = np.full((len(pi), 4), -1, np.int64)
            enc[:, 0] = -pi - 1
            for k, (i1, i2, i3) in {0: (0, None, None), 1: (1, None, None), 2: (2, None, None),
                                     3: (0, 1, None), 4: (1, 2, None), 5: (2, 0, None),
                                     6: (0, 1, 2)}.items():
                m = code == k
                enc[m, 1] = t[m, i1]
                if i2 is not None:
                    enc[m, 2] = t[m, i2]
                if i3 is not None:
                    enc[m, 3] = t[m, i3]
            # PT-derived point-point / point-edge pairs carry w = -1 (StiffGIPC/mlbvh.cu:560-640);
            # like the reference, a point close to a shared vertex or edge of several
            # triangles yields one pair per triangle
            out.append(enc)
            ccd.append(np.concatenate([(-pi - 1)[:, None], t.astype(np.int64)], 1))
    if len(surf_edges) > 1:
        mid = x[surf_edges].mean(1)
        hl = np.sqrt(((x[surf_edges[:, 0]] - x[surf_edges[:, 1]]) ** 2).sum(1)) * 0.5
        classes = _size_classes(hl)
        trees = [cKDTree(mid[m]) for m in classes]
        found = []
        for a, ma in enumerate(classes):
            for b in range(a, len(classes)):
                mb = classes[b]
                rq = float(hl[ma].max()) + float(hl[mb].max()) + gap
                if a == b:
                    pr = trees[a].query_pairs(rq, output_type="ndarray")
                    if len(pr):
                        found.append(np.stack([ma[pr[:, 0]], ma[pr[:, 1]]], 1))
                else:
                    lists = trees[a].query_ball_tree(trees[b], rq)
                    ia = np.repeat(np.arange(len(ma)), [len(l) for l in lists])
                    if len(ia):
                        ib = np.concatenate([np.asarray(l, np.int64) for l in lists])
                        found.append(np.stack([ma[ia], mb[ib]], 1))
        cand = np.concatenate(found) if found else np.zeros((0, 2), np.int64)
        cand = np.sort(cand, axis=1)
        cand = cand[np.lexsort((cand[:, 1], cand[:, 0]))]
        if len(cand):
            cand = np.sort(cand, axis=1)  # (self, other) with other > self, as _selfQuery_ee takes them
            ea, eb = surf_edges[cand[:, 0]], surf_edges[cand[:, 1]]
            keep = (ea[:, :, None] != eb[:, None, :]).all((1, 2))
            if inter_body_only and body is not None:
                keep &= body[ea[:, 0]] != body[eb[:, 0]]
            ea, eb, other = ea[keep], eb[keep], cand[keep, 1]
            a0, a1, b0, b1 = x[ea[:, 0]], x[ea[:, 1]], x[eb[:, 0]], x[eb[:, 1]]
            code = ee_type(a0, a1, b0, b1)
            d = np.full(len(ea), np.inf)
            m = code == 0; d[m] = d_pp(a0[m], b0[m])
            m = code == 1; d[m] = d_pp(a0[m], b1[m])
            m = code == 2; d[m] = d_pe(a0[m], b0[m], b1[m])
            m = code == 3; d[m] = d_pp(a1[m], b0[m])
            m = code == 4; d[m] = d_pp(a1[m], b1[m])
            m = code == 5; d[m] = d_pe(a1[m], b0[m], b1[m])
            m = code == 6; d[m] = d_pe(b0[m], a0[m], a1[m])
            m = code == 7; d[m] = d_pe(b1[m], a0[m], a1[m])
            m = code == 8; d[m] = d_ee(a0[m], a1[m], b0[m], b1[m])
            hit = d < dhat
            ea, eb, code, other = ea[hit], eb[hit], code[hit], other[hit]
            ep = eps_x(rest[ea[:, 0]], rest[ea[:, 1]], rest[eb[:, 0]], rest[eb[:, 1]])
            cr = np.cross(x[ea[:, 0]] - x[ea[:, 1]], x[eb[:, 0]] - x[eb[:, 1]])
            par = (cr * cr).sum(1) < ep
            # nearly parallel edges: the point-point / point-edge pair carries w = -(other edge) - 2
            # (add_e, StiffGIPC/mlbvh.cu:722); the mollified encodings stay off there (smooth = false)
            add_e = np.where(par, -other.astype(np.int64) - 2, -1)
            enc = np.zeros((len(ea), 4), np.int64)
            i0, i1, j0, j1 = ea[:, 0], ea[:, 1], eb[:, 0], eb[:, 1]
            table = {0: (i0, j0, None), 1: (i0, j1, None), 2: (i0, j0, j1),
                     3: (i1, j0, None), 4: (i1, j1, None), 5: (i1, j0, j1),
                     6: (j0, i0, i1), 7: (j1, i0, i1)}
            for k, (p, q, r) in table.items():
                m = code == k
                enc[m, 0] = -p[m] - 1
                enc[m, 1] = q[m]
                enc[m, 2] = -1 if r is None else r[m]
                enc[m, 3] = add_e[m]
            m = code == 8
            enc[m] = np.stack([i0[m], i1[m], j0[m], j1[m]], 1)
            out.append(enc)
            ccd.append(np.stack([i0, i1, j0, j1], 1))
    if not out:
        empty = np.zeros((0, 4), np.int32)
        return (empty, empty.copy()) if with_ccd else empty
    pairs = np.concatenate(out, 0).astype(np.int32)
    return (pairs, np.concatenate(ccd, 0).astype(np.int32)) if with_ccd else pairs


def ground_pairs(x, surf_verts, dhat, offset=-1.0):
    """``_GroundCollisionDetect`` (StiffGIPC/GIPC.cu:6420-6436): surface vertices within d-hat."""
    d = x[surf_verts, 1] - offset
    return surf_verts[d * d <= dhat].astype(np.int32)


# ----------------------------------------------------------------------------------------
# lagged friction (per frame)
# ----------------------------------------------------------------------------------------

def _barrier_lambda(d2, dhat, kappa):
    """Normal-force magnitude of the RANK-2 barrier (StiffGIPC/GIPC.cu:8484-8491)."""
    l = np.log(d2 / dhat)
    return -kappa * 2.0 * np.sqrt(d2) * (l * l * (2 * d2 - 2 * dhat) + 2 * l * (d2 - dhat) ** 2 / d2)


def lag_friction(x, pairs, gpairs, dhat, kappa, offset=-1.0):
    """Lagged normal forces, closest-point coordinates and tangent bases of the pairs.

    Restates ``_calFrictionLastH_DistAndTan`` and ``_calFrictionLastH_gd``
    (StiffGIPC/GIPC.cu:8362-8499) and the tangent/closest-point helpers of
    StiffGIPC/FrictionUtils.cuh:52-399.  Mollified pairs are skipped, as there.
    """
    lp, lam, coord, basis = [], [], [], []
    for pr in pairs:
        a, b, c, d = (int(v) for v in pr)
        if a >= 0:
            if d < 0:
                continue
            x0, x1, x2, x3 = x[a], x[b], x[c], x[d]
            n = np.cross(x1 - x0, x3 - x2)
            s = np.dot(x2 - x0, n)
            d2 = s * s / np.dot(n, n)
            e20, e01, e23 = x0 - x2, x1 - x0, x3 - x2
            A = np.array([[e01 @ e01, -(e23 @ e01)], [-(e23 @ e01), e23 @ e23]])
            r = np.array([-(e20 @ e01), e20 @ e23])
            gam = np.linalg.solve(A, r)
            t0 = e01 / np.linalg.norm(e01)
            cc = np.cross(np.cross(e01, e23), e01)
            bas = np.stack([t0, cc / np.linalg.norm(cc)], 1)
        else:
            p = -a - 1
            if c < 0:
                if b < 0:
                    continue
                x0, x1 = x[p], x[b]
                d2 = np.dot(x0 - x1, x0 - x1)
                gam = np.zeros(2)
                v01 = x1 - x0
                xc = np.array([0.0, -v01[2], v01[1]])
                yc = np.array([v01[2], 0.0, -v01[0]])
                t0 = xc if np.dot(xc, xc) > np.dot(yc, yc) else yc
                t1 = np.cross(v01, t0)
                bas = np.stack([t0 / np.linalg.norm(t0), t1 / np.linalg.norm(t1)], 1)
            elif d < 0:
                if b < 0:
                    continue
                x0, x1, x2 = x[p], x[b], x[c]
                e12 = x2 - x1
                d2 = np.dot(np.cross(x1 - x0, x2 - x0), np.cross(x1 - x0, x2 - x0)) / np.dot(e12, e12)
                gam = np.array([np.dot(x0 - x1, e12) / np.dot(e12, e12), 0.0])
                t0 = e12 / np.linalg.norm(e12)
                t1 = np.cross(e12, x0 - x1)
                bas = np.stack([t0, t1 / np.linalg.norm(t1)], 1)   # FrictionUtils.cuh:279-292
            else:
                x0, x1, x2, x3 = x[p], x[b], x[c], x[d]
                n = np.cross(x2 - x1, x3 - x1)
                s = np.dot(x0 - x1, n)
                d2 = s * s / np.dot(n, n)
                B = np.stack([x2 - x1, x3 - x1], 1)
                gam = np.linalg.solve(B.T @ B, B.T @ (x0 - x1))
                v12 = x2 - x1
                cc = np.cross(np.cross(v12, x3 - x1), v12)
                bas = np.stack([v12 / np.linalg.norm(v12), cc / np.linalg.norm(cc)], 1)
        lp.append(pr)
        lam.append(_barrier_lambda(d2, dhat, kappa))
        coord.append(gam)
        basis.append(bas)
    gd = x[gpairs, 1] - offset if len(gpairs) else np.zeros(0)
    d2g = gd * gd
    t = d2g - dhat
    gb = t * np.log(d2g / dhat) * -2.0 - (t * t) / d2g if len(gpairs) else np.zeros(0)
    glam = -kappa * 2.0 * np.sqrt(d2g) * gb
    if not lp:
        return (np.zeros((0, 4), np.int32), np.zeros(0), np.zeros((0, 2)), np.zeros((0, 3, 2)),
                gpairs.astype(np.int32), glam)
    return (np.asarray(lp, np.int32), np.asarray(lam), np.asarray(coord), np.asarray(basis),
            gpairs.astype(np.int32), glam)


def attach_contacts(sc, inter_body_only: bool = False) -> None:
    """Fill ``sc.pairs``, ``sc.ground_pairs`` and the lagged friction arrays in place."""
    p = sc.params
    sc.pairs = find_pairs(sc.vertexes, sc.rest_vertexes, sc.surf_tris, sc.surf_edges,
                          sc.surf_verts, p["dHat"], sc.body_of_vertex, inter_body_only)
    sc.ground_pairs = ground_pairs(sc.vertexes, sc.surf_verts, p["dHat"], p["ground_offset"])
    if p.get("frictionRate", 0.0) > 0.0:
        fp, fl, fc, fb, gp, gl = lag_friction(sc.o_vertexes, sc.pairs, sc.ground_pairs,
                                              p["dHat"], p["kappa"], p["ground_offset"])
        sc.fric_pairs, sc.fric_lambda, sc.fric_coord, sc.fric_basis = fp, fl, fc, fb
        sc.fric_gd_pairs, sc.fric_gd_lambda = gp, gl
