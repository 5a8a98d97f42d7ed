"""Seeded synthetic Newton systems in the layout of StiffGIPC's ``device_TetraData``.

The reference loads ``.msh``/``.obj`` meshes, sorts them with METIS into 16-vertex parts
and derives per-element data in ``initFEM`` (StiffGIPC/gl_main.cu:557-645).  None of
that is on the hot path; this module restates the derived quantities for procedurally
generated meshes so that the per-Newton-iteration linear system can be fed with the
same arrays the reference kernels read (StiffGIPC/device_fem_data.cuh:17-78):

* ``DmInverses`` — row-major 3x3 inverse of the rest edge matrix ``[x1-x0, x2-x0, x3-x0]``;
* ``volum`` — rest volume; ``masses`` — lumped ``rho*vol/4`` per tet corner;
* ``lengthRate = 4*mu_L/3`` and ``volumeRate = lambda_L + 5*mu_L/6`` from (E, nu)
  (StiffGIPC/gl_main.cu:609-617), i.e. the stable Neo-Hookean parameters;
* ``xTilta = x_prev + dt*v + dt^2*g`` (StiffGIPC/GIPC.cu:8073-8097);
* the MAS partition maps ``partId_map_real``/``real_map_partId`` and the vertex
  neighbour CSR built from tet and triangle edges (StiffGIPC/load_mesh.cpp:934-1040).

Contact pairs are produced by :mod:`sgipc.contacts` in the reference's int4 encoding.
Everything here is input preparation on the host; the assembled system and its solve
run on the GPU through the C ABI.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Optional

import numpy as np

GROUND_OFFSET = -1.0          # plane y = -1 with normal +y (StiffGIPC/GIPC.cu:8541-8549)
GROUND_NORMAL = (0.0, 1.0, 0.0)
GRAVITY = (0.0, -9.8, 0.0)
BANK = 16                     # MAS domain size (BANKSIZE, StiffGIPC/eigen_data.h:17)


@dataclasses.dataclass
class Scene:
    """One Newton system's inputs (host copies, float64 / int32 numpy arrays)."""

    name: str
    vertexes: np.ndarray          # (V,3) current Newton iterate x
    o_vertexes: np.ndarray        # (V,3) start-of-step positions (friction reference)
    rest_vertexes: np.ndarray     # (V,3) rest positions (mollifier eps, rest shapes)
    xTilta: np.ndarray            # (V,3) inertial target
    velocities: np.ndarray        # (V,3)
    masses: np.ndarray            # (V,)
    boundary_type: np.ndarray     # (V,) int32, 0 = free
    tets: np.ndarray              # (T,4) int32
    dm_inv: np.ndarray            # (T,3,3) row-major
    volum: np.ndarray             # (T,)
    length_rate: np.ndarray       # (T,)
    volume_rate: np.ndarray       # (T,)
    youngs: np.ndarray            # (T,) Young's modulus per tet (adjoint parameter)
    poisson: float
    tris: np.ndarray              # (F,3) cloth triangles
    tri_dm_inv: np.ndarray        # (F,2,2)
    area: np.ndarray              # (F,) area*thickness
    hinges: np.ndarray            # (Eh,2) hinge edge (tri_edges)
    hinge_adj: np.ndarray         # (Eh,2) opposite vertices (tri_edge_adj_vertex), -1 boundary
    hinge_q: np.ndarray           # (Eh,4,4) quadratic bending Q
    surf_tris: np.ndarray         # (S,3) collision surface triangles
    surf_edges: np.ndarray        # (E,2) collision surface edges
    surf_verts: np.ndarray        # (Sv,) collision surface vertices
    body_of_vertex: np.ndarray    # (V,) int32 body id
    part_map_real: np.ndarray     # (P*16,) position -> vertex or -1
    real_map_part: np.ndarray     # (V,) vertex -> position
    nbr_start: np.ndarray         # (V+1,) neighbour CSR
    nbr_list: np.ndarray          # (nnz,)
    params: Dict[str, float]
    pairs: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 4), np.int32))
    ground_pairs: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0,), np.int32))
    fric_pairs: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 4), np.int32))
    fric_lambda: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0,), np.float64))
    fric_coord: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 2), np.float64))
    fric_basis: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 3, 2), np.float64))
    fric_gd_pairs: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0,), np.int32))
    fric_gd_lambda: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0,), np.float64))
    soft_index: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0,), np.int32))
    soft_target: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 3), np.float64))

    @property
    def nv(self) -> int:
        return int(self.vertexes.shape[0])

    @property
    def nt(self) -> int:
        return int(self.tets.shape[0])

    def save(self, path: str) -> None:
        arrays = {k: v for k, v in dataclasses.asdict(self).items() if isinstance(v, np.ndarray)}
        np.savez_compressed(path, name=np.array(self.name), poisson=np.array(self.poisson),
                            params_keys=np.array(list(self.params.keys())),
                            params_vals=np.array(list(self.params.values()), np.float64), **arrays)

    @staticmethod
    def load(path: str) -> "Scene":
        z = np.load(path, allow_pickle=False)
        kw = {}
        for f in dataclasses.fields(Scene):
            if f.name in ("name", "poisson", "params"):
                continue
            kw[f.name] = z[f.name]
        params = {str(k): float(v) for k, v in zip(z["params_keys"], z["params_vals"])}
        return Scene(name=str(z["name"]), poisson=float(z["poisson"]), params=params, **kw)


# ----------------------------------------------------------------------------------------
# meshes
# ----------------------------------------------------------------------------------------

def lattice_tets(n: int, size: float, origin=(0.0, 0.0, 0.0)):
    """Regular n^3 vertex lattice over a cube of edge ``size``, 5 tets per cell.

    Cells alternate between the two mirror-image 5-tet splits so that faces match.
    Returns (verts (n^3,3), tets (5*(n-1)^3,4)) with positively oriented tets.
    """
    return box_lattice_tets((n, n, n), size / (n - 1), origin)


def box_lattice_tets(n, h: float, origin=(0.0, 0.0, 0.0)):
    """Regular nx x ny x nz vertex lattice of spacing h, 5 tets per cell (the split of
    :func:`lattice_tets`).  Returns (verts, tets) with positively oriented tets."""
    nx, ny, nz = (int(t) for t in n)
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    verts = h * np.stack([ii.ravel(), jj.ravel(), kk.ravel()], 1).astype(np.float64) + np.asarray(origin)

    def vid(i, j, k):
        return (i * ny + j) * nz + k

    ci, cj, ck = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), np.arange(nz - 1), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    corner = {}
    for a in (0, 1):
        for b in (0, 1):
            for d in (0, 1):
                corner[(a, b, d)] = vid(ci + a, cj + b, ck + d)
    even = ((ci + cj + ck) % 2) == 0
    # even split: corners at 000,110,101,011 + centre (100,010,001,111)
    ev = [((0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)),
          ((1, 1, 0), (0, 1, 0), (1, 0, 0), (1, 1, 1)),
          ((1, 0, 1), (1, 0, 0), (0, 0, 1), (1, 1, 1)),
          ((0, 1, 1), (0, 0, 1), (0, 1, 0), (1, 1, 1)),
          ((1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1))]
    # odd split: mirror in x
    od = [tuple((1 - p[0], p[1], p[2]) for p in t) for t in ev]
    tets = []
    for te, to in zip(ev, od):
        t_even = np.stack([corner[p] for p in te], 1)
        t_odd = np.stack([corner[p] for p in to], 1)
        tets.append(np.where(even[:, None], t_even, t_odd))
    tets = np.concatenate(tets, 0).astype(np.int64)
    tets = orient_tets(verts, tets)
    return verts, tets.astype(np.int32)


def orient_tets(verts, tets):
    x = verts[tets]
    d = np.einsum("ij,ij->i", np.cross(x[:, 1] - x[:, 0], x[:, 2] - x[:, 0]), x[:, 3] - x[:, 0])
    tets = tets.copy()
    neg = d < 0
    tets[neg, 1], tets[neg, 2] = tets[neg, 2].copy(), tets[neg, 1].copy()
    return tets


def tet_surface(tets: np.ndarray):
    """Boundary triangles (outward orientation), unique surface edges and vertices."""
    faces = np.concatenate([tets[:, [1, 2, 3]], tets[:, [0, 3, 2]],
                            tets[:, [0, 1, 3]], tets[:, [0, 2, 1]]], 0)
    key = np.sort(faces, 1)
    _, inv, cnt = np.unique(key, axis=0, return_inverse=True, return_counts=True)
    bnd = cnt[inv.ravel()] == 1
    tris = faces[bnd]
    edges = np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]], 0)
    edges = np.unique(np.sort(edges, 1), axis=0)
    sverts = np.unique(tris.ravel())
    return tris.astype(np.int32), edges.astype(np.int32), sverts.astype(np.int32)


def tri_mesh_edges(tris: np.ndarray):
    edges = np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]], 0)
    return np.unique(np.sort(edges, 1), axis=0).astype(np.int32)


def tet_rest_data(verts: np.ndarray, tets: np.ndarray):
    """DmInverses (row-major), rest volumes (StiffGIPC/gl_main.cu:587-600)."""
    x = verts[tets]
    dm = np.stack([x[:, 1] - x[:, 0], x[:, 2] - x[:, 0], x[:, 3] - x[:, 0]], 2)  # columns
    dm_inv = np.linalg.inv(dm)
    vol = np.abs(np.linalg.det(dm)) / 6.0
    return dm_inv, vol


def cloth_grid(n: int, size: float, origin=(0.0, 0.0, 0.0)):
    """n x n vertex grid over a size x size square in the x-z plane at height origin[1];
    2 (n-1)^2 triangles with alternating diagonals, normals along +y."""
    g = np.linspace(0.0, size, n)
    ii, kk = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    verts = np.stack([g[ii.ravel()], np.zeros(n * n), g[kk.ravel()]], 1) + np.asarray(origin, np.float64)
    c = np.arange(n - 1)
    ci, ck = np.meshgrid(c, c, indexing="ij")
    ci, ck = ci.ravel(), ck.ravel()
    v00, v10, v01, v11 = ci * n + ck, (ci + 1) * n + ck, ci * n + ck + 1, (ci + 1) * n + ck + 1
    even = ((ci + ck) % 2) == 0
    t1 = np.where(even[:, None], np.stack([v00, v01, v11], 1), np.stack([v00, v01, v10], 1))
    t2 = np.where(even[:, None], np.stack([v00, v11, v10], 1), np.stack([v01, v11, v10], 1))
    return verts, np.concatenate([t1, t2], 0).astype(np.int32)


def tri_rest_data(verts: np.ndarray, tris: np.ndarray, thickness: float):
    """triDmInverses (row-major 2x2) and area*thickness (StiffGIPC/gl_main.cu:619-640).

    As the reference's rest frame (femEnergy.cu:256-300), each triangle is rotated so that
    its unit normal n goes to +z (Rodrigues: R = I + [v]x + [v]x^2 / (1 + n.z), v = n x z;
    a half-turn about z when n = -z) and Dm = [u1 - u0, u2 - u0] of the rotated x, y."""
    x = verts[tris]
    e1, e2 = x[:, 1] - x[:, 0], x[:, 2] - x[:, 0]
    nrm = np.cross(e1, e2)
    area2 = np.linalg.norm(nrm, axis=1)
    n = nrm / area2[:, None]
    z = np.array([0.0, 0.0, 1.0])
    v = np.cross(n, z)
    c = n @ z
    K = np.zeros((len(tris), 3, 3))
    K[:, 0, 1], K[:, 0, 2], K[:, 1, 0] = -v[:, 2], v[:, 1], v[:, 2]
    K[:, 1, 2], K[:, 2, 0], K[:, 2, 1] = -v[:, 0], -v[:, 1], v[:, 0]
    anti = c + 1.0 == 0.0
    denom = np.where(anti, 1.0, 1.0 + c)
    R = np.eye(3)[None] + K + np.einsum("fij,fjk->fik", K, K) / denom[:, None, None]
    R[anti] = np.diag([-1.0, -1.0, 1.0])
    uv = np.einsum("fij,fvj->fvi", R, x)[:, :, :2]
    dm = np.stack([uv[:, 1] - uv[:, 0], uv[:, 2] - uv[:, 0]], 2)  # columns u0, u1
    return np.linalg.inv(dm), 0.5 * area2 * thickness


def hinge_topology(tris: np.ndarray):
    """tri_edges and tri_edge_adj_vertex: every mesh edge with the vertex opposite it in
    its first and second triangle (-1 for a boundary edge)."""
    e = np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]], 0)
    opp = np.concatenate([tris[:, 2], tris[:, 0], tris[:, 1]], 0)
    key = np.sort(e, 1)
    order = np.lexsort((np.arange(len(key)), key[:, 1], key[:, 0]))
    key, e, opp = key[order], e[order], opp[order]
    uniq, first, cnt = np.unique(key, axis=0, return_index=True, return_counts=True)
    edges = e[first]
    adj = np.full((len(uniq), 2), -1, np.int64)
    adj[:, 0] = opp[first]
    two = cnt == 2
    adj[two, 1] = opp[first[two] + 1]
    return edges.astype(np.int32), adj.astype(np.int32)


def quad_bending_q(rest: np.ndarray, edges: np.ndarray, adj: np.ndarray):
    """Constant 4x4 bending matrices of the quadratic bending model (Bergou et al., "A
    quadratic bending model for inextensible surfaces", 2006), as the reference's
    PrepareQuadBendingQ (StiffGIPC/femEnergy.cu:2492-2618) computes them: for hinge
    vertices [e0, e1, opposite 1, opposite 2], K = (c03 + c04, c01 + c02, -c01 - c03,
    -c02 - c04) with the cotangents of the angles at e0 and e1, Q = 3 / (A1 + A2) K K^T;
    boundary and degenerate hinges get Q = 0."""
    Q = np.zeros((len(edges), 4, 4))
    inner = adj[:, 1] >= 0
    if not inner.any():
        return Q
    v0, v1 = rest[edges[inner, 0]], rest[edges[inner, 1]]
    v2, v3 = rest[adj[inner, 0]], rest[adj[inner, 1]]
    e0, e1, e2, e3, e4 = v1 - v0, v2 - v0, v3 - v0, v2 - v1, v3 - v1

    def cot(a, b):
        cn = np.linalg.norm(np.cross(a, b), axis=1)
        return np.where(cn < 1e-12, 0.0, (a * b).sum(1) / np.where(cn < 1e-12, 1.0, cn))

    n01 = np.linalg.norm(np.cross(e0, e1), axis=1)
    n02 = np.linalg.norm(np.cross(e0, e2), axis=1)
    c01, c02, c03, c04 = cot(e0, e1), cot(e0, e2), cot(-e0, e3), cot(-e0, e4)
    K = np.stack([c03 + c04, c01 + c02, -c01 - c03, -c02 - c04], 1)
    asum = 0.5 * (n01 + n02)
    ok = (n01 >= 1e-12) & (n02 >= 1e-12) & (asum >= 1e-12)
    q = 3.0 / np.where(ok, asum, 1.0)[:, None, None] * K[:, :, None] * K[:, None, :]
    q[~ok] = 0.0
    q[~np.isfinite(q).all((1, 2))] = 0.0
    Q[inner] = q
    return Q


def cloth_stiffness(E: float, nu: float, strain_rate: float, bend_E: float, thickness: float):
    """(stretchStiff, shearStiff, bendStiff) of StiffGIPC/gl_main.cu:578-583."""
    stretch = E / (2.0 * (1.0 + nu))
    return stretch, 0.03 * stretch * strain_rate, bend_E * thickness ** 3 / (24.0 * (1.0 - nu * nu))


def snk_rates(E, nu):
    """(lengthRate, volumeRate) of the stable Neo-Hookean model, StiffGIPC/gl_main.cu:609-617."""
    E = np.asarray(E, np.float64)
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    return 4.0 * mu / 3.0, lam + 5.0 * mu / 6.0


def neighbour_csr(nv: int, tets: np.ndarray, tris: np.ndarray):
    """Vertex adjacency over tet and triangle edges (StiffGIPC/load_mesh.cpp:934-1040)."""
    e = []
    if len(tets):
        for a, b in ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)):
            e.append(tets[:, [a, b]])
    if len(tris):
        for a, b in ((0, 1), (1, 2), (2, 0)):
            e.append(tris[:, [a, b]])
    if not e:
        return np.zeros(nv + 1, np.int32), np.zeros(0, np.int32)
    e = np.unique(np.sort(np.concatenate(e, 0), 1), axis=0)
    both = np.concatenate([e, e[:, ::-1]], 0)
    order = np.lexsort((both[:, 1], both[:, 0]))
    both = both[order]
    start = np.zeros(nv + 1, np.int64)
    np.add.at(start, both[:, 0] + 1, 1)
    start = np.cumsum(start)
    return start.astype(np.int32), both[:, 1].astype(np.int32)


def _morton_key(p: np.ndarray) -> np.ndarray:
    lo = p.min(0)
    span = max(float((p.max(0) - lo).max()), 1e-30)
    q = np.clip(((p - lo) / span * 1023.0).round().astype(np.int64), 0, 1023)

    def spread(v):
        v = (v | (v << 16)) & 0x030000FF
        v = (v | (v << 8)) & 0x0300F00F
        v = (v | (v << 4)) & 0x030C30C3
        v = (v | (v << 2)) & 0x09249249
        return v

    return (spread(q[:, 0]) << 2) | (spread(q[:, 1]) << 1) | spread(q[:, 2])


def mas_partition(rest: np.ndarray, body: np.ndarray):
    """16-vertex MAS parts along a Morton curve, one body at a time.

    Stands in for the METIS ``*_sorted.16.part`` files (MeshProcess/metis_partition/
    src/metis_sort.cpp:25-219): a part never spans two bodies, each body's last part is
    padded with -1 to a multiple of 16, exactly the shape ``partId_map_real`` has in the
    reference (StiffGIPC/gl_main.cu:1066-1093).
    """
    nv = rest.shape[0]
    part_map = []
    for b in np.unique(body):
        ids = np.nonzero(body == b)[0]
        order = ids[np.argsort(_morton_key(rest[ids]), kind="stable")]
        pad = (-len(order)) % BANK
        part_map.append(order)
        if pad:
            part_map.append(-np.ones(pad, np.int64))
    part_map = np.concatenate(part_map).astype(np.int32)
    real_map = np.full(nv, -1, np.int32)
    pos = np.nonzero(part_map >= 0)[0]
    real_map[part_map[pos]] = pos
    return part_map, real_map


def ordered_partition(body: np.ndarray):
    """Part maps for vertices already numbered in part order: consecutive runs of 16
    within each body, the body's last part padded with -1."""
    nv = body.shape[0]
    part_map = []
    for b in np.unique(body):
        ids = np.nonzero(body == b)[0]
        part_map.append(ids)
        pad = (-len(ids)) % BANK
        if pad:
            part_map.append(-np.ones(pad, np.int64))
    part_map = np.concatenate(part_map).astype(np.int32)
    real_map = np.full(nv, -1, np.int32)
    pos = np.nonzero(part_map >= 0)[0]
    real_map[part_map[pos]] = pos
    return part_map, real_map


def suggest_kappa(bbox_diag2: float, dhat: float, mean_mass: float, min_kappa_coef: float = 1e11):
    """``GIPC::suggestKappa`` (StiffGIPC/GIPC.cu:9850-9866) with ``H_b`` of compute_H_b."""
    d = 1e-16 * bbox_diag2
    t = d - dhat
    hb = (math.log(d / dhat) * -2.0 - t * 4.0 / d) + 1.0 / (d * d) * (t * t)
    if mean_mass == 0.0:
        return min_kappa_coef / (4.0e-16 * bbox_diag2 * hb)
    return min_kappa_coef * mean_mass / (4.0e-16 * bbox_diag2 * hb)


# ----------------------------------------------------------------------------------------
# scene assembly
# ----------------------------------------------------------------------------------------

def inertial_target(x_prev, vel, btype, dt, apply_gravity=None):
    """``xTilta = x_prev + (dt v + dt^2 g)``, gravity on free vertices that take it
    (``_computeXTilta``, StiffGIPC/GIPC.cu:8073-8096; ``apply_gravity`` all ones when None)."""
    g = np.asarray(GRAVITY) * (dt * dt)
    on = np.asarray(btype) == 0
    if apply_gravity is not None:
        on &= np.asarray(apply_gravity) != 0
    return x_prev + (vel * dt + np.where(on[:, None], g[None, :], 0.0))


def _empty_cloth():
    return dict(tris=np.zeros((0, 3), np.int32), tri_dm_inv=np.zeros((0, 2, 2)),
                area=np.zeros(0), hinges=np.zeros((0, 2), np.int32),
                hinge_adj=np.zeros((0, 2), np.int32), hinge_q=np.zeros((0, 4, 4)))


def build_tet_scene(name: str, bodies: List[dict], dt: float, dhat_abs: float, density: float,
                    nu: float, mu_friction: float, seed: int, perturb: float,
                    kappa: Optional[float] = None, cloth: Optional[dict] = None) -> Scene:
    """Concatenate tet and cloth bodies, derive ``initFEM`` data and set up one Newton iterate.

    Each body dict holds ``verts`` and either ``tets`` with ``E`` (a soft solid) or
    ``tris`` (a cloth sheet), plus optional ``velocity`` (3,) and ``boundary`` flag.  A body
    with ``affine=True`` is the point set of an affine body: its ``tris`` are its contact
    surface only (no elements), its vertices are Dirichlet here (their motion is the body's,
    solved in body space) with unit mass on the kept diagonal.
    ``cloth`` gives the sheet material: ``thickness``, ``E``, ``bend_E``, ``density``,
    ``strain_rate`` (StiffGIPC/gl_main.cu:578-583, 619-640).  Vertex positions of the
    current iterate are the body's positions (``verts``) plus a seeded uniform perturbation of
    ``perturb`` metres; its rest shape is ``rest`` when given (a cloth posed away from its flat
    rest state), else ``verts``.
    """
    rng = np.random.default_rng(seed)
    verts, cur, tets, tris, atris, youngs, vel, btype, body_id = [], [], [], [], [], [], [], [], []
    off = 0
    for b, body in enumerate(bodies):
        v = np.asarray(body["verts"], np.float64)
        cur.append(v)
        verts.append(np.asarray(body.get("rest", v), np.float64))
        if body.get("affine"):
            atris.append(np.asarray(body["tris"], np.int64) + off)
        elif "tets" in body:
            t = np.asarray(body["tets"], np.int64) + off
            tets.append(t)
            youngs.append(np.full(len(t), float(body["E"])))
        else:
            tris.append(np.asarray(body["tris"], np.int64) + off)
        vel.append(np.tile(np.asarray(body.get("velocity", (0.0, 0.0, 0.0)), np.float64), (len(v), 1)))
        btype.append(np.full(len(v), 1 if body.get("affine") else int(body.get("boundary", 0)), np.int32))
        body_id.append(np.full(len(v), b, np.int32))
        off += len(v)
    rest = np.concatenate(verts)
    pose = np.concatenate(cur)
    tets = np.concatenate(tets).astype(np.int32) if tets else np.zeros((0, 4), np.int32)
    tris = np.concatenate(tris).astype(np.int64) if tris else np.zeros((0, 3), np.int64)
    atris = np.concatenate(atris).astype(np.int64) if atris else np.zeros((0, 3), np.int64)
    youngs = np.concatenate(youngs) if youngs else np.zeros(0)
    vel = np.concatenate(vel)
    btype = np.concatenate(btype)
    body_id = np.concatenate(body_id)
    nv = rest.shape[0]

    # renumber vertices in MAS part order, as the METIS-sorted meshes are, so that
    # real_map_partId is monotone (the reference's level-0 scatter assumes it,
    # StiffGIPC/MASPreconditioner.cu:1856-1867); bodies given with their own part ids (read
    # from .part files, or partitioned by sgipc.meshio) keep them and their numbering
    given = all("parts" in b for b in bodies)
    if given:
        offs, gparts = 0, []
        for body in bodies:
            p = np.asarray(body["parts"], np.int64)
            gparts.append(p - (p.min() if len(p) else 0) + offs)
            offs = int(gparts[-1].max()) + 1 if len(p) else offs
        gparts = np.concatenate(gparts)
        perm = np.arange(len(rest), dtype=np.int64)
    else:
        part_map, _ = mas_partition(rest, body_id)
        perm = part_map[part_map >= 0].astype(np.int64)
    inv = np.empty(nv, np.int64)
    inv[perm] = np.arange(nv)
    rest, pose, vel, btype, body_id = rest[perm], pose[perm], vel[perm], btype[perm], body_id[perm]
    tets = inv[tets].astype(np.int32)
    tris = inv[tris].astype(np.int32)
    atris = inv[atris].astype(np.int32)

    dm_inv, vol = tet_rest_data(rest, tets) if len(tets) else (np.zeros((0, 3, 3)), np.zeros(0))
    lr, vr = snk_rates(youngs, nu)
    masses = np.zeros(nv)
    np.add.at(masses, tets.ravel(), np.repeat(vol * density / 4.0, 4))
    if len(atris):
        masses[np.unique(atris)] = 1.0
    cl = _empty_cloth()
    stretch = shear = bend = srate = 0.0
    if len(tris):
        cloth = dict(dict(thickness=1e-3, E=1e6, bend_E=1e5, density=200.0, strain_rate=100.0), **(cloth or {}))
        tdm, tarea = tri_rest_data(rest, tris, cloth["thickness"])
        np.add.at(masses, tris.ravel(), np.repeat(tarea * cloth["density"] / 3.0, 3))
        hin, hadj = hinge_topology(tris)
        cl = dict(tris=tris, tri_dm_inv=tdm, area=tarea, hinges=hin, hinge_adj=hadj,
                  hinge_q=quad_bending_q(rest, hin, hadj))
        srate = cloth["strain_rate"]
        stretch, shear, bend = cloth_stiffness(cloth["E"], nu, srate, cloth["bend_E"], cloth["thickness"])

    x_prev = pose + rng.uniform(-perturb, perturb, rest.shape)
    x = x_prev.copy()
    g = np.asarray(GRAVITY)
    xt = inertial_target(x_prev, vel, btype, dt)

    stris, sedges, sverts = tet_surface(tets) if len(tets) else (np.zeros((0, 3), np.int32),
                                                                 np.zeros((0, 2), np.int32), np.zeros(0, np.int32))
    if len(tris):  # cloth sheets collide on both sides with every triangle, edge and vertex
        stris = np.concatenate([stris, tris]).astype(np.int32)
        sedges = np.unique(np.concatenate([sedges, tri_mesh_edges(tris)]), axis=0).astype(np.int32)
        sverts = np.unique(np.concatenate([sverts, tris.ravel()])).astype(np.int32)
    if len(atris):  # affine bodies collide with their surfaces
        stris = np.concatenate([stris, atris]).astype(np.int32)
        sedges = np.unique(np.concatenate([sedges, tri_mesh_edges(atris)]), axis=0).astype(np.int32)
        sverts = np.unique(np.concatenate([sverts, atris.ravel()])).astype(np.int32)
    nbr_start, nbr_list = neighbour_csr(nv, tets, tris)
    if given:
        from . import meshio
        part_map, real_map = meshio.part_maps(gparts)
    else:
        part_map, real_map = ordered_partition(body_id)

    lo = np.minimum(rest.min(0), x.min(0))
    hi = np.maximum(rest.max(0), x.max(0))
    bbox2 = float(((hi - lo) ** 2).sum())
    dhat = dhat_abs * dhat_abs
    mean_mass = float(masses.sum() / nv)
    if kappa is None:
        kappa = suggest_kappa(bbox2, dhat, mean_mass)
    params = dict(dt=dt, dHat=dhat, kappa=float(kappa), fDhat=1e-4 * bbox2, bboxDiag2=bbox2,
                  frictionRate=mu_friction, gd_frictionRate=mu_friction, ground_offset=GROUND_OFFSET,
                  stretchStiff=stretch, shearStiff=shear, strainRate=srate, bendStiff=bend,
                  motionRate=0.0, softRate=0.0, density=density, meanMass=mean_mass)
    return Scene(name=name, vertexes=x, o_vertexes=x_prev.copy(), rest_vertexes=rest,
                 xTilta=xt, velocities=vel, masses=masses, boundary_type=btype, tets=tets,
                 dm_inv=dm_inv, volum=vol, length_rate=lr, volume_rate=vr, youngs=youngs,
                 poisson=nu, surf_tris=stris, surf_edges=sedges, surf_verts=sverts,
                 body_of_vertex=body_id, part_map_real=part_map, real_map_part=real_map,
                 nbr_start=nbr_start, nbr_list=nbr_list, params=params, **cl)


def scene_from_files(bodies: List[dict], dt: float = 0.01, dhat_abs: float = 1e-3, density: float = 1000.0,
                     nu: float = 0.45, mu_friction: float = 0.2, seed: int = 0, perturb: float = 0.0,
                     kappa: Optional[float] = None, cloth: Optional[dict] = None, name: str = "files") -> Scene:
    """A Newton system of meshes read from files, as the reference's initScene loads them
    (StiffGIPC/gl_main.cu:1095-1438): each body names ``mesh`` (a ``.msh`` tet mesh or an
    ``.obj`` cloth), optionally ``part`` (its ``.part`` file; without one the vertices are
    partitioned and renumbered by :func:`sgipc.meshio.partition`), ``transform`` (4 x 4), and
    ``E`` (tets), ``velocity``, ``boundary`` as :func:`build_tet_scene` takes them."""
    from . import meshio
    loaded = []
    for b in bodies:
        v, e, p = meshio.load_body(b["mesh"], b.get("part"), b.get("transform"))
        d = {k: val for k, val in b.items() if k not in ("mesh", "part", "transform")}
        d["verts"], d["parts"] = v, p
        if e.shape[1] == 4:
            d["tets"] = e
            d.setdefault("E", 1e5)
        else:
            d["tris"] = e
        loaded.append(d)
    sc = build_tet_scene(name, loaded, dt=dt, dhat_abs=dhat_abs, density=density, nu=nu,
                         mu_friction=mu_friction, seed=seed, perturb=perturb, kappa=kappa, cloth=cloth)
    from . import contacts
    contacts.attach_contacts(sc)
    return sc


def scene_cube(n: int = 11, touching: bool = False, seed: int = 0) -> Scene:
    """The single-cube workload: one 0.1 m soft cube (n^3 lattice) dropped from 0.05 m (or touching)."""
    dhat_abs = 1e-3
    gap = 0.5 * dhat_abs if touching else 0.05
    v, t = lattice_tets(n, 0.1, (0.0, GROUND_OFFSET + gap, 0.0))
    sc = build_tet_scene("cube%d%s" % (n, "_touch" if touching else ""),
                         [dict(verts=v, tets=t, E=1e5)], dt=0.01, dhat_abs=dhat_abs,
                         density=1000.0, nu=0.4, mu_friction=0.0, seed=seed, perturb=1e-4)
    from . import contacts
    contacts.attach_contacts(sc)
    return sc


def scene_two_cubes(n: int = 21, seed: int = 1, friction: float = 0.2) -> Scene:
    """The two-cube workload: two stacked n^3 cubes, E = 1e5 / 1e6, nu = 0.45, mu = 0.2.

    The bottom cube rests 0.5 d-hat above the ground plane, the top cube 0.5 d-hat above
    the bottom one; the top cube's initial velocity has magnitude 1 m/s in a seeded
    random direction.  Both ground and cube-cube barrier/friction pairs are active.
    """
    dhat_abs = 1e-3
    size = 0.1
    gap = 0.5 * dhat_abs
    rng = np.random.default_rng(seed)
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    v0, t0 = lattice_tets(n, size, (0.0, GROUND_OFFSET + gap, 0.0))
    v1, t1 = lattice_tets(n, size, (0.0, GROUND_OFFSET + 2 * gap + size, 0.0))
    sc = build_tet_scene("two_cubes%d" % n,
                         [dict(verts=v0, tets=t0, E=1e5),
                          dict(verts=v1, tets=t1, E=1e6, velocity=tuple(d * 1.0))],
                         dt=0.01, dhat_abs=dhat_abs, density=1000.0, nu=0.45,
                         mu_friction=friction, seed=seed, perturb=1e-4)
    from . import contacts
    contacts.attach_contacts(sc)
    return sc


def scene_cloth_on_cube(n_cloth: int = 24, n_cube: int = 6, seed: int = 2, friction: float = 0.4) -> Scene:
    """A cloth sheet (n_cloth^2 grid, 0.2 m square, 1 mm thick, E 1e6, strain rate 100,
    the reference's cloth settings StiffGIPC/gl_main.cu:650-667) lying 0.5 d-hat above
    a soft 0.1 m cube (n_cube^3 lattice) that rests 0.5 d-hat above the ground, the sheet
    overhanging on every side.  Exercises the membrane, quadratic bending, cloth-solid
    barrier and friction terms together (a small stand-in for the cloth-over-sphere scene).
    """
    dhat_abs = 1e-3
    gap = 0.5 * dhat_abs
    v0, t0 = lattice_tets(n_cube, 0.1, (0.05, GROUND_OFFSET + gap, 0.05))
    vc, tc = cloth_grid(n_cloth, 0.2, (0.0, GROUND_OFFSET + 2 * gap + 0.1, 0.0))
    sc = build_tet_scene("cloth%d_cube%d" % (n_cloth, n_cube),
                         [dict(verts=v0, tets=t0, E=1e5), dict(verts=vc, tris=tc)],
                         dt=0.01, dhat_abs=dhat_abs, density=1000.0, nu=0.49, mu_friction=friction,
                         seed=seed, perturb=1e-5)
    from . import contacts
    contacts.attach_contacts(sc)
    return sc


def sphere_tets(n_cells: int = 4000, radius: float = 0.3, center=(0.0, 0.0, 0.0)):
    """A tet ball: the n_cells cells of a regular lattice whose centres lie nearest the ball's
    centre (ties by index), 5 tets each, the lattice spacing chosen so that n_cells cells fill
    the ball's volume.  Returns (verts, tets) with the unused lattice vertices dropped."""
    h = radius * (4.0 * math.pi / 3.0 / n_cells) ** (1.0 / 3.0)
    n = int(math.ceil(2.0 * radius / h)) + 2
    c0 = np.asarray(center, np.float64) - 0.5 * n * h
    verts, tets = lattice_tets(n + 1, n * h, c0)
    ncell = n ** 3
    cc = np.arange(n)
    ci, cj, ck = np.meshgrid(cc, cc, cc, indexing="ij")
    centre = c0 + h * (np.stack([ci.ravel(), cj.ravel(), ck.ravel()], 1) + 0.5)
    d = np.linalg.norm(centre - np.asarray(center), axis=1)
    keep = np.sort(np.argsort(d, kind="stable")[:n_cells])
    # lattice_tets lists the 5 tets of each split as whole-lattice blocks: tet k * ncell + c
    t = tets.reshape(5, ncell, 4)[:, keep].reshape(-1, 4)
    used, inv = np.unique(t, return_inverse=True)
    return verts[used], inv.reshape(-1, 4).astype(np.int32)


def cloth_roll(n: int = 256, length: float = 1.0, r0: float = 0.05, spacing: float = 4e-4,
               center=(0.0, 0.0, 0.0)):
    """An n x n cloth grid (length x length, :func:`cloth_grid`) rolled without stretch into
    an Archimedean spiral r = r0 + spacing theta / 2 pi about an axis along z through centre:
    the rows follow the spiral, so each layer lies ``spacing`` from the next.  With spacing
    below d-hat every layer is in contact with its neighbours (dense self-contact) and none
    crosses another.  Returns (verts, tris); the rest shape is the flat grid."""
    flat, tris = cloth_grid(n, length)
    a = spacing / (2.0 * math.pi)
    s = flat[:, 0]
    theta = (np.sqrt(r0 * r0 + 2.0 * a * s) - r0) / a  # arc length r0 t + a t^2 / 2 = s
    r = r0 + a * theta
    c = np.asarray(center, np.float64)
    verts = np.stack([c[0] + r * np.cos(theta), c[1] + r * np.sin(theta), c[2] + flat[:, 2] - 0.5 * length], 1)
    return verts, tris, flat


def scene_cloth_on_sphere(n_cloth: int = 256, sphere_cells: int = 4000, seed: int = 2,
                          friction: float = 0.2, contacts: bool = True) -> Scene:
    """The cloth-on-sphere workload: a 256 x 256 cloth (130 050 triangles; 1 m square, thickness 1 mm, membrane
    E 1e6 Pa, bending stiffness 1e-4) over a tet sphere (20 000 tets, radius 0.3 m, E 1e5 Pa)
    resting 0.5 d-hat above the ground, d-hat 5e-4 m.  The cloth lies rolled (:func:`cloth_roll`,
    layers 0.4 mm apart, about three turns) with its lowest layer 0.5 d-hat above the sphere's
    top and falls at 0.5 m/s: every layer touches the next, the dense self-contact of a draped,
    folded sheet.  Smaller n_cloth / sphere_cells give the same scene at parity-test sizes.
    With contacts=False the contact and friction arrays are left empty, for a caller that
    finds them on the GPU (``GIPC.buildCP`` and ``GIPC.buildFrictionSets``)."""
    dhat_abs = 5e-4
    radius = 0.3
    ctr = np.array([0.0, GROUND_OFFSET + radius + 0.5 * dhat_abs, 0.0])
    sv, st = sphere_tets(sphere_cells, radius, ctr)
    # the lattice's extent is not the ball's: put its lowest vertex 0.5 d-hat above the ground
    sv = sv + np.array([0.0, GROUND_OFFSET + 0.5 * dhat_abs - float(sv[:, 1].min()), 0.0])
    top = float(sv[:, 1].max())
    length = 1.0 * n_cloth / 256.0 if n_cloth < 256 else 1.0
    r0 = length / (2.0 * math.pi * 3.2)  # about three turns at any size
    spacing = 4e-4
    turns_r = r0 + spacing / (2 * math.pi) * ((math.sqrt(r0 * r0 + 2 * spacing / (2 * math.pi) * length) - r0)
                                             / (spacing / (2 * math.pi)))
    roll_c = (0.0, top + turns_r + 0.5 * dhat_abs, 0.0)
    cv, ct, flat = cloth_roll(n_cloth, length, r0, spacing, roll_c)
    bodies = [dict(verts=sv, tets=st, E=1e5), dict(verts=cv, tris=ct, velocity=(0.0, -0.5, 0.0), rest=flat)]
    sc = build_tet_scene("cloth%d_sphere%d" % (n_cloth, len(st)), bodies, dt=0.01, dhat_abs=dhat_abs,
                         density=1000.0, nu=0.4, mu_friction=friction, seed=seed, perturb=1e-6,
                         cloth=dict(thickness=1e-3, E=1e6, density=200.0, strain_rate=100.0, bend_E=1e5))
    sc.params["bendStiff"] = 1e-4
    if contacts:
        from . import contacts as _contacts
        _contacts.attach_contacts(sc)
    return sc


def scene_abd_boxes(nb: int = 500, seed: int = 3, edge: float = 0.05, density: float = 1000.0,
                    dt: float = 0.01, kappa_abd: float = 1e8) -> dict:
    """Affine bodies of the ABD configuration: nb boxes of 8 points and 5 tets (the
    2x2x2 lattice split), edge 0.05 m, at seeded positions in a 1 m cube, kappa_ABD 1e8
    (StiffGIPC/gipc/gipc.cu:18).  Returns the ABDSystem inputs: point_body, x_bar (points
    relative to the body centroid), the lumped dyadic mass (each tet's mass / 4 at its
    corners, abd_system.cu:527-600), volume, boundary_type, and one Newton iterate q
    (translation + slightly perturbed identity rows) with its q_tilde (gravity on the
    translation), plus the world positions x = J q."""
    rng = np.random.default_rng(seed)
    v, t = lattice_tets(2, edge)
    v = v - v.mean(0)
    _, vol_t = tet_rest_data(v, t)
    node_m = np.zeros(8)
    np.add.at(node_m, t.ravel(), np.repeat(vol_t * density / 4.0, 4))
    dm = np.concatenate([[node_m.sum()], (node_m[:, None] * v).sum(0),
                         np.einsum("p,pi,pj->ij", node_m, v, v).ravel()])
    point_body = np.repeat(np.arange(nb), 8).astype(np.int32)
    x_bar = np.tile(v, (nb, 1))
    centres = rng.uniform(0.0, 1.0, (nb, 3))
    A = np.eye(3)[None] + rng.normal(scale=1e-3, size=(nb, 3, 3))
    q = np.concatenate([centres, A.reshape(nb, 9)], 1)
    vel = rng.normal(scale=0.1, size=(nb, 3))
    q_prev = q.copy()
    q_prev[:, :3] -= dt * vel
    q_tilde = q_prev.copy()
    q_tilde[:, :3] += dt * vel + dt * dt * np.asarray(GRAVITY)
    x = (np.einsum("bij,bpj->bpi", A, x_bar.reshape(nb, 8, 3)) + centres[:, None]).reshape(-1, 3)
    return dict(point_body=point_body, x_bar=x_bar, dyadic_mass=np.tile(dm, (nb, 1)),
                volume=np.full(nb, vol_t.sum()), boundary_type=np.zeros(nb, np.int32),
                q=q, q_tilde=q_tilde, x=x, dt=dt, kappa=kappa_abd)


def scene_abd_on_bed(nb: int = 500, cells=(50, 8, 50), seed: int = 4, edge: float = 0.05, density: float = 1000.0,
                     dt: float = 0.01, kappa_abd: float = 1e8, dhat_abs: float = 1e-3, resting: float = 0.3,
                     bed_E: float = 1e5, contacts: bool = True):
    """The affine-bodies-on-a-bed workload: nb boxes (8 points, 12 surface triangles, edge
    0.05 m, kappa_ABD 1e8) at seeded positions over a soft tet bed (cells[0] x cells[1] x
    cells[2] lattice cells of 5 tets over a 1 m square, 100 000 tets by default, E 1e5 Pa)
    lying 0.5 d-hat above the ground.  A share ``resting`` of the boxes sits flat with its
    bottom 0.5 d-hat above the bed, the others are spread, without overlap, over the metre
    above it and fall at seeded velocities.

    Returns (scene, bodies).  In the scene the bed's vertices come first and the boxes' points
    follow from ``bodies["abd_first"]`` on, marked Dirichlet: their rows hold only the kept
    mass diagonal, and the contact terms that touch them go to the bodies through
    ``GIPC.contactPartition``.  ``bodies`` holds the ABDSystem inputs of
    :func:`scene_abd_boxes` with the points in the scene's order.  With contacts=False the
    contact arrays are left empty for the GPU pair search (body ids: the bed 0, box b b+1)."""
    rng = np.random.default_rng(seed)
    h = 1.0 / cells[0]
    base = GROUND_OFFSET + 0.5 * dhat_abs
    bv, bt = box_lattice_tets((cells[0] + 1, cells[1] + 1, cells[2] + 1), h, (0.0, base, 0.0))
    top = base + cells[1] * h
    cv, ct = lattice_tets(2, edge)
    cv = cv - cv.mean(0)
    cs_tris, _, _ = tet_surface(ct)
    _, vol_t = tet_rest_data(cv, ct)
    node_m = np.zeros(8)
    np.add.at(node_m, ct.ravel(), np.repeat(vol_t * density / 4.0, 4))
    dm = np.concatenate([[node_m.sum()], (node_m[:, None] * cv).sum(0),
                         np.einsum("p,pi,pj->ij", node_m, cv, cv).ravel()])
    # box centres: resting ones on the bed, the others in the metre above, no two within
    # edge + 2 d-hat of each other along every axis (boxes stay axis-aligned to within 1e-3)
    gap = edge + 2.0 * dhat_abs
    cen, rest_flag = [], []
    tries = 0
    while len(cen) < nb:
        tries += 1
        if tries > 200000:
            raise ValueError("no room for %d boxes" % nb)
        on = rng.uniform() < resting
        c = np.array([rng.uniform(0.5 * edge, 1.0 - 0.5 * edge),
                      top + 0.5 * dhat_abs + 0.5 * edge if on else rng.uniform(top + edge, top + 1.0),
                      rng.uniform(0.5 * edge, 1.0 - 0.5 * edge)])
        if cen:
            d = np.abs(np.asarray(cen) - c)
            if np.any((d < gap).all(1)):
                continue
        cen.append(c)
        rest_flag.append(on)
    cen = np.asarray(cen)
    rest_flag = np.asarray(rest_flag)
    A = np.tile(np.eye(3), (nb, 1, 1))
    fly = ~rest_flag
    A[fly] += rng.normal(scale=1e-3, size=(int(fly.sum()), 3, 3))
    vel = np.where(rest_flag[:, None], 0.0, rng.normal(scale=0.1, size=(nb, 3)))
    q = np.concatenate([cen, A.reshape(nb, 9)], 1)
    q_prev = q.copy()
    q_prev[:, :3] -= dt * vel
    q_tilde = q_prev.copy()
    q_tilde[:, :3] += dt * vel + dt * dt * np.asarray(GRAVITY)
    pts = np.einsum("bij,pj->bpi", A, cv) + cen[:, None]  # (nb, 8, 3)
    bodies_in = [dict(verts=bv, tets=bt, E=bed_E)]
    bodies_in += [dict(verts=pts[b], tris=cs_tris, affine=True) for b in range(nb)]
    sc = build_tet_scene("abd%d_bed%d" % (nb, len(bt)), bodies_in, dt=dt, dhat_abs=dhat_abs, density=density,
                         nu=0.4, mu_friction=0.0, seed=seed, perturb=0.0)
    nbed = len(bv)
    body = sc.body_of_vertex.astype(np.int64)
    if not (body[:nbed] == 0).all() or not (body[nbed:] > 0).all():
        raise AssertionError("the bed's vertices must come first")
    # each scene point: its box and its corner (matched by position; the corners are distinct)
    pb = body[nbed:] - 1
    x = sc.vertexes[nbed:]
    corner = np.argmin(((pts[pb] - x[:, None, :]) ** 2).sum(2), 1)
    bodies = dict(point_body=pb.astype(np.int32), x_bar=cv[corner], dyadic_mass=np.tile(dm, (nb, 1)),
                  volume=np.full(nb, vol_t.sum()), boundary_type=np.zeros(nb, np.int32), q=q, q_tilde=q_tilde,
                  x=x.copy(), dt=dt, kappa=kappa_abd, abd_first=nbed, resting=rest_flag)
    if contacts:
        from . import contacts as _contacts
        _contacts.attach_contacts(sc)
    return sc, bodies


SCENES = {
    "cube": scene_cube,
    "two_cubes": scene_two_cubes,
    "cloth_on_cube": scene_cloth_on_cube,
}
