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
    g = np.linspace(0.0, size, n)
    ii, jj, kk = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    verts = np.stack([g[ii.ravel()], g[jj.ravel()], g[kk.ravel()]], 1) + np.asarray(origin)

    def vid(i, j, k):
        return (i * n + j) * n + k

    c = np.arange(n - 1)
    ci, cj, ck = np.meshgrid(c, c, c, indexing="ij")
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

def _empty_cloth():
    return dict(tris=np.zeros((0, 3), np.int32), tri_dm_inv=np.zeros((0, 2, 2)),
                area=np.zeros(0), hinges=np.zeros((0, 2), np.int32),
                hinge_adj=np.zeros((0, 2), np.int32), hinge_q=np.zeros((0, 4, 4)))


def build_tet_scene(name: str, bodies: List[dict], dt: float, dhat_abs: float, density: float,
                    nu: float, mu_friction: float, seed: int, perturb: float,
                    kappa: Optional[float] = None) -> Scene:
    """Concatenate tet bodies, derive ``initFEM`` data and set up one Newton iterate.

    Each body dict holds ``verts``, ``tets``, ``E`` and optional ``velocity`` (3,) and
    ``boundary`` flag.  Vertex positions of the current iterate are the rest lattice plus
    a seeded uniform perturbation of ``perturb`` metres.
    """
    rng = np.random.default_rng(seed)
    verts, tets, youngs, vel, btype, body_id = [], [], [], [], [], []
    off = 0
    for b, body in enumerate(bodies):
        v = np.asarray(body["verts"], np.float64)
        t = np.asarray(body["tets"], np.int64) + off
        verts.append(v)
        tets.append(t)
        youngs.append(np.full(len(t), float(body["E"])))
        vel.append(np.tile(np.asarray(body.get("velocity", (0.0, 0.0, 0.0)), np.float64), (len(v), 1)))
        btype.append(np.full(len(v), int(body.get("boundary", 0)), np.int32))
        body_id.append(np.full(len(v), b, np.int32))
        off += len(v)
    rest = np.concatenate(verts)
    tets = np.concatenate(tets).astype(np.int32)
    youngs = np.concatenate(youngs)
    vel = np.concatenate(vel)
    btype = np.concatenate(btype)
    body_id = np.concatenate(body_id)
    nv = rest.shape[0]

    # renumber vertices in MAS part order, as the METIS-sorted meshes are, so that
    # real_map_partId is monotone (the reference's level-0 scatter assumes it,
    # StiffGIPC/MASPreconditioner.cu:1856-1867)
    part_map, _ = mas_partition(rest, body_id)
    perm = part_map[part_map >= 0].astype(np.int64)
    inv = np.empty(nv, np.int64)
    inv[perm] = np.arange(nv)
    rest, vel, btype, body_id = rest[perm], vel[perm], btype[perm], body_id[perm]
    tets = inv[tets].astype(np.int32)

    dm_inv, vol = tet_rest_data(rest, tets)
    lr, vr = snk_rates(youngs, nu)
    masses = np.zeros(nv)
    np.add.at(masses, tets.ravel(), np.repeat(vol * density / 4.0, 4))

    x_prev = rest + rng.uniform(-perturb, perturb, rest.shape)
    x = x_prev.copy()
    g = np.asarray(GRAVITY)
    xt = x_prev + dt * vel + np.where(btype[:, None] == 0, dt * dt * g[None, :], 0.0)

    stris, sedges, sverts = tet_surface(tets)
    nbr_start, nbr_list = neighbour_csr(nv, tets, np.zeros((0, 3), np.int32))
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
                  stretchStiff=0.0, shearStiff=0.0, strainRate=0.0, bendStiff=0.0,
                  motionRate=0.0, softRate=0.0, density=density, meanMass=mean_mass)
    return Scene(name=name, vertexes=x, o_vertexes=x_prev.copy(), rest_vertexes=rest,
                 xTilta=xt, velocities=vel, masses=masses, boundary_type=btype, tets=tets,
                 dm_inv=dm_inv, volum=vol, length_rate=lr, volume_rate=vr, youngs=youngs,
                 poisson=nu, surf_tris=stris, surf_edges=sedges, surf_verts=sverts,
                 body_of_vertex=body_id, part_map_real=part_map, real_map_part=real_map,
                 nbr_start=nbr_start, nbr_list=nbr_list, params=params, **_empty_cloth())


def scene_cube(n: int = 11, touching: bool = False, seed: int = 0) -> Scene:
    """Config C1: one 0.1 m soft cube (n^3 lattice) dropped from 0.05 m (or touching)."""
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
    """Config C2: two stacked n^3 cubes, E = 1e5 / 1e6, nu = 0.45, mu = 0.2.

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


SCENES = {
    "cube": scene_cube,
    "two_cubes": scene_two_cubes,
}
