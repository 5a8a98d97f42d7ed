"""Mesh and partition files of StiffGIPC scenes.

The reference reads Gmsh 2.2 tetrahedral meshes (``.msh``), Wavefront triangle meshes
(``.obj``) and the MAS partition files (``.part``) that its METIS step writes beside the
vertex-sorted copies of the meshes (``*_sorted.16.msh / .obj / .part``):

* :func:`read_msh` follows ``tetrahedra_obj::load_tetrahedraMesh`` (StiffGIPC/load_mesh.cpp:
  481-636): the ``$Nodes`` block (a count, then ``id x y z`` lines) and the ``$Elements`` block
  (a count, then lines whose last four integers are the 1-based tet vertices), with the
  optional 4 x 4 affine transform applied to every node;
* :func:`read_obj` follows ``load_triMesh`` (load_mesh.cpp:102-384): ``v x y z`` lines, and
  ``f`` lines whose polygons are fanned into triangles (first, k - 1, k), each vertex token's
  first integer being the 1-based vertex (``i``, ``i/j``, ``i/j/k``, ``i//k``);
* :func:`read_parts` follows ``load_parts`` (load_mesh.cpp:447-479): one part id per vertex;
* :func:`part_maps` follows ``setMAS_partition`` (StiffGIPC/gl_main.cu:1066-1093): part p owns
  MAS positions 16 p .. 16 p + 15, filled by its vertices in order, the rest padding (-1).

:func:`partition` stands in for the METIS k-way step of ``metis_sort``
(MeshProcess/metis_partition/src/metis_sort.cpp:25-219), which cuts a mesh into parts of at
most 16 vertices and renumbers the vertices part by part.  METIS is not part of this project;
here the parts come from recursive coordinate bisection: a vertex set is split across its
widest extent so that the first half takes a whole number of 16-vertex blocks, until one block
remains.  Every part then holds exactly 16 vertices except a body's last one, and the parts are
spatially compact, which is what the MAS's 16-node banks need.  :func:`sort_by_parts` renumbers a
mesh part by part, as the ``_sorted`` files are.
"""
from __future__ import annotations

import os
from typing import Optional, Tuple

import numpy as np

BANK = 16


def _transform(points: np.ndarray, transform: Optional[np.ndarray]) -> np.ndarray:
    if transform is None:
        return points
    T = np.asarray(transform, np.float64).reshape(4, 4)
    return points @ T[:3, :3].T + T[:3, 3]


# ------------------------------------------------------------------------------------------
# reading
# ------------------------------------------------------------------------------------------

def read_msh(path: str, transform: Optional[np.ndarray] = None) -> Tuple[np.ndarray, np.ndarray]:
    """(vertices (N, 3) float64, tets (T, 4) int32, 0-based) of a Gmsh 2.2 ASCII mesh."""
    with open(path) as f:
        lines = f.read().splitlines()
    verts, tets = None, None
    i = 0
    while i < len(lines):
        line = lines[i].strip()
        if line == "$Nodes":
            n = int(lines[i + 1].split()[0])
            rows = [lines[i + 2 + k].split() for k in range(n)]
            verts = np.array([[float(r[1]), float(r[2]), float(r[3])] for r in rows], np.float64).reshape(-1, 3)
            i += 2 + n
            continue
        if line == "$Elements":
            n = int(lines[i + 1].split()[0])
            rows = [lines[i + 2 + k].split() for k in range(n)]
            tets = np.array([[int(t) - 1 for t in r[-4:]] for r in rows], np.int64).reshape(-1, 4)
            break  # the reference stops at the first element block
        i += 1
    if verts is None or tets is None:
        raise ValueError("%s: no $Nodes / $Elements block" % path)
    if len(tets) and (tets.min() < 0 or tets.max() >= len(verts)):
        raise ValueError("%s: an element names a node that does not exist" % path)
    return _transform(verts, transform), tets.astype(np.int32)


def read_obj(path: str, transform: Optional[np.ndarray] = None) -> Tuple[np.ndarray, np.ndarray]:
    """(vertices (N, 3) float64, triangles (F, 3) int32, 0-based) of a Wavefront mesh;
    polygons are fanned into triangles."""
    verts, tris = [], []
    with open(path) as f:
        for line in f:
            if line.startswith("v "):
                p = line.split()
                verts.append((float(p[1]), float(p[2]), float(p[3])))
            elif line.startswith("f "):
                ids = [int(t.split("/")[0]) - 1 for t in line.split()[1:]]
                for k in range(2, len(ids)):
                    tris.append((ids[0], ids[k - 1], ids[k]))
    V = np.array(verts, np.float64).reshape(-1, 3)
    F = np.array(tris, np.int64).reshape(-1, 3)
    if len(F) and (F.min() < 0 or F.max() >= len(V)):
        raise ValueError("%s: a face names a vertex that does not exist" % path)
    return _transform(V, transform), F.astype(np.int32)


def read_parts(path: str, vertex_num: Optional[int] = None) -> np.ndarray:
    """Part id of every vertex (int32).  A count other than vertex_num is an error, as in
    load_parts."""
    with open(path) as f:
        parts = np.array(f.read().split(), np.int64)
    if vertex_num is not None and len(parts) != vertex_num:
        raise ValueError("%s: %d part ids for %d vertices" % (path, len(parts), vertex_num))
    return parts.astype(np.int32)


# ------------------------------------------------------------------------------------------
# writing
# ------------------------------------------------------------------------------------------

def write_msh(path: str, verts: np.ndarray, tets: np.ndarray) -> None:
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(verts))
        for k, p in enumerate(np.asarray(verts, np.float64)):
            f.write("%d %.17g %.17g %.17g\n" % (k + 1, p[0], p[1], p[2]))
        f.write("$EndNodes\n$Elements\n%d\n" % len(tets))
        for k, t in enumerate(np.asarray(tets, np.int64)):
            f.write("%d 4 0 %d %d %d %d\n" % (k + 1, t[0] + 1, t[1] + 1, t[2] + 1, t[3] + 1))
        f.write("$EndElements\n")


def write_obj(path: str, verts: np.ndarray, tris: np.ndarray) -> None:
    with open(path, "w") as f:
        for p in np.asarray(verts, np.float64):
            f.write("v %.17g %.17g %.17g\n" % (p[0], p[1], p[2]))
        for t in np.asarray(tris, np.int64):
            f.write("f %d %d %d\n" % (t[0] + 1, t[1] + 1, t[2] + 1))


def write_parts(path: str, parts: np.ndarray) -> None:
    with open(path, "w") as f:
        f.write("\n".join(str(int(p)) for p in parts) + "\n")


# ------------------------------------------------------------------------------------------
# partition
# ------------------------------------------------------------------------------------------

def partition(points: np.ndarray, block: int = BANK) -> np.ndarray:
    """Part id (int32, 0-based, in bisection order) of every point: recursive coordinate
    bisection into parts of ``block`` points, the last part taking the remainder."""
    pts = np.asarray(points, np.float64)
    n = len(pts)
    part = np.empty(n, np.int32)
    next_id = 0
    stack = [np.arange(n)]
    while stack:
        ids = stack.pop()
        if len(ids) <= block:
            part[ids] = next_id
            next_id += 1
            continue
        nb = (len(ids) + block - 1) // block
        left = ((nb + 1) // 2) * block
        span = pts[ids].max(0) - pts[ids].min(0)
        axis = int(np.argmax(span))
        # stable order along the axis (ties by index): a deterministic split
        order = ids[np.lexsort((ids, pts[ids, axis]))]
        stack.append(order[left:])   # popped second
        stack.append(order[:left])   # popped first: part ids follow the bisection order
    return part


def sort_by_parts(parts: np.ndarray) -> np.ndarray:
    """Permutation listing the vertices part by part (stable within a part): new vertex k is
    old vertex perm[k], as in metis_sort's sorted meshes."""
    return np.argsort(np.asarray(parts), kind="stable").astype(np.int64)


def part_maps(parts: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """``setMAS_partition`` (StiffGIPC/gl_main.cu:1066-1093) for part ids listed part by part:
    partId_map_real (16 positions per part, vertex or -1) and real_map_partId (position of every
    vertex).  Vertices of a part take its positions in order; a part of more than 16 vertices
    is an error (the MAS banks hold 16)."""
    parts = np.asarray(parts, np.int64)
    n = len(parts)
    if n == 0:
        return np.zeros(0, np.int32), np.zeros(0, np.int32)
    if np.any(np.diff(parts) < 0):
        raise ValueError("part ids must be listed part by part (a sorted mesh)")
    nparts = int(parts[-1]) + 1
    part_map = np.full(nparts * BANK, -1, np.int64)
    start = np.r_[0, np.nonzero(np.diff(parts))[0] + 1]
    index = np.arange(n) - np.repeat(start, np.diff(np.r_[start, n]))
    if index.max() >= BANK:
        raise ValueError("a part holds more than %d vertices" % BANK)
    part_map[BANK * parts + index] = np.arange(n)
    real_map = np.empty(n, np.int64)
    pos = np.nonzero(part_map >= 0)[0]
    real_map[part_map[pos]] = pos
    return part_map.astype(np.int32), real_map.astype(np.int32)


def edge_cut(parts: np.ndarray, edges: np.ndarray) -> float:
    """Fraction of mesh edges whose ends lie in different parts (the partition's cut)."""
    e = np.asarray(edges)
    return float(np.mean(parts[e[:, 0]] != parts[e[:, 1]])) if len(e) else 0.0


def sorted_copy(verts: np.ndarray, elems: np.ndarray, parts: np.ndarray):
    """(vertices, elements, part ids) renumbered part by part."""
    perm = sort_by_parts(parts)
    inv = np.empty(len(perm), np.int64)
    inv[perm] = np.arange(len(perm))
    return verts[perm], inv[np.asarray(elems, np.int64)].astype(np.int32), np.asarray(parts)[perm]


def load_body(path: str, part_path: Optional[str] = None, transform: Optional[np.ndarray] = None):
    """(vertices, elements, part ids) of one mesh file, renumbered part by part: with a
    ``.part`` file (the mesh is then already sorted, as the reference's ``_sorted`` meshes are)
    its ids, otherwise a :func:`partition` of the vertices."""
    ext = os.path.splitext(path)[1].lower()
    verts, elems = (read_msh if ext == ".msh" else read_obj)(path, transform)
    if part_path is not None:
        parts = read_parts(part_path, len(verts))
        parts = parts - parts.min() if len(parts) else parts
        return verts, elems, parts
    return sorted_copy(verts, elems, partition(verts))
