"""Mesh and partition files (``sgipc.meshio``) and scenes built from them.

* Round trips of the three formats the reference reads (.msh tet meshes, .obj cloths with
  polygons fanned into triangles, .part MAS partitions).
* The partition: parts of 16 vertices (one remainder part per body), deterministic, a
  renumbering part by part, the setMAS_partition maps, and an edge cut far below a random
  assignment's.
* The reference's own sorted meshes and their METIS .part files, where a checkout is present:
  they parse, their part maps hold at most 16 vertices per bank, and this partition's edge cut
  on the same meshes is compared with METIS's.
* A scene built from files assembles an SPD system with a connected MAS hierarchy.
"""
import os
import sys

import numpy as np
import pytest

import oracle
from sgipc import meshio, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ref_build  # noqa: E402  (only for the location of a reference checkout)

ASSETS = os.path.join(ref_build.CHECKOUT, "Assets", "sorted_mesh")


def _cube(n=6):
    v, t = scenes.lattice_tets(n, 0.1, (0.0, 0.0, 0.0))
    return np.asarray(v, np.float64), np.asarray(t, np.int32)


def _edges(elems):
    e = np.asarray(elems, np.int64)
    k = e.shape[1]
    pairs = np.concatenate([e[:, [a, b]] for a in range(k) for b in range(a + 1, k)])
    return np.unique(np.sort(pairs, 1), axis=0)


def test_msh_round_trip(tmp_path):
    v, t = _cube()
    p = str(tmp_path / "cube.msh")
    meshio.write_msh(p, v, t)
    v2, t2 = meshio.read_msh(p)
    assert np.array_equal(v2, v) and np.array_equal(t2, t)
    T = np.eye(4)
    T[:3, 3] = (1.0, -2.0, 0.5)
    T[0, 0] = 2.0
    v3, _ = meshio.read_msh(p, T)
    assert np.allclose(v3, v * [2.0, 1.0, 1.0] + [1.0, -2.0, 0.5], rtol=0, atol=1e-15)


def test_obj_fans_polygons_and_reads_slashed_tokens(tmp_path):
    p = tmp_path / "quad.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvn 0 0 1\n"
                 "f 1/1/1 2/2/1 3/3/1 4/4/1\nf 1//1 3//1 4//1\n")
    v, f = meshio.read_obj(str(p))
    assert v.shape == (4, 3)
    assert f.tolist() == [[0, 1, 2], [0, 2, 3], [0, 2, 3]]
    g, _ = scenes.cloth_grid(5, 0.2)
    q = str(tmp_path / "cloth.obj")
    tris = scenes.cloth_grid(5, 0.2)[1]
    meshio.write_obj(q, g, tris)
    g2, t2 = meshio.read_obj(q)
    assert np.array_equal(g2, g) and np.array_equal(t2, tris)


def test_parts_round_trip_and_count_check(tmp_path):
    p = str(tmp_path / "a.part")
    parts = np.repeat(np.arange(5), 16)[:70]
    meshio.write_parts(p, parts)
    assert np.array_equal(meshio.read_parts(p, 70), parts)
    with pytest.raises(ValueError):
        meshio.read_parts(p, 71)


def test_partition_blocks_order_and_maps():
    v, t = _cube(11)
    parts = meshio.partition(v)
    counts = np.bincount(parts)
    assert (counts == 16).sum() == len(counts) - 1 and counts[-1] == len(v) - 16 * (len(counts) - 1)
    assert np.array_equal(parts, meshio.partition(v))  # deterministic
    v2, t2, p2 = meshio.sorted_copy(v, t, parts)
    assert (np.diff(p2) >= 0).all()
    pm, rm = meshio.part_maps(p2)
    assert len(pm) == 16 * (p2.max() + 1)
    assert np.array_equal(pm[rm], np.arange(len(v2)))
    # setMAS_partition: part q's vertices take positions 16 q, 16 q + 1, ... in order
    for q in (0, 5, int(p2.max())):
        ids = np.nonzero(p2 == q)[0]
        assert np.array_equal(pm[16 * q:16 * q + len(ids)], ids)
        assert (pm[16 * q + len(ids):16 * (q + 1)] == -1).all()
    # spatially compact parts: far fewer cut edges than a random assignment of the same sizes
    rng = np.random.default_rng(0)
    e = _edges(t)
    assert meshio.edge_cut(parts, e) < 0.65 * meshio.edge_cut(rng.permutation(parts), e)
    with pytest.raises(ValueError):
        meshio.part_maps(np.zeros(17, np.int64))


def test_scene_from_files_assembles_spd_system(tmp_path):
    v, t = _cube(5)
    msh = str(tmp_path / "cube.msh")
    meshio.write_msh(msh, v, t)
    T = np.eye(4)
    T[1, 3] = -1.0 + 5e-4  # resting 0.5 d-hat above the ground plane y = -1
    sc = scenes.scene_from_files([dict(mesh=msh, transform=T, E=1e5)], perturb=1e-5, seed=3)
    assert sc.nv == len(v) and sc.nt == len(t)
    assert len(sc.ground_pairs) > 0
    b, rows, cols, vals, _ = oracle.assemble(sc)
    A = oracle.dense(rows, cols, vals, sc.nv)
    assert np.allclose(A, A.T, rtol=0, atol=1e-12 * np.abs(A).max())
    assert np.linalg.eigvalsh(A).min() > 0
    m = oracle.Mas(sc, rows, cols, vals)
    L, _, counts, _ = m.info()
    assert L >= 2 and counts[0] == len(sc.part_map_real)
    # the same mesh with an explicit part file: the numbering and maps follow the file
    parts = meshio.partition(v)
    v2, t2, p2 = meshio.sorted_copy(v, t, parts)
    msh2, prt = str(tmp_path / "cube_sorted.16.msh"), str(tmp_path / "cube_sorted.16.part")
    meshio.write_msh(msh2, v2, t2)
    meshio.write_parts(prt, p2)
    sc2 = scenes.scene_from_files([dict(mesh=msh2, part=prt, transform=T, E=1e5)])
    assert np.array_equal(sc2.part_map_real, meshio.part_maps(p2)[0])


@pytest.mark.skipif(not os.path.isdir(ASSETS), reason="no reference checkout")
@pytest.mark.parametrize("name", ["cube_sorted.16.msh", "bunny2_sorted.16.msh", "cloth_high_sorted.16.obj"])
def test_reference_sorted_meshes_and_their_partitions(name):
    """The reference's METIS-sorted meshes parse with their .part files; every bank holds at
    most 16 vertices; and this project's partition cuts no more edges than METIS's by more
    than a third on the same meshes."""
    path = os.path.join(ASSETS, name)
    verts, elems, parts = meshio.load_body(path, os.path.splitext(path)[0] + ".part")
    assert len(verts) == len(parts) and elems.max() < len(verts)
    pm, rm = meshio.part_maps(parts)
    assert np.array_equal(pm[rm], np.arange(len(verts)))
    if len(verts) > 64:
        e = _edges(elems)
        ours = meshio.edge_cut(meshio.partition(verts), e)
        metis = meshio.edge_cut(parts, e)
        assert ours < 1.34 * metis, (ours, metis)
