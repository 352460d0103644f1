"""Boundary regions, force fields, the JSON configuration and mesh files
(boundary/BoundaryCondition.h, config_parser.cpp): known answers on CPU, and the
mesh-driven set-up (buildGrids(coords, trifaces)) on the GPU."""
import json
import os
import struct

import numpy as np
import pytest

from robtop_b200 import boundary as B
from robtop_b200 import configs


def test_sphere_open_closed_complement():
    P = np.array([[0, 0, 0], [1, 0, 0], [1 + 1e-12, 0, 0], [0, 0, 1.5]], np.float64)
    assert B.Sphere((0, 0, 0), 1.0).contains(P).tolist() == [True, False, False, False]
    assert B.Sphere((0, 0, 0), 1.0, closed=True).contains(P).tolist() == [True, True, True, False]
    assert B.Sphere((0, 0, 0), 1.0, complement=True).contains(P).tolist() == [False, True, True, True]


def test_box_corners_in_any_order():
    P = np.array([[0.5, 0.5, 0.5], [1, 0.5, 0.5], [2, 0.5, 0.5]], np.float64)
    b = B.Box((1, 1, 1), (0, 0, 0))  # corners given max-first
    assert b.contains(P).tolist() == [True, False, False]
    assert B.Box((0, 0, 0), (1, 1, 1), closed=True).contains(P).tolist() == [True, True, False]


def test_halfspace_orientation():
    """Plane through p1, p2, p3; the positive side is where (p2 - p1) x (p3 - p1) points."""
    h = B.HalfSpace((0, 0, 36.8), (1, 0, 36.8), (0, 1, 36.8))  # normal +z
    P = np.array([[5, 5, 40], [5, 5, 36.8], [5, 5, 30]], np.float64)
    assert h.contains(P).tolist() == [True, False, False]
    assert B.HalfSpace((0, 0, 36.8), (1, 0, 36.8), (0, 1, 36.8), closed=True).contains(P).tolist() == [True, True, False]
    assert B.HalfSpace((0, 0, 36.8), (0, 1, 36.8), (1, 0, 36.8)).contains(P).tolist() == [False, False, True]


def test_cylinder_and_union():
    c = B.Cylinder((0, 0, 0), 1.0, (0, 0, 2))
    P = np.array([[0, 0, 1], [0.99, 0, 0], [0, 0, 2.01], [1.0, 0, 1], [0, 0, -0.01]], np.float64)
    assert c.contains(P).tolist() == [True, True, False, False, False]
    u = B.Union([B.Sphere((5, 0, 0), 1), c])
    assert u.contains(np.array([[5, 0, 0], [0, 0, 1], [3, 0, 0]], np.float64)).tolist() == [True, True, False]
    assert not B.Union().contains(np.zeros((1, 3))).any()


def test_force_fields():
    reg = {"type": "sphere", "center": [0, 0, 0], "radius": 10}
    P = np.array([[1.0, 2.0, 0.5], [20, 0, 0]])
    f = B.parse_field({"type": "const", "norm": 2.0, "direction": [0, 0, -3], "region": reg})
    np.testing.assert_allclose(f.at(P), [[0, 0, -2], [0, 0, 0]])
    f = B.parse_field({"type": "RadialNormConstDir", "center": [1, 2, 0], "direction": [1, 0, 0], "amplifier": 3,
                       "dampRatio": 0.5, "region": reg})
    r = np.linalg.norm(np.array([1, 2, 0]) - P[0])
    np.testing.assert_allclose(f.at(P)[0], [3 * np.exp(-r ** 1.0), 0, 0])
    f = B.parse_field({"type": "ConstNormRadialDir", "center": [1, 2, 3.5], "norm": 4, "region": reg})
    np.testing.assert_allclose(f.at(P)[0], [0, 0, 4])
    f = B.parse_field({"type": "Twist", "AxisStart": [0, 0, 0], "AxisEnd": [0, 0, 2], "amplifier": 0.5,
                       "region": reg})
    v = f.at(np.array([[2.0, 0, 1]]))[0]
    np.testing.assert_allclose(v, [0, -1.0, 0])  # (p - a) x (b - a) normalised, |(p - a) x axis| * 0.5 = 1
    assert B.parse_field({"type": "gradient", "region": reg}) is None
    with pytest.raises(ValueError):
        B.parse_field({"type": "spiral", "region": reg})


def test_parse_config_sums_fields_and_unions_regions(tmp_path):
    doc = {"model": "part.obj",
           "fixedarea": [{"type": "halfspace", "p1": [0, 0, 8], "p2": [1, 0, 8], "p3": [0, 1, 8]},
                         {"type": "box", "p": [0, 0, 0], "q": [1, 1, 1], "closed": True}],
           "loadarea": [{"type": "sphere", "center": [4, 4, 0], "radius": 2}],
           "force": [{"type": "const", "norm": 1, "direction": [0, 0, -1],
                      "region": {"type": "sphere", "center": [4, 4, 0], "radius": 2}},
                     {"type": "const", "norm": 2, "direction": [1, 0, 0],
                      "region": {"type": "box", "p": [3, 3, -1], "q": [5, 5, 1]}}]}
    path = tmp_path / "config1.json"
    path.write_text(json.dumps(doc))
    cfg = B.parse_config(str(path))
    P = np.array([[4, 4, 0.5], [0.5, 0.5, 0.5], [4, 4, 9], [7, 7, 4]], np.float64)
    assert cfg.fixed(P).tolist() == [False, True, True, False]
    assert cfg.load(P).tolist() == [True, False, False, False]
    np.testing.assert_allclose(cfg.force(P)[0], [2, 0, -1])
    assert cfg.model_path() == os.path.join(str(tmp_path), "part.obj")
    with pytest.raises(ValueError):
        B.parse_config({"fixedarea": [{"type": "torus"}]})


def test_mesh_readers_roundtrip(tmp_path):
    v, f = configs.box_mesh((0, 0, 0), (2, 1, 1))
    # OBJ with quads, texture/normal indices and a negative (relative) index
    obj = tmp_path / "box.obj"
    lines = ["# box"] + [f"v {x} {y} {z}" for x, y, z in v]
    quads = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (2, 3, 7, 6), (0, 4, 7, 3), (1, 2, 6, 5)]
    for q in quads:
        lines.append("f " + " ".join(f"{i + 1}/1/1" for i in q[:3]) + f" {q[3] - 8}")
    obj.write_text("\n".join(lines) + "\n")
    vo, fo = B.read_mesh(str(obj))
    np.testing.assert_array_equal(vo, v)
    assert fo.shape == (12, 3)
    # the fanned quads cover the same surface: equal signed volume
    vol = lambda V, F: np.einsum("ij,ij->i", V[F[:, 0]], np.cross(V[F[:, 1]], V[F[:, 2]])).sum() / 6  # noqa: E731
    assert abs(vol(vo.astype(float), fo) - 2.0) < 1e-6
    # binary and ASCII STL
    tri = v[f]
    stlb = tmp_path / "box_b.stl"
    with open(stlb, "wb") as fh:
        fh.write(b"\0" * 80 + struct.pack("<I", len(f)))
        for t in tri:
            fh.write(struct.pack("<12fH", 0, 0, 0, *t.reshape(-1), 0))
    stla = tmp_path / "box_a.stl"
    stla.write_text("solid box\n" + "".join(
        "facet normal 0 0 0\nouter loop\n" + "".join(f"vertex {x} {y} {z}\n" for x, y, z in t) + "endloop\nendfacet\n"
        for t in tri) + "endsolid box\n")
    for p in (stlb, stla):
        vs, fs = B.read_mesh(str(p))
        assert len(vs) == 8 and fs.shape == (12, 3)
        assert abs(vol(vs.astype(float), fs) - 2.0) < 1e-6


def test_closest_points_normals_and_shell():
    """Closest surface points against brute force, outward normals of a sphere mesh, and the
    shell elements of a box: those within shell_width element lengths of the surface."""
    v, f = configs.icosphere(2, (0, 0, 0), 1.0)
    rng = np.random.default_rng(3)
    P = rng.standard_normal((200, 3))
    P *= (rng.random(200) * 1.6 + 0.2)[:, None] / np.linalg.norm(P, axis=1, keepdims=True)
    q, d2, t = B.closest_points(P, v, f)
    T = v.astype(np.float64)[f]
    brute = np.full(len(P), np.inf)
    for k in range(len(f)):
        qq = B._closest_on_triangles(P, *(np.repeat(T[k:k + 1, j], len(P), 0) for j in range(3)))
        brute = np.minimum(brute, ((qq - P) ** 2).sum(1))
    np.testing.assert_allclose(d2, brute, atol=1e-12)
    n = B.outward_normals(P, v, f)
    assert ((n * P).sum(1) / np.linalg.norm(P, axis=1)).min() > 0.98  # outward, close to radial
    bv, bf = configs.box_mesh((0, 0, 0), (10, 10, 10))
    sh = B.shell_elements(np.ones((10, 10, 10), np.uint8), (0, 0, 0), (1.0, 1.0, 1.0), bv, bf, 3.0)
    assert sh.sum() == 1000 - 4 ** 3 and sh[5, 5, 5] == 0 and sh[0, 5, 5] == 1


@pytest.mark.gpu
def test_build_grids_from_mesh_and_config(tmp_path):
    """buildGrids(coords, trifaces): voxelise, then flag surface nodes by the configuration's
    regions evaluated at mesh-frame positions; run two OC iterations."""
    import oracle as O
    import robtop_b200.optimization as OPT

    v, f = configs.box_mesh((0, 0, 0), (24, 12, 12))
    obj = tmp_path / "beam.obj"
    obj.write_text("\n".join([f"v {x} {y} {z}" for x, y, z in v] + [f"f {a + 1} {b + 1} {c + 1}" for a, b, c in f]))
    doc = {"model": "beam.obj",
           "fixedarea": [{"type": "halfspace", "p1": [1, 0, 0], "p2": [1, 0, 1], "p3": [1, 1, 0], "closed": True}],
           "loadarea": [{"type": "box", "p": [23, -1, -1], "q": [25, 13, 1]}],
           "force": [{"type": "const", "norm": 1.0, "direction": [0, 0, -1],
                      "region": {"type": "box", "p": [23, -1, -1], "q": [25, 13, 1]}}]}
    (tmp_path / "config1.json").write_text(json.dumps(doc))
    rec = OPT.run_config(str(tmp_path / "config1.json"), gridreso=31, max_iter=2, volRatio=0.5)
    assert len(rec) == 2 and all(np.isfinite(rec))
    G = OPT.getGrids()
    # the cube and the solid cells are the oracle voxeliser's
    R, bmin, bmax, unit = O.voxel_box(v, 31)
    assert G[0].n_valid_elements() == O.bits_total(O.voxelize_solid(v, f, R, bmin, unit))
    # supports: surface nodes with x <= 1 in the mesh frame (the plane's positive side is -x)
    g0 = G[0]
    vx, vy = g0.nx + 1, g0.ny + 1
    surf = G.surface_nodes().astype(bool) & g0.getVact().astype(bool)
    ids = np.flatnonzero(surf)
    x = float(bmin[0]) + (ids % vx) * ((float(bmax[0]) - float(bmin[0])) / R)  # buildGrids' positions
    assert set(OPT._state["fixed_ids"].tolist()) == set(ids[x <= 1.0].tolist())
    assert len(OPT._state["load_ids"]) > 0
    # the shell (3 element lengths of the surface) stays solid through the OC updates
    eact = g0.getEact().reshape(g0.nz, g0.ny, g0.nx)
    h = (bmax.astype(np.float64) - bmin.astype(np.float64)) / R
    sh = B.shell_elements(eact, bmin.astype(np.float64), h, v, f, 3.0).ravel().astype(bool)
    assert sh.any() and np.all(g0.getRho()[sh] == 1.0)
