"""Solid mesh voxeliser on the GPU against the oracle's restatement of the reference's
solid voxeliser (voxelizer/cpu_voxelizer.cpp:245-322, voxelizer/voxelize_solid.cu:80-150):
bit-exact on closed, rotated, merged, open and degenerate meshes at every cube size path
(R < 32 rows share words, R >= 32 row words), plus the genFromMesh boundary."""
import numpy as np
import pytest

import oracle as O
import robtop_b200 as rb
from robtop_b200 import configs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = rb.Context(0)
    yield c
    c.close()


def _oracle_bits(v, f, prefer):
    R, bmin, bmax, unit = O.voxel_box(v, prefer)
    return O.voxelize_solid(v, f, R, bmin, unit), R, np.stack([bmin, bmax])


def _meshes():
    s3 = configs.icosphere(3, radius=1.0)
    t = configs.torus(1.0, 0.35, 40, 20)
    return {
        "sphere": configs.icosphere(4, radius=1.0),
        "sphere_rotated": (configs.rigid_transform(s3[0], 11, (0.3, -0.2, 0.1)), s3[1]),
        "torus_rotated": (configs.rigid_transform(t[0], 12), t[1]),
        "box_half_voxel": configs.box_mesh((0.1, 0.1, 0.1), (0.9, 0.9, 0.9)),
        "box_flat": configs.box_mesh((0.0, 0.0, 0.0), (1.0, 0.37, 0.61)),
        "two_spheres": configs.merge_meshes(configs.icosphere(2, (0, 0, 0), 0.5), configs.icosphere(3, (1.3, 0.2, 0.1), 0.6)),
    }


@pytest.mark.parametrize("prefer", [7, 31, 63, 200])
@pytest.mark.parametrize("name", sorted(_meshes()))
def test_voxelize_bit_exact(ctx, name, prefer):
    v, f = _meshes()[name]
    ob, R, box = _oracle_bits(v, f, prefer)
    gb, gR, gbox = rb.voxelize_mesh(ctx, v, f, prefer)
    assert gR == R == rb.lib().rt_voxel_resolution(prefer)
    np.testing.assert_array_equal(gbox, box)
    diff = np.count_nonzero(gb != ob)
    assert diff == 0, f"{diff} of {ob.size} words differ"
    if name != "box_flat":
        assert O.bits_total(O.word_reverse(gb)) > 0


def test_open_and_degenerate_meshes_bit_exact(ctx):
    """Non-closed input flips rows by the same XOR rule; zero-area triangles are skipped."""
    rng = np.random.default_rng(4)
    v = rng.random((60, 3)).astype(np.float32)
    f = rng.integers(0, 60, (80, 3)).astype(np.int32)
    f[:5, 1] = f[:5, 0]  # degenerate: repeated vertex
    for prefer in (15, 63):
        ob, R, _ = _oracle_bits(v, f, prefer)
        gb, gR, _ = rb.voxelize_mesh(ctx, v, f, prefer)
        np.testing.assert_array_equal(gb, ob)


def test_empty_face_list(ctx):
    v, _ = configs.box_mesh()
    gb, R, _ = rb.voxelize_mesh(ctx, v, np.zeros((0, 3), np.int32), 31)
    assert R == 32 and not gb.any()


def test_invalid_meshes_are_rejected(ctx):
    v, f = configs.box_mesh()
    bad = f.copy()
    bad[3, 2] = 8  # one past the last vertex
    with pytest.raises(rb.RTError):
        rb.voxelize_mesh(ctx, v, bad, 31)
    with pytest.raises(ValueError):
        rb.voxelize_mesh(ctx, v, f, 0)
    vn = v.copy()
    vn[2, 1] = np.nan
    with pytest.raises(rb.RTError):
        rb.voxelize_mesh(ctx, vn, f, 31)


def test_hierarchy_from_mesh_equals_hierarchy_from_bits(ctx):
    """genFromMesh(pcoords, faces) = voxelise + word reverse + genFromMesh(solid_bit, reso)."""
    v, f = configs.merge_meshes(configs.icosphere(3, (0, 0, 0), 1.0), configs.icosphere(2, (1.5, 0.0, 0.2), 0.4))
    G1 = rb.HierarchyGrid(ctx, rb.default_params())
    G1.genFromTriMesh(v, f, 63)
    ob, R, _ = _oracle_bits(v, f, 63)
    G2 = rb.HierarchyGrid(ctx, rb.default_params())
    G2.genFromMesh(O.word_reverse(ob), R)
    assert G1.n_grid() == G2.n_grid()
    for i in range(G1.n_grid()):
        np.testing.assert_array_equal(G1[i].getEact(), G2[i].getEact())
    G1.close()
    G2.close()
