"""Seeded synthetic domains with the shapes of the benchmark configurations.

Each builder returns a dict with the dense element activity ``eact[nz,ny,nx]``,
the density ``rho[nz,ny,nx]`` (float32), support flags ``vfix[nz+1,ny+1,nx+1]``,
the load set (dense node ids + unit outward normals), an optional fixed load
``fload[3, nv]`` and the work mode.  Support / load flags follow the
reference's rule (Grid::computeProjectionMatrix, grid/Grid.cpp:1291-1403): only
surface nodes (mark_surface_nodes_kernel, grid/Grid.cu:2005-2039) can be
supports or loads, and a support node is never a load node.  No public dataset
is involved: every input is generated here from fixed seeds.
"""
from __future__ import annotations

import numpy as np

from ._capi import MODE_NSCF, MODE_NSFF, MODE_WSCF, MODE_WSFF  # noqa: F401


def surface_nodes(eact):
    """Numpy restatement of the surface-node rule (used only for building inputs)."""
    nz, ny, nx = eact.shape
    pad = np.zeros((nz + 2, ny + 2, nx + 2), bool)
    pad[1:-1, 1:-1, 1:-1] = eact.astype(bool)
    # s[c][b][a] = element at node offset (a-1, b-1, c-1)
    s = {}
    for c in (0, 1):
        for b in (0, 1):
            for a in (0, 1):
                s[(a, b, c)] = pad[c:c + nz + 1, b:b + ny + 1, a:a + nx + 1]
    ax = np.zeros((nz + 1, ny + 1, nx + 1), bool)
    ay = np.zeros_like(ax)
    az = np.zeros_like(ax)
    for i in (0, 1):
        for j in (0, 1):
            ax |= s[(0, i, j)] & s[(1, i, j)]
            ay |= s[(i, 0, j)] & s[(i, 1, j)]
            az |= s[(i, j, 0)] & s[(i, j, 1)]
    return ~ax | ~ay | ~az


def node_active(eact):
    nz, ny, nx = eact.shape
    pad = np.zeros((nz + 2, ny + 2, nx + 2), bool)
    pad[1:-1, 1:-1, 1:-1] = eact.astype(bool)
    v = np.zeros((nz + 1, ny + 1, nx + 1), bool)
    for c in (0, 1):
        for b in (0, 1):
            for a in (0, 1):
                v |= pad[c:c + nz + 1, b:b + ny + 1, a:a + nx + 1]
    return v


def _flags(eact, in_fixed, in_load):
    nz, ny, nx = eact.shape
    z, y, x = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    surf = surface_nodes(eact) & node_active(eact)
    fix = surf & in_fixed(x, y, z)
    load = surf & ~fix & in_load(x, y, z)
    return fix.astype(np.uint8), np.flatnonzero(load.ravel()).astype(np.int32)


def smoothed_density(shape, seed, rho_min=1e-3, sigma=4.0, sharpness=8.0):
    """rho = rho_min + (1 - rho_min) * sigmoid(8 g), g a seeded N(0,1) field (Philox),
    Gaussian-smoothed with sigma voxels (truncate 4 sigma, reflect), standardised."""
    from scipy.ndimage import gaussian_filter

    g = np.random.Generator(np.random.Philox(seed)).standard_normal(shape)
    g = gaussian_filter(g, sigma=sigma, mode="reflect", truncate=4.0)
    g = (g - g.mean()) / g.std()
    return (rho_min + (1 - rho_min) / (1 + np.exp(-sharpness * g))).astype(np.float32)


def cantilever(nx=64, ny=32, nz=32, rho=0.4):
    """64x32x32 cantilever: x=0 face clamped, total load 1.0 in -z spread evenly
    over the nodes of the bottom edge (z=0) of the x=nx face; fixed load (wsff)."""
    eact = np.ones((nz, ny, nx), np.uint8)
    vfix, load = _flags(eact, lambda x, y, z: x == 0, lambda x, y, z: (x == nx) & (z == 0))
    nv = (nx + 1) * (ny + 1) * (nz + 1)
    fload = np.zeros((3, nv))
    fload[2, load] = -1.0 / load.size
    normals = np.tile([0.0, 0.0, -1.0], (load.size, 1))
    return dict(name=f"cantilever_{nx}x{ny}x{nz}", eact=eact, rho=np.full(eact.shape, rho, np.float32), vfix=vfix,
                load_nodes=load, normals=normals, fload=fload, mode=MODE_WSFF)


def worst_case_box(nx=128, ny=128, nz=64, seed=0, rho_min=1e-3):
    """128x128x64 worst-case configuration: smoothed random density, z=0 clamped,
    loadable set = all top-face nodes (z=nz), free direction (wsff)."""
    eact = np.ones((nz, ny, nx), np.uint8)
    vfix, load = _flags(eact, lambda x, y, z: z == 0, lambda x, y, z: z == nz)
    normals = np.tile([0.0, 0.0, 1.0], (load.size, 1))
    return dict(name=f"worstcase_{nx}x{ny}x{nz}", eact=eact, rho=smoothed_density(eact.shape, seed, rho_min),
                vfix=vfix, load_nodes=load, normals=normals, fload=None, mode=MODE_WSFF)


def arch(nx=511, ny=256, nz=256, tunnel=96, pad=16, rho=0.4):
    """511x256x256 arch: solid box minus a cylindrical tunnel of radius 96 voxels
    along x centred at (y=128, z=0); four 16x16-voxel support pads at the bottom
    corners; loadable set = top face, load normal-constrained (wscf)."""
    z, y = np.meshgrid(np.arange(nz) + 0.5, np.arange(ny) + 0.5, indexing="ij")
    keep = ((y - ny / 2) ** 2 + z ** 2) >= tunnel ** 2
    eact = np.broadcast_to(keep[:, :, None], (nz, ny, nx)).astype(np.uint8).copy()
    fx = lambda x, y, z: (z == 0) & ((x <= pad) | (x >= nx - pad)) & ((y <= pad) | (y >= ny - pad))
    vfix, load = _flags(eact, fx, lambda x, y, z: z == nz)
    normals = np.tile([0.0, 0.0, 1.0], (load.size, 1))
    return dict(name=f"arch_{nx}x{ny}x{nz}", eact=eact, rho=np.where(eact, rho, 0).astype(np.float32), vfix=vfix,
                load_nodes=load, normals=normals, fload=None, mode=MODE_WSCF)


def free_block(nx=16, ny=8, nz=8, seed=3, mode=MODE_NSFF):
    """Unsupported block with the top face loadable (no-support modes)."""
    eact = np.ones((nz, ny, nx), np.uint8)
    vfix = np.zeros((nz + 1, ny + 1, nx + 1), np.uint8)
    _, load = _flags(eact, lambda x, y, z: np.zeros_like(x, bool), lambda x, y, z: z == nz)
    normals = np.tile([0.0, 0.0, 1.0], (load.size, 1))
    # moderate contrast: an unsupported body with floating stiff islands has many
    # near-rigid modes that no V-cycle preconditioner resolves quickly
    rho = smoothed_density(eact.shape, seed, rho_min=0.05, sigma=2.0, sharpness=2.0)
    return dict(name=f"free_{nx}x{ny}x{nz}", eact=eact, rho=rho, vfix=vfix, load_nodes=load, normals=normals,
                fload=None, mode=mode)


def batch_instances(n=12, lo=48, hi=160, seed=1):
    """Per-axis sizes drawn uniformly from {lo..hi} (seeded); cantilever BCs."""
    rng = np.random.Generator(np.random.Philox(seed))
    sizes = rng.integers(lo, hi + 1, size=(n, 3))
    return [tuple(int(v) for v in s) for s in sizes]


# ----------------------------------------------------------------------------
# closed triangle meshes for the voxeliser (outward-facing, counter-clockwise)
# ----------------------------------------------------------------------------
def icosphere(subdiv=3, center=(0.0, 0.0, 0.0), radius=1.0):
    """Icosahedron refined ``subdiv`` times, vertices pushed to the sphere: 20 * 4^subdiv triangles."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = np.array(v, np.float64)
    verts /= np.linalg.norm(verts, axis=1, keepdims=True)
    faces = np.array(f, np.int64)
    for _ in range(subdiv):
        edges = np.sort(np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]]), axis=1)
        uniq, inv = np.unique(edges, axis=0, return_inverse=True)
        mid = verts[uniq[:, 0]] + verts[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = verts.shape[0]
        verts = np.concatenate([verts, mid])
        nf = faces.shape[0]
        m01, m12, m20 = (base + inv.reshape(-1)[k * nf:(k + 1) * nf] for k in range(3))
        a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
        faces = np.concatenate([np.stack([a, m01, m20], 1), np.stack([b, m12, m01], 1), np.stack([c, m20, m12], 1),
                                np.stack([m01, m12, m20], 1)])
    return (verts * radius + np.asarray(center, np.float64)).astype(np.float32), faces.astype(np.int32)


def torus(R=1.0, r=0.35, n=48, m=24, center=(0.0, 0.0, 0.0)):
    """Torus around the z axis, n x m quads split into 2 n m triangles."""
    i, j = np.meshgrid(np.arange(n), np.arange(m), indexing="ij")
    u, w = 2 * np.pi * i / n, 2 * np.pi * j / m
    verts = np.stack([(R + r * np.cos(w)) * np.cos(u), (R + r * np.cos(w)) * np.sin(u), r * np.sin(w)], -1)
    verts = verts.reshape(-1, 3) + np.asarray(center, np.float64)
    idx = lambda a, b: (a % n) * m + (b % m)  # noqa: E731
    q00, q10, q11, q01 = idx(i, j), idx(i + 1, j), idx(i + 1, j + 1), idx(i, j + 1)
    faces = np.concatenate([np.stack([q00, q10, q11], -1).reshape(-1, 3), np.stack([q00, q11, q01], -1).reshape(-1, 3)])
    return verts.astype(np.float32), faces.astype(np.int32)


def box_mesh(lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    """Axis-aligned box, 12 triangles."""
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    c = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], np.float64)
    verts = lo + c * (hi - lo)
    faces = [(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4), (2, 3, 7), (2, 7, 6), (0, 4, 7),
             (0, 7, 3), (1, 2, 6), (1, 6, 5)]
    return verts.astype(np.float32), np.array(faces, np.int32)


def rigid_transform(verts, seed, shift=(0.0, 0.0, 0.0)):
    """A seeded random rotation of the vertices about their centroid, then a shift."""
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    v = np.asarray(verts, np.float64)
    c = v.mean(0)
    return ((v - c) @ q.T + c + np.asarray(shift, np.float64)).astype(np.float32)


def merge_meshes(*meshes):
    """Disjoint union of (verts, faces) pairs."""
    vs, fs, base = [], [], 0
    for v, f in meshes:
        vs.append(np.asarray(v, np.float32))
        fs.append(np.asarray(f, np.int32) + base)
        base += len(v)
    return np.concatenate(vs), np.concatenate(fs)
