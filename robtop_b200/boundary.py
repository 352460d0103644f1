"""Boundary-condition regions, force fields and the JSON benchmark configuration.

Restates the reference's region and field types and its configuration parser:

* regions (``boundary/BoundaryCondition.h:379-568``, static forms ``:1-370``): sphere, box,
  half space (through three points), cylinder; ``closed`` adds the boundary, ``complement``
  negates; a list of regions is their union (``rangeUnion::generate``);
* force fields (``boundary/BoundaryCondition.h:570-740``): ``const``,
  ``RadialNormConstDir``, ``ConstNormRadialDir``, ``RadialNormRadialDir``, ``Twist``, each
  restricted to its own region; the fields of a configuration add up (``Field_t::at``);
* the configuration file (``config_parser.cpp:140-434``): ``fixedarea`` and ``loadarea``
  region lists, a ``force`` field list and the ``model`` mesh name;
* mesh files read by ``config_parser_t::readMesh`` (``config_parser.cpp:401-425``, OpenMesh):
  Wavefront OBJ and STL (ASCII or binary), polygons fanned into triangles.

Every predicate and field is vectorised over an ``[n, 3]`` array of positions.  Host-side
set-up only: the flags and loads it produces go to the device through ``HierarchyGrid``.
Errors raise ``ValueError`` where the reference prints and exits.
"""
from __future__ import annotations

import json
import os
import struct

import numpy as np

SMALL = 1e-8  # range_t::small_value


def _vec(d, key, default=None):
    if key not in d:
        if default is None:
            raise ValueError(f"missing member \"{key}\"")
        return np.asarray(default, np.float64)
    v = d[key]
    if not isinstance(v, (list, tuple)) or len(v) > 3 or not all(isinstance(x, (int, float)) for x in v):
        raise ValueError(f"\"{key}\" should be an array of at most 3 numbers")
    out = np.zeros(3)
    out[:len(v)] = v
    return out


class Region:
    """A region: ``contains(P)`` -> bool[n] for positions ``P[n, 3]``."""

    closed = False
    complement = False

    def _inside(self, P):
        raise NotImplementedError

    def contains(self, P):
        return self._inside(np.atleast_2d(np.asarray(P, np.float64))) ^ self.complement

    def __call__(self, p):
        return bool(self.contains(np.asarray(p, np.float64).reshape(1, 3))[0])


class Sphere(Region):
    """sphereRange_t: |p - c|^2 < r^2, or within small_value of it when closed."""

    def __init__(self, center, radius, closed=False, complement=False):
        self.c, self.r2 = np.asarray(center, np.float64), float(radius) ** 2
        self.closed, self.complement = closed, complement

    def _inside(self, P):
        d2 = ((P - self.c) ** 2).sum(1)
        return (d2 < self.r2) | (self.closed & (d2 - self.r2 < SMALL))


class Box(Region):
    """boxRange_t (an iso-cuboid spanned by two corners): strictly inside, or on a face when closed."""

    def __init__(self, p, q, closed=False, complement=False):
        p, q = np.asarray(p, np.float64), np.asarray(q, np.float64)
        self.lo, self.hi = np.minimum(p, q), np.maximum(p, q)
        self.closed, self.complement = closed, complement

    def _inside(self, P):
        strict = np.all((P > self.lo) & (P < self.hi), 1)
        if not self.closed:
            return strict
        return np.all((P >= self.lo) & (P <= self.hi), 1)


class HalfSpace(Region):
    """halfSpaceRange_t through p1, p2, p3: the side the normal (p2 - p1) x (p3 - p1) points to
    (the points are counter-clockwise seen from it), plus the plane itself when closed."""

    def __init__(self, p1, p2, p3, closed=False, complement=False):
        self.p1 = np.asarray(p1, np.float64)
        self.n = np.cross(np.asarray(p2, np.float64) - self.p1, np.asarray(p3, np.float64) - self.p1)
        self.closed, self.complement = closed, complement

    def _inside(self, P):
        s = (P - self.p1) @ self.n
        return (s > 0) | (self.closed & (s == 0))


class Cylinder(Region):
    """cylinderRange_t: 0 <= (p - c).z <= |h| along the unit axis z = h / |h|, and distance
    from the axis below the radius (no closed / complement forms)."""

    def __init__(self, bottom_center, radius, height_vector):
        self.c, self.r = np.asarray(bottom_center, np.float64), float(radius)
        h = np.asarray(height_vector, np.float64)
        self.H = float(np.linalg.norm(h))
        self.z = h / self.H

    def _inside(self, P):
        d = P - self.c
        proj = d @ self.z
        devi = np.linalg.norm(np.cross(d, self.z), axis=1)
        return (proj <= self.H) & (proj >= 0) & (devi < self.r)


class Union(Region):
    """rangeUnion::generate: inside any member (an empty union contains nothing)."""

    def __init__(self, regions=()):
        self.regions = list(regions)

    def _inside(self, P):
        out = np.zeros(P.shape[0], bool)
        for r in self.regions:
            out |= r.contains(P)
        return out


def parse_region(d):
    """One region object (config_parser.cpp:48-138 and :140-236)."""
    if not isinstance(d, dict) or not isinstance(d.get("type"), str):
        raise ValueError("a region should have a member \"type\": \"box\" / \"sphere\" / \"halfspace\" / \"cylinder\"")
    closed = bool(d.get("closed", False)) if isinstance(d.get("closed", False), bool) else False
    comp = bool(d.get("complement", False)) if isinstance(d.get("complement", False), bool) else False
    t = d["type"]
    if t == "box":
        return Box(_vec(d, "p"), _vec(d, "q"), closed, comp)
    if t == "sphere":
        r = d.get("radius")
        if not isinstance(r, (int, float)):
            raise ValueError("a sphere needs a numeric \"radius\"")
        return Sphere(_vec(d, "center", (0, 0, 0)), r, closed, comp)
    if t == "halfspace":
        return HalfSpace(_vec(d, "p1"), _vec(d, "p2"), _vec(d, "p3"), closed, comp)
    if t == "cylinder":
        return Cylinder(_vec(d, "bottomCenter"), float(d["radius"]), _vec(d, "heightVector"))
    raise ValueError(f"unknown region type \"{t}\"")


def _unit(v):
    n = np.linalg.norm(v, axis=-1, keepdims=True)
    return v / np.where(n > 0, n, 1.0)


class Field:
    """A force field restricted to a region (rangeField_t): norm(p) * direction(p) inside, 0 outside."""

    def __init__(self, region, norm, direction):
        self.region, self.norm, self.direction = region, norm, direction

    def at(self, P):
        P = np.atleast_2d(np.asarray(P, np.float64))
        out = self.norm(P)[:, None] * self.direction(P)
        out[~self.region.contains(P)] = 0.0
        return out


def parse_field(d):
    """One force-field object (config_parser.cpp:238-367)."""
    if not isinstance(d, dict) or "region" not in d:
        raise ValueError("a force field needs a \"region\"")
    region = parse_region(d["region"])
    t = d.get("type")
    if not isinstance(t, str):
        raise ValueError("a force field should have a member \"type\"")
    if t == "const":
        nf, dirv = float(d["norm"]), _unit(_vec(d, "direction"))
        return Field(region, lambda P: np.full(P.shape[0], nf), lambda P: np.tile(dirv, (P.shape[0], 1)))
    if t in ("RadialNormConstDir", "RadialNormRadialDir"):
        nc = _vec(d, "center") if t == "RadialNormConstDir" else _vec(d, "NormCenter")
        amp, damp = float(d.get("amplifier", 1.0)), float(d.get("dampRatio", 1.0))
        norm = lambda P: amp * np.exp(-np.linalg.norm(nc - P, axis=1) ** (damp * 2))  # noqa: E731
        if t == "RadialNormConstDir":
            dirv = _unit(_vec(d, "direction"))
            return Field(region, norm, lambda P: np.tile(dirv, (P.shape[0], 1)))
        dc = _vec(d, "DirCenter")
        return Field(region, norm, lambda P: _unit(dc - P))
    if t == "ConstNormRadialDir":
        c, nr = _vec(d, "center"), float(d["norm"])
        return Field(region, lambda P: np.full(P.shape[0], nr), lambda P: _unit(c - P))
    if t == "Twist":
        a, b, amp = _vec(d, "AxisStart"), _vec(d, "AxisEnd"), float(d["amplifier"])
        ax = _unit(b - a)
        norm = lambda P: np.linalg.norm(np.cross(P - a, ax), axis=1) * amp  # noqa: E731
        return Field(region, norm, lambda P: _unit(np.cross(P - a, b - a)))
    if t == "gradient":  # parsed and ignored by the reference
        return None
    raise ValueError(f"unknown force field type \"{t}\"")


class Config:
    """A parsed benchmark configuration: ``fixed(P)``, ``load(P)``, ``force(P)`` and the model file."""

    def __init__(self, fixed, load, fields, model=None, directory=""):
        self.fixed_area, self.load_area, self.fields = fixed, load, fields
        self.model, self.directory = model, directory

    def fixed(self, P):
        return self.fixed_area.contains(P)

    def load(self, P):
        return self.load_area.contains(P)

    def force(self, P):
        P = np.atleast_2d(np.asarray(P, np.float64))
        out = np.zeros_like(P)
        for f in self.fields:
            out += f.at(P)
        return out

    def model_path(self):
        return os.path.join(self.directory, self.model) if self.model else None


def parse_config(src):
    """config_parser_t::parse_benchmark_configuration (config_parser.cpp:369-399): ``src`` is a
    path to the JSON file or its parsed dict."""
    directory = ""
    if isinstance(src, (str, os.PathLike)):
        directory = os.path.dirname(os.path.abspath(src))
        with open(src) as fh:
            src = json.load(fh)
    if not isinstance(src, dict):
        raise ValueError("the configuration should be a JSON object")

    def region_list(key):
        v = src.get(key, [])
        if not isinstance(v, list):
            raise ValueError(f"{key} should be a list of region objects")
        return Union(parse_region(r) for r in v)

    forces = src.get("force", [])
    if not isinstance(forces, list):
        raise ValueError("force should be a list of field objects")
    fields = [f for f in (parse_field(x) for x in forces) if f is not None]
    return Config(region_list("fixedarea"), region_list("loadarea"), fields, src.get("model"), directory)


# ----------------------------------------------------------------------------
# mesh files
# ----------------------------------------------------------------------------
def read_mesh(path):
    """Vertices float32 [n, 3] and triangles int32 [m, 3] of an OBJ or STL file
    (polygons are fanned from their first vertex)."""
    ext = os.path.splitext(path)[1].lower()
    if ext == ".obj":
        return _read_obj(path)
    if ext == ".stl":
        return _read_stl(path)
    raise ValueError(f"unsupported mesh format {ext}")


def _read_obj(path):
    verts, faces = [], []
    with open(path) as fh:
        for line in fh:
            t = line.split()
            if not t:
                continue
            if t[0] == "v" and len(t) >= 4:
                verts.append([float(t[1]), float(t[2]), float(t[3])])
            elif t[0] == "f" and len(t) >= 4:
                idx = []
                for s in t[1:]:
                    i = int(s.split("/")[0])
                    idx.append(i - 1 if i > 0 else len(verts) + i)
                faces.extend([idx[0], idx[k], idx[k + 1]] for k in range(1, len(idx) - 1))
    v = np.asarray(verts, np.float32).reshape(-1, 3)
    f = np.asarray(faces, np.int32).reshape(-1, 3)
    if f.size and (f.min() < 0 or f.max() >= len(v)):
        raise ValueError("face index out of range")
    return v, f


def _read_stl(path):
    with open(path, "rb") as fh:
        data = fh.read()
    tris = None
    if len(data) >= 84:
        n = struct.unpack_from("<I", data, 80)[0]
        if 84 + 50 * n == len(data):
            rec = np.frombuffer(data, np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")]), n, 84)
            tris = rec["v"].reshape(-1, 3)
    if tris is None:
        pts = [[float(x) for x in line.split()[1:4]] for line in data.decode("ascii", "replace").splitlines()
               if line.strip().startswith("vertex")]
        tris = np.asarray(pts, np.float32).reshape(-1, 3)
    # weld identical vertices so shared edges are shared in the index list
    v, inv = np.unique(tris, axis=0, return_inverse=True)
    return v.astype(np.float32), inv.reshape(-1, 3).astype(np.int32)


# ----------------------------------------------------------------------------
# distances to the mesh surface: outward normals of load nodes, shell elements
# ----------------------------------------------------------------------------
def _closest_on_triangles(P, A, B, C):
    """Closest points of points P[k] on triangles (A[k], B[k], C[k]) (Voronoi-region tests)."""
    ab, ac, ap = B - A, C - A, P - A
    d1, d2 = (ab * ap).sum(1), (ac * ap).sum(1)
    bp = P - B
    d3, d4 = (ab * bp).sum(1), (ac * bp).sum(1)
    cp = P - C
    d5, d6 = (ab * cp).sum(1), (ac * cp).sum(1)
    va, vb, vc = d3 * d6 - d5 * d4, d5 * d2 - d1 * d6, d1 * d4 - d3 * d2
    out = np.empty_like(P)
    done = np.zeros(len(P), bool)

    def put(mask, val):
        m = mask & ~done
        out[m] = val[m] if val.ndim == 2 else val
        done[:] |= m

    put((d1 <= 0) & (d2 <= 0), A)
    put((d3 >= 0) & (d4 <= d3), B)
    with np.errstate(divide="ignore", invalid="ignore"):
        put((vc <= 0) & (d1 >= 0) & (d3 <= 0), A + ab * (d1 / (d1 - d3))[:, None])
        put((d6 >= 0) & (d5 <= d6), C)
        put((vb <= 0) & (d2 >= 0) & (d6 <= 0), A + ac * (d2 / (d2 - d6))[:, None])
        put((va <= 0) & ((d4 - d3) >= 0) & ((d5 - d6) >= 0),
            B + (C - B) * ((d4 - d3) / ((d4 - d3) + (d5 - d6)))[:, None])
        den = va + vb + vc
        put(np.ones(len(P), bool), A + ab * (vb / den)[:, None] + ac * (vc / den)[:, None])
    return out


def closest_points(points, verts, faces):
    """For each point: the closest point on the triangle mesh, its squared distance and the
    triangle (the AABB-tree query of Grid::outwardNormal, grid/Grid.cpp:1404-1423).  Candidates
    are the triangles whose centroid lies within (distance to the nearest centroid + the
    largest centroid-to-vertex radius), found with a k-d tree."""
    from scipy.spatial import cKDTree

    P = np.atleast_2d(np.asarray(points, np.float64))
    V = np.asarray(verts, np.float64)
    F = np.asarray(faces, np.int64)
    T = V[F]  # [m, 3, 3]
    cen = T.mean(1)
    rad = np.sqrt(((T - cen[:, None, :]) ** 2).sum(2).max(1)).max()
    tree = cKDTree(cen)
    d0, _ = tree.query(P)
    best_q = np.zeros_like(P)
    best_d = np.full(len(P), np.inf)
    best_t = np.zeros(len(P), np.int64)
    cands = tree.query_ball_point(P, d0 + rad + 1e-12)
    idx_p = np.repeat(np.arange(len(P)), [len(c) for c in cands])
    idx_t = np.fromiter((t for c in cands for t in c), np.int64, count=len(idx_p))
    for s in range(0, len(idx_p), 1 << 20):
        ip, it = idx_p[s:s + (1 << 20)], idx_t[s:s + (1 << 20)]
        q = _closest_on_triangles(P[ip], T[it, 0], T[it, 1], T[it, 2])
        d = ((q - P[ip]) ** 2).sum(1)
        order = np.lexsort((d, ip))  # per point, smallest distance first
        first = np.ones(len(order), bool)
        first[1:] = ip[order][1:] != ip[order][:-1]
        sel = order[first]
        upd = d[sel] < best_d[ip[sel]]
        tgt = ip[sel][upd]
        best_d[tgt], best_q[tgt], best_t[tgt] = d[sel][upd], q[sel][upd], it[sel][upd]
    return best_q, best_d, best_t


def outward_normals(points, verts, faces):
    """Grid::outwardNormal (grid/Grid.cpp:1404-1423): the unit vector from the point to its
    closest surface point, oriented along that triangle's normal (the triangle's own normal
    when the point lies on the surface, within 1e-6)."""
    P = np.atleast_2d(np.asarray(points, np.float64))
    q, d2, t = closest_points(P, verts, faces)
    V = np.asarray(verts, np.float64)
    F = np.asarray(faces, np.int64)[t]
    tn = np.cross(V[F[:, 1]] - V[F[:, 0]], V[F[:, 2]] - V[F[:, 0]])
    p2c = q - P
    ln = np.sqrt(d2)
    on = ln < 1e-6
    sgn = np.where((p2c * tn).sum(1) < 0, -1.0, 1.0)
    out = np.where(on[:, None], tn / np.linalg.norm(tn, axis=1, keepdims=True),
                   p2c / np.where(on, 1.0, ln * sgn)[:, None])
    return out


def shell_elements(eact, origin, h, verts, faces, shell_width):
    """HierarchyGrid::setSolidShellElement (grid/Grid.cpp:67-137): solid elements whose centre
    lies within shell_width * h of the mesh surface.  ``eact[nz, ny, nx]`` dense level-0
    activity, element (x, y, z) centred at origin + (x + 1/2, y + 1/2, z + 1/2) h."""
    from scipy.ndimage import binary_erosion

    eact = np.asarray(eact).astype(bool)
    out = np.zeros(eact.shape, np.uint8)
    if not eact.any():
        return out
    hv = np.asarray(h, np.float64)
    w = float(shell_width) * float(np.max(hv))
    # the mesh surface lies within a voxel of the solid's boundary: only elements within
    # ceil(shell_width) + 2 cells of a void cell or the box edge can be closer than w to it
    k = int(np.ceil(w / float(np.min(hv)))) + 2
    core = binary_erosion(np.pad(eact, 1), iterations=k)[1:-1, 1:-1, 1:-1]
    z, y, x = np.nonzero(eact & ~core)
    cen = np.asarray(origin, np.float64) + (np.stack([x, y, z], 1) + 0.5) * hv
    _, d2, _ = closest_points(cen, verts, faces)
    inside = d2 < w * w
    out[z[inside], y[inside], x[inside]] = 1
    return out
