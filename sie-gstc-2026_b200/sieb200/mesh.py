"""Triangle meshes: MeshData, RWG edge numbering, sphere generators, OBJ I/O.

MeshData mirrors include/sie_mom/mesh/spherical_surface.hpp:10-15. Edge
numbering (first appearance over (face, local edge (le, le+1 mod 3)), key
(min, max)) is computed by the library (sieb200_build_edges), the contract of
src/sie_mom/mesh/obj_mesh_loader.cpp:360-386.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _lib


@dataclass
class MeshData:
    vertices: np.ndarray      # (nV, 3) float64
    faces: np.ndarray         # (nF, 3) int32, CCW seen from the exterior
    edges: np.ndarray         # (nE, 2) int32, (min, max)
    faces_edges: np.ndarray   # (nF, 3) int32

    @property
    def num_faces(self) -> int:
        return int(self.faces.shape[0])

    @property
    def num_edges(self) -> int:
        return int(self.edges.shape[0])

    def as_c(self) -> _lib.Mesh:
        m = _lib.Mesh()
        m.vertices = self.vertices.ctypes.data
        m.num_vertices = self.vertices.shape[0]
        m.faces = self.faces.ctypes.data
        m.num_faces = self.faces.shape[0]
        m.faces_edges = self.faces_edges.ctypes.data
        m.num_edges = self.edges.shape[0]
        return m


def build_edges(faces: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    faces = np.ascontiguousarray(faces, dtype=np.int32)
    nf = faces.shape[0]
    edges = np.zeros((3 * nf, 2), dtype=np.int32)
    fe = np.zeros((nf, 3), dtype=np.int32)
    ne = ctypes.c_int64()
    _lib.check(_lib.lib().sieb200_build_edges(faces.ctypes.data, nf, edges.ctypes.data,
                                               fe.ctypes.data, ctypes.byref(ne)))
    return edges[: ne.value].copy(), fe


def make_mesh(vertices: np.ndarray, faces: np.ndarray) -> MeshData:
    v = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 3)
    f = np.ascontiguousarray(faces, dtype=np.int32).reshape(-1, 3)
    edges, fe = build_edges(f)
    return MeshData(v, f, edges, fe)


def _normalize(v: np.ndarray) -> np.ndarray:
    # math_utils.cuh:139-142: multiply by the reciprocal length
    inv = 1.0 / np.sqrt(v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1] + v[..., 2] * v[..., 2])
    return v * inv[..., None]


def _orient_outward(vertices: np.ndarray, faces: np.ndarray, center=(0.0, 0.0, 0.0)) -> None:
    v0, v1, v2 = (vertices[faces[:, i]] for i in range(3))
    n = np.cross(v1 - v0, v2 - v0)
    c = (v0 + v1 + v2) / 3.0 - np.asarray(center)
    flip = np.einsum("ij,ij->i", n, c) < 0
    faces[flip, 1], faces[flip, 2] = faces[flip, 2].copy(), faces[flip, 1].copy()


def icosphere(radius: float, level: int) -> MeshData:
    """Icosahedral sphere with 20*4^level faces, built as
    src/sie_mom/mesh/spherical_surface.cpp:19-80 does (same vertex and face
    order, float radius), then oriented CCW outward and edge-numbered."""
    phi = (1.0 + np.sqrt(5.0)) / 2.0
    V = [np.array(p, dtype=np.float64) for p in [
        (-1, phi, 0), (1, phi, 0), (-1, -phi, 0), (1, -phi, 0), (0, -1, phi), (0, 1, phi),
        (0, -1, -phi), (0, 1, -phi), (phi, 0, -1), (phi, 0, 1), (-phi, 0, -1), (-phi, 0, 1)]]
    V = [_normalize(v) for v in V]
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
         (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache: dict[tuple[int, int], int] = {}

        def mid(i: int, j: int) -> int:
            key = (min(i, j), max(i, j))
            if key in cache:
                return cache[key]
            m = _normalize((V[i] + V[j]) * 0.5)
            V.append(m)
            cache[key] = len(V) - 1
            return cache[key]

        nf = []
        for a, b, c in F:
            ab = mid(a, b)
            bc = mid(b, c)
            ca = mid(c, a)
            nf += [(a, ab, ca), (ab, b, bc), (ca, bc, c), (ab, bc, ca)]
        F = nf
    r = float(np.float32(radius))
    verts = np.array(V) * r
    faces = np.array(F, dtype=np.int32)
    _orient_outward(verts, faces)
    return make_mesh(verts, faces)


def geodesic_sphere(radius: float, frequency: int) -> MeshData:
    """Class-I geodesic sphere: each icosahedron face split into frequency^2
    triangles on a barycentric grid and projected to the sphere
    (20 * frequency^2 faces, 30 * frequency^2 edges)."""
    base = icosphere(1.0, 0)
    n = int(frequency)
    key_index: dict[tuple, int] = {}
    verts: list[np.ndarray] = []

    def vid(face: np.ndarray, i: int, j: int) -> int:
        # barycentric (n-i-j, i, j) over the face's corners; canonical key by
        # sorted (corner, weight) pairs so shared edges and corners dedupe.
        w = {int(face[0]): n - i - j, int(face[1]): i, int(face[2]): j}
        key = tuple(sorted((c, wt) for c, wt in w.items() if wt > 0))
        if key not in key_index:
            p = sum(base.vertices[c] * (wt / n) for c, wt in w.items())
            verts.append(_normalize(p) * radius)
            key_index[key] = len(verts) - 1
        return key_index[key]

    faces = []
    for face in base.faces:
        for i in range(n):
            for j in range(n - i):
                a, b, c = vid(face, i, j), vid(face, i + 1, j), vid(face, i, j + 1)
                faces.append((a, b, c))
                if i + j < n - 1:
                    faces.append((vid(face, i + 1, j), vid(face, i + 1, j + 1), vid(face, i, j + 1)))
    v = np.array(verts)
    f = np.array(faces, dtype=np.int32)
    _orient_outward(v, f)
    return make_mesh(v, f)


def revolved_spindle(arc_radius: float = 1.5, half_angle_deg: float = 60.0, n_axial: int = 50,
                     n_azimuth: int = 100) -> MeshData:
    """Circular-arc spindle (ogive) surface of revolution, structured mesh.

    The generating arc has radius arc_radius and spans +-half_angle about the
    equator; the profile r(z) = sqrt(R^2 - z^2) - (R - rmax) with
    rmax = R (1 - cos(alpha)) and half length R sin(alpha)
    (src/sie_mom/mesh/circular_ogive.py:13-60 geometry). Tips are single
    vertices on the axis.
    """
    R = float(arc_radius)
    a = np.deg2rad(half_angle_deg)
    rmax = R * (1.0 - np.cos(a))
    half = R * np.sin(a)
    zs = np.linspace(-half, half, n_axial + 1)
    verts = [np.array([0.0, 0.0, -half])]
    rings = []
    for z in zs[1:-1]:
        r = np.sqrt(R * R - z * z) - (R - rmax)
        ring = []
        for k in range(n_azimuth):
            t = 2 * np.pi * k / n_azimuth
            verts.append(np.array([r * np.cos(t), r * np.sin(t), z]))
            ring.append(len(verts) - 1)
        rings.append(ring)
    verts.append(np.array([0.0, 0.0, half]))
    top = len(verts) - 1
    faces = []
    for k in range(n_azimuth):
        faces.append((0, rings[0][(k + 1) % n_azimuth], rings[0][k]))
    for r0, r1 in zip(rings[:-1], rings[1:]):
        for k in range(n_azimuth):
            k1 = (k + 1) % n_azimuth
            faces.append((r0[k], r0[k1], r1[k1]))
            faces.append((r0[k], r1[k1], r1[k]))
    for k in range(n_azimuth):
        faces.append((rings[-1][k], rings[-1][(k + 1) % n_azimuth], top))
    v = np.array(verts)
    f = np.array(faces, dtype=np.int32)
    _orient_outward(v, f)
    return make_mesh(v, f)


def _obj_index(token: str, seen: int, where: str) -> int:
    """obj_mesh_loader.cpp:26-66: 1-based or negative (relative) index before any '/'."""
    text = token.split("/", 1)[0]
    if not text:
        raise ValueError(f"{where}: face has an empty vertex index")
    try:
        raw = int(text)
    except ValueError:
        raise ValueError(f"{where}: invalid face vertex index '{text}'") from None
    if raw == 0:
        raise ValueError(f"{where}: invalid face vertex index '{text}'")
    if raw > 0:
        return raw - 1
    if not 0 <= seen + raw < seen:
        raise ValueError(f"{where}: relative face vertex index is out of range")
    return seen + raw


def load_obj(path: str | Path) -> MeshData:
    """Vertices (v) and triangular faces (f) in file order, winding preserved,
    with the line-level checks and messages of ObjMeshLoader
    (src/sie_mom/mesh/obj_mesh_loader.cpp:90-152): three coordinates per
    vertex, exactly three indices per face (a trailing '#' comment ends the
    face), no empty, zero or out-of-range index, at least one vertex and one
    face, finite coordinates."""
    path = str(path)
    try:
        text = Path(path).read_text()
    except OSError:
        raise RuntimeError(f"Failed to open OBJ file: {path}") from None
    verts, faces = [], []
    for number, line in enumerate(text.splitlines(), 1):
        parts = line.split()
        if not parts or parts[0].startswith("#"):
            continue
        where = f"{path}:{number}"
        if parts[0] == "v":
            try:
                verts.append([float(x) for x in parts[1:4]])
                if len(parts) < 4:
                    raise ValueError
            except ValueError:
                raise RuntimeError(f"{where}: vertex requires three coordinates") from None
        elif parts[0] == "f":
            tokens = []
            for t in parts[1:]:
                if t.startswith("#"):
                    break
                tokens.append(t)
            if len(tokens) != 3:
                raise RuntimeError(f"{where}: only triangular faces are supported")
            try:
                faces.append([_obj_index(t, len(verts), where) for t in tokens])
            except ValueError as e:
                raise RuntimeError(str(e)) from None
    if not verts:
        raise RuntimeError(f"Invalid OBJ mesh {path}: no vertices")
    if not faces:
        raise RuntimeError(f"Invalid OBJ mesh {path}: no faces")
    v = np.array(verts, dtype=np.float64)
    if not np.isfinite(v).all():
        raise RuntimeError(f"Invalid OBJ mesh {path}: non-finite vertex coordinate")
    return make_mesh(v, np.array(faces, dtype=np.int32))


def save_obj(mesh: MeshData, path: str | Path) -> None:
    with open(path, "w") as fh:
        for v in mesh.vertices:
            fh.write(f"v {v[0]:.17g} {v[1]:.17g} {v[2]:.17g}\n")
        for f in mesh.faces:
            fh.write(f"f {f[0] + 1} {f[1] + 1} {f[2] + 1}\n")


def infer_sphere_radius(mesh: MeshData, max_relative_spread: float = 1e-4) -> float:
    """Mean vertex radius of a sphere mesh centred at the origin
    (include/sie_mom/mesh/mesh_utils.hpp:156-182)."""
    r = np.sqrt((np.asarray(mesh.vertices, dtype=np.float64) ** 2).sum(axis=1))
    if not (np.isfinite(r).all() and (r > 0).all()):
        raise RuntimeError("sphere mesh contains a non-finite or zero-radius vertex")
    radius = float(np.sum(r.astype(np.longdouble)) / r.size)
    if (r.max() - r.min()) / radius > max_relative_spread:
        raise RuntimeError("mesh vertices do not lie on a common spherical radius")
    return radius
