"""Test infrastructure only: ctypes access to the CPU oracle (sieoracle.c) and,
when it has been built, to the reference harness (_ref/libsieref.so).

Only tests/, the smoke check and bench.py's CPU-baseline leg import this.
"""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libsieoracle.so"
REF_SO = HERE / "_ref" / "libsieref.so"

_P = ctypes.c_void_p
_f = ctypes.c_float
_d = ctypes.c_double
_i = ctypes.c_int

_ASSEMBLE = [_i, _P, _P, _P, _i, _i, _i, _f, _f, _f, _f, _f, _f, _f, _f, _f, _f, _P, _i, _i, _P, _i, _i, _i]


def _build_oracle() -> None:
    src = HERE / "sieoracle.c"
    if ORACLE_SO.exists() and ORACLE_SO.stat().st_mtime >= src.stat().st_mtime:
        return
    subprocess.run(["make", "-s", "-C", str(HERE), str(ORACLE_SO)], check=True,
                   capture_output=True)


_FIELDS = [_P, _P, _P, _i, _i, _P, _P, _i, _P, _d, _d, _d, _d, _d, _i, _P, _P]


def oracle() -> ctypes.CDLL:
    _build_oracle()
    lib = ctypes.CDLL(str(ORACLE_SO))
    lib.so_rule.argtypes = [_i, _P, _P]
    lib.so_build_edges.argtypes = [_P, _i, _P, _P]
    lib.so_wilton.argtypes = [_P, _P, _P]
    lib.so_pair_blocks.argtypes = [_P, _P, _i, _i, _i, _f, _f, _f, _P]
    lib.so_pair_blocks_n.argtypes = [_P, _P, _i, _i, _i, _f, _f, _f, _i, _P]
    lib.so_gauss_legendre.argtypes = [_i, _P, _P]
    lib.so_assemble.argtypes = _ASSEMBLE
    lib.so_assemble_rows.argtypes = _ASSEMBLE[:20] + [_P, _i, _P, _i, _P, _i, _i, _i]
    lib.so_rhs.argtypes = [_i, _i, _P, _P, _P, _i, _i, _i, _P, _P, _i, _d, _d, _i, _d, _d, _P, _i, _d, _d]
    lib.so_far_field.argtypes = [_P, _P, _i, _i, _P, _P, _d, _d, _i, _P, _P, _P, _P, _P, _P]
    lib.so_surface_fields.argtypes = _FIELDS
    lib.so_incident_fields.argtypes = [_i, _P, _P, _i, _d, _d, _i, _P, _P, _P]
    return lib


def reference() -> ctypes.CDLL | None:
    if not REF_SO.exists():
        return None
    lib = ctypes.CDLL(str(REF_SO))
    lib.ref_dunavant.argtypes = [_i, _P, _P]
    lib.ref_icosphere.argtypes = [_f, _i, ctypes.POINTER(_i), ctypes.POINTER(_i), ctypes.POINTER(_i),
                                  _P, _P, _P, _P]
    lib.ref_wilton.argtypes = [_P, _P, _P]
    lib.ref_phi0.argtypes = [_P, _P]
    lib.ref_phi0.restype = _d
    lib.ref_pair_blocks.argtypes = [_P, _P, _i, _i, _i, _f, _f, _f, _P]
    lib.ref_pair_blocks_n.argtypes = [_P, _P, _i, _i, _i, _f, _f, _f, _i, _P]
    lib.ref_gauss_legendre.argtypes = [_i, _P, _P]
    lib.ref_incident_fields.argtypes = [_i, _P, _P, _i, _d, _d, _i, _P, _P, _P]
    lib.ref_rhs_dipole.argtypes = [_i, _P, _P, _P, _i, _i, _i, _P, _P, _i, _d, _d, _i, _d, _d, _P, _i, _d, _d]
    lib.ref_assemble.argtypes = _ASSEMBLE
    lib.ref_rhs_plane_wave.argtypes = [_i, _P, _P, _P, _i, _i, _i, _P, _P, _d, _d, _i, _d, _d, _P, _i, _d, _d]
    lib.ref_surface_fields.argtypes = _FIELDS
    lib.ref_lu_solve.argtypes = [_i, _P, _P, _P, _i, _i]
    lib.ref_lu_solve.restype = _d
    lib.ref_max_threads.restype = _i
    return lib


REF_GPU_SO = HERE / "_ref" / "libsieref_gpu.so"


def reference_gpu() -> ctypes.CDLL | None:
    """The reference's own GPU dielectric solver (oracle/ref_gpu_harness.cu,
    make -C oracle ref_gpu), or None when it has not been built."""
    if not REF_GPU_SO.exists():
        return None
    lib = ctypes.CDLL(str(REF_GPU_SO))
    lib.ref_gpu_last_error.restype = ctypes.c_char_p
    lib.ref_gpu_solve_dielectric.argtypes = [_P, _i, _P, _i, _P, _P, _i, _d, _d, _i, _P, _P]
    lib.ref_gpu_solve_dielectric.restype = _i
    return lib


def reference_gpu_dielectric(lib, mesh, frequency_hz: float, eps_r: float, rule: int):
    """(physical interior-oriented currents [J, M], timings dict) of the
    reference's solve_dielectric_dense for an x-polarised plane wave along +z."""
    V = np.ascontiguousarray(mesh.vertices, dtype=np.float64)
    F = np.ascontiguousarray(mesh.faces, dtype=np.int32)
    E = np.ascontiguousarray(mesh.edges, dtype=np.int32)
    FE = np.ascontiguousarray(mesh.faces_edges, dtype=np.int32)
    ne = E.shape[0]
    cur = np.zeros(2 * ne, np.complex128)
    t = np.zeros(6)
    rc = lib.ref_gpu_solve_dielectric(_p(V), V.shape[0], _p(F), F.shape[0], _p(E), _p(FE), ne, float(frequency_hz),
                                      float(eps_r), int(rule), _p(cur), _p(t))
    if rc != 0:
        raise RuntimeError("reference GPU solve failed: " + lib.ref_gpu_last_error().decode(errors="replace"))
    return cur, {"device_preparation_seconds": t[0], "assembly_seconds": t[1], "solve_seconds": t[2],
                 "residual_seconds": t[3], "call_seconds": t[4], "relative_residual": t[5]}


def _p(a):
    return None if a is None else a.ctypes.data


def dimension(kind: int, ne: int) -> int:
    return ne * (1, 2, 4)[kind]


def kernel_scalars(kind: int, frequency_hz: float, eps_r=(1.0, 1.0), mu_r=(1.0, 1.0),
                   threshold_lambda0: float = 0.1, eps0: float | None = None,
                   mu0: float | None = None) -> dict:
    """The float kernel arguments the reference solvers pass
    (pec_solver.cu:338-359, dielectric_solver.cu:312-321, gstc_sie.cu:281-290):
    eps_r/mu_r = (interior, exterior)."""
    if eps0 is None:
        eps0 = 8.8541878188e-12 if kind == 2 else 8.8541878128e-12
    if mu0 is None:
        mu0 = 1.25663706127e-6 if kind == 2 else 1.25663706212e-6
    omega = 2.0 * np.pi * frequency_hz
    k1 = omega * np.sqrt(mu_r[0] * mu0 * eps_r[0] * eps0)
    k2 = omega * np.sqrt(mu_r[1] * mu0 * eps_r[1] * eps0)
    if kind == 2:
        thr = threshold_lambda0 * (1.0 / np.sqrt(mu0 * eps0)) / frequency_hz
    else:
        thr = threshold_lambda0 * 2.0 * np.pi / (omega * np.sqrt(mu0 * eps0))
    if kind == 0:
        k1 = k2
    return dict(k1=k1, k2=k2, mu_r1=mu_r[0], mu_r2=mu_r[1], eps_r1=eps_r[0], eps_r2=eps_r[1],
                mu0=mu0, eps0=eps0, omega=omega, thr=thr)


def assemble(lib, kind: int, mesh, rule: int, scalars: dict, tensors=None, uniform=False,
             basis=0, threads=0, fn="so_assemble", variant: int = 0, line_points: int = 0) -> np.ndarray:
    """variant 1: rotated (n x RWG) testing, N-EFIE (kind 0) or N-PMCHWT
    (kind 1), surface nTL form; variant 2: N-MFIE (kind 0) or N-Muller
    (kind 1); line_points > 0 selects the line nTL form A with that many
    Gauss-Legendre points (N-EFIE, N-PMCHWT, N-Muller)."""
    V = np.ascontiguousarray(mesh.vertices, dtype=np.float64)
    F = np.ascontiguousarray(mesh.faces, dtype=np.int32)
    FE = np.ascontiguousarray(mesh.faces_edges, dtype=np.int32)
    ne = int(mesh.edges.shape[0])
    N = dimension(kind, ne)
    Z = np.zeros((N, N), dtype=np.complex128, order="F")
    t = None if tensors is None else np.ascontiguousarray(tensors, dtype=np.complex128)
    s = scalars
    getattr(lib, fn)(kind, _p(V), _p(F), _p(FE), F.shape[0], ne, rule, s["k1"], s["k2"], s["mu_r1"],
                     s["mu_r2"], s["eps_r1"], s["eps_r2"], s["mu0"], s["eps0"], s["omega"], s["thr"],
                     _p(t), int(uniform), int(basis), _p(Z), int(threads), int(variant), int(line_points))
    return Z


def assemble_rows(lib, kind: int, mesh, rule: int, scalars: dict, rows, tensors=None, uniform=False, basis=0,
                  threads=0, variant: int = 0, line_points: int = 0) -> np.ndarray:
    """Rows `rows` of the matrix assemble() gives (len(rows) x N), computed
    from the test faces that hold their edges only."""
    V = np.ascontiguousarray(mesh.vertices, dtype=np.float64)
    F = np.ascontiguousarray(mesh.faces, dtype=np.int32)
    FE = np.ascontiguousarray(mesh.faces_edges, dtype=np.int32)
    ne = int(mesh.edges.shape[0])
    N = dimension(kind, ne)
    rows = np.asarray(rows, dtype=np.int64)
    rowmap = np.full(N, -1, np.int32)
    rowmap[rows] = np.arange(rows.size, dtype=np.int32)
    edges = np.unique(rows % ne)
    faces = np.unique(np.nonzero(np.isin(FE, edges).any(axis=1))[0]).astype(np.int32)
    out = np.zeros((rows.size, N), dtype=np.complex128, order="F")
    t = None if tensors is None else np.ascontiguousarray(tensors, dtype=np.complex128)
    s = scalars
    rc = lib.so_assemble_rows(kind, _p(V), _p(F), _p(FE), F.shape[0], ne, rule, s["k1"], s["k2"], s["mu_r1"],
                              s["mu_r2"], s["eps_r1"], s["eps_r2"], s["mu0"], s["eps0"], s["omega"], s["thr"],
                              _p(t), int(uniform), int(basis), _p(faces), faces.size, _p(rowmap), rows.size,
                              _p(out), int(threads), int(variant), int(line_points))
    if rc != 0:
        raise ValueError("oracle assembly: invalid rule")
    return out


def rhs(lib, kind: int, mesh, rule: int, source: dict, k: float, eta: float, mu0: float,
        eps0: float, variant: int = 0, eps_r_src: float = 1.0, mu_r_src: float = 1.0) -> np.ndarray:
    """source: {'kind': 0|1, 'a': (3,), 'b': (3,), 'is_magnetic': bool, 'region': 1|2};
    variant as for assemble(); eps_r_src, mu_r_src: the source region's medium
    (used by N-Muller)."""
    V = np.ascontiguousarray(mesh.vertices, dtype=np.float64)
    F = np.ascontiguousarray(mesh.faces, dtype=np.int32)
    FE = np.ascontiguousarray(mesh.faces_edges, dtype=np.int32)
    ne = int(mesh.edges.shape[0])
    b = np.zeros(dimension(kind, ne), dtype=np.complex128)
    a = np.ascontiguousarray(source["a"], dtype=np.float64)
    bb = np.ascontiguousarray(source["b"], dtype=np.float64)
    lib.so_rhs(kind, source["kind"], _p(V), _p(F), _p(FE), F.shape[0], ne, rule, _p(a), _p(bb),
               int(source.get("is_magnetic", 0)), k, eta, source["region"], mu0, eps0, _p(b),
               int(variant), float(eps_r_src), float(mu_r_src))
    return b


def far_field(lib, mesh, j, m, k0, eta0, r_hat, theta_hat, phi_hat):
    V = np.ascontiguousarray(mesh.vertices, dtype=np.float64)
    F = np.ascontiguousarray(mesh.faces, dtype=np.int32)
    j = np.ascontiguousarray(j, dtype=np.complex128)
    m = None if m is None else np.ascontiguousarray(m, dtype=np.complex128)
    rh, th, ph = (np.ascontiguousarray(x, dtype=np.float64) for x in (r_hat, theta_hat, phi_hat))
    nd = rh.shape[0]
    ft = np.zeros(nd, np.complex128)
    fp = np.zeros(nd, np.complex128)
    U = np.zeros(nd)
    rc = lib.so_far_field(_p(V), _p(F), F.shape[0], int(mesh.edges.shape[0]), _p(j), _p(m), k0, eta0,
                          nd, _p(rh), _p(th), _p(ph), _p(ft), _p(fp), _p(U))
    if rc != 0:
        raise ValueError("oracle far field: edge numbering mismatch")
    return ft, fp, U


def surface_fields(lib, mesh, j, m, points, frequency_hz, eps_r=1.0, mu_r=1.0, eps0=8.8541878188e-12,
                   mu0=1.25663706127e-6, rule=17):
    """(E, H) surface-integral terms (nobs x 3 complex) from the C
    restatement (lib = oracle()) or the reference harness (lib = reference())."""
    V = np.ascontiguousarray(mesh.vertices, dtype=np.float64)
    F = np.ascontiguousarray(mesh.faces, dtype=np.int32)
    FE = np.ascontiguousarray(mesh.faces_edges, dtype=np.int32)
    j = np.ascontiguousarray(j, dtype=np.complex128)
    m = None if m is None else np.ascontiguousarray(m, dtype=np.complex128)
    P = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
    E = np.zeros((P.shape[0], 3), np.complex128)
    H = np.zeros((P.shape[0], 3), np.complex128)
    fn = lib.so_surface_fields if hasattr(lib, "so_surface_fields") else lib.ref_surface_fields
    rc = fn(_p(V), _p(F), _p(FE), F.shape[0], int(mesh.edges.shape[0]), _p(j), _p(m), P.shape[0], _p(P),
            float(frequency_hz), float(eps_r), float(mu_r), float(eps0), float(mu0), int(rule), _p(E), _p(H))
    if rc != 0:
        raise ValueError("surface fields: invalid quadrature rule")
    return E, H


def incident_fields(lib, source: dict, k: float, eta: float, points):
    """Incident (E, H) at points (n x 3 complex) of a source dict as for rhs()
    (plane-wave direction normalised here, as the library prepares it), from
    the C restatement (lib = oracle()) or the reference's functors
    (lib = reference())."""
    P = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
    a = np.ascontiguousarray(source["a"], dtype=np.float64)
    b = np.ascontiguousarray(source["b"], dtype=np.float64)
    if source["kind"] == 0:
        b = b / np.linalg.norm(b)
    E = np.zeros((P.shape[0], 3), np.complex128)
    H = np.zeros((P.shape[0], 3), np.complex128)
    fn = lib.so_incident_fields if hasattr(lib, "so_incident_fields") else lib.ref_incident_fields
    fn(int(source["kind"]), _p(a), _p(b), int(source.get("is_magnetic", 0)), float(k), float(eta), P.shape[0],
       _p(P), _p(E), _p(H))
    return E, H


# ------------------------------------------------------------------ meshes
# The synthetic spheres of the benchmark workloads, generated here without
# the library so that the reference arm of the benchmark and the checks that
# compare against it never load libsieb200.so. Construction (the same as the
# library's generator, asserted vertex- and index-equal by the tests):
# SphericalSurface's icosahedron (src/sie_mom/mesh/spherical_surface.cpp:19-80),
# each face split on a barycentric grid of the given frequency, projected to
# the sphere by multiplying with the reciprocal length, faces oriented CCW
# outward, RWG edges numbered by first appearance (so_build_edges).

class OracleMesh:
    def __init__(self, vertices: np.ndarray, faces: np.ndarray):
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float64)
        self.faces = np.ascontiguousarray(faces, dtype=np.int32)
        nf = self.faces.shape[0]
        fe = np.zeros((nf, 3), np.int32)
        tmp = np.zeros((3 * nf, 2), np.int32)
        ne = oracle().so_build_edges(_p(self.faces), nf, _p(tmp), _p(fe))
        self.edges = tmp[:ne].copy()
        self.faces_edges = fe

    @property
    def num_faces(self) -> int:
        return int(self.faces.shape[0])

    @property
    def num_edges(self) -> int:
        return int(self.edges.shape[0])


def _unit(v: np.ndarray) -> np.ndarray:
    inv = 1.0 / np.sqrt(v[..., 0] * v[..., 0] + v[..., 1] * v[..., 1] + v[..., 2] * v[..., 2])
    return v * inv[..., None]


def _outward(vertices: np.ndarray, faces: np.ndarray) -> None:
    v0, v1, v2 = (vertices[faces[:, i]] for i in range(3))
    n = np.cross(v1 - v0, v2 - v0)
    c = (v0 + v1 + v2) / 3.0
    flip = np.einsum("ij,ij->i", n, c) < 0
    faces[flip, 1], faces[flip, 2] = faces[flip, 2].copy(), faces[flip, 1].copy()


def _icosahedron():
    phi = (1.0 + np.sqrt(5.0)) / 2.0
    V = np.array([(-1, phi, 0), (1, phi, 0), (-1, -phi, 0), (1, -phi, 0), (0, -1, phi), (0, 1, phi),
                  (0, -1, -phi), (0, 1, -phi), (phi, 0, -1), (phi, 0, 1), (-phi, 0, -1), (-phi, 0, 1)],
                 dtype=np.float64)
    F = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
                  (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
                  (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)], dtype=np.int32)
    V = _unit(V)
    _outward(V, F)
    return V, F


def geodesic_sphere(radius: float, frequency: int) -> OracleMesh:
    """Class-I geodesic sphere: 20 n^2 faces, 30 n^2 edges."""
    BV, BF = _icosahedron()
    n = int(frequency)
    index: dict[tuple, int] = {}
    verts: list[np.ndarray] = []

    def vid(face, i: int, j: int) -> int:
        corners = ((int(face[0]), n - i - j), (int(face[1]), i), (int(face[2]), j))
        key = tuple(sorted((c, w) for c, w in corners if w > 0))
        if key not in index:
            p = 0
            for c, w in corners:
                p = p + BV[c] * (w / n)
            verts.append(_unit(p) * radius)
            index[key] = len(verts) - 1
        return index[key]

    faces = []
    for face in BF:
        for i in range(n):
            for j in range(n - i):
                faces.append((vid(face, i, j), vid(face, i + 1, j), vid(face, i, j + 1)))
                if i + j < n - 1:
                    faces.append((vid(face, i + 1, j), vid(face, i + 1, j + 1), vid(face, i, j + 1)))
    V = np.array(verts)
    F = np.array(faces, dtype=np.int32)
    _outward(V, F)
    return OracleMesh(V, F)


def icosphere(radius: float, level: int) -> OracleMesh:
    """SphericalSurface(radius, level): 20 * 4^level faces, midpoints
    normalised, float radius (spherical_surface.cpp:19-80)."""
    BV, _ = _icosahedron()
    V = list(BV)
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
         (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
         (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache: dict[tuple[int, int], int] = {}

        def mid(i: int, j: int) -> int:
            key = (min(i, j), max(i, j))
            if key not in cache:
                V.append(_unit((V[i] + V[j]) * 0.5))
                cache[key] = len(V) - 1
            return cache[key]

        nf = []
        for a, b, c in F:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (ab, b, bc), (ca, bc, c), (ab, bc, ca)]
        F = nf
    verts = np.array(V) * float(np.float32(radius))
    faces = np.array(F, dtype=np.int32)
    _outward(verts, faces)
    return OracleMesh(verts, faces)
