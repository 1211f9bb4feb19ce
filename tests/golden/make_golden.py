"""Regenerate tests/golden/golden.npz from the reference implementation itself.

Run in a checkout that has the reference sources, named by the first
argument or the SIE_REFERENCE environment variable:
    python tests/golden/make_golden.py /path/to/reference

Sources of truth:
  * oracle/_ref/libsieref.so: the reference's own host-compiled quadrature
    (include/sie_mom/cuda/*.cuh, USE_DOUBLE_PRECISION) behind
    oracle/ref_harness.cpp, built by oracle/Makefile. Gives Dunavant rules,
    icosphere meshes (SphericalSurface), Wilton potentials, face-pair blocks,
    assembled Z and right-hand sides in ref-compat mode.
  * applications/anisotropic_gstc_sphere/plot_far_field.py imported from the
    reference (matplotlib stubbed, plotting unused): far-field vectors of a
    seeded current vector.
Everything is seeded; the file holds only small cases (icosphere level 0).
"""

from __future__ import annotations

import subprocess
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "sie-gstc-2026_b200"))

from oracle import oracle as O  # noqa: E402


class _Mesh:
    def __init__(self, V, F, E, FE):
        self.vertices, self.faces, self.edges, self.faces_edges = V, F, E, FE


def ref_icosphere(ref, radius, level):
    import ctypes
    nv, nf, ne = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    ref.ref_icosphere(radius, level, ctypes.byref(nv), ctypes.byref(nf), ctypes.byref(ne),
                      None, None, None, None)
    V = np.zeros((nv.value, 3))
    F = np.zeros((nf.value, 3), np.int32)
    E = np.zeros((ne.value, 2), np.int32)
    FE = np.zeros((nf.value, 3), np.int32)
    ref.ref_icosphere(radius, level, ctypes.byref(nv), ctypes.byref(nf), ctypes.byref(ne),
                      V.ctypes.data, F.ctypes.data, E.ctypes.data, FE.ctypes.data)
    return _Mesh(V, F, E, FE)


def reference_far_field(refdir: Path, mesh, currents, frequency_hz, theta, phi):
    mpl = types.ModuleType("matplotlib")
    mpl.use = lambda *a, **k: None
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", types.ModuleType("matplotlib.pyplot"))
    sys.path[:0] = [str(refdir / "src"), str(refdir / "applications/anisotropic_gstc_sphere")]
    import plot_far_field as pff  # the reference's own evaluator

    with tempfile.TemporaryDirectory() as tmp:
        path = Path(tmp) / "currents.bin"
        currents.astype(np.complex128).tofile(path)
        ev = pff.MetasurfaceFarFieldEvaluator(pff.TriangleMesh(mesh.vertices, mesh.faces), path,
                                              frequency_hz)
        st, ct, sp, cp = np.sin(theta), np.cos(theta), np.sin(phi), np.cos(phi)
        r_hat = np.column_stack([st * cp, st * sp, ct])
        th_hat = np.column_stack([ct * cp, ct * sp, -st])
        ph_hat = np.column_stack([-sp, cp, np.zeros_like(sp)])
        ft, fp, U = ev.evaluate_directions(r_hat, th_hat, ph_hat)
        return r_hat, th_hat, ph_hat, ft, fp, U, ev.k0, ev.eta0


def reference_dir() -> Path:
    """The reference checkout: first argument, else $SIE_REFERENCE."""
    import os
    d = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SIE_REFERENCE")
    if not d:
        raise SystemExit("name the reference checkout: make_golden.py /path/to/reference (or set SIE_REFERENCE)")
    return Path(d)


def main() -> None:
    refdir = reference_dir()
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref", f"REF={refdir}"], check=True)
    ref = O.reference()
    assert ref is not None, "reference harness did not build"
    out: dict[str, np.ndarray] = {}

    for rule in range(1, 21):
        n = ref.ref_dunavant(rule, None, None)
        p = np.zeros(2 * n, np.float32)
        w = np.zeros(n, np.float32)
        ref.ref_dunavant(rule, p.ctypes.data, w.ctypes.data)
        out[f"rule{rule}_points"], out[f"rule{rule}_weights"] = p, w

    meshes = {"L0": ref_icosphere(ref, 1.0, 0), "L1r05": ref_icosphere(ref, 0.5, 1)}
    for name, m in meshes.items():
        out[f"ico_{name}_V"], out[f"ico_{name}_F"] = m.vertices, m.faces
        out[f"ico_{name}_E"], out[f"ico_{name}_FE"] = m.edges, m.faces_edges

    # Wilton potentials: observation points around and on a source triangle.
    rng = np.random.default_rng(1234)
    tri = meshes["L0"].vertices[meshes["L0"].faces[0]]
    c = tri.mean(0)
    n = np.cross(tri[1] - tri[0], tri[2] - tri[0])
    n /= np.linalg.norm(n)
    pts = [c, c + 0.1 * n, c - 0.3 * n, tri[0] * 0.6 + tri[1] * 0.3 + tri[2] * 0.1 + 0.02 * n,
           c + rng.normal(size=3) * 0.5, c + 2.0 * n + rng.normal(size=3)]
    W = np.zeros((len(pts), 12))
    for i, r in enumerate(pts):
        r = np.ascontiguousarray(r, dtype=np.float64)
        ref.ref_wilton(r.ctypes.data, np.ascontiguousarray(tri).ctypes.data, W[i].ctypes.data)
    out["wilton_tri"], out["wilton_points"], out["wilton_values"] = tri, np.array(pts), W

    # Dense matrices and right-hand sides on icosphere L0 (30 edges), rule 5,
    # free-space k0 = 2 pi (f = c0), as the reference kernels assemble them.
    c0 = 299792458.0
    L0 = meshes["L0"]
    tens = (rng.standard_normal((20, 32)) + 1j * rng.standard_normal((20, 32)))
    uniform = (rng.standard_normal(32) + 1j * rng.standard_normal(32))
    out["gstc_tensors_L0"], out["gstc_tensors_uniform"] = tens, uniform
    cases = {
        "pec": (0, dict(eps_r=(1.0, 1.0), mu_r=(1.0, 1.0)), None, False, 0),
        "pmchwt": (1, dict(eps_r=(4.0, 1.0), mu_r=(1.0, 1.0)), None, False, 0),
        "gstc_face": (2, dict(eps_r=(1.0, 1.0), mu_r=(1.0, 1.0)), tens, False, 0),
        "gstc_sph_uniform": (2, dict(eps_r=(2.0, 1.0), mu_r=(1.0, 1.0)), uniform, True, 1),
    }
    for name, (kind, media, t, uni, basis) in cases.items():
        s = O.kernel_scalars(kind, c0, **media, threshold_lambda0=0.1)
        Z = O.assemble(ref, kind, L0, 5, s, tensors=t, uniform=uni, basis=basis, threads=1,
                       fn="ref_assemble")
        out[f"Z_{name}_L0"] = Z
        eps0, mu0 = s["eps0"], s["mu0"]
        omega = s["omega"]
        k = omega * np.sqrt(mu0 * eps0 * media["eps_r"][1] * media["mu_r"][1])
        eta = np.sqrt(mu0 * media["mu_r"][1] / (eps0 * media["eps_r"][1]))
        b = np.zeros(Z.shape[0], np.complex128)
        E0 = np.array([1.0, 0.0, 0.0])
        kh = np.array([0.0, 0.0, 1.0])
        ref.ref_rhs_plane_wave(kind, L0.vertices.ctypes.data, L0.faces.ctypes.data,
                               L0.faces_edges.ctypes.data, 20, 30, 5, E0.ctypes.data, kh.ctypes.data,
                               k, eta, 2, mu0, eps0, b.ctypes.data, 0, 1.0, 1.0)
        out[f"b_{name}_L0"] = b

    # Far field of a seeded [J1, M1, J2, M2] vector on icosphere L1 r=0.5.
    L1 = meshes["L1r05"]
    ne = L1.edges.shape[0]
    cur = rng.standard_normal(4 * ne) + 1j * rng.standard_normal(4 * ne)
    theta = np.linspace(0.0, np.pi, 19)
    phi = np.linspace(0.0, 2 * np.pi, 19)
    rh, th, ph, ft, fp, U, k0, eta0 = reference_far_field(refdir, L1, cur, c0, theta, phi)
    out.update(ff_currents=cur, ff_r_hat=rh, ff_theta_hat=th, ff_phi_hat=ph, ff_f_theta=ft,
               ff_f_phi=fp, ff_U=U, ff_k0=np.array(k0), ff_eta0=np.array(eta0))

    np.savez_compressed(Path(__file__).with_name("golden.npz"), **out)
    print("wrote", Path(__file__).with_name("golden.npz"))


if __name__ == "__main__":
    main()
