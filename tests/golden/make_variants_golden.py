"""Regenerate tests/golden/variants_golden.npz: the rotated-testing
formulations (N-EFIE, N-MFIE, N-PMCHWT, N-Muller; surface nTL form B and line
form A) as the reference computes them.

Run in a checkout that has the reference sources and the harness built
(make -C oracle):
    python tests/golden/make_variants_golden.py

Source of truth: oracle/_ref/libsieref.so, the reference's own quadrature
(calculateDoubleQuadrature_nTL_nTK, calculateSingularPartQuadrature_nTL_nTK,
calculateFormAQuadrature_nTL_nTK and its singular part, gauss_legendre_rule,
calculateMassMatrixQuadrature, calculateExcitationQuadrature<NxRWG>) in the
loops of n_pmchwt_kernel / n_muller_kernel
(src/sie_mom/solvers/dielectric/dielectric_kernels.cu:155-489) and
assemble_pec_n_efie/n_mfie_operator_kernel (src/sie_mom/solvers/pec_solver.cu:113-240),
driven by oracle/ref_harness.cpp. Meshes come from golden.npz (the
reference's icospheres). Everything is small and deterministic.
"""

from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402

C0 = 299792458.0
OUT = Path(__file__).resolve().parent / "variants_golden.npz"

# name -> (kind, variant, media, Gauss-Legendre points of the line form A; 0: surface form B)
CASES = {
    "n_efie": (0, 1, {}, 0),
    "n_mfie": (0, 2, {}, 0),
    "n_pmchwt": (1, 1, dict(eps_r=(4.0, 1.0), mu_r=(1.0, 1.0)), 0),
    "n_muller": (1, 2, dict(eps_r=(2.5, 1.0), mu_r=(1.5, 1.0)), 0),
    "n_efie_line": (0, 1, {}, 20),
    "n_pmchwt_line": (1, 1, dict(eps_r=(4.0, 1.0), mu_r=(1.0, 1.0)), 10),
    "n_muller_line": (1, 2, dict(eps_r=(2.5, 1.0), mu_r=(1.5, 1.0)), 7),
}


class _Mesh:
    def __init__(self, g, name):
        self.vertices = g[f"ico_{name}_V"]
        self.faces = g[f"ico_{name}_F"].astype(np.int32)
        self.edges = g[f"ico_{name}_E"].astype(np.int32)
        self.faces_edges = g[f"ico_{name}_FE"].astype(np.int32)


def main() -> None:
    ref = O.reference()
    if ref is None:
        raise SystemExit("build the reference harness first: make -C oracle")
    g = dict(np.load(ROOT / "tests" / "golden" / "golden.npz"))
    L0 = _Mesh(g, "L0")
    L1 = _Mesh(g, "L1r05")
    out = {}
    # The line-form cases use the icosahedron scaled to radius 0.3 at 3 C0
    # (same electrical size): at unit scale the reference's line form gives
    # non-finite values (kept below as Z_n_efie_line_unit_L0).
    L0s = _Mesh(g, "L0")
    L0s.vertices = 0.3 * L0s.vertices
    for name, (kind, variant, media, line_points) in CASES.items():
        # frequency C0 (lambda0 = 1 m) with a 1.5 lambda0 threshold on the
        # unit icosahedron: self and neighbouring pairs take the extracted path.
        mesh, freq = (L0s, 3 * C0) if line_points else (L0, C0)
        s = O.kernel_scalars(kind, freq, **media, threshold_lambda0=1.5)
        out[f"Z_{name}_L0"] = O.assemble(ref, kind, mesh, 5, s, fn="ref_assemble", variant=variant,
                                         threads=1, line_points=line_points)
        if name == "n_efie_line":
            su = O.kernel_scalars(kind, C0, **media, threshold_lambda0=1.5)
            out["Z_n_efie_line_unit_L0"] = O.assemble(ref, kind, L0, 5, su, fn="ref_assemble",
                                                      variant=variant, threads=1, line_points=line_points)
        eps_r = media.get("eps_r", (1.0, 1.0))
        mu_r = media.get("mu_r", (1.0, 1.0))
        regions = (2, 1) if kind == 1 else (2,)
        for region in regions:
            er, mr = eps_r[region - 1], mu_r[region - 1]
            k = s["omega"] * math.sqrt(s["mu0"] * s["eps0"] * er * mr)
            eta = math.sqrt(s["mu0"] * mr / (s["eps0"] * er))
            b = np.zeros(O.dimension(kind, L0.edges.shape[0]), np.complex128)
            E0 = np.array([1.0, 0.0, 0.0])
            kh = np.array([0.0, 0.0, 1.0])
            ref.ref_rhs_plane_wave(kind, mesh.vertices.ctypes.data, mesh.faces.ctypes.data,
                                   mesh.faces_edges.ctypes.data, L0.faces.shape[0], L0.edges.shape[0], 5,
                                   E0.ctypes.data, kh.ctypes.data, k, eta, region, s["mu0"], s["eps0"],
                                   b.ctypes.data, variant, er, mr)
            out[f"b_{name}_L0_region{region}"] = b
    # Face-pair nTL/nTK blocks on icosphere L1 (r = 0.5): self, edge
    # neighbour, vertex neighbour and far pairs, rule 6, 0.3 lambda0 at 2 C0.
    s = O.kernel_scalars(1, 2 * C0, eps_r=(4.0, 1.0), threshold_lambda0=0.3)
    pairs = np.array([[0, 0], [0, 1], [0, 5], [3, 7], [10, 30], [17, 62]], np.int32)
    blocks = np.zeros((pairs.shape[0], 72))
    for p, (m, n) in enumerate(pairs):
        ref.ref_pair_blocks_n(L1.vertices.ctypes.data, L1.faces.ctypes.data, int(m), int(n), 6,
                              s["k1"], s["k2"], s["thr"], 0, blocks[p].ctypes.data)
    blocks_line = np.zeros((pairs.shape[0], 72))
    for p, (m, n) in enumerate(pairs):
        ref.ref_pair_blocks_n(L1.vertices.ctypes.data, L1.faces.ctypes.data, int(m), int(n), 6,
                              s["k1"], s["k2"], s["thr"], 12, blocks_line[p].ctypes.data)
    # Incident fields of the reference's source functors at seeded points
    # (plane wave, electric and magnetic dipoles; k, eta of a medium 3 / 1.5).
    rng = np.random.default_rng(77)
    P = rng.uniform(-1.0, 1.0, (40, 3))
    k = 2 * np.pi * C0 * np.sqrt(1.25663706127e-6 * 1.5 * 8.8541878188e-12 * 3.0)
    eta = np.sqrt(1.25663706127e-6 * 1.5 / (8.8541878188e-12 * 3.0))
    srcs = [(0, [0.0, 2.0, 0.0], [1.0, 0.0, 0.0], 0), (1, [0.2, 0.0, 1.0], [0.1, 0.05, 0.0], 1),
            (1, [0.0, 1.0, 0.0], [0.0, 0.0, 0.2], 0)]
    for q, (kind, a, b, mag) in enumerate(srcs):
        E = np.zeros((P.shape[0], 3), np.complex128)
        H = np.zeros((P.shape[0], 3), np.complex128)
        a = np.array(a)
        b = np.array(b)
        ref.ref_incident_fields(kind, a.ctypes.data, b.ctypes.data, mag, float(k), float(eta), P.shape[0],
                                P.ctypes.data, E.ctypes.data, H.ctypes.data)
        out[f"inc{q}_E"] = E
        out[f"inc{q}_H"] = H
        out[f"inc{q}_source"] = np.concatenate(([kind, mag], a, b))
    out["inc_points"] = P
    # Dipole right-hand sides on the unit icosahedron, every formulation and
    # testing variant, interior and exterior sources (rule 5, f = C0).
    for kind, variant, region, mag in [(0, 0, 2, 0), (0, 1, 2, 1), (0, 2, 2, 0), (1, 0, 1, 1), (1, 1, 1, 0),
                                       (1, 2, 1, 1), (1, 2, 2, 0), (2, 0, 1, 0), (2, 0, 2, 1)]:
        er, mr = (2.5, 1.5) if region == 1 else (1.0, 1.0)
        kd = 2 * np.pi * C0 * np.sqrt(1.25663706212e-6 * mr * 8.8541878128e-12 * er)
        etad = np.sqrt(1.25663706212e-6 * mr / (8.8541878128e-12 * er))
        mom = np.array([0.3, -0.2, 1.0])
        pos = np.array([0.1, 0.0, 0.05]) if region == 1 else np.array([0.4, 1.8, -0.3])
        bd = np.zeros(O.dimension(kind, L0.edges.shape[0]), np.complex128)
        ref.ref_rhs_dipole(kind, L0.vertices.ctypes.data, L0.faces.ctypes.data, L0.faces_edges.ctypes.data,
                           L0.faces.shape[0], L0.edges.shape[0], 5, mom.ctypes.data, pos.ctypes.data, mag,
                           float(kd), float(etad), region, 1.25663706212e-6, 8.8541878128e-12, bd.ctypes.data,
                           variant, er, mr)
        out[f"bdip_{kind}_{variant}_{region}_{mag}"] = bd
    out["inc_k_eta"] = np.array([k, eta])
    out["pair_n_index"] = pairs
    out["pair_n_blocks"] = blocks
    out["pair_n_blocks_line12"] = blocks_line
    # The reference's Gauss-Legendre rules on [0, 1] (gauss_legendre_rule.cpp).
    for n in range(1, 21):
        t = np.zeros(n)
        w = np.zeros(n)
        ref.ref_gauss_legendre(n, t.ctypes.data, w.ctypes.data)
        out[f"gl{n}_nodes"] = t
        out[f"gl{n}_weights"] = w
    out["pair_n_scalars"] = np.array([s["k1"], s["k2"], s["thr"]], np.float32)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
