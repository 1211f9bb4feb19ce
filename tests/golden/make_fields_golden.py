"""Regenerate tests/golden/fields_golden.npz from the reference implementation.

Run in a checkout that has the reference sources and oracle/_ref built
(python -c "import __graft_entry__ as g; g.build()"):
    python tests/golden/make_fields_golden.py

Source of truth: ref_surface_fields in oracle/_ref/libsieref.so, which runs the
reference's own per-face helpers calculateScatterFieldQuadrature and
calculateScatterFieldSingular (include/sie_mom/cuda/dunavant_quadrature.cuh:
1634-1770, compiled from the reference headers) in the loop of
compute_scattered_fields_kernel (sie_kernels_utils.cuh:21-140) with the
constants of surface_current_fields.cu:96-112 and :255-275. The mesh is the
reference's own SphericalSurface (ref_icosphere). Everything is seeded.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1]))

from make_golden import ref_icosphere  # noqa: E402
from oracle import oracle as O  # noqa: E402

# Observation points around a unit sphere: far, within 0.1 lambda of the
# surface (extracted quadrature + Wilton part for the nearby faces), inside.
POINTS = np.array([
    [0.0, 0.0, 3.0], [2.0, -1.0, 0.5], [0.2, 0.1, 1.05], [0.5, 0.5, 0.72],
    [0.0, 0.0, 0.9], [0.3, -0.6, 0.2], [-0.7, 0.1, 0.75], [0.05, 0.02, 0.0],
])
CASES = [  # (name, frequency, eps_r, mu_r, rule)
    ("vac_r5", 299792458.0 / 4.0, 1.0, 1.0, 5),
    ("diel_r7", 299792458.0 / 3.0, 2.5, 1.2, 7),
]


def main() -> None:
    ref = O.reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libsieref.so is missing: build it first")
    mesh = ref_icosphere(ref, 1.0, 1)
    rng = np.random.default_rng(20261203)
    ne = mesh.edges.shape[0]
    J = rng.standard_normal(ne) + 1j * rng.standard_normal(ne)
    M = rng.standard_normal(ne) + 1j * rng.standard_normal(ne)
    out = {"V": mesh.vertices, "F": mesh.faces, "Ed": mesh.edges, "FE": mesh.faces_edges, "J": J, "M": M,
           "points": POINTS, "eps0": 8.8541878188e-12, "mu0": 1.25663706127e-6}
    for name, f, er, mr, rule in CASES:
        E, H = O.surface_fields(ref, mesh, J, M, POINTS, f, er, mr, rule=rule)
        out[f"{name}_params"] = np.array([f, er, mr, rule])
        out[f"{name}_E"], out[f"{name}_H"] = E, H
    np.savez_compressed(HERE / "fields_golden.npz", **out)
    print("wrote", HERE / "fields_golden.npz")


if __name__ == "__main__":
    main()
