"""Regenerate tests/golden/records_golden.npz from the reference's own
surface-record preparation (src/sie_mom/gstc/tensor_io.py, imported from the
reference checkout; pure numpy/scipy).

    python tests/golden/make_records_golden.py /path/to/reference   (or $SIE_REFERENCE)

Seeded inputs: 64 reciprocal lossless maps with an ill-scaled spectrum, 32
reciprocal complex maps, 16 diagonal lossless maps; each case stores the four
(2, 2, F) blocks and the reference's (F, 32) records and diagnostics.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

REF = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SIE_REFERENCE", ""))
OUT = Path(__file__).resolve().parent / "records_golden.npz"
ETA = 376.730313668


def lossless_maps(rng, F, spread):
    """Balanced maps B with B^H = -B and reciprocity: ee, mm = i (real
    symmetric), em real, me = -em^T; returned in physical units."""
    out = np.zeros((F, 4, 4), complex)
    for f in range(F):
        q, _ = np.linalg.qr(rng.normal(size=(2, 2)))
        s_ee = (q * rng.uniform(0.2, 2.0, 2) * np.array([1.0, spread])) @ q.T
        q, _ = np.linalg.qr(rng.normal(size=(2, 2)))
        s_mm = (q * rng.uniform(0.2, 2.0, 2)) @ q.T
        em = rng.normal(size=(2, 2))
        B = np.zeros((4, 4), complex)
        B[:2, :2] = 1j * s_ee
        B[2:, 2:] = 1j * s_mm
        B[:2, 2:] = em
        B[2:, :2] = -em.T
        M = B.copy()
        M[:2, :2] /= ETA
        M[2:, 2:] *= ETA
        out[f] = M
    return out


def complex_maps(rng, F):
    out = np.zeros((F, 4, 4), complex)
    for f in range(F):
        a = rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2))
        b = rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2))
        em = rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2))
        B = np.zeros((4, 4), complex)
        B[:2, :2] = a + a.T + 3 * np.eye(2)
        B[2:, 2:] = b + b.T + 3 * np.eye(2)
        B[:2, 2:] = em
        B[2:, :2] = -em.T
        M = B.copy()
        M[:2, :2] /= ETA
        M[2:, 2:] *= ETA
        out[f] = M
    return out


def main() -> None:
    if not str(REF) or str(REF) == ".":
        raise SystemExit("name the reference checkout: make_records_golden.py /path/to/reference (or set SIE_REFERENCE)")
    sys.path.insert(0, str(REF / "src"))
    from sie_mom.gstc import SurfaceParameters
    from sie_mom.gstc.tensor_io import prepare_tensor_records
    rng = np.random.default_rng(2026)
    diag = np.zeros((16, 4, 4), complex)
    for f in range(16):
        diag[f] = np.diag(1j * rng.uniform(0.5, 2.0, 4) * np.array([1 / ETA, 1 / ETA, ETA, ETA]))
    cases = {
        "lossless": (lossless_maps(rng, 64, 1e-5), "reciprocal_lossless", "general"),
        "complex": (complex_maps(rng, 32), "reciprocal_complex", "general"),
        "diagonal": (diag, "reciprocal_lossless", "diagonal"),
    }
    out = {}
    for name, (maps, method, structure) in cases.items():
        m = np.moveaxis(maps, 0, -1)
        p = SurfaceParameters(m[:2, :2], m[:2, 2:], m[2:, :2], m[2:, 2:])
        records, diag_out = prepare_tensor_records(p, maps.shape[0], reference_impedance=ETA,
                                                   extraction_method=method, tensor_structure=structure)
        out[f"{name}_maps"] = maps
        out[f"{name}_records"] = records
        out[f"{name}_condition"] = diag_out["maximum_map_condition_number"]
    out["eta"] = ETA
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
