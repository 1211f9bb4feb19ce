"""File formats of the SIE-GSTC applications (little-endian binaries).

face_tensors.bin  per face 32 complex values (Y then Z, 4x4 row-major each),
                  complex64 or complex128, told apart by the file size
                  (include/sie_mom/gstc_utils.hpp:158-210)
currents.bin      physical RWG coefficients [J1, M1, J2, M2] as interleaved
                  float64 pairs (anisotropic_sphere_app.cpp:519-549)
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np


def load_face_tensors(path: str | Path, num_faces: int) -> np.ndarray:
    """(num_faces, 32) complex128 records; complex64 files are widened."""
    path = str(path)
    try:
        data = Path(path).read_bytes()
    except OSError:
        raise RuntimeError(f"Could not open tensor file: {path}") from None
    values = num_faces * 32 * 2
    f32, f64 = values * 4, values * 8
    if len(data) not in (f32, f64):
        raise RuntimeError(f"Tensor file size mismatch. Expected {f32} or {f64} bytes, got {len(data)}")
    raw = np.frombuffer(data, dtype="<f4" if len(data) == f32 else "<f8").astype(np.float64)
    return (raw[0::2] + 1j * raw[1::2]).reshape(num_faces, 32)


def save_face_tensors(path: str | Path, tensors, single: bool = False) -> None:
    t = np.ascontiguousarray(tensors, dtype=np.complex64 if single else np.complex128).reshape(-1)
    Path(path).write_bytes(t.astype("<c8" if single else "<c16").tobytes())


def write_physical_currents(path: str | Path, currents) -> None:
    if sys.byteorder != "little":
        raise RuntimeError("currents.bin export currently requires a little-endian host")
    c = np.ascontiguousarray(currents, dtype=np.complex128).reshape(-1)
    Path(path).write_bytes(c.astype("<c16").tobytes())


def read_physical_currents(path: str | Path) -> np.ndarray:
    return np.frombuffer(Path(path).read_bytes(), dtype="<c16").astype(np.complex128)
