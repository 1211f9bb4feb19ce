"""Surface-parameter record preparation on the device, for loops that rebuild
the GSTC records every step (adjoint design, sweeps): the checks, the
impedance-balanced inversion and the 32-value record layout of
src/sie_mom/gstc/tensor_io.py:13-132. On a CUDA device one library kernel
(sieb200_prepare_records, one thread per face: balanced map, constraint
defects, one-sided Jacobi singular values, pivoted 4x4 inverse, residuals)
does the per-face work; on the CPU the same steps run batched in torch.

Records: per face the row-major 4x4 map [[Y_ee, Y_em], [Y_me, Y_mm]] followed
by its full inverse (complex128), the layout face_tensors.bin and the
assembly read.
"""

from __future__ import annotations

import math

import numpy as np

CONSTRAINT_TOLERANCE = 1e-10
INVERSE_TOLERANCE = 1e-8


def _torch():
    import torch
    return torch


def _blocks(parameters):
    if isinstance(parameters, dict):
        return [parameters[k] for k in ("Y_ee", "Y_em", "Y_me", "Y_mm")]
    return [getattr(parameters, k) for k in ("Y_ee", "Y_em", "Y_me", "Y_mm")]


def prepare_tensor_records(parameters, face_count: int, *, reference_impedance: float, extraction_method: str,
                           tensor_structure: str, device=None, hermitian_solver: str = "auto"):
    """(records, diagnostics): records a (face_count, 32) complex128 tensor on
    `device` (default: the current CUDA device). parameters: an object or dict
    with Y_ee, Y_em, Y_me, Y_mm of shape (2, 2, face_count) (numpy arrays or
    tensors). Raises ValueError with the reference's messages: reciprocity,
    losslessness (extraction_method "reciprocal_lossless"), diagonal
    structure (tensor_structure "diagonal"), numerical singularity
    (s_min <= 4 eps s_max) and the two-sided inverse residual (1e-8).
    On CUDA the library's record kernel inverts every map by pivoted
    elimination (hermitian_solver is not used there); on the CPU lossless
    maps are inverted as the Hermitian system (i B) X = i I by LDL^H
    (hermitian_solver "lu" forces LU), the others by LU."""
    torch = _torch()
    dev = torch.device(device) if device is not None else torch.device("cuda")
    eta = float(reference_impedance)
    if not math.isfinite(eta) or eta <= 0:
        raise ValueError("reference_impedance must be finite and positive")
    blocks = []
    for name, b in zip(("Y_ee", "Y_em", "Y_me", "Y_mm"), _blocks(parameters)):
        t = torch.as_tensor(b, device=dev)
        if tuple(t.shape) != (2, 2, face_count) or not (t.is_complex() or t.is_floating_point()) or \
                not bool(torch.isfinite(torch.view_as_real(t) if t.is_complex() else t).all()):
            raise ValueError(f"surface block {name} must be finite with shape (2, 2, {face_count})")
        blocks.append(t.to(torch.complex128))
    top = torch.cat((blocks[0], blocks[1]), dim=1)
    bottom = torch.cat((blocks[2], blocks[3]), dim=1)
    matrix = torch.cat((top, bottom), dim=0).permute(2, 0, 1).contiguous()  # (F, 4, 4)
    if dev.type == "cuda":
        return _prepare_on_device(matrix, face_count, eta, extraction_method, tensor_structure, dev)
    # impedance balance: eta on the Y_ee block, 1/eta on the Y_mm block
    balanced = matrix.clone()
    balanced[:, :2, :2] *= eta
    balanced[:, 2:, 2:] /= eta
    if not bool(torch.isfinite(torch.view_as_real(balanced)).all()):
        raise ValueError("impedance-balanced surface maps must be finite")
    tiny = torch.finfo(torch.float64).tiny
    scale = torch.clamp(balanced.abs().amax(dim=(1, 2)), min=tiny)

    def rel(defect):
        return float((defect.abs().amax(dim=(1, 2)) / scale).max())

    reciprocity = max(rel(balanced[:, :2, :2] - balanced[:, :2, :2].transpose(1, 2)),
                      rel(balanced[:, 2:, 2:] - balanced[:, 2:, 2:].transpose(1, 2)),
                      rel(balanced[:, 2:, :2] + balanced[:, :2, 2:].transpose(1, 2)))
    losslessness = rel(balanced + balanced.conj().transpose(1, 2))
    if reciprocity > CONSTRAINT_TOLERANCE:
        raise ValueError("surface maps do not satisfy reciprocity")
    if extraction_method == "reciprocal_lossless" and losslessness > CONSTRAINT_TOLERANCE:
        raise ValueError("surface maps do not satisfy losslessness")
    if tensor_structure == "diagonal":
        off = balanced.clone()
        idx = torch.arange(4, device=dev)
        off[:, idx, idx] = 0
        if rel(off) > CONSTRAINT_TOLERANCE:
            raise ValueError("surface maps do not satisfy the configured diagonal structure")
    sv = torch.linalg.svdvals(balanced)
    singular = sv[:, -1] <= 4 * np.finfo(float).eps * sv[:, 0]
    if bool(singular.any()):
        first = int(torch.nonzero(singular)[0, 0])
        raise ValueError(f"surface map is numerically singular at {int(singular.sum())} faces "
                         f"(first face index {first}); the current SIE interface requires its full inverse")
    eye = torch.eye(4, dtype=torch.complex128, device=dev).expand(face_count, 4, 4)
    try:
        ldl = hermitian_solver == "ldl" or (hermitian_solver == "auto" and dev.type == "cpu")
        if extraction_method == "reciprocal_lossless" and ldl:
            # B^H = -B, so i B is Hermitian and (i B) X = i I gives B^-1.
            LD, piv = torch.linalg.ldl_factor(1j * balanced, hermitian=True)
            binv = torch.linalg.ldl_solve(LD, piv, 1j * eye, hermitian=True)
        elif extraction_method == "reciprocal_lossless":
            # The same system by LU: torch has no complex Hermitian LDL^H solve
            # on CUDA. The two-sided residual check below holds either way.
            binv = torch.linalg.solve(1j * balanced, 1j * eye)
        else:
            binv = torch.linalg.inv(balanced)
    except RuntimeError as error:
        raise ValueError("surface map is singular; the current SIE interface requires its full inverse") from error
    inverse = binv.clone()
    inverse[:, :2, :2] *= eta
    inverse[:, 2:, 2:] /= eta
    if not bool(torch.isfinite(torch.view_as_real(inverse)).all()):
        raise ValueError("surface map inverse must be finite")
    balanced_inverse = inverse.clone()
    balanced_inverse[:, :2, :2] /= eta
    balanced_inverse[:, 2:, 2:] *= eta
    residual = float(max(torch.linalg.matrix_norm(balanced @ balanced_inverse - eye).max(),
                         torch.linalg.matrix_norm(balanced_inverse @ balanced - eye).max()))
    if not math.isfinite(residual) or residual > INVERSE_TOLERANCE:
        raise ValueError(f"surface map inversion residual {residual:.3g} exceeds {INVERSE_TOLERANCE}")
    physical_residual = float(torch.linalg.matrix_norm(matrix @ inverse - eye).max())
    if not math.isfinite(physical_residual):
        raise ValueError("physical surface map inversion residual must be finite")
    records = torch.cat((matrix.reshape(-1, 16), inverse.reshape(-1, 16)), dim=1)
    return records, {
        "all_tensors_finite": True,
        "relative_constraint_tolerance": CONSTRAINT_TOLERANCE,
        "balanced_inverse_tolerance": INVERSE_TOLERANCE,
        "maximum_relative_reciprocity_residual": reciprocity,
        "maximum_relative_skew_hermitian_residual": losslessness,
        "maximum_map_condition_number": float((sv[:, 0] / sv[:, -1]).max()),
        "maximum_balanced_inverse_residual": residual,
        "maximum_inverse_residual": physical_residual,
    }


def _prepare_on_device(matrix, face_count: int, eta: float, extraction_method: str, tensor_structure: str, dev):
    """The checks and inversion by the library's record kernel
    (sieb200_prepare_records, one thread per face), then the reference's
    tolerances and messages in the reference's order."""
    import ctypes
    from . import _lib
    from .solvers import Context, default_context
    torch = _torch()
    ctx = default_context() if (dev.index or 0) == 0 else Context(dev.index)
    records = torch.empty((face_count, 32), dtype=torch.complex128, device=dev)
    diag = torch.empty((face_count, 8), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    _lib.check(_lib.lib().sieb200_prepare_records(ctx.handle, face_count, matrix.data_ptr(), ctypes.c_double(eta),
                                                  records.data_ptr(), diag.data_ptr()))
    d = diag.cpu().numpy()
    flags = d[:, 7].astype(np.int64)
    if (flags & 1).any():
        raise ValueError("impedance-balanced surface maps must be finite")
    reciprocity = float(d[:, 0].max()) if face_count else 0.0
    losslessness = float(d[:, 1].max()) if face_count else 0.0
    if reciprocity > CONSTRAINT_TOLERANCE:
        raise ValueError("surface maps do not satisfy reciprocity")
    if extraction_method == "reciprocal_lossless" and losslessness > CONSTRAINT_TOLERANCE:
        raise ValueError("surface maps do not satisfy losslessness")
    if tensor_structure == "diagonal" and face_count and float(d[:, 2].max()) > CONSTRAINT_TOLERANCE:
        raise ValueError("surface maps do not satisfy the configured diagonal structure")
    singular = d[:, 4] <= 4 * np.finfo(float).eps * d[:, 3]
    if singular.any():
        raise ValueError(f"surface map is numerically singular at {int(singular.sum())} faces "
                         f"(first face index {int(np.flatnonzero(singular)[0])}); the current SIE interface "
                         "requires its full inverse")
    if (flags & 2).any():
        raise ValueError("surface map is singular; the current SIE interface requires its full inverse")
    if (flags & 4).any():
        raise ValueError("surface map inverse must be finite")
    if (flags & 8).any():
        raise ValueError("impedance-balanced inverse must be finite")
    residual = float(d[:, 5].max()) if face_count else 0.0
    if not math.isfinite(residual) or residual > INVERSE_TOLERANCE:
        raise ValueError(f"surface map inversion residual {residual:.3g} exceeds {INVERSE_TOLERANCE}")
    physical_residual = float(d[:, 6].max()) if face_count else 0.0
    if not math.isfinite(physical_residual):
        raise ValueError("physical surface map inversion residual must be finite")
    return records, {
        "all_tensors_finite": True,
        "relative_constraint_tolerance": CONSTRAINT_TOLERANCE,
        "balanced_inverse_tolerance": INVERSE_TOLERANCE,
        "maximum_relative_reciprocity_residual": reciprocity,
        "maximum_relative_skew_hermitian_residual": losslessness,
        "maximum_map_condition_number": float((d[:, 3] / d[:, 4]).max()) if face_count else 0.0,
        "maximum_balanced_inverse_residual": residual,
        "maximum_inverse_residual": physical_residual,
    }
