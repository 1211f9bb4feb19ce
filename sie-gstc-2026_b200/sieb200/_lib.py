"""ctypes binding of libsieb200.so (declarations: include/sieb200.h).

The library is the only compute path: importing this module on a machine
without the built library tries to build it with nvcc and raises if that is
impossible. There is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path

import numpy as np

from . import _build

OK, INVALID_ARG, OVERFLOW, SINGULAR, NONFINITE, NOT_CONVERGED, CUDA_ERROR, TIMEOUT, NO_DEVICE, \
    OUT_OF_MEMORY, UNSUPPORTED = range(11)
VARIANT_T, VARIANT_N, VARIANT_N_JUMP = 0, 1, 2
NTL_SURFACE, NTL_LINE = 0, 1
PEC_EFIE, PMCHWT, GSTC = 0, 1, 2
ABI_VERSION = 3  # SIEB200_ABI_VERSION of include/sieb200.h
SOLVER_LU_FP64, SOLVER_LU_CUSOLVER, SOLVER_MIXED_IR, SOLVER_GMRES_C64 = 0, 1, 2, 3

_STATUS_NAMES = {
    INVALID_ARG: "invalid argument", OVERFLOW: "overflow", SINGULAR: "singular matrix",
    NONFINITE: "non-finite value", NOT_CONVERGED: "not converged", CUDA_ERROR: "CUDA error",
    TIMEOUT: "timeout", NO_DEVICE: "no CUDA device", OUT_OF_MEMORY: "out of device memory",
    UNSUPPORTED: "unsupported option",
}


class SiebError(RuntimeError):
    """Error raised for a non-zero status of the C ABI."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class InvalidArgument(SiebError, ValueError):
    pass


class Mesh(ctypes.Structure):
    _fields_ = [("vertices", ctypes.c_void_p), ("num_vertices", ctypes.c_int64),
                ("faces", ctypes.c_void_p), ("num_faces", ctypes.c_int64),
                ("faces_edges", ctypes.c_void_p), ("num_edges", ctypes.c_int64)]


class Options(ctypes.Structure):
    _fields_ = [("formulation", ctypes.c_int), ("frequency_hz", ctypes.c_double),
                ("eps_r_interior", ctypes.c_double), ("mu_r_interior", ctypes.c_double),
                ("eps_r_exterior", ctypes.c_double), ("mu_r_exterior", ctypes.c_double),
                ("quadrature_rule", ctypes.c_int), ("singularity_threshold_lambda0", ctypes.c_double),
                ("vacuum_permittivity", ctypes.c_double), ("vacuum_permeability", ctypes.c_double),
                ("basis", ctypes.c_int), ("tensors_are_uniform", ctypes.c_int),
                ("compute_residual", ctypes.c_int), ("solver", ctypes.c_int),
                ("tolerance", ctypes.c_double), ("max_iterations", ctypes.c_int),
                ("restart", ctypes.c_int), ("variant", ctypes.c_int), ("ntl_form", ctypes.c_int),
                ("line_quadrature_points", ctypes.c_int)]


class Source(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("region", ctypes.c_int), ("a", ctypes.c_double * 3),
                ("b", ctypes.c_double * 3), ("is_magnetic", ctypes.c_int)]


class Metrics(ctypes.Structure):
    _fields_ = [("matrix_dimension", ctypes.c_int64), ("dense_matrix_bytes", ctypes.c_int64),
                ("assembly_seconds", ctypes.c_double), ("factorization_seconds", ctypes.c_double),
                ("solve_seconds", ctypes.c_double), ("residual_seconds", ctypes.c_double),
                ("residual_computed", ctypes.c_int), ("rhs_norm", ctypes.c_double),
                ("absolute_residual", ctypes.c_double), ("relative_residual", ctypes.c_double),
                ("maximum_coefficient", ctypes.c_double * 4), ("refinement_iterations", ctypes.c_int),
                ("solver", ctypes.c_int)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["maximum_coefficient"] = list(self.maximum_coefficient)
        return d


class SweepInstance(ctypes.Structure):
    _fields_ = [("mesh", Mesh), ("tensors", ctypes.c_void_p), ("opt", Options), ("source", Source * 2),
                ("currents_out", ctypes.c_void_p), ("metrics", ctypes.POINTER(Metrics))]


_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_SIGNATURES = {
    "sieb200_last_error": ([], ctypes.c_char_p),
    "sieb200_version": ([], ctypes.c_int),
    "sieb200_ctx_create": ([ctypes.c_int, ctypes.POINTER(_P)], ctypes.c_int),
    "sieb200_ctx_destroy": ([_P], ctypes.c_int),
    "sieb200_ctx_synchronize": ([_P], ctypes.c_int),
    "sieb200_ctx_stream": ([_P], _P),
    "sieb200_quadrature_rule": ([ctypes.c_int, _P, _P], ctypes.c_int),
    "sieb200_build_edges": ([_P, _I64, _P, _P, ctypes.POINTER(_I64)], ctypes.c_int),
    "sieb200_options_default": ([ctypes.c_int, ctypes.POINTER(Options)], ctypes.c_int),
    "sieb200_solve_pec_dense": ([_P, ctypes.POINTER(Mesh), ctypes.POINTER(Options),
                                 ctypes.POINTER(Source), _P, ctypes.POINTER(Metrics)], ctypes.c_int),
    "sieb200_solve_dielectric_dense": ([_P, ctypes.POINTER(Mesh), ctypes.POINTER(Options),
                                        ctypes.POINTER(Source), _P, ctypes.POINTER(Metrics)], ctypes.c_int),
    "sieb200_solve_gstc_dense_batch": ([_P, ctypes.POINTER(Mesh), _P, ctypes.POINTER(Options),
                                        ctypes.POINTER(Source), ctypes.c_int, _P, ctypes.POINTER(Metrics)],
                                       ctypes.c_int),
    "sieb200_assemble_matrix": ([_P, ctypes.POINTER(Mesh), ctypes.POINTER(Options), _P, _P,
                                 ctypes.c_int], ctypes.c_int),
    "sieb200_assemble_rhs": ([_P, ctypes.POINTER(Mesh), ctypes.POINTER(Options), ctypes.POINTER(Source),
                              ctypes.c_int, _P, ctypes.c_int], ctypes.c_int),
    "sieb200_dense_solver_create": ([_P, _I64, ctypes.c_int, ctypes.POINTER(_P)], ctypes.c_int),
    "sieb200_dense_solver_destroy": ([_P], ctypes.c_int),
    "sieb200_dense_solver_factorize": ([_P, _P, _I64], ctypes.c_int),
    "sieb200_dense_solver_solve": ([_P, _I64, _P, _I64, ctypes.c_double, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "sieb200_dense_solver_solve_adjoint": ([_P, _I64, _P, _I64, ctypes.c_double, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "sieb200_matvec": ([_P, _I64, _P, _I64, ctypes.c_int, _P, ctypes.c_double, _P], ctypes.c_int),
    "sieb200_matvec_noalloc": ([_P, _I64, _P, _I64, ctypes.c_int, _P, ctypes.c_double, _P], ctypes.c_int),
    "sieb200_gstc_tensor_gradient": ([_P, _P, _P, _P, _P, ctypes.c_int, _P], ctypes.c_int),
    "sieb200_matvec_matrix_free": ([_P, _P, _P, _P, _P, _P, ctypes.c_int], ctypes.c_int),
    "sieb200_surface_fields": ([_P, _P, _P, _P, _I64, _P, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                ctypes.c_double, ctypes.c_double, ctypes.c_int, _P, _P], ctypes.c_int),
    "sieb200_far_field_matrix": ([_P, _P, ctypes.c_double, ctypes.c_double, _I64, _P, _P, _P, ctypes.c_int, _P],
                                 ctypes.c_int),
    "sieb200_incident_fields": ([_P, _P, _P, _I64, _P, _P, _P], ctypes.c_int),
    "sieb200_profile_enable": ([_P, ctypes.c_int], ctypes.c_int),
    "sieb200_fp64_fma_peak": ([_P, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "sieb200_fp64_mma_peak": ([_P, ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "sieb200_profile_timeline": ([_P, _I64, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_I64)], ctypes.c_int),
    "sieb200_launch_count": ([], ctypes.c_int64),
    "sieb200_profile_read": ([_P, ctypes.c_int, ctypes.POINTER(_I64), ctypes.POINTER(ctypes.c_double),
                              ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "sieb200_solve_gstc_sweep": ([_P, _P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)],
                                 ctypes.c_int),
    "sieb200_prepare_records": ([_P, _I64, _P, ctypes.c_double, _P, _P], ctypes.c_int),
    "sieb200_zgemm": ([_P, _I64, _I64, _I64, _P, _I64, _P, _I64, _P, _I64, _P, _P], ctypes.c_int),
    "sieb200_gemm_tf32_sub": ([_P, _I64, _I64, ctypes.c_int, _P, _P, _P, _I64, ctypes.c_int], ctypes.c_int),
    "sieb200_gemm_tf32_sub_shifted": ([_P, _I64, _I64, ctypes.c_int, _P, _P, _P, _I64, ctypes.c_int, _I64],
                                      ctypes.c_int),
    "sieb200_far_field": ([_P, ctypes.POINTER(Mesh), _P, _P, ctypes.c_double, ctypes.c_double, _I64,
                           _P, _P, _P, _P, _P, _P], ctypes.c_int),
}

_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


def library_path() -> Path:
    return _build.LIB


def lib() -> ctypes.CDLL:
    """Load (building first if needed) libsieb200.so and bind its C ABI."""
    global _lib
    with _lock:
        if _lib is None:
            path = _build.build()
            handle = ctypes.CDLL(str(path))
            for name, (args, res) in _SIGNATURES.items():
                fn = getattr(handle, name)
                fn.argtypes = args
                fn.restype = res
            if handle.sieb200_version() != ABI_VERSION:
                raise RuntimeError(f"{path} implements C ABI version {handle.sieb200_version()}, this binding "
                                   f"needs {ABI_VERSION}: rebuild the library")
            _lib = handle
        return _lib


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


def check(status: int) -> int:
    if status in (OK,):
        return status
    msg = lib().sieb200_last_error().decode(errors="replace")
    if status == INVALID_ARG:
        raise InvalidArgument(status, msg)
    raise SiebError(status, msg)


def ptr(a: np.ndarray | None) -> int | None:
    if a is None:
        return None
    return a.ctypes.data


def default_options(formulation: int) -> Options:
    o = Options()
    check(lib().sieb200_options_default(formulation, ctypes.byref(o)))
    return o
