"""Reference-shaped solver API over the C ABI.

Names, argument meaning and error behaviour follow the SIE-GSTC solver's C++
API (paths relative to that project):
    solve_pec_dense           include/sie_mom/solvers/pec_solver.hpp:57-61
    solve_dielectric_dense    include/sie_mom/solvers/dielectric/dielectric_solver.hpp:92-96
    solve_gstc_dense          include/sie_mom/solvers/gstc_sie.hpp:214-219
    solve_gstc_dense_batch    include/sie_mom/solvers/gstc_sie.hpp:226-239
    DenseLuSolver             include/sie_mom/cuda/dense_lu_solver.cuh:17-184
Invalid inputs raise ValueError (the reference's std::invalid_argument);
singular or non-finite results raise SiebError (std::runtime_error).
"""

from __future__ import annotations

import ctypes
import threading
import weakref
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from .mesh import MeshData

SOLVERS = {"lu_fp64": _lib.SOLVER_LU_FP64, "lu_cusolver": _lib.SOLVER_LU_CUSOLVER,
           "mixed_ir": _lib.SOLVER_MIXED_IR, "gmres_c64": 3}


@dataclass
class IsotropicMedium:
    relative_permittivity: float = 1.0
    relative_permeability: float = 1.0


INTERIOR, EXTERIOR = 1, 2


@dataclass
class PlaneWaveExcitation:
    electric_amplitude: Sequence[float] = (1.0, 0.0, 0.0)
    propagation_direction: Sequence[float] = (0.0, 0.0, 1.0)
    region: int = EXTERIOR

    def as_c(self) -> _lib.Source:
        s = _lib.Source()
        s.kind, s.region, s.is_magnetic = 0, int(self.region), 0
        s.a[:] = [float(x) for x in self.electric_amplitude]
        s.b[:] = [float(x) for x in self.propagation_direction]
        return s


@dataclass
class DipoleExcitation:
    effective_moment: Sequence[float] = (0.0, 0.0, 1.0)
    position: Sequence[float] = (0.0, 0.0, 0.0)
    is_magnetic: bool = False
    region: int = INTERIOR

    def as_c(self) -> _lib.Source:
        s = _lib.Source()
        s.kind, s.region, s.is_magnetic = 1, int(self.region), int(bool(self.is_magnetic))
        s.a[:] = [float(x) for x in self.effective_moment]
        s.b[:] = [float(x) for x in self.position]
        return s


# PecFormulation (pec_solver.hpp:12) and DielectricFormulation
# (dielectric_solver.hpp:15-19) by enum name, plus the applications' CLI
# spellings (pec_sphere_app.cpp:83-92, pmchwt_app.cpp:158-167).
PEC_FORMULATIONS = {"TEfie": _lib.VARIANT_T, "NEfie": _lib.VARIANT_N, "NMfie": _lib.VARIANT_N_JUMP,
                    "t-efie": _lib.VARIANT_T, "n-efie": _lib.VARIANT_N, "n-mfie": _lib.VARIANT_N_JUMP,
                    "t": _lib.VARIANT_T, "n": _lib.VARIANT_N}
DIELECTRIC_FORMULATIONS = {"T_PMCHWT": _lib.VARIANT_T, "N_PMCHWT": _lib.VARIANT_N,
                           "N_Muller": _lib.VARIANT_N_JUMP, "t": _lib.VARIANT_T, "n": _lib.VARIANT_N,
                           "muller": _lib.VARIANT_N_JUMP}
NTL_FORMS = {"Surface": _lib.NTL_SURFACE, "Line": _lib.NTL_LINE, "surface": _lib.NTL_SURFACE,
             "line": _lib.NTL_LINE}


@dataclass
class PecOptions:
    frequency_hz: float = 0.0
    exterior: IsotropicMedium = field(default_factory=IsotropicMedium)
    quadrature_rule: int = 7
    singularity_threshold_lambda0: float = 0.1
    compute_residual: bool = True
    formulation: str = "TEfie"
    ntl_form: str = "Surface"
    line_quadrature_points: int = 20
    vacuum_permittivity: float = 8.8541878128e-12
    vacuum_permeability: float = 1.25663706212e-6
    solver: str = "lu_cusolver"
    tolerance: float = 1e-10
    max_iterations: int = 50


@dataclass
class DielectricOptions:
    frequency_hz: float = 0.0
    interior: IsotropicMedium = field(default_factory=IsotropicMedium)
    exterior: IsotropicMedium = field(default_factory=IsotropicMedium)
    quadrature_rule: int = 17
    singularity_threshold_lambda0: float = 0.1
    compute_residual: bool = True
    vacuum_permittivity: float = 8.8541878128e-12
    vacuum_permeability: float = 1.25663706212e-6
    formulation: str = "T_PMCHWT"
    ntl_form: str = "Surface"
    line_quadrature_points: int = 20
    solver: str = "lu_cusolver"
    tolerance: float = 1e-10
    max_iterations: int = 50


@dataclass
class GstcSieOptions:
    frequency_hz: float = 0.0
    interior: IsotropicMedium = field(default_factory=IsotropicMedium)
    exterior: IsotropicMedium = field(default_factory=IsotropicMedium)
    quadrature_rule: int = 17
    singularity_threshold_lambda0: float = 0.1
    tensors_are_uniform: bool = False
    compute_residual: bool = True
    basis: str = "face"
    vacuum_permittivity: float = 8.8541878188e-12
    vacuum_permeability: float = 1.25663706127e-6
    solver: str = "lu_cusolver"
    tolerance: float = 1e-10
    max_iterations: int = 50


def to_c_options(opt, formulation: int) -> _lib.Options:
    o = _lib.default_options(formulation)
    o.frequency_hz = float(opt.frequency_hz)
    if formulation != _lib.PEC_EFIE:
        o.eps_r_interior = float(opt.interior.relative_permittivity)
        o.mu_r_interior = float(opt.interior.relative_permeability)
    o.eps_r_exterior = float(opt.exterior.relative_permittivity)
    o.mu_r_exterior = float(opt.exterior.relative_permeability)
    o.quadrature_rule = int(opt.quadrature_rule)
    o.singularity_threshold_lambda0 = float(opt.singularity_threshold_lambda0)
    o.vacuum_permittivity = float(opt.vacuum_permittivity)
    o.vacuum_permeability = float(opt.vacuum_permeability)
    o.compute_residual = int(bool(opt.compute_residual))
    if opt.solver not in SOLVERS:
        raise ValueError(f"unknown solver {opt.solver!r}; choose one of {sorted(SOLVERS)}")
    o.solver = SOLVERS[opt.solver]
    o.tolerance = float(opt.tolerance)
    o.max_iterations = int(opt.max_iterations)
    if formulation != _lib.GSTC:
        table = PEC_FORMULATIONS if formulation == _lib.PEC_EFIE else DIELECTRIC_FORMULATIONS
        if opt.formulation not in table:
            raise ValueError(f"unknown formulation {opt.formulation!r}; choose one of {sorted(table)}")
        if opt.ntl_form not in NTL_FORMS:
            raise ValueError("ntl_form must be 'Surface' or 'Line'")
        o.variant = table[opt.formulation]
        o.ntl_form = NTL_FORMS[opt.ntl_form]
        o.line_quadrature_points = int(opt.line_quadrature_points)
        line_integrated = (o.variant == _lib.VARIANT_N if formulation == _lib.PEC_EFIE
                           else o.variant != _lib.VARIANT_T)
        if o.ntl_form == _lib.NTL_LINE and line_integrated and \
                not 1 <= int(opt.line_quadrature_points) <= 20:
            # pec_solver.cu:91-95, dielectric_solver.cu:116-122
            raise ValueError("Gauss-Legendre point count must be in [1, 20]")
    if formulation == _lib.GSTC:
        if opt.basis not in ("face", "spherical"):
            raise ValueError("unsupported GSTC basis type")
        o.basis = 0 if opt.basis == "face" else 1
        o.tensors_are_uniform = int(bool(opt.tensors_are_uniform))
    return o


class Context:
    """One CUDA stream plus reusable device workspaces (sieb200_ctx)."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        _lib.check(_lib.lib().sieb200_ctx_create(int(device), ctypes.byref(self._h)))
        self.device = device
        # Solvers made on this context; closed before it (they use its stream).
        self._solvers = weakref.WeakSet()

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    @property
    def stream(self) -> int:
        return _lib.lib().sieb200_ctx_stream(self._h) or 0

    def synchronize(self) -> None:
        _lib.check(_lib.lib().sieb200_ctx_synchronize(self._h))

    def profile(self, enable: bool = True, timeline: bool = False) -> None:
        """Start (and reset) or stop event timing of the library's hot kernels;
        with timeline=True every span is also kept with its start and end."""
        mode = (2 if timeline else 1) if enable else 0
        _lib.check(_lib.lib().sieb200_profile_enable(self._h, mode))

    def fp64_fma_peak(self) -> float:
        """Measured FP64 FMA throughput of this context's device, TFLOP/s."""
        t = ctypes.c_double()
        _lib.check(_lib.lib().sieb200_fp64_fma_peak(self._h, ctypes.byref(t)))
        return t.value

    def fp64_mma_peak(self) -> float:
        """Measured FP64 tensor-core (mma.sync .f64) throughput, TFLOP/s."""
        t = ctypes.c_double()
        _lib.check(_lib.lib().sieb200_fp64_mma_peak(self._h, ctypes.byref(t)))
        return t.value

    def profile_timeline(self) -> list:
        """[(kernel kind, start_ms, end_ms)] of the spans since profile(timeline=True),
        times relative to that call (kinds as in profile_read)."""
        count = ctypes.c_int64()
        _lib.check(_lib.lib().sieb200_profile_timeline(self._h, 0, None, None, None, ctypes.byref(count)))
        n = count.value
        kinds = (ctypes.c_int * max(n, 1))()
        t0 = (ctypes.c_double * max(n, 1))()
        t1 = (ctypes.c_double * max(n, 1))()
        _lib.check(_lib.lib().sieb200_profile_timeline(self._h, n, kinds, t0, t1, ctypes.byref(count)))
        return [(kinds[i], t0[i], t1[i]) for i in range(min(n, count.value))]

    def profile_read(self, kernel: int) -> dict:
        """kernel 0: split-TF32 trailing GEMM, 1: triangular solves, 2: FP64 matvec
        and complex GEMM, 3: diagonal-block LU, 4: block-step panels (L21 and U12),
        5: multi-right-hand-side block triangular solves,
        6: whole mixed factorizations, 7: whole refined solves."""
        n = ctypes.c_int64()
        ms, fl, by = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _lib.check(_lib.lib().sieb200_profile_read(self._h, int(kernel), ctypes.byref(n), ctypes.byref(ms),
                                                   ctypes.byref(fl), ctypes.byref(by)))
        return {"launches": n.value, "ms": ms.value, "flops": fl.value, "bytes": by.value}

    def close(self) -> None:
        if self._h:
            for solver in list(self._solvers):
                solver.close()
            _lib.lib().sieb200_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_tls = threading.local()


def default_context() -> Context:
    ctx = getattr(_tls, "ctx", None)
    if ctx is None:
        ctx = Context(0)
        _tls.ctx = ctx
    return ctx


@dataclass
class SolveResult:
    currents: np.ndarray
    metrics: dict


def _metrics(m: _lib.Metrics) -> dict:
    return m.as_dict()


def solve_pec_dense(mesh: MeshData, options: PecOptions, source, ctx: Optional[Context] = None) -> SolveResult:
    ctx = ctx or default_context()
    o = to_c_options(options, _lib.PEC_EFIE)
    out = np.zeros(mesh.num_edges, dtype=np.complex128)
    m = _lib.Metrics()
    src = source.as_c()
    _lib.check(_lib.lib().sieb200_solve_pec_dense(ctx.handle, ctypes.byref(mesh.as_c()), ctypes.byref(o),
                                                  ctypes.byref(src), out.ctypes.data, ctypes.byref(m)))
    return SolveResult(out, _metrics(m))


def solve_dielectric_dense(mesh: MeshData, options: DielectricOptions, source,
                           ctx: Optional[Context] = None) -> SolveResult:
    ctx = ctx or default_context()
    o = to_c_options(options, _lib.PMCHWT)
    out = np.zeros(2 * mesh.num_edges, dtype=np.complex128)
    m = _lib.Metrics()
    src = source.as_c()
    _lib.check(_lib.lib().sieb200_solve_dielectric_dense(ctx.handle, ctypes.byref(mesh.as_c()),
                                                         ctypes.byref(o), ctypes.byref(src),
                                                         out.ctypes.data, ctypes.byref(m)))
    return SolveResult(out, _metrics(m))


@dataclass
class GstcExcitationCase:
    interior: Optional[object] = None
    exterior: Optional[object] = None


def _tensor_array(mesh: MeshData, tensors, uniform: bool) -> np.ndarray:
    t = np.ascontiguousarray(np.asarray(tensors, dtype=np.complex128).reshape(-1))
    expected = 32 if uniform else 32 * mesh.num_faces
    if t.size != expected:
        raise ValueError(f"GSTC tensor count mismatch: expected {expected}, got {t.size}")
    return t


def solve_gstc_dense_batch(mesh: MeshData, tensors, options: GstcSieOptions,
                           cases: Sequence[GstcExcitationCase], ctx: Optional[Context] = None):
    ctx = ctx or default_context()
    if len(cases) == 0:
        raise ValueError("SIE batch must contain at least one excitation case")
    o = to_c_options(options, _lib.GSTC)
    t = _tensor_array(mesh, tensors, options.tensors_are_uniform)
    srcs = (_lib.Source * (2 * len(cases)))()
    for c, case in enumerate(cases):
        for slot, s in enumerate((case.interior, case.exterior)):
            if s is None:
                srcs[2 * c + slot].kind = -1
            else:
                srcs[2 * c + slot] = s.as_c()
    N = 4 * mesh.num_edges
    out = np.zeros((len(cases), N), dtype=np.complex128)
    ms = (_lib.Metrics * len(cases))()
    _lib.check(_lib.lib().sieb200_solve_gstc_dense_batch(
        ctx.handle, ctypes.byref(mesh.as_c()), t.ctypes.data, ctypes.byref(o), srcs, len(cases),
        out.ctypes.data, ms))
    return [SolveResult(out[c], _metrics(ms[c])) for c in range(len(cases))]


def solve_gstc_dense(mesh: MeshData, tensors, options: GstcSieOptions, source,
                     ctx: Optional[Context] = None) -> SolveResult:
    case = GstcExcitationCase(interior=source if source.region == INTERIOR else None,
                              exterior=source if source.region == EXTERIOR else None)
    return solve_gstc_dense_batch(mesh, tensors, options, [case], ctx)[0]


@dataclass
class SweepInstance:
    """One system of a batched sweep: a mesh, its tensor records, GSTC
    options and up to one interior and one exterior source."""
    mesh: MeshData
    tensors: object
    options: "GstcSieOptions"
    exterior: Optional[object] = None
    interior: Optional[object] = None


def solve_gstc_sweep_batched(instances: Sequence[SweepInstance], concurrency="auto",
                             ctx: Optional[Context] = None):
    """All instances in one library call (sieb200_solve_gstc_sweep): largest
    first over `concurrency` lanes that run concurrently on the GPU, each
    lane's trailing GEMMs on its share of the SMs. concurrency "auto" takes
    the autotuned lane count for these sizes (sieb200.autotune). Returns
    (list of SolveResult in input order, wall seconds)."""
    ctx = ctx or default_context()
    if len(instances) == 0:
        raise ValueError("a sweep needs at least one instance")
    if concurrency == "auto":
        from .autotune import sweep_concurrency
        concurrency = sweep_concurrency([4 * inst.mesh.num_edges for inst in instances], ctx=ctx)
    arr = (_lib.SweepInstance * len(instances))()
    keep = []
    outs = []
    metrics = (_lib.Metrics * len(instances))()
    for i, inst in enumerate(instances):
        if inst.interior is None and inst.exterior is None:
            raise ValueError(f"sweep instance {i}: at least one incident region is required")
        t = _tensor_array(inst.mesh, inst.tensors, inst.options.tensors_are_uniform)
        out = np.zeros(4 * inst.mesh.num_edges, dtype=np.complex128)
        keep.append(t)
        outs.append(out)
        a = arr[i]
        a.mesh = inst.mesh.as_c()
        a.tensors = t.ctypes.data
        a.opt = to_c_options(inst.options, _lib.GSTC)
        for slot, src in enumerate((inst.interior, inst.exterior)):
            if src is None:
                a.source[slot].kind = -1
            else:
                a.source[slot] = src.as_c()
        a.currents_out = out.ctypes.data
        a.metrics = ctypes.pointer(metrics[i])
    secs = ctypes.c_double()
    _lib.check(_lib.lib().sieb200_solve_gstc_sweep(ctx.handle, arr, len(instances), int(concurrency),
                                                   ctypes.byref(secs)))
    return [SolveResult(outs[i], metrics[i].as_dict()) for i in range(len(instances))], secs.value


def _formulation_of(options) -> int:
    if isinstance(options, PecOptions):
        return _lib.PEC_EFIE
    if isinstance(options, DielectricOptions):
        return _lib.PMCHWT
    if isinstance(options, GstcSieOptions):
        return _lib.GSTC
    raise TypeError("options must be PecOptions, DielectricOptions or GstcSieOptions")


def system_dimension(options, mesh: MeshData) -> int:
    return {0: 1, 1: 2, 2: 4}[_formulation_of(options)] * mesh.num_edges


def assemble_matrix(mesh: MeshData, options, tensors=None, ctx: Optional[Context] = None) -> np.ndarray:
    """Dense eta0-scaled system matrix, column-major (returned as a numpy
    array with Fortran order)."""
    ctx = ctx or default_context()
    f = _formulation_of(options)
    o = to_c_options(options, f)
    N = system_dimension(options, mesh)
    Z = np.zeros((N, N), dtype=np.complex128, order="F")
    t = _tensor_array(mesh, tensors, options.tensors_are_uniform) if f == _lib.GSTC else None
    _lib.check(_lib.lib().sieb200_assemble_matrix(ctx.handle, ctypes.byref(mesh.as_c()), ctypes.byref(o),
                                                  _lib.ptr(t), Z.ctypes.data, 0))
    return Z


def assemble_matrix_device(mesh: MeshData, options, out_ptr: int, tensors=None,
                           ctx: Optional[Context] = None) -> None:
    """Assemble into caller-owned device memory (N*N complex128, ld = N)."""
    ctx = ctx or default_context()
    f = _formulation_of(options)
    o = to_c_options(options, f)
    t = _tensor_array(mesh, tensors, options.tensors_are_uniform) if f == _lib.GSTC else None
    _lib.check(_lib.lib().sieb200_assemble_matrix(ctx.handle, ctypes.byref(mesh.as_c()), ctypes.byref(o),
                                                  _lib.ptr(t), out_ptr, 1))


def assemble_rhs(mesh: MeshData, options, sources: Sequence, ctx: Optional[Context] = None) -> np.ndarray:
    """One column per source, shape (N, nsrc), column-major."""
    ctx = ctx or default_context()
    f = _formulation_of(options)
    o = to_c_options(options, f)
    N = system_dimension(options, mesh)
    arr = (_lib.Source * len(sources))(*[s.as_c() for s in sources])
    B = np.zeros((N, len(sources)), dtype=np.complex128, order="F")
    _lib.check(_lib.lib().sieb200_assemble_rhs(ctx.handle, ctypes.byref(mesh.as_c()), ctypes.byref(o),
                                               arr, len(sources), B.ctypes.data, 0))
    return B


def incident_fields(observation_points, source, options, ctx: Optional[Context] = None):
    """Incident (E, H) of one source at observation points, each (n, 3)
    complex128 (evaluate_incident_fields, src/sie_mom/excitation/excitation.cu:158-210);
    the source's wavenumber and impedance come from its region's medium in
    options."""
    ctx = ctx or default_context()
    o = to_c_options(options, _formulation_of(options))
    pts = np.ascontiguousarray(observation_points, dtype=np.float64).reshape(-1, 3)
    E = np.zeros((pts.shape[0], 3), dtype=np.complex128)
    H = np.zeros((pts.shape[0], 3), dtype=np.complex128)
    src = source.as_c()
    _lib.check(_lib.lib().sieb200_incident_fields(ctx.handle, ctypes.byref(o), ctypes.byref(src), pts.shape[0],
                                                  pts.ctypes.data, E.ctypes.data, H.ctypes.data))
    return E, H


def matvec_matrix_free(mesh: MeshData, options, x: np.ndarray, tensors=None,
                       ctx: Optional[Context] = None) -> np.ndarray:
    """y = Z x with Z recomputed by the quadrature kernels, never stored
    (sie_kernels_matvec.cuh:9-327 counterpart; host vectors)."""
    ctx = ctx or default_context()
    f = _formulation_of(options)
    o = to_c_options(options, f)
    N = system_dimension(options, mesh)
    xv = np.ascontiguousarray(x, dtype=np.complex128).reshape(-1)
    if xv.size != N:
        raise ValueError(f"x must have {N} entries")
    y = np.zeros(N, dtype=np.complex128)
    t = _tensor_array(mesh, tensors, options.tensors_are_uniform) if f == _lib.GSTC else None
    _lib.check(_lib.lib().sieb200_matvec_matrix_free(ctx.handle, ctypes.byref(mesh.as_c()), ctypes.byref(o),
                                                     _lib.ptr(t), xv.ctypes.data, y.ctypes.data, 0))
    return y


class DenseLuSolver:
    """Factorize once, solve many (dense_lu_solver.cuh:17-184).

    Works on device memory addresses (e.g. torch tensors' data_ptr()).
    "lu_cusolver" factors in place; "lu_fp64" (own complex128 LU) and
    "mixed_ir" keep the matrix intact and refine every solve to `tolerance`
    against it."""

    def __init__(self, n: int, method: str = "lu_cusolver", ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        if method not in SOLVERS:
            raise ValueError(f"unknown method {method!r}")
        self._h = ctypes.c_void_p()
        _lib.check(_lib.lib().sieb200_dense_solver_create(self.ctx.handle, int(n), SOLVERS[method],
                                                          ctypes.byref(self._h)))
        self.ctx._solvers.add(self)
        self.n = n
        self.last_iterations = 0

    def factorize(self, a_ptr: int, lda: Optional[int] = None) -> None:
        _lib.check(_lib.lib().sieb200_dense_solver_factorize(self._h, a_ptr, int(lda or self.n)))

    def solve(self, b_ptr: int, nrhs: int = 1, ldb: Optional[int] = None, tolerance: float = 1e-10,
              max_iterations: int = 50, adjoint: bool = False) -> int:
        it = ctypes.c_int(0)
        fn = (_lib.lib().sieb200_dense_solver_solve_adjoint if adjoint
              else _lib.lib().sieb200_dense_solver_solve)
        _lib.check(fn(self._h, int(nrhs), b_ptr, int(ldb or self.n), float(tolerance),
                      int(max_iterations), ctypes.byref(it)))
        self.last_iterations = it.value
        return it.value

    def close(self) -> None:
        # A solver whose context is already closed has nothing left to free.
        if self._h and self.ctx.handle:
            _lib.lib().sieb200_dense_solver_destroy(self._h)
        self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def zgemm(m: int, nc: int, k: int, a_ptr: int, x_ptr: int, c_ptr: int, lda: Optional[int] = None,
          ldx: Optional[int] = None, ldc: Optional[int] = None, alpha: complex = 1.0, beta: complex = 0.0,
          ctx: Optional[Context] = None) -> None:
    """C = alpha A X + beta C on device complex128 data (column-major)."""
    ctx = ctx or default_context()
    al = (ctypes.c_double * 2)(complex(alpha).real, complex(alpha).imag)
    be = (ctypes.c_double * 2)(complex(beta).real, complex(beta).imag)
    _lib.check(_lib.lib().sieb200_zgemm(ctx.handle, int(m), int(nc), int(k), a_ptr, int(lda or m), x_ptr,
                                        int(ldx or k), c_ptr, int(ldc or m), al, be))


def matvec(n: int, a_ptr: int, x_ptr: int, y_ptr: int, lda: Optional[int] = None, prec: int = 0,
           beta: float = 0.0, ctx: Optional[Context] = None) -> None:
    ctx = ctx or default_context()
    _lib.check(_lib.lib().sieb200_matvec(ctx.handle, int(n), a_ptr, int(lda or n), int(prec), x_ptr,
                                         float(beta), y_ptr))
