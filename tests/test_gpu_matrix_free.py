"""GPU: the matrix-free product (Z recomputed by the quadrature kernels and
contracted on the fly) and the GMRES solver on a complex64 copy of Z.

The reference pins its matrix-free GSTC product against its dense matrix at
1e-4 (tests/cpp/test_matvec_consistency.cu:484) in single precision; here
both sides are the same FP64 arithmetic, so the bound is 1e-12 relative.
GMRES_C64 must reach the requested relative residual against the FP64 Z
(1e-10) and agree with the cuSOLVER FP64 currents to 1e-8."""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
C0 = 299792458.0


def _cases():
    import sieb200
    m = sieb200.icosphere(1.0, 2)
    rng = np.random.default_rng(4)
    rec = sieb200.omega_records(*(rng.uniform(0.5, 2.0, m.num_faces) for _ in range(3))).numpy()
    return [
        ("pec", m, sieb200.PecOptions(frequency_hz=0.5 * C0, quadrature_rule=5), None),
        ("pmchwt", m, sieb200.DielectricOptions(frequency_hz=0.5 * C0, quadrature_rule=5,
                                                interior=sieb200.IsotropicMedium(4.0, 1.0)), None),
        ("gstc", m, sieb200.GstcSieOptions(frequency_hz=0.5 * C0, quadrature_rule=5), rec),
        ("gstc-uniform", m, sieb200.GstcSieOptions(frequency_hz=0.5 * C0, quadrature_rule=5,
                                                   tensors_are_uniform=True, basis="spherical"), rec[0]),
    ]


@pytest.mark.parametrize("idx", range(4))
def test_matrix_free_matches_dense(idx, gpu_ctx):
    import sieb200
    name, m, o, t = _cases()[idx]
    Z = sieb200.assemble_matrix(m, o, t, ctx=gpu_ctx)
    rng = np.random.default_rng(idx)
    x = rng.standard_normal(Z.shape[0]) + 1j * rng.standard_normal(Z.shape[0])
    y = sieb200.matvec_matrix_free(m, o, x, tensors=t, ctx=gpu_ctx)
    ref = Z @ x
    assert np.linalg.norm(y - ref) <= 1e-12 * np.linalg.norm(ref), name
    y2 = sieb200.matvec_matrix_free(m, o, x, tensors=t, ctx=gpu_ctx)
    assert np.array_equal(y, y2)  # deterministic: no atomics


def test_gmres_c64_dense_solver(gpu_ctx):
    import torch
    import sieb200
    n = 700
    rng = np.random.default_rng(9)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 4.0 * math.sqrt(n) * np.eye(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    Z = torch.from_numpy(A.T.copy()).cuda()
    s = sieb200.DenseLuSolver(n, "gmres_c64", ctx=gpu_ctx)
    s.factorize(Z.data_ptr())
    for adjoint, M in [(False, A), (True, A.conj().T)]:
        x = torch.from_numpy(b.copy()).cuda()
        torch.cuda.synchronize()
        s.solve(x.data_ptr(), tolerance=1e-11, max_iterations=200, adjoint=adjoint)
        gpu_ctx.synchronize()
        assert np.linalg.norm(M @ x.cpu().numpy() - b) / np.linalg.norm(b) <= 1e-11
    s.close()


def test_gmres_c64_small_pmchwt_solve(gpu_ctx):
    """GMRES_C64 is the unfactored option (Jacobi only): on a small system it
    reaches the FP64 residual target and the cuSOLVER currents."""
    import sieb200
    m = sieb200.icosphere(0.5, 1)
    o = sieb200.DielectricOptions(frequency_hz=C0, quadrature_rule=5, interior=sieb200.IsotropicMedium(4.0, 1.0))
    ref = sieb200.solve_dielectric_dense(m, o, sieb200.PlaneWaveExcitation(), ctx=gpu_ctx)
    o.solver = "gmres_c64"
    o.max_iterations = 2000
    got = sieb200.solve_dielectric_dense(m, o, sieb200.PlaneWaveExcitation(), ctx=gpu_ctx)
    assert got.metrics["relative_residual"] <= 1e-10
    assert np.linalg.norm(got.currents - ref.currents) / np.linalg.norm(ref.currents) < 1e-8
