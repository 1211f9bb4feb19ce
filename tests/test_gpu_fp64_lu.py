"""GPU: the own FP64 LU (SIEB200_SOLVER_LU_FP64: butterfly transform, blocked
LU without pivoting in complex128 with this library's diagonal-block, panel
and FP64 GEMM kernels, FP64 refinement against the intact matrix).

Tolerances: against numpy's FP64 solve 1e-12 on random well-conditioned
systems (ragged sizes, several right-hand sides); against the oracle's FP64
currents 1e-10 (the reference's own parity bar for the FP64 path); against
the cuSOLVER batch 1e-10."""

import math

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
C0 = 299792458.0


def _dev(a):
    import torch
    return torch.from_numpy(np.asfortranarray(a).T.copy()).cuda()


def _host(t, rows, cols):
    # the tensor is (cols, rows): column-major storage of a rows x cols matrix
    a = t.cpu().numpy().T
    assert a.shape == (rows, cols)
    return a


@pytest.mark.parametrize("diag", ["split_panels", "split_steps", "fused_steps", "split_compact"])
@pytest.mark.parametrize("n,nrhs", [(5, 1), (50, 2), (130, 1), (997, 3), (2100, 1)])
def test_fp64_lu_matches_numpy(n, nrhs, diag, gpu_ctx, monkeypatch):
    """Against numpy at 1e-12, with the diagonal block's update in its own
    kernel or inside the LU kernel, and the elimination synchronised per
    panel or per step."""
    import torch
    import sieb200
    monkeypatch.setenv("SIEB200_DIAG_SPLIT", "0" if diag.startswith("fused") else "1")
    monkeypatch.setenv("SIEB200_DIAG_PANELS", "1" if diag.endswith("panels") else "0")
    monkeypatch.setenv("SIEB200_DIAG_COMPACT", "1" if diag.endswith("compact") else "0")
    rng = np.random.default_rng(n)
    A = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    A += np.diag(2.0 + rng.uniform(0, 1, n))
    B = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    dA, dB = _dev(A), _dev(B)
    s = sieb200.DenseLuSolver(n, "lu_fp64", ctx=gpu_ctx)
    torch.cuda.synchronize()
    s.factorize(dA.data_ptr())
    s.solve(dB.data_ptr(), nrhs=nrhs, tolerance=1e-14, max_iterations=5)
    X = _host(dB, n, nrhs)
    Xo = np.linalg.solve(A, B)
    assert np.linalg.norm(X - Xo) / np.linalg.norm(Xo) < 1e-12
    assert np.array_equal(_host(dA, n, n), A)  # the matrix is left intact
    with pytest.raises(sieb200.InvalidArgument, match="conjugate-transpose"):
        s.solve(dB.data_ptr(), nrhs=nrhs, adjoint=True)
    s.close()


def test_fp64_lu_pmchwt_matches_oracle(gpu_ctx, oracle_lib):
    import sieb200
    m = sieb200.icosphere(0.5, 2)
    o = sieb200.DielectricOptions(frequency_hz=C0, quadrature_rule=7, solver="lu_fp64",
                                  interior=sieb200.IsotropicMedium(4.0, 1.0))
    r = sieb200.solve_dielectric_dense(m, o, sieb200.PlaneWaveExcitation(), ctx=gpu_ctx)
    s = O.kernel_scalars(1, C0, eps_r=(4.0, 1.0))
    Z = O.assemble(oracle_lib, 1, m, 7, s)
    k = s["omega"] * math.sqrt(s["mu0"] * s["eps0"])
    eta = math.sqrt(s["mu0"] / s["eps0"])
    b = O.rhs(oracle_lib, 1, m, 7, dict(kind=0, a=[1, 0, 0], b=[0, 0, 1], region=2), k, eta, s["mu0"], s["eps0"])
    x = np.linalg.solve(Z, b)
    x[m.num_edges:] *= eta
    assert np.linalg.norm(r.currents - x) / np.linalg.norm(x) < 1e-10
    assert r.metrics["relative_residual"] < 1e-10


def test_fp64_lu_gstc_batch_matches_cusolver(gpu_ctx):
    import sieb200
    m = sieb200.icosphere(1.0, 2)
    rng = np.random.default_rng(9)
    t = 0.3 * (rng.standard_normal((m.num_faces, 32)) + 1j * rng.standard_normal((m.num_faces, 32)))
    cases = [sieb200.GstcExcitationCase(exterior=sieb200.PlaneWaveExcitation()),
             sieb200.GstcExcitationCase(interior=sieb200.DipoleExcitation(region=sieb200.INTERIOR))]
    res = {}
    for solver in ("lu_cusolver", "lu_fp64"):
        o = sieb200.GstcSieOptions(frequency_hz=C0, quadrature_rule=5, solver=solver)
        res[solver] = sieb200.solve_gstc_dense_batch(m, t, o, cases, ctx=gpu_ctx)
    for a, b in zip(res["lu_fp64"], res["lu_cusolver"]):
        assert np.linalg.norm(a.currents - b.currents) / np.linalg.norm(b.currents) < 1e-10
        assert a.metrics["relative_residual"] < 1e-10
