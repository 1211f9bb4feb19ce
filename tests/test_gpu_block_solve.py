"""GPU: the multi-right-hand-side mixed solve (tensor-core block triangular
solves inside a batched FGMRES) and the FP64 complex GEMM it refines with.

Tolerances: both FP64 GEMM kernels <= 1e-13 (max-entry error over the
largest entry) against numpy; every column of a block solve reaches the requested relative
residual (1e-10, with the FP64 GEMM) and agrees with numpy's FP64 solution
to <= 1e-9 (forward error bounded by the condition of these systems times
the residual), as does the column-by-column solve it replaces."""

import os

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
C0 = 299792458.0


def _dev(a):
    import torch
    return torch.from_numpy(np.asfortranarray(a).T.copy()).cuda()  # column-major storage


def _host(t, rows, cols):
    # the tensor is (cols, rows): column-major storage of a rows x cols matrix
    a = t.cpu().numpy().T
    assert a.shape == (rows, cols)
    return a


@pytest.mark.parametrize("kernel", ["dmma", "fma"])
@pytest.mark.parametrize("m,nc,k", [(1, 1, 1), (130, 7, 77), (1000, 64, 999), (257, 33, 300), (64, 1, 2000),
                                    (600, 700, 64)])
def test_zgemm_matches_numpy(m, nc, k, kernel, gpu_ctx, monkeypatch):
    """Both FP64 complex GEMM kernels: the tensor-core one (mma.sync .f64)
    and the FMA one (SIEB200_ZGEMM_DMMA=0)."""
    import torch
    import sieb200
    monkeypatch.setenv("SIEB200_ZGEMM_DMMA", "1" if kernel == "dmma" else "0")
    rng = np.random.default_rng(m + 7 * nc + k)
    A = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
    X = rng.standard_normal((k, nc)) + 1j * rng.standard_normal((k, nc))
    C = rng.standard_normal((m, nc)) + 1j * rng.standard_normal((m, nc))
    alpha, beta = 0.5 - 1.25j, -1.0 + 0.5j
    dA, dX, dC = _dev(A), _dev(X), _dev(C)
    torch.cuda.synchronize()
    sieb200.zgemm(m, nc, k, dA.data_ptr(), dX.data_ptr(), dC.data_ptr(), alpha=alpha, beta=beta, ctx=gpu_ctx)
    ref = alpha * (A @ X) + beta * C
    assert rel_err(_host(dC, m, nc), ref) < 1e-13
    # beta = 0 must not read C (filled with NaN here)
    dC.fill_(float("nan"))
    torch.cuda.synchronize()
    sieb200.zgemm(m, nc, k, dA.data_ptr(), dX.data_ptr(), dC.data_ptr(), alpha=1.0, beta=0.0, ctx=gpu_ctx)
    assert rel_err(_host(dC, m, nc), A @ X) < 1e-13


def _system(n, seed):
    rng = np.random.default_rng(seed)
    A = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    A += np.diag(2.0 + rng.uniform(0, 1, n) + 1j * rng.uniform(-1, 1, n))
    return A


def _solve(A, B, method="mixed_ir", per_column=False, gpu_ctx=None):
    import torch
    import sieb200
    n, nrhs = B.shape
    dA = _dev(A)
    dB = _dev(B)
    s = sieb200.DenseLuSolver(n, method, ctx=gpu_ctx)
    torch.cuda.synchronize()
    s.factorize(dA.data_ptr())
    old = os.environ.get("SIEB200_PER_COLUMN_SOLVE")
    os.environ["SIEB200_PER_COLUMN_SOLVE"] = "1" if per_column else "0"
    try:
        s.solve(dB.data_ptr(), nrhs=nrhs, tolerance=1e-10, max_iterations=60)
    finally:
        if old is None:
            del os.environ["SIEB200_PER_COLUMN_SOLVE"]
        else:
            os.environ["SIEB200_PER_COLUMN_SOLVE"] = old
    X = _host(dB, n, nrhs)
    s.close()
    return X


@pytest.mark.parametrize("packs", ["split", "three"])
@pytest.mark.parametrize("lookahead", ["1", "0"])
@pytest.mark.parametrize("n,nrhs", [(50, 2), (130, 7), (997, 64), (2100, 17), (4099, 33)])
def test_block_solve_matches_numpy(n, nrhs, lookahead, packs, gpu_ctx, monkeypatch):
    """Block triangular solves with the lookahead (each diagonal block takes
    the previous step's update itself, beside the trailing GEMM on another
    stream) and without (SIEB200_BLOCK_LOOKAHEAD=0), on split [hi | lo]
    packs (default) and on three-product packs (SIEB200_BLOCK_HILO=0)."""
    monkeypatch.setenv("SIEB200_BLOCK_LOOKAHEAD", lookahead)
    monkeypatch.setenv("SIEB200_BLOCK_HILO", "0" if packs == "three" else "1")
    A = _system(n, n)
    rng = np.random.default_rng(n + 1)
    B = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    X = _solve(A, B, gpu_ctx=gpu_ctx)
    Xo = np.linalg.solve(A, B)
    for c in range(nrhs):
        assert np.linalg.norm(A @ X[:, c] - B[:, c]) / np.linalg.norm(B[:, c]) <= 1e-10
        assert np.linalg.norm(X[:, c] - Xo[:, c]) / np.linalg.norm(Xo[:, c]) < 1e-9
    Xc = _solve(A, B, per_column=True, gpu_ctx=gpu_ctx)
    assert np.linalg.norm(X - Xc) / np.linalg.norm(Xc) < 1e-9


def test_block_solve_after_refactorization(gpu_ctx, monkeypatch):
    """The packed factors follow a new factorization of the same solver, and
    a change of pack layout between solves (the packs are rebuilt)."""
    import torch
    import sieb200
    n, nrhs = 700, 5
    rng = np.random.default_rng(3)
    B = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    s = sieb200.DenseLuSolver(n, "mixed_ir", ctx=gpu_ctx)
    for seed, hilo in ((1, "1"), (2, "1"), (1, "0"), (1, "1")):
        monkeypatch.setenv("SIEB200_BLOCK_HILO", hilo)
        A = _system(n, seed)
        dA, dB = _dev(A), _dev(B)
        torch.cuda.synchronize()
        s.factorize(dA.data_ptr())
        s.solve(dB.data_ptr(), nrhs=nrhs, tolerance=1e-10, max_iterations=60)
        X = _host(dB, n, nrhs)
        Xo = np.linalg.solve(A, B)
        assert np.linalg.norm(X - Xo) / np.linalg.norm(Xo) < 1e-9
    s.close()


def test_gstc_batch_of_plane_waves_mixed_matches_fp64(gpu_ctx):
    """16 plane waves over a theta grid in one batch: the mixed block solve
    equals the FP64 cuSOLVER batch, every case at relative residual <= 1e-10."""
    import sieb200
    m = sieb200.icosphere(1.0, 2)
    rng = np.random.default_rng(12)
    nf = m.num_faces
    B, X, chi = (rng.uniform(-2, 2, nf) for _ in range(3))
    bad = np.abs(chi ** 2 - B * X) < 0.25
    while bad.any():
        B[bad], X[bad], chi[bad] = (rng.uniform(-2, 2, int(bad.sum())) for _ in range(3))
        bad = np.abs(chi ** 2 - B * X) < 0.25
    t = sieb200.omega_records(B, X, chi).numpy().reshape(nf, 32)
    th = np.linspace(0.0, np.pi, 16)
    cases = [sieb200.GstcExcitationCase(exterior=sieb200.PlaneWaveExcitation(
        electric_amplitude=(np.cos(a), 0.0, -np.sin(a)), propagation_direction=(np.sin(a), 0.0, np.cos(a))))
        for a in th]
    out = {}
    for solver in ("lu_cusolver", "mixed_ir"):
        o = sieb200.GstcSieOptions(frequency_hz=C0, quadrature_rule=5, solver=solver)
        out[solver] = sieb200.solve_gstc_dense_batch(m, t, o, cases, ctx=gpu_ctx)
    for a, b in zip(out["mixed_ir"], out["lu_cusolver"]):
        assert np.linalg.norm(a.currents - b.currents) / np.linalg.norm(b.currents) < 1e-9
        assert a.metrics["relative_residual"] <= 1e-10
        assert b.metrics["relative_residual"] <= 1e-10
