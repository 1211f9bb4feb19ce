"""GPU parity: the CUDA path through the C ABI against the oracle and the
golden fixtures made from the reference.

Tolerances: assembled Z and right-hand sides <= 1e-12 (max-entry error
relative to the largest entry: FP64 with the reference's float demotions
mirrored, differing only in summation order); solved currents and far fields
of the FP64 paths <= 1e-10 relative."""

import math

import numpy as np
import pytest

from conftest import GoldenMesh, rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu
C0 = 299792458.0
Z_TOL = 1e-12
X_TOL = 1e-10


def _mesh(g):
    import sieb200
    return sieb200.make_mesh(g.vertices, g.faces)


def _opts(kind, freq, rule, thr=0.1, eps_r=(1.0, 1.0), mu_r=(1.0, 1.0), basis="face", uniform=False,
          solver="lu_cusolver"):
    import sieb200
    if kind == 0:
        return sieb200.PecOptions(frequency_hz=freq, quadrature_rule=rule, singularity_threshold_lambda0=thr,
                                  exterior=sieb200.IsotropicMedium(eps_r[1], mu_r[1]), solver=solver)
    cls = sieb200.DielectricOptions if kind == 1 else sieb200.GstcSieOptions
    kw = dict(frequency_hz=freq, quadrature_rule=rule, singularity_threshold_lambda0=thr,
              interior=sieb200.IsotropicMedium(eps_r[0], mu_r[0]),
              exterior=sieb200.IsotropicMedium(eps_r[1], mu_r[1]), solver=solver)
    if kind == 2:
        kw.update(basis=basis, tensors_are_uniform=uniform)
    return cls(**kw)


@pytest.mark.parametrize("name", ["pec", "pmchwt", "gstc_face", "gstc_sph_uniform"])
def test_assembly_matches_reference_golden(name, golden, gpu_ctx, mesh_l0):
    import sieb200
    kind = {"pec": 0, "pmchwt": 1}.get(name, 2)
    eps = {"pmchwt": (4.0, 1.0), "gstc_sph_uniform": (2.0, 1.0)}.get(name, (1.0, 1.0))
    t = {"gstc_face": golden["gstc_tensors_L0"], "gstc_sph_uniform": golden["gstc_tensors_uniform"]}.get(name)
    o = _opts(kind, C0, 5, eps_r=eps, basis="spherical" if name == "gstc_sph_uniform" else "face",
              uniform=name == "gstc_sph_uniform")
    m = _mesh(mesh_l0)
    Z = sieb200.assemble_matrix(m, o, tensors=t, ctx=gpu_ctx)
    assert rel_err(Z, golden[f"Z_{name}_L0"]) < Z_TOL
    b = sieb200.assemble_rhs(m, o, [sieb200.PlaneWaveExcitation()], ctx=gpu_ctx)[:, 0]
    assert rel_err(b, golden[f"b_{name}_L0"]) < Z_TOL


@pytest.mark.parametrize("kernel", ["per_point", "flat"])
@pytest.mark.parametrize("kind,rule,thr,level", [
    (0, 7, 0.1, 2), (0, 5, 0.35, 1), (1, 17, 0.1, 1), (1, 4, 0.3, 1), (2, 5, 0.3, 1), (2, 17, 0.1, 1),
    (1, 8, 0.1, 1), (0, 20, 0.2, 1)])
def test_assembly_matches_oracle(kind, rule, thr, level, kernel, gpu_ctx, oracle_lib, monkeypatch):
    """Both regular-pass kernels (a test point per lane where its lanes stay
    busy, or the flat point-pair kernel: SIEB200_ASM_PER_POINT=0) against the
    oracle's assembly."""
    import sieb200
    monkeypatch.setenv("SIEB200_ASM_PER_POINT", "1" if kernel == "per_point" else "0")
    m = sieb200.icosphere(0.5, level)
    eps = (4.0, 1.0) if kind == 1 else (2.5, 1.0)
    freq = 2 * C0 if kind == 2 else C0
    rng = np.random.default_rng(11 + kind)
    t = rng.standard_normal((m.num_faces, 32)) + 1j * rng.standard_normal((m.num_faces, 32))
    o = _opts(kind, freq, rule, thr=thr, eps_r=eps)
    Z = sieb200.assemble_matrix(m, o, tensors=t if kind == 2 else None, ctx=gpu_ctx)
    s = O.kernel_scalars(kind, freq, eps_r=eps, threshold_lambda0=thr)
    Zo = O.assemble(oracle_lib, kind, m, rule, s, tensors=t if kind == 2 else None)
    assert rel_err(Z, Zo) < Z_TOL


def test_gstc_spherical_basis_and_interior_source(gpu_ctx, oracle_lib):
    import sieb200
    m = sieb200.icosphere(1.0, 1)
    rng = np.random.default_rng(5)
    t = rng.standard_normal((m.num_faces, 32)) + 1j * rng.standard_normal((m.num_faces, 32))
    o = _opts(2, C0, 7, eps_r=(3.0, 1.0), basis="spherical")
    Z = sieb200.assemble_matrix(m, o, tensors=t, ctx=gpu_ctx)
    s = O.kernel_scalars(2, C0, eps_r=(3.0, 1.0))
    assert rel_err(Z, O.assemble(oracle_lib, 2, m, 7, s, tensors=t, basis=1)) < Z_TOL
    dip = sieb200.DipoleExcitation(effective_moment=(0.3, 0.0, 1.0), position=(0.1, 0.0, 0.05),
                                   is_magnetic=True, region=sieb200.INTERIOR)
    b = sieb200.assemble_rhs(m, o, [dip], ctx=gpu_ctx)[:, 0]
    omega = 2 * math.pi * C0
    k = omega * math.sqrt(s["mu0"] * s["eps0"] * 3.0)
    eta = math.sqrt(s["mu0"] / (s["eps0"] * 3.0))
    bo = O.rhs(oracle_lib, 2, m, 7, dict(kind=1, a=[0.3, 0, 1.0], b=[0.1, 0, 0.05], is_magnetic=1, region=1),
               k, eta, s["mu0"], s["eps0"])
    assert rel_err(b, bo) < Z_TOL


def _oracle_solution(oracle_lib, kind, m, rule, eps, freq, tensors=None):
    s = O.kernel_scalars(kind, freq, eps_r=eps)
    Z = O.assemble(oracle_lib, kind, m, rule, s, tensors=tensors)
    k = s["omega"] * math.sqrt(s["mu0"] * s["eps0"] * eps[1])
    eta = math.sqrt(s["mu0"] / (s["eps0"] * eps[1]))
    b = O.rhs(oracle_lib, kind, m, rule, dict(kind=0, a=[1, 0, 0], b=[0, 0, 1], region=2), k, eta,
              s["mu0"], s["eps0"])
    x = np.linalg.solve(Z, b)
    ne = m.num_edges
    eta0 = math.sqrt(s["mu0"] / s["eps0"])
    for blk in range(1, {0: 1, 1: 2, 2: 4}[kind], 2):
        x[blk * ne:(blk + 1) * ne] *= eta0
    return x


@pytest.mark.parametrize("solver", ["lu_cusolver"])
def test_pec_solve_matches_oracle(solver, gpu_ctx, oracle_lib):
    import sieb200
    m = sieb200.icosphere(1.0, 2)
    r = sieb200.solve_pec_dense(m, _opts(0, C0, 5, solver=solver), sieb200.PlaneWaveExcitation(), ctx=gpu_ctx)
    x = _oracle_solution(oracle_lib, 0, m, 5, (1.0, 1.0), C0)
    assert np.linalg.norm(r.currents - x) / np.linalg.norm(x) < X_TOL
    assert r.metrics["relative_residual"] < 1e-10


def test_dielectric_solve_matches_oracle(gpu_ctx, oracle_lib):
    import sieb200
    m = sieb200.icosphere(0.5, 1)
    r = sieb200.solve_dielectric_dense(m, _opts(1, C0, 7, eps_r=(4.0, 1.0)), sieb200.PlaneWaveExcitation(),
                                       ctx=gpu_ctx)
    x = _oracle_solution(oracle_lib, 1, m, 7, (4.0, 1.0), C0)
    assert np.linalg.norm(r.currents - x) / np.linalg.norm(x) < X_TOL
    assert r.metrics["relative_residual"] < 1e-10


def test_gstc_batch_matches_oracle_and_single(gpu_ctx, oracle_lib):
    import sieb200
    m = sieb200.icosphere(1.0, 1)
    rng = np.random.default_rng(3)
    t = rng.standard_normal((m.num_faces, 32)) + 1j * rng.standard_normal((m.num_faces, 32))
    o = _opts(2, C0, 5)
    pw = sieb200.PlaneWaveExcitation()
    pw2 = sieb200.PlaneWaveExcitation(electric_amplitude=(0, 1, 0), propagation_direction=(1, 0, 0))
    dip = sieb200.DipoleExcitation(region=sieb200.INTERIOR)
    cases = [sieb200.GstcExcitationCase(exterior=pw), sieb200.GstcExcitationCase(interior=dip, exterior=pw2)]
    rb = sieb200.solve_gstc_dense_batch(m, t, o, cases, ctx=gpu_ctx)
    x = _oracle_solution(oracle_lib, 2, m, 5, (1.0, 1.0), C0, tensors=t)
    assert np.linalg.norm(rb[0].currents - x) / np.linalg.norm(x) < X_TOL
    single = sieb200.solve_gstc_dense(m, t, o, pw, ctx=gpu_ctx)
    assert np.linalg.norm(single.currents - rb[0].currents) / np.linalg.norm(x) < 1e-12
    # superposition: case 2 = interior-only + exterior-only solves (excitation_test.cu:288-346)
    ri = sieb200.solve_gstc_dense(m, t, o, dip, ctx=gpu_ctx)
    re = sieb200.solve_gstc_dense(m, t, o, pw2, ctx=gpu_ctx)
    ref = ri.currents + re.currents
    assert np.linalg.norm(rb[1].currents - ref) / np.linalg.norm(ref) < 1e-10
    for r in rb:
        assert r.metrics["relative_residual"] < 1e-10


def test_far_field_matches_reference_script(golden, gpu_ctx):
    import sieb200
    g = GoldenMesh(golden, "L1r05")
    m = _mesh(g)
    ne = m.num_edges
    cur = golden["ff_currents"]
    ft, fp, U = sieb200.far_field(m, cur[2 * ne:3 * ne], cur[3 * ne:], float(golden["ff_k0"]),
                                  float(golden["ff_eta0"]), golden["ff_r_hat"], golden["ff_theta_hat"],
                                  golden["ff_phi_hat"], ctx=gpu_ctx)
    assert rel_err(ft, golden["ff_f_theta"]) < X_TOL
    assert rel_err(fp, golden["ff_f_phi"]) < X_TOL
    assert rel_err(U, golden["ff_U"]) < X_TOL


def test_matvec_matches_numpy(gpu_ctx):
    import torch
    import sieb200
    rng = np.random.default_rng(0)
    n = 1000
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y0 = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    dA = torch.from_numpy(np.asfortranarray(A).T.copy()).cuda()  # column-major storage
    dx = torch.from_numpy(x).cuda()
    dy = torch.from_numpy(y0).cuda()
    gpu_ctx.synchronize()
    torch.cuda.synchronize()
    sieb200.matvec(n, dA.data_ptr(), dx.data_ptr(), dy.data_ptr(), beta=-1.0, ctx=gpu_ctx)
    assert rel_err(dy.cpu().numpy(), A @ x - y0) < 1e-13
    dA32 = dA.to(torch.complex64)
    dy.zero_()
    torch.cuda.synchronize()
    sieb200.matvec(n, dA32.data_ptr(), dx.data_ptr(), dy.data_ptr(), prec=1, ctx=gpu_ctx)
    A32 = A.astype(np.complex64).astype(np.complex128)
    assert rel_err(dy.cpu().numpy(), A32 @ x) < 1e-12


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("n,lda", [(256, 256), (257, 260), (1000, 1003), (2049, 2050), (6016, 6016)])
def test_matvec_tma_staged_matches_numpy(n, lda, prec, gpu_ctx):
    """The TMA-staged matvec (16 KB tiles of 128 rows through a shared-memory
    ring) over ragged row tiles, ragged column chunks and padded leading
    dimensions, against numpy and against the per-thread-load kernel
    (SIEB200_GEMV_TMA=0). Tolerances: 1e-13 (FP64 accumulation either way)."""
    import os
    import torch
    import sieb200
    rng = np.random.default_rng(n + lda + prec)
    A = rng.standard_normal((lda, n)) + 1j * rng.standard_normal((lda, n))
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y0 = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    dt = torch.complex128 if prec == 0 else torch.complex64
    dA = torch.from_numpy(np.asfortranarray(A).T.copy()).to(dt).cuda()  # column-major, leading dimension lda
    Ah = A[:n].astype(np.complex64).astype(np.complex128) if prec else A[:n]
    dx = torch.from_numpy(x).cuda()
    out = {}
    for tma in ("1", "0"):
        dy = torch.from_numpy(y0).cuda()
        torch.cuda.synchronize()
        os.environ["SIEB200_GEMV_TMA"] = tma
        try:
            sieb200.matvec(n, dA.data_ptr(), dx.data_ptr(), dy.data_ptr(), beta=-1.0, prec=prec, lda=lda,
                           ctx=gpu_ctx)
        finally:
            del os.environ["SIEB200_GEMV_TMA"]
        out[tma] = dy.cpu().numpy()
        assert rel_err(out[tma], Ah @ x - y0) < 1e-13
    assert rel_err(out["1"], out["0"]) < 1e-13
