"""GPU parity at the benchmark configurations' sizes, against the oracle
(the C restatement of the reference's quadrature, whose small-case values are
pinned to the reference's own host build and fixtures).

* PEC sphere, radius 1 m, 1280 faces / 1920 edges (SphericalSurface(1, 3)),
  T-EFIE, k = 2 pi, Dunavant rule 5, threshold 0.1 lambda0, x-polarised plane
  wave along +z: the whole Z and b, the FP64 and mixed currents, the 181-point
  bistatic RCS cuts, and the matrix-free product.
* T-PMCHWT sphere, radius 0.5 m, eps_r = 4, 2000 faces / 3000 edges: the
  whole Z at rule 5 and the mixed currents against the oracle's FP64
  solution; sampled rows of Z at rule 17 (the benchmark's rule).
* SIE-GSTC sphere, radius 1 m, 2880 faces / 4320 edges (N = 17280, the size
  of the 64-right-hand-side workload), per-face lossless omega records: sampled
  rows of Z at rule 17.

Tolerances: Z, b and rows <= 1e-12 (max-entry error over the largest entry);
FP64 currents and far fields <= 1e-10; mixed currents <= 1e-9 with the
relative residual <= 1e-10; matrix-free product <= 1e-12 (norm-wise)."""

import math

import numpy as np
import pytest

from conftest import rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu
C0 = 299792458.0
Z_TOL = 1e-12
X_TOL = 1e-10


def _pec_options(solver="lu_cusolver"):
    import sieb200
    return sieb200.PecOptions(frequency_hz=C0, quadrature_rule=5, singularity_threshold_lambda0=0.1,
                              solver=solver)


@pytest.fixture(scope="module")
def config1(oracle_lib):
    """Oracle Z, b and FP64 currents of the PEC workload."""
    import sieb200
    m = sieb200.icosphere(1.0, 3)
    s = O.kernel_scalars(0, C0)
    Zo = O.assemble(oracle_lib, 0, m, 5, s)
    k = s["omega"] * math.sqrt(s["mu0"] * s["eps0"])
    eta = math.sqrt(s["mu0"] / s["eps0"])
    bo = O.rhs(oracle_lib, 0, m, 5, dict(kind=0, a=[1, 0, 0], b=[0, 0, 1], region=2), k, eta, s["mu0"],
               s["eps0"])
    xo = np.linalg.solve(Zo, bo)
    return m, Zo, bo, xo, k, eta


def test_config1_pec_matrix_and_rhs(config1, gpu_ctx):
    import sieb200
    m, Zo, bo, _, _, _ = config1
    assert m.num_faces == 1280 and m.num_edges == 1920
    o = _pec_options()
    assert rel_err(sieb200.assemble_matrix(m, o, ctx=gpu_ctx), Zo) < Z_TOL
    assert rel_err(sieb200.assemble_rhs(m, o, [sieb200.PlaneWaveExcitation()], ctx=gpu_ctx)[:, 0], bo) < Z_TOL


@pytest.mark.parametrize("solver,tol", [("lu_cusolver", X_TOL), ("mixed_ir", 1e-9)])
def test_config1_pec_currents_and_rcs(solver, tol, config1, gpu_ctx, oracle_lib):
    import sieb200
    m, _, _, xo, k, eta = config1
    r = sieb200.solve_pec_dense(m, _pec_options(solver), sieb200.PlaneWaveExcitation(), ctx=gpu_ctx)
    assert np.linalg.norm(r.currents - xo) / np.linalg.norm(xo) < tol
    assert r.metrics["relative_residual"] < 1e-10
    # bistatic RCS over 181 theta in the phi = 0 and phi = 90 degree cuts
    th = np.linspace(0.0, np.pi, 181)
    for phi in (0.0, np.pi / 2):
        ph = np.full_like(th, phi)
        r_hat, t_hat, p_hat = sieb200.spherical_frames(th, ph)
        ft, fp, U = sieb200.far_field(m, r.currents, None, k, eta, r_hat, t_hat, p_hat, ctx=gpu_ctx)
        fto, fpo, Uo = O.far_field(oracle_lib, m, xo, None, k, eta, r_hat, t_hat, p_hat)
        rcs = 4 * np.pi * (np.abs(ft) ** 2 + np.abs(fp) ** 2)
        rcs_o = 4 * np.pi * (np.abs(fto) ** 2 + np.abs(fpo) ** 2)
        assert rel_err(rcs, rcs_o) < 10 * tol
        # both components against the larger field (F_phi vanishes in the phi = 0 cut)
        scale = max(np.abs(fto).max(), np.abs(fpo).max())
        assert max(np.abs(ft - fto).max(), np.abs(fp - fpo).max()) < tol * scale


def test_config1_matrix_free_product(config1, gpu_ctx):
    import sieb200
    m, Zo, _, _, _, _ = config1
    rng = np.random.default_rng(21)
    x = rng.standard_normal(m.num_edges) + 1j * rng.standard_normal(m.num_edges)
    y = sieb200.matvec_matrix_free(m, _pec_options(), x, ctx=gpu_ctx)
    yo = Zo @ x
    assert np.linalg.norm(y - yo) / np.linalg.norm(yo) < Z_TOL


def test_gstc_matrix_free_product_matches_oracle(gpu_ctx, oracle_lib):
    import sieb200
    m = sieb200.icosphere(1.0, 2)
    rng = np.random.default_rng(22)
    t = rng.standard_normal((m.num_faces, 32)) + 1j * rng.standard_normal((m.num_faces, 32))
    o = sieb200.GstcSieOptions(frequency_hz=C0, quadrature_rule=5, basis="spherical",
                               interior=sieb200.IsotropicMedium(2.0, 1.0))
    s = O.kernel_scalars(2, C0, eps_r=(2.0, 1.0))
    Zo = O.assemble(oracle_lib, 2, m, 5, s, tensors=t, basis=1)
    x = rng.standard_normal(Zo.shape[0]) + 1j * rng.standard_normal(Zo.shape[0])
    y = sieb200.matvec_matrix_free(m, o, x, tensors=t, ctx=gpu_ctx)
    yo = Zo @ x
    assert np.linalg.norm(y - yo) / np.linalg.norm(yo) < Z_TOL


def _pmchwt_options(rule, solver="lu_cusolver"):
    import sieb200
    return sieb200.DielectricOptions(frequency_hz=C0, quadrature_rule=rule, solver=solver,
                                     interior=sieb200.IsotropicMedium(4.0, 1.0))


def test_config2_pmchwt_rule5_matrix_and_mixed_currents(gpu_ctx, oracle_lib):
    import sieb200
    m = sieb200.geodesic_sphere(0.5, 10)
    assert m.num_faces == 2000 and m.num_edges == 3000
    s = O.kernel_scalars(1, C0, eps_r=(4.0, 1.0))
    Zo = O.assemble(oracle_lib, 1, m, 5, s)
    assert rel_err(sieb200.assemble_matrix(m, _pmchwt_options(5), ctx=gpu_ctx), Zo) < Z_TOL
    k = s["omega"] * math.sqrt(s["mu0"] * s["eps0"])
    eta = math.sqrt(s["mu0"] / s["eps0"])
    bo = O.rhs(oracle_lib, 1, m, 5, dict(kind=0, a=[1, 0, 0], b=[0, 0, 1], region=2), k, eta, s["mu0"],
               s["eps0"])
    xo = np.linalg.solve(Zo, bo)
    del Zo
    xo[m.num_edges:] *= eta
    r = sieb200.solve_dielectric_dense(m, _pmchwt_options(5, "mixed_ir"), sieb200.PlaneWaveExcitation(),
                                       ctx=gpu_ctx)
    assert np.linalg.norm(r.currents - xo) / np.linalg.norm(xo) < 1e-9
    assert r.metrics["relative_residual"] < 1e-10


def _sample_rows(rng, ne, blocks, per_block=3):
    edges = rng.choice(ne, per_block, replace=False)
    return np.concatenate([edges + b * ne for b in range(blocks)])


def test_config2_pmchwt_rule17_sampled_rows(gpu_ctx, oracle_lib):
    import sieb200
    m = sieb200.geodesic_sphere(0.5, 10)
    Z = sieb200.assemble_matrix(m, _pmchwt_options(17), ctx=gpu_ctx)
    s = O.kernel_scalars(1, C0, eps_r=(4.0, 1.0))
    rows = _sample_rows(np.random.default_rng(17), m.num_edges, 2, 4)
    R = O.assemble_rows(oracle_lib, 1, m, 17, s, rows)
    assert rel_err(Z[rows], R) < Z_TOL


def test_config3_size_gstc_rule17_sampled_rows(gpu_ctx, oracle_lib):
    import sieb200
    m = sieb200.geodesic_sphere(1.0, 12)
    assert m.num_edges == 4320
    rng = np.random.default_rng(33)
    nf = m.num_faces
    # lossless omega records (B, X, chi uniform in [-2, 2], maps with
    # |chi^2 - B X| < 0.25 redrawn so that every Lambda is well invertible)
    B, X, chi = (rng.uniform(-2, 2, nf) for _ in range(3))
    bad = np.abs(chi ** 2 - B * X) < 0.25
    while bad.any():
        B[bad], X[bad], chi[bad] = (rng.uniform(-2, 2, int(bad.sum())) for _ in range(3))
        bad = np.abs(chi ** 2 - B * X) < 0.25
    t = sieb200.omega_records(B, X, chi).numpy().reshape(nf, 32)
    o = sieb200.GstcSieOptions(frequency_hz=C0, quadrature_rule=17)
    Z = sieb200.assemble_matrix(m, o, tensors=t, ctx=gpu_ctx)
    s = O.kernel_scalars(2, C0)
    rows = _sample_rows(rng, m.num_edges, 4, 2)
    R = O.assemble_rows(oracle_lib, 2, m, 17, s, rows, tensors=t)
    assert rel_err(Z[rows], R) < Z_TOL


def _rcs_vs_mie(m, currents_j, currents_m, eps_r, ctx):
    """Relative RMS difference of the bistatic RCS (phi = 0 and 90 degree
    cuts, 181 theta each) from the Mie series."""
    import sieb200
    from oracle import mie
    th = np.linspace(0.0, np.pi, 181)
    k = 2 * math.pi * C0 * math.sqrt(1.25663706212e-6 * 8.8541878128e-12)
    eta = math.sqrt(1.25663706212e-6 / 8.8541878128e-12)
    num = den = 0.0
    for phi in (0.0, np.pi / 2):
        ph = np.full_like(th, phi)
        r_hat, t_hat, p_hat = sieb200.spherical_frames(th, ph)
        ft, fp, _ = sieb200.far_field(m, currents_j, currents_m, k, eta, r_hat, t_hat, p_hat, ctx=ctx)
        rcs = 4 * np.pi * (np.abs(ft) ** 2 + np.abs(fp) ** 2)
        ref = mie.bistatic_rcs(k, float(np.linalg.norm(m.vertices, axis=1).mean()), eps_r, th, ph)
        num += float(np.sum((rcs - ref) ** 2))
        den += float(np.sum(ref ** 2))
    return math.sqrt(num / den)


def test_config1_rcs_against_mie(gpu_ctx):
    """Discretization error of the PEC workload's bistatic RCS against the
    Mie series of a perfectly conducting sphere: about 1 % on 1280 faces at
    ka = 2 pi (the oracle's solution shows the same; not a parity bar)."""
    import sieb200
    m = sieb200.icosphere(1.0, 3)
    r = sieb200.solve_pec_dense(m, _pec_options("mixed_ir"), sieb200.PlaneWaveExcitation(), ctx=gpu_ctx)
    err = _rcs_vs_mie(m, r.currents, None, None, gpu_ctx)
    assert err < 0.03, err


def test_config2_rcs_against_mie(gpu_ctx):
    """The benchmark system (2000 faces, rule 17, mixed solve): bistatic RCS
    against the Mie series of the eps_r = 4 sphere."""
    import sieb200
    m = sieb200.geodesic_sphere(0.5, 10)
    r = sieb200.solve_dielectric_dense(m, _pmchwt_options(17, "mixed_ir"), sieb200.PlaneWaveExcitation(),
                                       ctx=gpu_ctx)
    ne = m.num_edges
    err = _rcs_vs_mie(m, r.currents[:ne], r.currents[ne:], 4.0, gpu_ctx)
    assert err < 0.03, err
