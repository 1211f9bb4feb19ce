"""GPU parity of the rotated-testing formulations (N-EFIE, N-MFIE, N-PMCHWT,
N-Muller; surface nTL form B and line form A) through the C ABI, against the
golden fixtures made from the reference and against the oracle.

Tolerances as for the tangential formulations: assembled Z and right-hand
sides <= 1e-12 (max-entry error relative to the largest entry); solved
currents <= 1e-10 relative."""

import math
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu
C0 = 299792458.0
Z_TOL = 1e-12
X_TOL = 1e-10
VG = Path(__file__).resolve().parent / "golden" / "variants_golden.npz"
CASES = {
    "n_efie": (0, "NEfie", {}),
    "n_mfie": (0, "NMfie", {}),
    "n_pmchwt": (1, "N_PMCHWT", dict(eps_r=(4.0, 1.0), mu_r=(1.0, 1.0))),
    "n_muller": (1, "N_Muller", dict(eps_r=(2.5, 1.0), mu_r=(1.5, 1.0))),
}
VARIANT = {"n_efie": 1, "n_mfie": 2, "n_pmchwt": 1, "n_muller": 2}
# line form A: case -> (base case, Gauss-Legendre points); the fixtures use
# the icosahedron scaled to radius 0.3 at 3 C0.
LINE = {"n_efie_line": ("n_efie", 20), "n_pmchwt_line": ("n_pmchwt", 10), "n_muller_line": ("n_muller", 7)}


@pytest.fixture(scope="module")
def vgolden():
    return dict(np.load(VG))


def _opts(name, freq, rule, thr, solver="lu_cusolver", ntl_form="Surface", line_points=20):
    import sieb200
    kind, form, media = CASES[name]
    eps_r = media.get("eps_r", (1.0, 1.0))
    mu_r = media.get("mu_r", (1.0, 1.0))
    if kind == 0:
        return sieb200.PecOptions(frequency_hz=freq, quadrature_rule=rule, singularity_threshold_lambda0=thr,
                                  exterior=sieb200.IsotropicMedium(eps_r[1], mu_r[1]), solver=solver,
                                  formulation=form, ntl_form=ntl_form, line_quadrature_points=line_points)
    return sieb200.DielectricOptions(frequency_hz=freq, quadrature_rule=rule, singularity_threshold_lambda0=thr,
                                     interior=sieb200.IsotropicMedium(eps_r[0], mu_r[0]),
                                     exterior=sieb200.IsotropicMedium(eps_r[1], mu_r[1]), solver=solver,
                                     formulation=form, ntl_form=ntl_form, line_quadrature_points=line_points)


@pytest.mark.parametrize("name", sorted(CASES))
def test_variant_assembly_matches_reference_golden(name, vgolden, gpu_ctx, mesh_l0):
    import sieb200
    kind = CASES[name][0]
    m = sieb200.make_mesh(mesh_l0.vertices, mesh_l0.faces)
    o = _opts(name, C0, 5, 1.5)
    Z = sieb200.assemble_matrix(m, o, ctx=gpu_ctx)
    assert rel_err(Z, vgolden[f"Z_{name}_L0"]) < Z_TOL
    for region in ((2, 1) if kind == 1 else (2,)):
        src = sieb200.PlaneWaveExcitation(region=region)
        b = sieb200.assemble_rhs(m, o, [src], ctx=gpu_ctx)[:, 0]
        assert rel_err(b, vgolden[f"b_{name}_L0_region{region}"]) < Z_TOL, region


@pytest.mark.parametrize("name,rule,thr,level", [
    ("n_efie", 7, 0.35, 1), ("n_efie", 7, 0.1, 2), ("n_mfie", 5, 0.35, 1), ("n_pmchwt", 4, 0.3, 1),
    ("n_pmchwt", 17, 0.1, 1), ("n_muller", 6, 0.3, 1)])
def test_variant_assembly_matches_oracle(name, rule, thr, level, gpu_ctx, oracle_lib):
    import sieb200
    kind, _, media = CASES[name]
    m = sieb200.icosphere(0.5, level)
    Z = sieb200.assemble_matrix(m, _opts(name, C0, rule, thr), ctx=gpu_ctx)
    s = O.kernel_scalars(kind, C0, **media, threshold_lambda0=thr)
    Zo = O.assemble(oracle_lib, kind, m, rule, s, variant=VARIANT[name])
    assert rel_err(Z, Zo) < Z_TOL


@pytest.mark.parametrize("name", ["n_pmchwt", "n_mfie"])
def test_variant_matrix_free_matches_assembled(name, gpu_ctx):
    import sieb200
    m = sieb200.icosphere(0.5, 1)
    o = _opts(name, C0, 5, 0.3)
    Z = sieb200.assemble_matrix(m, o, ctx=gpu_ctx)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(Z.shape[0]) + 1j * rng.standard_normal(Z.shape[0])
    y = sieb200.matvec_matrix_free(m, o, x, ctx=gpu_ctx)
    assert rel_err(y, Z @ x) < 1e-12


def _oracle_solution(oracle_lib, name, m, rule, freq, thr):
    kind, _, media = CASES[name]
    eps_r = media.get("eps_r", (1.0, 1.0))
    mu_r = media.get("mu_r", (1.0, 1.0))
    s = O.kernel_scalars(kind, freq, **media, threshold_lambda0=thr)
    Z = O.assemble(oracle_lib, kind, m, rule, s, variant=VARIANT[name])
    k = s["omega"] * math.sqrt(s["mu0"] * s["eps0"] * eps_r[1] * mu_r[1])
    eta = math.sqrt(s["mu0"] * mu_r[1] / (s["eps0"] * eps_r[1]))
    b = O.rhs(oracle_lib, kind, m, rule, dict(kind=0, a=[1, 0, 0], b=[0, 0, 1], region=2), k, eta,
              s["mu0"], s["eps0"], variant=VARIANT[name], eps_r_src=eps_r[1], mu_r_src=mu_r[1])
    x = np.linalg.solve(Z, b)
    if kind == 1:
        x[m.num_edges:] *= math.sqrt(s["mu0"] / s["eps0"])
    return x


@pytest.mark.parametrize("name,solver", [("n_efie", "lu_cusolver"), ("n_mfie", "lu_cusolver"),
                                         ("n_pmchwt", "lu_cusolver"), ("n_pmchwt", "mixed_ir"),
                                         ("n_muller", "lu_cusolver")])
def test_variant_solve_matches_oracle(name, solver, gpu_ctx, oracle_lib):
    import sieb200
    m = sieb200.icosphere(0.5, 2)
    o = _opts(name, C0, 5, 0.1, solver=solver)
    src = sieb200.PlaneWaveExcitation()
    r = (sieb200.solve_pec_dense if CASES[name][0] == 0 else sieb200.solve_dielectric_dense)(m, o, src,
                                                                                            ctx=gpu_ctx)
    x = _oracle_solution(oracle_lib, name, m, 5, C0, 0.1)
    # The mixed solver refines until the relative residual is below its
    # tolerance (1e-10), so its forward error is bounded by cond(Z) * 1e-10.
    tol = 1e-9 if solver == "mixed_ir" else X_TOL
    assert np.linalg.norm(r.currents - x) / np.linalg.norm(x) < tol
    assert r.metrics["relative_residual"] <= 1e-10


@pytest.mark.parametrize("name", sorted(LINE))
def test_line_form_assembly_matches_reference_golden(name, vgolden, gpu_ctx, mesh_l0):
    import sieb200
    base, lp = LINE[name]
    m = sieb200.make_mesh(0.3 * mesh_l0.vertices, mesh_l0.faces)
    Z = sieb200.assemble_matrix(m, _opts(base, 3 * C0, 5, 1.5, ntl_form="Line", line_points=lp), ctx=gpu_ctx)
    assert rel_err(Z, vgolden[f"Z_{name}_L0"]) < Z_TOL


@pytest.mark.parametrize("name,rule,thr", [("n_efie_line", 7, 0.35), ("n_pmchwt_line", 6, 0.3),
                                           ("n_muller_line", 5, 0.3)])
def test_line_form_assembly_matches_oracle(name, rule, thr, gpu_ctx, oracle_lib):
    import sieb200
    base, lp = LINE[name]
    kind, _, media = CASES[base]
    m = sieb200.icosphere(0.5, 1)
    o = _opts(base, C0, rule, thr, ntl_form="Line", line_points=lp)
    Z = sieb200.assemble_matrix(m, o, ctx=gpu_ctx)
    s = O.kernel_scalars(kind, C0, **media, threshold_lambda0=thr)
    Zo = O.assemble(oracle_lib, kind, m, rule, s, variant=VARIANT[base], line_points=lp)
    assert rel_err(Z, Zo) < Z_TOL
    rng = np.random.default_rng(9)
    x = rng.standard_normal(Z.shape[0]) + 1j * rng.standard_normal(Z.shape[0])
    assert rel_err(sieb200.matvec_matrix_free(m, o, x, ctx=gpu_ctx), Z @ x) < 1e-12


def test_invalid_line_options_are_refused(gpu_ctx):
    import sieb200
    m = sieb200.icosphere(0.5, 0)
    with pytest.raises(ValueError, match="Gauss-Legendre"):
        sieb200.assemble_matrix(m, _opts("n_pmchwt", C0, 5, 0.1, ntl_form="Line", line_points=21), ctx=gpu_ctx)
    with pytest.raises(ValueError, match="requires N-EFIE"):
        sieb200.assemble_matrix(m, _opts("n_mfie", C0, 5, 0.1, ntl_form="Line"), ctx=gpu_ctx)
    o = sieb200.DielectricOptions(frequency_hz=C0, ntl_form="Line")
    with pytest.raises(ValueError, match="N-PMCHWT or N-Muller"):
        sieb200.assemble_matrix(m, o, ctx=gpu_ctx)
