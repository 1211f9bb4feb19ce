"""GPU: surface-integral field values (sieb200_surface_fields) against the
reference's values (tests/golden/fields_golden.npz) and the C oracle.

Tolerance: 1e-12 relative to the largest field value of a case (the kernel
sums faces in another order than the reference's per-thread strides and tree
reduction, and contracts multiply-adds; the branch choice per face uses the
same float distance and threshold). Repeated calls are bit-identical."""

from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
FIX = Path(__file__).resolve().parent / "golden" / "fields_golden.npz"


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def _mesh(g):
    import sieb200
    return sieb200.MeshData(np.ascontiguousarray(g["V"]), g["F"].astype(np.int32), g["Ed"].astype(np.int32),
                            g["FE"].astype(np.int32))


@pytest.mark.parametrize("case", ["vac_r5", "diel_r7"])
def test_fields_match_reference_golden(case, gpu_ctx):
    import sieb200
    g = np.load(FIX)
    f, er, mr, rule = g[f"{case}_params"]
    E, H = sieb200.evaluate_surface_integral_fields(
        _mesh(g), g["J"], g["M"], g["points"], float(f), sieb200.IsotropicMedium(float(er), float(mr)), int(rule),
        float(g["eps0"]), float(g["mu0"]), ctx=gpu_ctx)
    assert _rel(E, g[f"{case}_E"]) < 1e-12
    assert _rel(H, g[f"{case}_H"]) < 1e-12


def test_fields_match_oracle_and_are_deterministic(gpu_ctx, oracle_lib):
    import sieb200
    m = sieb200.icosphere(0.5, 3)
    rng = np.random.default_rng(11)
    ne = m.num_edges
    J = rng.standard_normal(ne) + 1j * rng.standard_normal(ne)
    M = rng.standard_normal(ne) + 1j * rng.standard_normal(ne)
    d = rng.standard_normal((40, 3))
    pts = d / np.linalg.norm(d, axis=1)[:, None] * rng.uniform(0.2, 2.0, (40, 1))
    f = 299792458.0 / 1.5
    med = sieb200.IsotropicMedium(2.0, 1.0)
    E, H = sieb200.evaluate_surface_integral_fields(m, J, M, pts, f, med, 7, ctx=gpu_ctx)
    Eo, Ho = O.surface_fields(oracle_lib, m, J, M, pts, f, 2.0, 1.0, rule=7)
    assert _rel(E, Eo) < 1e-12 and _rel(H, Ho) < 1e-12
    E2, H2 = sieb200.evaluate_surface_integral_fields(m, J, M, pts, f, med, 7, ctx=gpu_ctx)
    assert np.array_equal(E, E2) and np.array_equal(H, H2)
    # no magnetic currents: the same as zeros
    E3, H3 = sieb200.evaluate_surface_integral_fields(m, J, None, pts, f, med, 7, ctx=gpu_ctx)
    E4, H4 = sieb200.evaluate_surface_integral_fields(m, J, np.zeros(ne), pts, f, med, 7, ctx=gpu_ctx)
    assert np.array_equal(E3, E4) and np.array_equal(H3, H4)


def test_fields_validation_mirrors_reference(gpu_ctx):
    import sieb200
    m = sieb200.icosphere(1.0, 0)
    J = np.ones(m.num_edges, complex)
    pts = np.array([[0.0, 0.0, 2.0]])
    ev = sieb200.evaluate_surface_integral_fields
    with pytest.raises(sieb200.InvalidArgument):
        ev(m, J, J, pts, -1.0, ctx=gpu_ctx)
    with pytest.raises(sieb200.InvalidArgument):
        ev(m, J, J, pts, 1e8, sieb200.IsotropicMedium(0.0, 1.0), ctx=gpu_ctx)
    with pytest.raises(sieb200.InvalidArgument):
        ev(m, J, J, pts, 1e8, quadrature_rule=21, ctx=gpu_ctx)
    with pytest.raises(sieb200.InvalidArgument):
        ev(m, J, J, np.array([[0.0, np.nan, 2.0]]), 1e8, ctx=gpu_ctx)
    with pytest.raises(ValueError):
        ev(m, J[:-1], J, pts, 1e8, ctx=gpu_ctx)
    E, H = ev(m, J, J, np.zeros((0, 3)), 1e8, ctx=gpu_ctx)
    assert E.shape == (0, 3) and H.shape == (0, 3)
