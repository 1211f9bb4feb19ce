"""CPU: the rotated-testing formulations (N-EFIE, N-MFIE, N-PMCHWT, N-Muller;
surface nTL form B and line form A) of the oracle pinned against the reference: the golden
fixtures of tests/golden/make_variants_golden.py and the live reference
harness when it is built. Plus the option mapping of the Python front end."""

import math
from pathlib import Path

import numpy as np
import pytest

from conftest import GoldenMesh, rel_err
from oracle import oracle as O

C0 = 299792458.0
VG = Path(__file__).resolve().parent / "golden" / "variants_golden.npz"
CASES = {
    "n_efie": (0, 1, {}, 0),
    "n_mfie": (0, 2, {}, 0),
    "n_pmchwt": (1, 1, dict(eps_r=(4.0, 1.0), mu_r=(1.0, 1.0)), 0),
    "n_muller": (1, 2, dict(eps_r=(2.5, 1.0), mu_r=(1.5, 1.0)), 0),
    "n_efie_line": (0, 1, {}, 20),
    "n_pmchwt_line": (1, 1, dict(eps_r=(4.0, 1.0), mu_r=(1.0, 1.0)), 10),
    "n_muller_line": (1, 2, dict(eps_r=(2.5, 1.0), mu_r=(1.5, 1.0)), 7),
}


@pytest.fixture(scope="module")
def vgolden():
    return dict(np.load(VG))


def test_fixture_mixes_extracted_and_regular_pairs(golden):
    # 1.5 lambda0 at lambda0 = 1 m on the unit icosahedron: some pairs are
    # extracted, some are not, so both paths are in the fixtures.
    m = GoldenMesh(golden, "L0")
    c = m.vertices[m.faces].mean(axis=1)
    d = np.linalg.norm(c[:, None, :] - c[None, :, :], axis=-1)
    near = (d < 1.5).sum()
    assert m.faces.shape[0] < near < m.faces.shape[0] ** 2


@pytest.mark.parametrize("line_points,key", [(0, "pair_n_blocks"), (12, "pair_n_blocks_line12")])
def test_pair_blocks_n_match_reference(line_points, key, golden, vgolden, oracle_lib):
    m = GoldenMesh(golden, "L1r05")
    k1, k2, thr = (float(x) for x in vgolden["pair_n_scalars"])
    for (a, b), ref in zip(vgolden["pair_n_index"], vgolden[key]):
        out = np.zeros(72)
        oracle_lib.so_pair_blocks_n(m.vertices.ctypes.data, m.faces.ctypes.data, int(a), int(b), 6, k1, k2,
                                    thr, line_points, out.ctypes.data)
        assert rel_err(out, ref) < 1e-13, (a, b)
    # self pair: nTK is zero, nTL is not
    self_blocks = vgolden["pair_n_blocks"][0].reshape(4, 9, 2)
    assert np.all(self_blocks[2:] == 0.0) and np.abs(self_blocks[:2]).max() > 0


@pytest.mark.parametrize("name", sorted(CASES))
def test_variant_matrix_and_rhs_match_reference_golden(name, vgolden, oracle_lib, mesh_l0):
    kind, variant, media, lp = CASES[name]
    mesh, freq = (_scaled(mesh_l0, 0.3), 3 * C0) if lp else (mesh_l0, C0)
    s = O.kernel_scalars(kind, freq, **media, threshold_lambda0=1.5)
    Z = O.assemble(oracle_lib, kind, mesh, 5, s, variant=variant, line_points=lp)
    assert rel_err(Z, vgolden[f"Z_{name}_L0"]) < 1e-13
    eps_r = media.get("eps_r", (1.0, 1.0))
    mu_r = media.get("mu_r", (1.0, 1.0))
    for region in ((2, 1) if kind == 1 else (2,)):
        er, mr = eps_r[region - 1], mu_r[region - 1]
        k = s["omega"] * math.sqrt(s["mu0"] * s["eps0"] * er * mr)
        eta = math.sqrt(s["mu0"] * mr / (s["eps0"] * er))
        b = O.rhs(oracle_lib, kind, mesh, 5, dict(kind=0, a=[1, 0, 0], b=[0, 0, 1], region=region), k,
                  eta, s["mu0"], s["eps0"], variant=variant, eps_r_src=er, mu_r_src=mr)
        assert rel_err(b, vgolden[f"b_{name}_L0_region{region}"]) < 1e-13, region
    if lp:
        # the line form changes nTL only: not the same matrix as the surface form
        Zb = O.assemble(oracle_lib, kind, mesh, 5, s, variant=variant)
        assert rel_err(Z, Zb) > 1e-4


def _scaled(mesh, f):
    class _M:
        pass
    m = _M()
    m.vertices = np.ascontiguousarray(mesh.vertices * f)
    m.faces, m.edges, m.faces_edges = mesh.faces, mesh.edges, mesh.faces_edges
    return m


def test_line_form_at_unit_scale_is_non_finite_like_the_reference(vgolden, oracle_lib, mesh_l0):
    # At unit scale the reference's line form is not finite: on a testing edge
    # that lies on a source edge (R0 < 1e-8) the regularisation
    # sqrt(R^2 + 1e-16) is lost in rounding once R^2 > ~0.9, and log1p(-1)
    # follows (semi_analytic_integrals.cuh:120-136). The oracle reproduces the
    # same non-finite entries and agrees on the finite ones.
    ref = vgolden["Z_n_efie_line_unit_L0"]
    s = O.kernel_scalars(0, C0, threshold_lambda0=1.5)
    Z = O.assemble(oracle_lib, 0, mesh_l0, 5, s, variant=1, line_points=20)
    fin = np.isfinite(ref)
    assert not fin.all()
    assert np.array_equal(np.isfinite(Z), fin)
    assert rel_err(Z[fin], ref[fin]) < 1e-13


@pytest.mark.parametrize("name", sorted(CASES))
def test_variant_oracle_matches_live_reference_harness(name, golden, oracle_lib, ref_lib):
    kind, variant, media, lp = CASES[name]
    m = GoldenMesh(golden, "L1r05")
    s = O.kernel_scalars(kind, 2 * C0, **media, threshold_lambda0=0.3)
    Zo = O.assemble(oracle_lib, kind, m, 4, s, variant=variant, line_points=lp)
    Zr = O.assemble(ref_lib, kind, m, 4, s, fn="ref_assemble", variant=variant, threads=1, line_points=lp)
    assert rel_err(Zo, Zr) < 1e-13


def test_rotated_formulations_differ_from_tangential(vgolden, golden, oracle_lib, mesh_l0):
    # A check that the fixtures exercise new code: N-PMCHWT is not T-PMCHWT.
    s = O.kernel_scalars(1, C0, eps_r=(4.0, 1.0), threshold_lambda0=1.5)
    Zt = O.assemble(oracle_lib, 1, mesh_l0, 5, s, variant=0)
    assert rel_err(Zt, vgolden["Z_n_pmchwt_L0"]) > 0.1


def test_gauss_legendre_rules_match_reference(vgolden, oracle_lib):
    # The library's table (numpy's leggauss on [0, 1]) against the reference's
    # gauss_legendre_rule: the float-rounded values the kernels use are equal.
    for n in range(1, 21):
        t = np.zeros(n, np.float32)
        w = np.zeros(n, np.float32)
        assert oracle_lib.so_gauss_legendre(n, t.ctypes.data, w.ctypes.data) == n
        assert np.array_equal(t, vgolden[f"gl{n}_nodes"].astype(np.float32)), n
        assert np.array_equal(w, vgolden[f"gl{n}_weights"].astype(np.float32)), n
        assert abs(float(vgolden[f"gl{n}_weights"].sum()) - 1.0) < 1e-14
    assert oracle_lib.so_gauss_legendre(21, None, None) == -1


def test_line_form_constant_potential_vanishes_on_closed_edges(golden):
    # ntl_form_a_line_geometry_test.cpp: with phi_0 = 1 the testing-edge sum
    # sum_e sum_q L_e w_q (tau_j . nu_e) vanishes (the divergence of a
    # rotated RWG integrates to zero over its face). Checked on every face of
    # the level-1 icosphere with the 20-point rule.
    from oracle import oracle as Ol
    lib = Ol.oracle()
    t = np.zeros(20, np.float32)
    w = np.zeros(20, np.float32)
    lib.so_gauss_legendre(20, t.ctypes.data, w.ctypes.data)
    m = GoldenMesh(golden, "L1r05")
    for f in range(m.faces.shape[0]):
        v = m.vertices[m.faces[f]]
        cr = np.cross(v[1] - v[0], v[2] - v[0])
        n = cr / np.linalg.norm(cr)
        for j in range(3):
            fv = v[(j + 2) % 3]
            tot, absum = 0.0, 0.0
            for e in range(3):
                a, b = v[e], v[(e + 1) % 3]
                E = b - a
                L = np.linalg.norm(E)
                nu = np.cross(E, n) / L
                for q in range(20):
                    r = a + float(t[q]) * E
                    c = L * float(w[q]) * np.dot(np.cross(r - fv, n), nu)
                    tot += c
                    absum += abs(c)
            assert abs(tot) <= 1e-8 * absum


def test_python_options_map_reference_formulation_names():
    import sieb200
    from sieb200 import _lib
    from sieb200.solvers import to_c_options
    o = to_c_options(sieb200.DielectricOptions(frequency_hz=1e9, formulation="N_PMCHWT"), _lib.PMCHWT)
    assert (o.variant, o.ntl_form) == (_lib.VARIANT_N, _lib.NTL_SURFACE)
    o = to_c_options(sieb200.DielectricOptions(frequency_hz=1e9, formulation="muller", ntl_form="line"),
                     _lib.PMCHWT)
    assert (o.variant, o.ntl_form) == (_lib.VARIANT_N_JUMP, _lib.NTL_LINE)
    o = to_c_options(sieb200.PecOptions(frequency_hz=1e9, formulation="NMfie"), _lib.PEC_EFIE)
    assert o.variant == _lib.VARIANT_N_JUMP
    assert to_c_options(sieb200.PecOptions(frequency_hz=1e9), _lib.PEC_EFIE).variant == _lib.VARIANT_T
    with pytest.raises(ValueError):
        to_c_options(sieb200.DielectricOptions(frequency_hz=1e9, formulation="X"), _lib.PMCHWT)
    with pytest.raises(ValueError):
        to_c_options(sieb200.PecOptions(frequency_hz=1e9, formulation="NEfie", ntl_form="line",
                                        line_quadrature_points=21), _lib.PEC_EFIE)


def test_incident_fields_match_reference_functors(vgolden, oracle_lib):
    # so_incident_fields (the oracle of sieb200_incident_fields) against the
    # reference's PlaneWave / DipoleSource functors (source_functors.cuh:14-130).
    P = vgolden["inc_points"]
    k, eta = (float(x) for x in vgolden["inc_k_eta"])
    for q in range(3):
        src = vgolden[f"inc{q}_source"]
        spec = dict(kind=int(src[0]), is_magnetic=int(src[1]), a=src[2:5], b=src[5:8])
        E, H = O.incident_fields(oracle_lib, spec, k, eta, P)
        assert rel_err(E, vgolden[f"inc{q}_E"]) < 1e-14 and rel_err(H, vgolden[f"inc{q}_H"]) < 1e-14, q


def test_incident_fields_match_live_reference(vgolden, oracle_lib, ref_lib):
    rng = np.random.default_rng(5)
    P = rng.uniform(-2, 2, (30, 3))
    for spec in (dict(kind=0, a=[0, 0, 1.5], b=[0.6, 0.8, 0.0]), dict(kind=1, a=[1, 2, 3], b=[0, 0, 0], is_magnetic=1)):
        Eo, Ho = O.incident_fields(oracle_lib, spec, 7.0, 300.0, P)
        Er, Hr = O.incident_fields(ref_lib, spec, 7.0, 300.0, P)
        assert rel_err(Eo, Er) < 1e-14 and rel_err(Ho, Hr) < 1e-14


@pytest.mark.parametrize("name,rule,thr,freq", [("n_pmchwt", 1, 0.3, 2), ("n_muller", 20, 0.1, 1),
                                                ("n_efie_line", 3, 0.5, 1), ("n_mfie", 13, 0.6, 1),
                                                ("n_pmchwt_line", 2, 0.3, 2)])
def test_variant_oracle_matches_harness_across_rules(name, rule, thr, freq, golden, oracle_lib, ref_lib):
    # Dunavant rules 1-20 (one point up to 79), thresholds from self pairs
    # only to most neighbours.
    kind, variant, media, lp = CASES[name]
    m = GoldenMesh(golden, "L1r05")
    s = O.kernel_scalars(kind, freq * C0, **media, threshold_lambda0=thr)
    Zo = O.assemble(oracle_lib, kind, m, rule, s, variant=variant, line_points=lp)
    Zr = O.assemble(ref_lib, kind, m, rule, s, fn="ref_assemble", variant=variant, threads=1, line_points=lp)
    assert np.isfinite(Zr).all()
    assert rel_err(Zo, Zr) < 1e-13


@pytest.mark.parametrize("kind,variant,region,mag", [(0, 0, 2, 0), (0, 1, 2, 1), (0, 2, 2, 0), (1, 0, 1, 1),
                                                     (1, 1, 1, 0), (1, 2, 1, 1), (1, 2, 2, 0), (2, 0, 1, 0),
                                                     (2, 0, 2, 1)])
def test_dipole_rhs_matches_reference(kind, variant, region, mag, vgolden, oracle_lib, mesh_l0):
    # The oracle's dipole right-hand sides (every formulation, testing variant
    # and region) against the reference's DipoleSource through its own
    # calculateExcitationQuadrature and the RHS placements.
    er, mr = (2.5, 1.5) if region == 1 else (1.0, 1.0)
    mu0, eps0 = 1.25663706212e-6, 8.8541878128e-12
    k = 2 * math.pi * C0 * math.sqrt(mu0 * mr * eps0 * er)
    eta = math.sqrt(mu0 * mr / (eps0 * er))
    pos = [0.1, 0.0, 0.05] if region == 1 else [0.4, 1.8, -0.3]
    b = O.rhs(oracle_lib, kind, mesh_l0, 5, dict(kind=1, a=[0.3, -0.2, 1.0], b=pos, is_magnetic=mag, region=region),
              k, eta, mu0, eps0, variant=variant, eps_r_src=er, mu_r_src=mr)
    assert rel_err(b, vgolden[f"bdip_{kind}_{variant}_{region}_{mag}"]) < 1e-13
