"""CPU: the oracle pinned against the reference (golden fixtures made from the
reference's own code, and the live reference harness when it is built), plus
the host-side logic of the product that needs no GPU."""

import math

import numpy as np
import pytest

from conftest import GoldenMesh, rel_err
from oracle import oracle as O

C0 = 299792458.0


def test_dunavant_rules_match_reference_bit_exact(golden, oracle_lib):
    for rule in range(1, 21):
        p_ref, w_ref = golden[f"rule{rule}_points"], golden[f"rule{rule}_weights"]
        n = oracle_lib.so_rule(rule, None, None)
        p = np.zeros(2 * n, np.float32)
        w = np.zeros(n, np.float32)
        oracle_lib.so_rule(rule, p.ctypes.data, w.ctypes.data)
        assert n == w_ref.size
        assert np.array_equal(p, p_ref) and np.array_equal(w, w_ref), rule
    # published point counts (rule 5 = 7, 7 = 13, 17 = 61, 20 = 79)
    assert [oracle_lib.so_rule(r, None, None) for r in (1, 5, 7, 13, 17, 20)] == [1, 7, 13, 37, 61, 79]


def test_dunavant_weights_sum_to_one_and_integrate_exactly(oracle_lib):
    # triangle_dunavant_rule_test.cpp: rule of degree d integrates x^a y^b, a+b <= d.
    degree = {1: 1, 2: 2, 3: 3, 4: 4, 5: 5, 7: 7, 17: 17}
    for rule, d in degree.items():
        n = oracle_lib.so_rule(rule, None, None)
        p = np.zeros(2 * n, np.float32)
        w = np.zeros(n, np.float32)
        oracle_lib.so_rule(rule, p.ctypes.data, w.ctypes.data)
        x, y, w = p[0::2].astype(float), p[1::2].astype(float), w.astype(float)
        assert abs(w.sum() - 1.0) < 1e-6
        for a in range(d + 1):
            for b in range(d + 1 - a):
                exact = 2.0 * math.factorial(a) * math.factorial(b) / math.factorial(a + b + 2)
                assert abs((w * x**a * y**b).sum() - exact) < 2e-6, (rule, a, b)


def test_edge_numbering_matches_reference(golden, oracle_lib):
    for name in ("L0", "L1r05"):
        m = GoldenMesh(golden, name)
        fe = np.zeros_like(m.faces)
        e = np.zeros((3 * m.faces.shape[0], 2), np.int32)
        ne = oracle_lib.so_build_edges(m.faces.ctypes.data, m.faces.shape[0], e.ctypes.data, fe.ctypes.data)
        assert ne == m.edges.shape[0]
        assert np.array_equal(fe, m.faces_edges) and np.array_equal(e[:ne], m.edges)


def _wilton(lib, r, tri):
    out = np.zeros(12)
    lib.so_wilton(np.ascontiguousarray(r, dtype=float).ctypes.data,
                  np.ascontiguousarray(tri, dtype=float).ctypes.data, out.ctypes.data)
    return out


def test_wilton_potentials_match_reference(golden, oracle_lib):
    tri = golden["wilton_tri"]
    for r, ref in zip(golden["wilton_points"], golden["wilton_values"]):
        got = _wilton(oracle_lib, r, tri)
        assert rel_err(got, ref) < 1e-13


def test_phi0_closed_forms(oracle_lib):
    # Known answers of tests/cpp/semi_analytic_test.cpp:19-155 (equilateral
    # triangle, side 1, in z = 0).
    s3 = math.sqrt(3.0)
    tri = np.array([[0, 0, 0], [1, 0, 0], [0.5, s3 / 2, 0]], dtype=float)
    c = np.array([0.5, s3 / 6, 0.0])
    cases = [
        (c, s3 * math.log(2 + s3)),
        (np.array([0.0, -0.5, 0.0]), 0.47636237419365196),
        (c + [0, 0, 0.25], 1.2111344892951112),
        (c + [0, 0, 10.0], 0.04328324600959819),
        (np.array([0.0, 0.0, 0.25]), 0.7250473223433905),
        (np.array([0.5, 0.0, 0.0]), 1.6162320698995925042),
    ]
    for r, expected in cases:
        assert abs(_wilton(oracle_lib, r, tri)[0] - expected) < 1e-12 * abs(expected), r


@pytest.mark.parametrize("name", ["pec", "pmchwt", "gstc_face", "gstc_sph_uniform"])
def test_oracle_matrix_and_rhs_match_reference_golden(name, golden, oracle_lib, mesh_l0):
    kind = {"pec": 0, "pmchwt": 1}.get(name, 2)
    media = {"pmchwt": dict(eps_r=(4.0, 1.0), mu_r=(1.0, 1.0)),
             "gstc_sph_uniform": dict(eps_r=(2.0, 1.0), mu_r=(1.0, 1.0))}.get(name, {})
    s = O.kernel_scalars(kind, C0, **media)
    t = {"gstc_face": golden["gstc_tensors_L0"], "gstc_sph_uniform": golden["gstc_tensors_uniform"]}.get(name)
    Z = O.assemble(oracle_lib, kind, mesh_l0, 5, s, tensors=t, uniform=name == "gstc_sph_uniform",
                   basis=1 if name == "gstc_sph_uniform" else 0)
    assert rel_err(Z, golden[f"Z_{name}_L0"]) < 1e-13
    eps_r = media.get("eps_r", (1.0, 1.0))
    k = s["omega"] * math.sqrt(s["mu0"] * s["eps0"] * eps_r[1])
    eta = math.sqrt(s["mu0"] / (s["eps0"] * eps_r[1]))
    b = O.rhs(oracle_lib, kind, mesh_l0, 5, dict(kind=0, a=[1, 0, 0], b=[0, 0, 1], region=2), k, eta,
              s["mu0"], s["eps0"])
    assert rel_err(b, golden[f"b_{name}_L0"]) < 1e-13


def test_oracle_far_field_matches_reference_script(golden, oracle_lib):
    m = GoldenMesh(golden, "L1r05")
    ne = m.edges.shape[0]
    cur = golden["ff_currents"]
    ft, fp, U = O.far_field(oracle_lib, m, cur[2 * ne:3 * ne], cur[3 * ne:], float(golden["ff_k0"]),
                            float(golden["ff_eta0"]), golden["ff_r_hat"], golden["ff_theta_hat"],
                            golden["ff_phi_hat"])
    assert rel_err(ft, golden["ff_f_theta"]) < 1e-12
    assert rel_err(fp, golden["ff_f_phi"]) < 1e-12
    assert rel_err(U, golden["ff_U"]) < 1e-12


@pytest.mark.parametrize("kind,rule", [(0, 7), (1, 4), (2, 3)])
def test_oracle_matches_live_reference_harness(kind, rule, golden, oracle_lib, ref_lib):
    m = GoldenMesh(golden, "L1r05")
    media = dict(eps_r=(4.0, 1.0), mu_r=(1.0, 1.0)) if kind == 1 else {}
    # threshold 0.3 lambda0 so that edge-adjacent pairs take the singular path too
    s = O.kernel_scalars(kind, 2 * C0, **media, threshold_lambda0=0.3)
    rng = np.random.default_rng(7)
    t = rng.standard_normal((m.faces.shape[0], 32)) + 1j * rng.standard_normal((m.faces.shape[0], 32))
    Zo = O.assemble(oracle_lib, kind, m, rule, s, tensors=t if kind == 2 else None)
    Zr = O.assemble(ref_lib, kind, m, rule, s, tensors=t if kind == 2 else None, fn="ref_assemble")
    assert rel_err(Zo, Zr) < 1e-13


def test_python_icosphere_matches_reference(golden):
    import sieb200
    for name, (r, lv) in {"L0": (1.0, 0), "L1r05": (0.5, 1)}.items():
        g = GoldenMesh(golden, name)
        m = sieb200.icosphere(r, lv)
        assert np.array_equal(m.faces, g.faces)
        assert np.abs(m.vertices - g.vertices).max() < 1e-15
        assert np.array_equal(m.edges, g.edges) and np.array_equal(m.faces_edges, g.faces_edges)


def test_geodesic_sphere_counts():
    import sieb200
    m = sieb200.geodesic_sphere(0.5, 4)
    assert m.num_faces == 20 * 16 and m.num_edges == 30 * 16
    assert np.allclose(np.linalg.norm(m.vertices, axis=1), 0.5)
    v0, v1, v2 = (m.vertices[m.faces[:, i]] for i in range(3))
    n = np.cross(v1 - v0, v2 - v0)
    assert (np.einsum("ij,ij->i", n, (v0 + v1 + v2) / 3) > 0).all()
