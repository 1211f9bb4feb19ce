"""CPU: the rotated-testing formulations (N-EFIE, N-MFIE, N-PMCHWT, N-Muller,
surface nTL form) of the oracle pinned against the reference: the golden
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
    "n_efie": (0, 1, {}),
    "n_mfie": (0, 2, {}),
    "n_pmchwt": (1, 1, dict(eps_r=(4.0, 1.0), mu_r=(1.0, 1.0))),
    "n_muller": (1, 2, dict(eps_r=(2.5, 1.0), mu_r=(1.5, 1.0))),
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


def test_pair_blocks_n_match_reference(golden, vgolden, oracle_lib):
    m = GoldenMesh(golden, "L1r05")
    k1, k2, thr = (float(x) for x in vgolden["pair_n_scalars"])
    for (a, b), ref in zip(vgolden["pair_n_index"], vgolden["pair_n_blocks"]):
        out = np.zeros(72)
        oracle_lib.so_pair_blocks_n(m.vertices.ctypes.data, m.faces.ctypes.data, int(a), int(b), 6, k1, k2,
                                    thr, out.ctypes.data)
        assert rel_err(out, ref) < 1e-13, (a, b)
    # self pair: nTK is zero, nTL is not
    self_blocks = vgolden["pair_n_blocks"][0].reshape(4, 9, 2)
    assert np.all(self_blocks[2:] == 0.0) and np.abs(self_blocks[:2]).max() > 0


@pytest.mark.parametrize("name", sorted(CASES))
def test_variant_matrix_and_rhs_match_reference_golden(name, vgolden, oracle_lib, mesh_l0):
    kind, variant, media = CASES[name]
    s = O.kernel_scalars(kind, C0, **media, threshold_lambda0=1.5)
    Z = O.assemble(oracle_lib, kind, mesh_l0, 5, s, variant=variant)
    assert rel_err(Z, vgolden[f"Z_{name}_L0"]) < 1e-13
    eps_r = media.get("eps_r", (1.0, 1.0))
    mu_r = media.get("mu_r", (1.0, 1.0))
    for region in ((2, 1) if kind == 1 else (2,)):
        er, mr = eps_r[region - 1], mu_r[region - 1]
        k = s["omega"] * math.sqrt(s["mu0"] * s["eps0"] * er * mr)
        eta = math.sqrt(s["mu0"] * mr / (s["eps0"] * er))
        b = O.rhs(oracle_lib, kind, mesh_l0, 5, dict(kind=0, a=[1, 0, 0], b=[0, 0, 1], region=region), k,
                  eta, s["mu0"], s["eps0"], variant=variant, eps_r_src=er, mu_r_src=mr)
        assert rel_err(b, vgolden[f"b_{name}_L0_region{region}"]) < 1e-13, region


@pytest.mark.parametrize("name", sorted(CASES))
def test_variant_oracle_matches_live_reference_harness(name, golden, oracle_lib, ref_lib):
    kind, variant, media = CASES[name]
    m = GoldenMesh(golden, "L1r05")
    s = O.kernel_scalars(kind, 2 * C0, **media, threshold_lambda0=0.3)
    Zo = O.assemble(oracle_lib, kind, m, 4, s, variant=variant)
    Zr = O.assemble(ref_lib, kind, m, 4, s, fn="ref_assemble", variant=variant, threads=1)
    assert rel_err(Zo, Zr) < 1e-13


def test_rotated_formulations_differ_from_tangential(vgolden, golden, oracle_lib, mesh_l0):
    # A check that the fixtures exercise new code: N-PMCHWT is not T-PMCHWT.
    s = O.kernel_scalars(1, C0, eps_r=(4.0, 1.0), threshold_lambda0=1.5)
    Zt = O.assemble(oracle_lib, 1, mesh_l0, 5, s, variant=0)
    assert rel_err(Zt, vgolden["Z_n_pmchwt_L0"]) > 0.1


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
