"""The oracle's Mie series (oracle/mie.py) against the reference's own
spherical-wave collocation solution of the benchmark's dielectric sphere
(tests/golden/mie_golden.npz, made by tests/golden/make_mie_golden.py) and
against the closed-form small-sphere and large-sphere limits."""

from pathlib import Path

import numpy as np

from oracle import mie

GOLDEN = Path(__file__).resolve().parent / "golden" / "mie_golden.npz"


def test_mie_matches_reference_collocation():
    g = np.load(GOLDEN)
    ft, fp = mie.far_field_moduli(float(g["k0"]), float(g["radius"]), float(g["eps_r"]), g["theta"], g["phi"])
    rt, rp = np.abs(g["r_E_theta"]), np.abs(g["r_E_phi"])
    # the collocation solution is accurate to ~3e-7 (n_max = 15 on a 40 x 40 grid)
    assert np.abs(ft - rt).max() / rt.max() < 1e-6
    assert np.abs(fp - rp).max() / rp.max() < 1e-6


def test_mie_limits():
    k, a = 1.0, 0.01
    # Rayleigh backscatter: 4 pi k^4 a^6 |(eps-1)/(eps+2)|^2, PEC 9 pi k^4 a^6
    assert abs(mie.bistatic_rcs(k, a, 4.0, np.pi, 0.0) / (4 * np.pi * k ** 4 * a ** 6 * 0.25) - 1) < 1e-4
    assert abs(mie.bistatic_rcs(k, a, None, np.pi, 0.0) / (9 * np.pi * k ** 4 * a ** 6) - 1) < 1e-4
    # small PEC sphere at theta = 90 degrees: the H-plane (phi = 90) cross
    # section is 4 times the E-plane one (amplitudes 1 - cos/2 and cos - 1/2);
    # backscatter alone cannot tell a_n from b_n
    e = mie.bistatic_rcs(k, a, None, np.pi / 2, 0.0)
    h = mie.bistatic_rcs(k, a, None, np.pi / 2, np.pi / 2)
    assert abs(h / e - 4.0) < 1e-3
    # dielectric Rayleigh sphere: the E-plane cross section vanishes at 90 degrees
    assert mie.bistatic_rcs(k, a, 4.0, np.pi / 2, 0.0) < 1e-6 * mie.bistatic_rcs(k, a, 4.0, np.pi / 2, np.pi / 2)
    # optical limit of the monostatic PEC cross section: pi a^2
    assert abs(mie.bistatic_rcs(1.0, 60.0, None, np.pi, 0.0, n_max=120) / (np.pi * 60 ** 2) - 1) < 1e-2
