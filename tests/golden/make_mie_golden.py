"""Regenerate tests/golden/mie_golden.npz from the reference's own
spherical-wave collocation solver (src/spherical_expansion/solver.py:53,
imported from the reference checkout), which pins the oracle's Mie series
(oracle/mie.py).

    python tests/golden/make_mie_golden.py /path/to/reference   (or $SIE_REFERENCE)

Case: the dielectric sphere of the T-PMCHWT benchmark (radius 0.5 m,
eps_r = 4, mu_r = 1, k0 = 2 pi, x-polarised unit plane wave along +z) as a
GSTC sphere whose surface susceptibilities are all zero, n_max = 15 on a
40 x 40 collocation grid (the reference test's settings). Stored: the
scattered E_theta and E_phi times r at r = 1e6 m (Hankel-function SVWFs) on a
theta grid in three phi cuts, and the solver's relative residual.
"""

from __future__ import annotations

import contextlib
import io
import os
import sys
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent / "mie_golden.npz"


def main() -> None:
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SIE_REFERENCE")
    if not ref:
        raise SystemExit("name the reference checkout: make_mie_golden.py /path/to/reference (or set SIE_REFERENCE)")
    sys.path.insert(0, str(Path(ref) / "src"))
    from spherical_expansion.solver import solve_collocation
    from spherical_expansion.svwf_sphere import compute_fields

    c0 = 299792458.0
    radius, eps_r = 0.5, 4.0
    mu0 = 1.25663706212e-6
    eps0 = 8.8541878128e-12
    eta0 = np.sqrt(mu0 / eps0)
    k0 = 2.0 * np.pi
    k1 = k0 * np.sqrt(eps_r)
    eta1 = eta0 / np.sqrt(eps_r)
    with contextlib.redirect_stdout(io.StringIO()):
        a, b, c, d, metrics = solve_collocation(
            n_max=15, k0=k0, eta0=eta0, k1=k1, eta1=eta1, radius=radius,
            gstc_params={"Y": 0.0, "Chi": 0.0, "Gamma": 0.0, "Z": 0.0},
            n_theta=40, n_phi=40, row_scale=True, return_metrics=True)
    theta = np.radians(np.arange(5.0, 180.0, 10.0))
    phis = np.array([0.0, np.pi / 4, np.pi / 2])
    th, ph = np.meshgrid(theta, phis, indexing="ij")
    r_obs = 1.0e6
    r = np.full(th.size, r_obs)
    E, _ = compute_fields(k=k0, r=r, theta=th.ravel(), phi=ph.ravel(), a_coeffs=a, b_coeffs=b, kind=3, eta=eta0,
                          grid=False)
    np.savez_compressed(
        OUT, radius=radius, eps_r=eps_r, k0=k0, r_obs=r_obs, theta=th.ravel(), phi=ph.ravel(),
        r_E_theta=r_obs * E[1], r_E_phi=r_obs * E[2], residual_rel=float(metrics["residual_rel"]))
    print(f"wrote {OUT} (collocation relative residual {metrics['residual_rel']:.2e})")


if __name__ == "__main__":
    main()
