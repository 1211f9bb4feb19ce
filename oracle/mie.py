"""Test infrastructure only: Mie series for plane-wave scattering by a
homogeneous sphere (dielectric, or perfectly conducting) in vacuum.

Written from the mathematics (Bohren & Huffman, "Absorption and Scattering of
Light by Small Particles", 1983, sections 4.4 and 4.8), with Riccati-Bessel
functions psi_n(z) = z j_n(z) and xi_n(z) = z h_n^(1)(z) from scipy:

  a_n = [m psi_n(mx) psi_n'(x) - mu1 psi_n(x) psi_n'(mx)]
        / [m psi_n(mx) xi_n'(x) - mu1 xi_n(x) psi_n'(mx)]
  b_n = [mu1 psi_n(mx) psi_n'(x) - m psi_n(x) psi_n'(mx)]
        / [mu1 psi_n(mx) xi_n'(x) - m xi_n(x) psi_n'(mx)]
  (relative permeability mu1 inside, 1 outside; m = sqrt(eps_r mu1);
  B&H eqs. 4.53-4.54 multiplied through by x)
  PEC (the limit m -> infinity of the above): a_n = psi_n'(x) / xi_n'(x),
  b_n = psi_n(x) / xi_n(x)

  S1(theta) = sum_n (2n+1)/(n(n+1)) (a_n pi_n + b_n tau_n)
  S2(theta) = sum_n (2n+1)/(n(n+1)) (a_n tau_n + b_n pi_n)

with pi_n, tau_n by the upward recurrence in mu = cos(theta). For an x-polarised
wave travelling along +z, |E_theta| r -> |S2 cos(phi)| / k and
|E_phi| r -> |S1 sin(phi)| / k far away, so the bistatic radar cross section
is sigma = (4 pi / k^2) (|S2|^2 cos^2 phi + |S1|^2 sin^2 phi). These moduli do
not depend on the time convention; the MoM far fields are compared through
them.

Pinned against the reference's own spherical-wave collocation solver
(src/spherical_expansion/solver.py:53, the dielectric sphere as a GSTC sphere
with zero surface susceptibilities) through tests/golden/mie_golden.npz.
"""

from __future__ import annotations

import numpy as np
from scipy.special import spherical_jn, spherical_yn


def _riccati(n: np.ndarray, z):
    """psi_n(z), psi_n'(z), xi_n(z), xi_n'(z) (xi only for real z)."""
    j = spherical_jn(n, z)
    jp = spherical_jn(n, z, derivative=True)
    psi = z * j
    dpsi = j + z * jp
    if np.iscomplexobj(z):
        return psi, dpsi, None, None
    y = spherical_yn(n, z)
    yp = spherical_yn(n, z, derivative=True)
    xi = z * (j + 1j * y)
    dxi = (j + 1j * y) + z * (jp + 1j * yp)
    return psi, dpsi, xi, dxi


def coefficients(x: float, eps_r: complex | None, mu_r: complex = 1.0, n_max: int | None = None):
    """Mie coefficients a_n, b_n (n = 1..n_max) for size parameter x = k a;
    eps_r None: perfectly conducting sphere."""
    if n_max is None:
        n_max = int(np.ceil(x + 4.05 * x ** (1.0 / 3.0) + 2)) + 6
    n = np.arange(1, n_max + 1)
    psi, dpsi, xi, dxi = _riccati(n, x)
    if eps_r is None:
        return dpsi / dxi, psi / xi
    m = np.sqrt(complex(eps_r) * complex(mu_r))
    mx = m * x
    jm = spherical_jn(n, mx)
    jmp = spherical_jn(n, mx, derivative=True)
    psim = mx * jm
    dpsim = jm + mx * jmp
    mu1 = complex(mu_r)
    a = (m * psim * dpsi - mu1 * psi * dpsim) / (m * psim * dxi - mu1 * xi * dpsim)
    b = (mu1 * psim * dpsi - m * psi * dpsim) / (mu1 * psim * dxi - m * xi * dpsim)
    return a, b


def amplitudes(theta: np.ndarray, a: np.ndarray, b: np.ndarray):
    """S1(theta), S2(theta)."""
    mu = np.cos(np.asarray(theta, dtype=np.float64))
    n_max = a.size
    pi_prev = np.zeros_like(mu)
    pi_n = np.ones_like(mu)
    S1 = np.zeros(mu.shape, np.complex128)
    S2 = np.zeros(mu.shape, np.complex128)
    for n in range(1, n_max + 1):
        if n > 1:
            pi_next = ((2 * n - 1) * mu * pi_n - n * pi_prev) / (n - 1)
            pi_prev, pi_n = pi_n, pi_next
        tau_n = n * mu * pi_n - (n + 1) * pi_prev
        f = (2 * n + 1) / (n * (n + 1))
        S1 += f * (a[n - 1] * pi_n + b[n - 1] * tau_n)
        S2 += f * (a[n - 1] * tau_n + b[n - 1] * pi_n)
    return S1, S2


def far_field_moduli(k: float, radius: float, eps_r, theta, phi, mu_r=1.0, n_max=None):
    """|F_theta| and |F_phi| (scattered field times r, far away) for a unit
    x-polarised plane wave along +z."""
    a, b = coefficients(k * radius, eps_r, mu_r, n_max)
    S1, S2 = amplitudes(theta, a, b)
    phi = np.asarray(phi, dtype=np.float64)
    return np.abs(S2 * np.cos(phi)) / k, np.abs(S1 * np.sin(phi)) / k


def bistatic_rcs(k: float, radius: float, eps_r, theta, phi, mu_r=1.0, n_max=None):
    """sigma(theta, phi) in m^2 for a unit incident field."""
    ft, fp = far_field_moduli(k, radius, eps_r, theta, phi, mu_r, n_max)
    return 4.0 * np.pi * (ft ** 2 + fp ** 2)
