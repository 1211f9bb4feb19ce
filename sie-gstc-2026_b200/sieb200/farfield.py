"""Far-field projection and bistatic RCS on the GPU.

MetasurfaceFarFieldEvaluator mirrors
applications/anisotropic_gstc_sphere/plot_far_field.py:118-265 (Schelkunoff
N and L vectors at the script's 7-point rule, F_theta, F_phi, radiation
intensity U, radiated power and directivity); the sums run in
sieb200_far_field.
"""

from __future__ import annotations

import numpy as np

from . import _lib
from .mesh import MeshData
from .solvers import Context, default_context

SPEED_OF_LIGHT = 299792458.0
VACUUM_PERMITTIVITY = 8.8541878188e-12
VACUUM_PERMEABILITY = 1.25663706127e-6
VACUUM_IMPEDANCE = float(np.sqrt(VACUUM_PERMEABILITY / VACUUM_PERMITTIVITY))


def spherical_frames(theta: np.ndarray, phi: np.ndarray):
    theta = np.asarray(theta, dtype=np.float64).ravel()
    phi = np.asarray(phi, dtype=np.float64).ravel()
    st, ct, sp, cp = np.sin(theta), np.cos(theta), np.sin(phi), np.cos(phi)
    r_hat = np.column_stack([st * cp, st * sp, ct])
    theta_hat = np.column_stack([ct * cp, ct * sp, -st])
    phi_hat = np.column_stack([-sp, cp, np.zeros_like(sp)])
    return r_hat, theta_hat, phi_hat


def far_field(mesh: MeshData, j_exterior: np.ndarray, m_exterior: np.ndarray | None, k0: float,
              eta0: float, r_hat, theta_hat, phi_hat, ctx: Context | None = None):
    ctx = ctx or default_context()
    j = np.ascontiguousarray(j_exterior, dtype=np.complex128)
    m = None if m_exterior is None else np.ascontiguousarray(m_exterior, dtype=np.complex128)
    rh = np.ascontiguousarray(r_hat, dtype=np.float64).reshape(-1, 3)
    th = np.ascontiguousarray(theta_hat, dtype=np.float64).reshape(-1, 3)
    ph = np.ascontiguousarray(phi_hat, dtype=np.float64).reshape(-1, 3)
    nd = rh.shape[0]
    if j.size != mesh.num_edges or (m is not None and m.size != mesh.num_edges):
        raise ValueError("current vectors must have one coefficient per mesh edge")
    ft = np.zeros(nd, dtype=np.complex128)
    fp = np.zeros(nd, dtype=np.complex128)
    U = np.zeros(nd, dtype=np.float64)
    import ctypes
    _lib.check(_lib.lib().sieb200_far_field(ctx.handle, ctypes.byref(mesh.as_c()), j.ctypes.data,
                                            _lib.ptr(m), float(k0), float(eta0), nd, rh.ctypes.data,
                                            th.ctypes.data, ph.ctypes.data, ft.ctypes.data,
                                            fp.ctypes.data, U.ctypes.data))
    return ft, fp, U


def evaluate_surface_integral_fields(mesh: MeshData, electric_currents, magnetic_currents, observation_points,
                                     frequency_hz: float, medium=None, quadrature_rule: int = 17,
                                     vacuum_permittivity: float = VACUUM_PERMITTIVITY,
                                     vacuum_permeability: float = VACUUM_PERMEABILITY,
                                     ctx: Context | None = None):
    """The positive surface-integral terms Q_E = +j w mu L[J] + K[M] and
    Q_H = -K[J] + j w eps L[M] at observation points, as
    evaluate_surface_integral_fields (surface_current_fields.hpp:12-44) returns
    them: (E, H), each (npoints, 3) complex128. electric/magnetic_currents:
    one physical RWG coefficient per edge (M, not M / eta0; None = 0);
    medium: an IsotropicMedium (relative constants, default vacuum). Not the
    scattered or total fields by themselves: F_total = F_incident - Q in the
    region the currents radiate into."""
    import ctypes
    ctx = ctx or default_context()
    eps_r = 1.0 if medium is None else float(medium.relative_permittivity)
    mu_r = 1.0 if medium is None else float(medium.relative_permeability)
    j = np.ascontiguousarray(electric_currents, dtype=np.complex128).ravel()
    m = None if magnetic_currents is None else np.ascontiguousarray(magnetic_currents, dtype=np.complex128).ravel()
    if j.size != mesh.num_edges or (m is not None and m.size != mesh.num_edges):
        raise ValueError("field evaluation requires one electric and magnetic coefficient per mesh edge")
    pts = np.ascontiguousarray(observation_points, dtype=np.float64).reshape(-1, 3)
    E = np.zeros((pts.shape[0], 3), dtype=np.complex128)
    H = np.zeros((pts.shape[0], 3), dtype=np.complex128)
    _lib.check(_lib.lib().sieb200_surface_fields(ctx.handle, ctypes.byref(mesh.as_c()), j.ctypes.data, _lib.ptr(m),
                                                 pts.shape[0], pts.ctypes.data, float(frequency_hz), eps_r, mu_r,
                                                 float(vacuum_permittivity), float(vacuum_permeability),
                                                 int(quadrature_rule), E.ctypes.data, H.ctypes.data))
    return E, H


class MetasurfaceFarFieldEvaluator:
    """Exterior-current radiation pattern evaluator (plot_far_field.py:118-265).

    currents: [J_int, M_int, J_ext, M_ext] physical coefficients (GSTC), or
    pass j_exterior / m_exterior directly."""

    def __init__(self, mesh: MeshData, frequency_hz: float, currents: np.ndarray | None = None,
                 j_exterior: np.ndarray | None = None, m_exterior: np.ndarray | None = None):
        self.mesh = mesh
        self.frequency_hz = frequency_hz
        self.omega = 2.0 * np.pi * frequency_hz
        self.k0 = self.omega / SPEED_OF_LIGHT
        self.eta0 = VACUUM_IMPEDANCE
        ne = mesh.num_edges
        if currents is not None:
            c = np.asarray(currents, dtype=np.complex128).ravel()
            if c.size != 4 * ne:
                raise ValueError(f"currents has {c.size} elements; expected {4 * ne}")
            j_exterior, m_exterior = c[2 * ne: 3 * ne], c[3 * ne: 4 * ne]
        if j_exterior is None:
            raise ValueError("either currents or j_exterior is required")
        self.j = j_exterior
        self.m = m_exterior

    def evaluate_directions(self, r_hat, theta_hat, phi_hat):
        return far_field(self.mesh, self.j, self.m, self.k0, self.eta0, r_hat, theta_hat, phi_hat)

    def compute_total_power_and_directivity(self, num_theta: int = 91, num_phi: int = 181):
        theta_vals = np.linspace(0.0, np.pi, num_theta)
        phi_vals = np.linspace(0.0, 2.0 * np.pi, num_phi, endpoint=False)
        th, ph = np.meshgrid(theta_vals, phi_vals, indexing="ij")
        r_hat, theta_hat, phi_hat = spherical_frames(th.ravel(), ph.ravel())
        _, _, U = self.evaluate_directions(r_hat, theta_hat, phi_hat)
        u_grid = U.reshape(num_theta, num_phi)
        dtheta = theta_vals[1] - theta_vals[0]
        dphi = phi_vals[1] - phi_vals[0]
        w = np.ones(num_theta)
        w[0] = w[-1] = 0.5
        p_rad = float(np.sum(u_grid * np.sin(theta_vals)[:, None] * w[:, None]) * dtheta * dphi)
        d = 4.0 * np.pi * u_grid / p_rad
        d_max = float(np.max(d))
        return p_rad, d_max, float(10.0 * np.log10(max(d_max, 1e-12))), theta_vals, phi_vals, d


def bistatic_rcs(mesh: MeshData, j_exterior, m_exterior, k0: float, eta0: float, theta, phi,
                 incident_amplitude: float = 1.0):
    """sigma = 4 pi (|F_theta|^2 + |F_phi|^2) / |E0|^2 for the exterior
    currents (PEC: m_exterior = None)."""
    r_hat, theta_hat, phi_hat = spherical_frames(theta, phi)
    ft, fp, _ = far_field(mesh, j_exterior, m_exterior, k0, eta0, r_hat, theta_hat, phi_hat)
    return 4.0 * np.pi * (np.abs(ft) ** 2 + np.abs(fp) ** 2) / incident_amplitude ** 2
