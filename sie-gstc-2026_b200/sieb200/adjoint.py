"""Adjoint gradients of SIE-GSTC solutions with respect to the per-face
surface-parameter records (no counterpart in the reference, which has no
adjoint).

The GSTC system Z(p) x = b depends on the records p (32 complex values per
face: the 4x4 map Lambda row-major, then its inverse) only through the
jump-condition mass blocks of each face, and linearly. For a real objective
L(x), with g = dL/dx in torch's convention (x.grad),

    Z^H lambda = g,          dL/dp = -conj(lambda^H (dZ/dp) x),

so a gradient costs one conjugate-transpose solve with the factors of the
forward solve plus one contraction kernel (sieb200_gstc_tensor_gradient).
`gstc_solve` wraps assembly, factorization, solve and this backward pass in a
torch.autograd.Function, so objectives written in torch (for example the
far-field power in a cone, through the explicit far-field operator of
`far_field_matrix`) differentiate end to end with respect to whatever
parameterization produced the records (e.g. `omega_records`).

Torch is used here for device buffers and for autograd bookkeeping; the
assembly, factorizations, solves and contractions run in libsieb200.
"""

from __future__ import annotations

import ctypes
import math
from typing import Optional

import numpy as np

from . import _lib
from .mesh import MeshData
from .solvers import (Context, DenseLuSolver, GstcSieOptions, assemble_matrix_device, default_context,
                      to_c_options)

C0 = 299792458.0


def _torch():
    import torch
    return torch


def tensor_gradient(mesh: MeshData, options: GstcSieOptions, lam, x, ctx: Optional[Context] = None):
    """s[f, k] = lambda^H (dZ / d record[f, k]) x for device complex128 torch
    vectors lam and x (length 4 * num_edges); returns a (num_faces, 32)
    complex128 device tensor."""
    torch = _torch()
    ctx = ctx or default_context()
    o = to_c_options(options, _lib.GSTC)
    n = 4 * mesh.num_edges
    if lam.numel() != n or x.numel() != n:
        raise ValueError(f"lambda and x must have {n} entries")
    lam = lam.detach().to(dtype=torch.complex128).contiguous()
    x = x.detach().to(dtype=torch.complex128).contiguous()
    s = torch.empty((mesh.num_faces, 32), dtype=torch.complex128, device=lam.device)
    torch.cuda.synchronize()
    _lib.check(_lib.lib().sieb200_gstc_tensor_gradient(ctx.handle, ctypes.byref(mesh.as_c()), ctypes.byref(o),
                                                       lam.data_ptr(), x.data_ptr(), 1, s.data_ptr()))
    return s


def far_field_matrix(mesh: MeshData, k0: float, eta0: float, r_hat, theta_hat, phi_hat,
                     ctx: Optional[Context] = None):
    """Explicit far-field operator on the device: A (2 ndir, 2 num_edges)
    complex128 with [F_theta; F_phi] = A [J_ext; M_ext] (physical exterior
    currents), the projection of applications/anisotropic_gstc_sphere/
    plot_far_field.py:118-220."""
    torch = _torch()
    ctx = ctx or default_context()
    rh = np.ascontiguousarray(r_hat, dtype=np.float64).reshape(-1, 3)
    th = np.ascontiguousarray(theta_hat, dtype=np.float64).reshape(-1, 3)
    ph = np.ascontiguousarray(phi_hat, dtype=np.float64).reshape(-1, 3)
    nd = rh.shape[0]
    A = torch.empty((2 * nd, 2 * mesh.num_edges), dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    _lib.check(_lib.lib().sieb200_far_field_matrix(ctx.handle, ctypes.byref(mesh.as_c()), float(k0), float(eta0),
                                                   nd, rh.ctypes.data, th.ctypes.data, ph.ctypes.data, 1,
                                                   A.data_ptr()))
    return A


def omega_records(B, X, chi):
    """Records of lossless omega-type bianisotropic faces (torch, differentiable):
    Lambda = [[jB I, K], [K, jX I]] with K = [[0, chi], [-chi, 0]], then its
    inverse (src/sie_mom/gstc/omega_biisotropic.py:410-435,
    applications/omega_biisotropic_sphere/prepare_sie_inputs.py:77-93).
    B, X, chi: real tensors of shape (F,); returns (F, 32) complex128."""
    torch = _torch()
    B, X, chi = (torch.as_tensor(v, dtype=torch.float64) for v in (B, X, chi))
    F = B.shape[0]
    z = torch.zeros_like(B)
    jB = torch.complex(z, B)
    jX = torch.complex(z, X)
    c = torch.complex(chi, z)
    zc = torch.complex(z, z)
    rows = [
        torch.stack([jB, zc, zc, c], -1),
        torch.stack([zc, jB, -c, zc], -1),
        torch.stack([zc, c, jX, zc], -1),
        torch.stack([-c, zc, zc, jX], -1),
    ]
    lam = torch.stack(rows, -2)  # (F, 4, 4)
    inv = torch.linalg.inv(lam)
    return torch.cat([lam.reshape(F, 16), inv.reshape(F, 16)], -1)


def cone_directions(half_angle_deg: float, n_theta: int = 8, n_phi: int = 16):
    """Gauss-Legendre in cos(theta) x uniform phi samples of a cone about +z:
    unit vectors r_hat, theta_hat, phi_hat (n, 3) and solid-angle weights (n,)."""
    ct0 = math.cos(math.radians(half_angle_deg))
    xg, wg = np.polynomial.legendre.leggauss(n_theta)
    ct = 0.5 * (1.0 - ct0) * xg + 0.5 * (1.0 + ct0)
    wct = 0.5 * (1.0 - ct0) * wg
    phis = (np.arange(n_phi) + 0.5) * (2.0 * np.pi / n_phi)
    T, P = np.meshgrid(np.arccos(ct), phis, indexing="ij")
    W = np.repeat(wct[:, None] * (2.0 * np.pi / n_phi), n_phi, axis=1)
    st, ctt, sp, cp = np.sin(T), np.cos(T), np.sin(P), np.cos(P)
    r = np.stack([st * cp, st * sp, ctt], -1).reshape(-1, 3)
    t = np.stack([ctt * cp, ctt * sp, -st], -1).reshape(-1, 3)
    p = np.stack([-sp, cp, np.zeros_like(sp)], -1).reshape(-1, 3)
    return r, t, p, W.reshape(-1)


class _GstcSolve:
    """Holder so that the autograd function is created once torch is imported."""
    fn = None


def _autograd_function():
    if _GstcSolve.fn is not None:
        return _GstcSolve.fn
    torch = _torch()

    class GstcSolve(torch.autograd.Function):
        @staticmethod
        def forward(fctx, records, b, mesh, options, method, tolerance, ctx):
            n = 4 * mesh.num_edges
            Z = torch.empty((n, n), dtype=torch.complex128, device="cuda")
            rec = records.detach().to("cpu", torch.complex128).numpy()
            assemble_matrix_device(mesh, options, Z.data_ptr(), tensors=rec, ctx=ctx)
            solver = DenseLuSolver(n, method, ctx=ctx)
            solver.factorize(Z.data_ptr())
            x = b.detach().to("cuda", torch.complex128).clone().contiguous()
            torch.cuda.synchronize()
            solver.solve(x.data_ptr(), tolerance=tolerance, max_iterations=60)
            ctx.synchronize()
            fctx.solver, fctx.Z = solver, Z  # the mixed method refines against Z
            fctx.mesh, fctx.options, fctx.ctx, fctx.tolerance = mesh, options, ctx, tolerance
            fctx.rec_shape, fctx.rec_device = records.shape, records.device
            fctx.save_for_backward(x)
            return x.clone()

        @staticmethod
        def backward(fctx, grad_x):
            (x,) = fctx.saved_tensors
            lam = grad_x.detach().to("cuda", torch.complex128).clone().contiguous()
            torch.cuda.synchronize()
            fctx.solver.solve(lam.data_ptr(), tolerance=fctx.tolerance, max_iterations=60, adjoint=True)
            fctx.ctx.synchronize()
            s = tensor_gradient(fctx.mesh, fctx.options, lam, x, ctx=fctx.ctx)
            g = -s.conj()
            if fctx.options.tensors_are_uniform:
                g = g.sum(0)
            return g.reshape(fctx.rec_shape).to(fctx.rec_device), None, None, None, None, None, None

    _GstcSolve.fn = GstcSolve
    return GstcSolve


def gstc_solve(records, b, mesh: MeshData, options: GstcSieOptions, method: str = "mixed_ir",
               tolerance: float = 1e-10, ctx: Optional[Context] = None):
    """Scaled solution x of Z(records) x = b on the device, differentiable
    with respect to `records` (torch complex tensor, (F, 32) or (32,) for
    uniform tensors). b: the right-hand side (e.g. sieb200.assemble_rhs)."""
    ctx = ctx or default_context()
    return _autograd_function().apply(records, b, mesh, options, method, tolerance, ctx)


def physical_exterior(x, mesh: MeshData, options: GstcSieOptions):
    """(J_ext, M_ext) physical currents from the scaled solution x (the M blocks
    carry eta0 as in sieb200_solve_gstc_dense_batch)."""
    ne = mesh.num_edges
    eta0 = math.sqrt(options.vacuum_permeability / options.vacuum_permittivity)
    return x[2 * ne:3 * ne], x[3 * ne:4 * ne] * eta0


class FarFieldConeObjective:
    """L = sum_d w_d U(r_d), U = (|F_theta|^2 + |F_phi|^2) / (2 eta0), over a
    cone of directions, as a torch function of the scaled GSTC solution."""

    def __init__(self, mesh: MeshData, options: GstcSieOptions, half_angle_deg: float = 10.0,
                 n_theta: int = 8, n_phi: int = 16, ctx: Optional[Context] = None):
        torch = _torch()
        self.mesh, self.options = mesh, options
        self.eta0 = math.sqrt(options.vacuum_permeability / options.vacuum_permittivity)
        k0 = 2.0 * math.pi * options.frequency_hz / C0
        r, t, p, w = cone_directions(half_angle_deg, n_theta, n_phi)
        self.A = far_field_matrix(mesh, k0, self.eta0, r, t, p, ctx=ctx)
        self.w = torch.as_tensor(w, dtype=torch.float64, device="cuda")
        self.nd = r.shape[0]

    def __call__(self, x):
        torch = _torch()
        j, m = physical_exterior(x, self.mesh, self.options)
        F = self.A @ torch.cat([j, m])
        U = (F[: self.nd].abs() ** 2 + F[self.nd:].abs() ** 2) / (2.0 * self.eta0)
        return (self.w * U).sum()
