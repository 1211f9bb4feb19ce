"""GPU adjoint gradients against an FP64 host adjoint built entirely from the
oracle, and against central finite differences on 50 random parameters.

The host gradient (no GPU code): records r(theta) of lossless omega faces
(Lambda = [[jB I, K], [K', jX I]], K = [[0, chi], [-chi, 0]], and the inverse),
Z(r) and b from the oracle's C restatement of the reference's assembly, x =
Z^-1 b (LAPACK), the cone objective L = sum_d w_d (|F_theta|^2 + |F_phi|^2) /
(2 eta0) with F from the oracle's restatement of the reference far-field
projection (as an explicit matrix), and

    dL/dtheta_k = -(1 / eta0) Re(lambda^H (dZ/dtheta_k) x),
    Z^H lambda = A_P^H W F,

where A_P maps x to the far fields, W holds the weights, dZ/dtheta_k is the
mass-block part of Z with records dr/dtheta_k (Z is linear in the records;
dLambda^-1 = -Lambda^-1 dLambda Lambda^-1), computed as (Z(s dr) - Z(0)) / s
with s = 1e6 so that the Calderon part cancels exactly.

Tolerances: GPU (cuSOLVER FP64 and mixed) against the host adjoint, each
component within 1e-6 of its own magnitude plus 1e-9 of the largest (the
FP64 gradient agrees to ~1e-10); fourth-order central differences
(h = 5e-5) on 50 random parameters within 1e-6 of each component plus 1e-8
of the largest (the floor covers the objective's rounding divided by h for
the smallest components)."""

import math

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
C0 = 299792458.0


def _records(B, X, chi):
    nf = B.size
    L = np.zeros((nf, 4, 4), np.complex128)
    L[:, 0, 0] = L[:, 1, 1] = 1j * B
    L[:, 2, 2] = L[:, 3, 3] = 1j * X
    L[:, 0, 3] = chi
    L[:, 1, 2] = -chi
    L[:, 2, 1] = chi
    L[:, 3, 0] = -chi
    Li = np.linalg.inv(L)
    return L, Li, np.concatenate([L.reshape(nf, 16), Li.reshape(nf, 16)], 1)


def _dlambda(kind):
    d = np.zeros((4, 4), np.complex128)
    if kind == 0:
        d[0, 0] = d[1, 1] = 1j
    elif kind == 1:
        d[2, 2] = d[3, 3] = 1j
    else:
        d[0, 3], d[1, 2], d[2, 1], d[3, 0] = 1, -1, 1, -1
    return d


def _setup():
    import sieb200
    m = sieb200.icosphere(1.0, 1)
    o = sieb200.GstcSieOptions(frequency_hz=0.5 * C0, quadrature_rule=5)
    rng = np.random.default_rng(31)
    nf = m.num_faces
    B, X, chi = (rng.uniform(-2, 2, nf) for _ in range(3))
    bad = np.abs(chi ** 2 - B * X) < 0.25
    while bad.any():
        B[bad], X[bad], chi[bad] = (rng.uniform(-2, 2, int(bad.sum())) for _ in range(3))
        bad = np.abs(chi ** 2 - B * X) < 0.25
    return m, o, (B, X, chi)


def _host_gradient(m, o, params, ks, oracle_lib):
    """FP64 host adjoint gradient for the parameter indices ks, and L."""
    import sieb200
    B, X, chi = params
    nf, ne = m.num_faces, m.num_edges
    _, Lami, rec = _records(B, X, chi)
    s = O.kernel_scalars(2, o.frequency_hz)
    Z = O.assemble(oracle_lib, 2, m, 5, s, tensors=rec)
    k = s["omega"] * math.sqrt(s["mu0"] * s["eps0"])
    eta_src = math.sqrt(s["mu0"] / s["eps0"])
    b = O.rhs(oracle_lib, 2, m, 5, dict(kind=0, a=[1, 0, 0], b=[0, 0, 1], region=2), k, eta_src, s["mu0"], s["eps0"])
    x = np.linalg.solve(Z, b)
    eta0 = math.sqrt(o.vacuum_permeability / o.vacuum_permittivity)
    k0 = 2.0 * math.pi * o.frequency_hz / C0
    r, t, p, w = sieb200.cone_directions(10.0, 8, 16)
    nd = r.shape[0]
    # far-field operator of the exterior (J, M) currents, column by column
    A = np.zeros((2 * nd, 2 * ne), np.complex128)
    for c in range(2 * ne):
        j = np.zeros(ne, np.complex128)
        mm = np.zeros(ne, np.complex128)
        (j if c < ne else mm)[c % ne] = 1.0
        ft, fp, _ = O.far_field(oracle_lib, m, j, mm, k0, eta0, r, t, p)
        A[:nd, c], A[nd:, c] = ft, fp
    P = np.zeros((2 * ne, 4 * ne), np.complex128)
    P[np.arange(ne), 2 * ne + np.arange(ne)] = 1.0
    P[ne + np.arange(ne), 3 * ne + np.arange(ne)] = eta0
    AP = A @ P
    F = AP @ x
    W = np.concatenate([w, w])
    L = float(np.sum(W * np.abs(F) ** 2) / (2.0 * eta0))
    lam = np.linalg.solve(Z.conj().T, AP.conj().T @ (W * F))
    Z0 = O.assemble(oracle_lib, 2, m, 5, s, tensors=np.zeros_like(rec))
    scale = 1e6
    g = {}
    for kk in ks:
        kind, f = divmod(int(kk), nf)
        dL = _dlambda(kind)
        drec = np.zeros_like(rec)
        drec[f, :16] = dL.reshape(-1)
        drec[f, 16:] = (-Lami[f] @ dL @ Lami[f]).reshape(-1)
        dZ = (O.assemble(oracle_lib, 2, m, 5, s, tensors=scale * drec) - Z0) / scale
        g[int(kk)] = -(1.0 / eta0) * float(np.real(lam.conj() @ (dZ @ x)))
    return g, L


def _gpu_gradient(m, o, params, method, gpu_ctx):
    import torch
    import sieb200
    B, X, chi = (torch.tensor(v, dtype=torch.float64, requires_grad=True) for v in params)
    b = torch.from_numpy(sieb200.assemble_rhs(m, o, [sieb200.PlaneWaveExcitation()], ctx=gpu_ctx)[:, 0].copy()).cuda()
    obj = sieb200.FarFieldConeObjective(m, o, half_angle_deg=10.0, ctx=gpu_ctx)
    x = sieb200.gstc_solve(sieb200.omega_records(B, X, chi), b, m, o, method=method, tolerance=1e-13, ctx=gpu_ctx)
    L = obj(x)
    L.backward()
    return np.concatenate([B.grad.numpy(), X.grad.numpy(), chi.grad.numpy()]), float(L.detach()), obj, b


@pytest.fixture(scope="module")
def adjoint_case(oracle_lib):
    m, o, params = _setup()
    ks = np.random.default_rng(50).choice(3 * m.num_faces, 50, replace=False)
    g_host, L_host = _host_gradient(m, o, params, ks, oracle_lib)
    return m, o, params, ks, g_host, L_host


@pytest.mark.parametrize("method", ["lu_cusolver", "mixed_ir"])
def test_gpu_gradient_matches_fp64_host_adjoint(method, adjoint_case, gpu_ctx):
    m, o, params, ks, g_host, L_host = adjoint_case
    g, L, _, _ = _gpu_gradient(m, o, params, method, gpu_ctx)
    assert abs(L - L_host) <= 1e-9 * abs(L_host)
    gmax = max(abs(v) for v in g_host.values())
    for kk in ks:
        ref = g_host[int(kk)]
        assert abs(g[kk] - ref) <= 1e-6 * abs(ref) + 1e-9 * gmax, (kk, g[kk], ref)


def test_gpu_gradient_matches_central_differences_on_50_parameters(adjoint_case, gpu_ctx):
    import torch
    import sieb200
    m, o, params, ks, g_host, _ = adjoint_case
    g, _, obj, b = _gpu_gradient(m, o, params, "lu_cusolver", gpu_ctx)
    flat = np.concatenate(params)
    nf = m.num_faces

    def L_of(v):
        rec = sieb200.omega_records(v[:nf], v[nf:2 * nf], v[2 * nf:])
        with torch.no_grad():
            x = sieb200.gstc_solve(rec, b, m, o, method="lu_cusolver", ctx=gpu_ctx)
            return float(obj(x))

    gmax = np.abs(g).max()
    h = 5e-5

    def shifted(kk, d):
        v = flat.copy()
        v[kk] += d
        return L_of(v)

    for kk in ks:
        # fourth-order central difference: near-singular faces make the
        # second-order one's truncation error reach 1e-5 at h = 1e-5
        fd = (8 * (shifted(kk, h) - shifted(kk, -h)) - (shifted(kk, 2 * h) - shifted(kk, -2 * h))) / (12 * h)
        assert abs(fd - g[kk]) <= 1e-6 * abs(g[kk]) + 1e-8 * gmax, (kk, fd, g[kk])
