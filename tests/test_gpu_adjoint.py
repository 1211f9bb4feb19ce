"""GPU: adjoint gradients of SIE-GSTC solutions with respect to the per-face
tensor records, and the explicit far-field operator.

Pins (the reference has no adjoint, so parity is against the derivative of
this library's own assembly, itself pinned to the reference):
  * the contraction s = lambda^H (dZ/dp) x equals the central difference of
    the assembled matrix (exact for a linear dependence; tolerance 1e-9
    relative, set by FP64 rounding of Z);
  * the far-field operator reproduces sieb200_far_field to 1e-12;
  * gradients of a far-field cone objective through gstc_solve match central
    finite differences of the objective to 1e-6 relative (FP64 cuSOLVER
    solves), and the mixed-precision solver's gradient matches the FP64 one
    to 1e-8 relative."""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
C0 = 299792458.0


def _case(level=1, seed=0, uniform=False, basis="face"):
    import sieb200
    m = sieb200.icosphere(1.0, level)
    o = sieb200.GstcSieOptions(frequency_hz=0.5 * C0, quadrature_rule=5, basis=basis,
                               tensors_are_uniform=uniform)
    rng = np.random.default_rng(seed)
    nf = 1 if uniform else m.num_faces
    B, X, chi = (rng.uniform(-2, 2, nf) for _ in range(3))
    return m, o, (B, X, chi)


def _records_np(params):
    import sieb200
    return sieb200.omega_records(*params).numpy()


@pytest.mark.parametrize("uniform,basis", [(False, "face"), (False, "spherical"), (True, "face")])
def test_contraction_equals_matrix_derivative(uniform, basis, gpu_ctx):
    import torch
    import sieb200
    m, o, params = _case(1, 3, uniform, basis)
    rec = _records_np(params).reshape(-1)
    n = 4 * m.num_edges
    rng = np.random.default_rng(5)
    lam = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    s = sieb200.tensor_gradient(m, o, torch.from_numpy(lam).cuda(), torch.from_numpy(x).cuda(),
                                ctx=gpu_ctx).cpu().numpy()
    if uniform:
        s = s.sum(0, keepdims=True)
    for k in rng.choice(rec.size, 12, replace=False):
        h = 1.0  # Z is linear in the record: the central difference is exact
        rp, rm = rec.copy(), rec.copy()
        rp[k] += h
        rm[k] -= h
        dZ = (sieb200.assemble_matrix(m, o, rp, ctx=gpu_ctx) - sieb200.assemble_matrix(m, o, rm, ctx=gpu_ctx)) / (2 * h)
        ref = lam.conj() @ (dZ @ x)
        got = s.reshape(-1)[k]
        scale = np.linalg.norm(lam) * np.linalg.norm(dZ) * np.linalg.norm(x)
        assert abs(got - ref) <= 1e-9 * scale, (k, got, ref)
    # also the imaginary direction (complex-linear dependence)
    k = int(rng.integers(rec.size))
    rp = rec.copy()
    rp[k] += 1j
    dZ = sieb200.assemble_matrix(m, o, rp, ctx=gpu_ctx) - sieb200.assemble_matrix(m, o, rec, ctx=gpu_ctx)
    ref = lam.conj() @ (dZ @ x)
    assert abs(1j * s.reshape(-1)[k] - ref) <= 1e-9 * np.linalg.norm(lam) * np.linalg.norm(dZ) * np.linalg.norm(x)


def test_far_field_matrix_matches_far_field(gpu_ctx):
    import sieb200
    m = sieb200.icosphere(1.0, 2)
    rng = np.random.default_rng(1)
    ne = m.num_edges
    j = rng.standard_normal(ne) + 1j * rng.standard_normal(ne)
    mm = rng.standard_normal(ne) + 1j * rng.standard_normal(ne)
    r, t, p, _ = sieb200.cone_directions(40.0, 4, 6)
    k0, eta0 = 2 * math.pi, 376.73
    ft, fp, _ = sieb200.far_field(m, j, mm, k0, eta0, r, t, p, ctx=gpu_ctx)
    A = sieb200.far_field_matrix(m, k0, eta0, r, t, p, ctx=gpu_ctx).cpu().numpy()
    F = A @ np.concatenate([j, mm])
    nd = r.shape[0]
    assert np.linalg.norm(F[:nd] - ft) <= 1e-12 * np.linalg.norm(ft)
    assert np.linalg.norm(F[nd:] - fp) <= 1e-12 * np.linalg.norm(fp)


def _objective_and_grad(m, o, params, method, gpu_ctx):
    import torch
    import sieb200
    B, X, chi = (torch.tensor(v, dtype=torch.float64, requires_grad=True) for v in params)
    b = torch.from_numpy(sieb200.assemble_rhs(m, o, [sieb200.PlaneWaveExcitation()], ctx=gpu_ctx)[:, 0].copy()).cuda()
    obj = sieb200.FarFieldConeObjective(m, o, half_angle_deg=10.0, ctx=gpu_ctx)
    x = sieb200.gstc_solve(sieb200.omega_records(B, X, chi), b, m, o, method=method, tolerance=1e-13,
                           ctx=gpu_ctx)
    L = obj(x)
    L.backward()
    return float(L.detach()), np.concatenate([B.grad.numpy(), X.grad.numpy(), chi.grad.numpy()]), obj, b


def test_gradient_matches_central_differences(gpu_ctx):
    import torch
    import sieb200
    m, o, params = _case(1, 11)
    L0, g, obj, b = _objective_and_grad(m, o, params, "lu_cusolver", gpu_ctx)
    assert L0 > 0
    flat = np.concatenate(params)
    nf = m.num_faces
    rng = np.random.default_rng(12)

    def L_of(v):
        rec = sieb200.omega_records(v[:nf], v[nf:2 * nf], v[2 * nf:])
        with torch.no_grad():
            x = sieb200.gstc_solve(rec, b, m, o, method="lu_cusolver", ctx=gpu_ctx)
            return float(obj(x))

    for k in rng.choice(flat.size, 6, replace=False):
        h = 1e-5
        vp, vm = flat.copy(), flat.copy()
        vp[k] += h
        vm[k] -= h
        fd = (L_of(vp) - L_of(vm)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * np.abs(g).max(), (k, fd, g[k])


def test_mixed_gradient_matches_fp64(gpu_ctx):
    m, o, params = _case(2, 21)
    L64, g64, _, _ = _objective_and_grad(m, o, params, "lu_cusolver", gpu_ctx)
    Lmx, gmx, _, _ = _objective_and_grad(m, o, params, "mixed_ir", gpu_ctx)
    assert abs(Lmx - L64) <= 1e-10 * abs(L64)
    assert np.linalg.norm(gmx - g64) <= 1e-8 * np.linalg.norm(g64)
