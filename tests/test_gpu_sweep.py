"""GPU: a sweep of uneven GSTC spheres at different frequencies through
sieb200.parallel.solve_gstc_sweep equals the instances solved one by one
(bit-identical: same kernels, same order), on one rank."""

from types import SimpleNamespace

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
C0 = 299792458.0


def test_sweep_matches_individual_solves(gpu_ctx):
    import sieb200
    from sieb200.parallel import solve_gstc_sweep
    rng = np.random.default_rng(3)
    insts = []
    for level, ka in [(1, 1.0), (2, 2.0), (1, 3.0)]:
        m = sieb200.icosphere(1.0, level)
        rec = sieb200.omega_records(*(rng.uniform(0.5, 2.0, m.num_faces) for _ in range(3))).numpy()
        o = sieb200.GstcSieOptions(frequency_hz=ka * C0 / (2 * np.pi), quadrature_rule=5, solver="mixed_ir")
        cases = [sieb200.GstcExcitationCase(exterior=sieb200.PlaneWaveExcitation())]
        insts.append(SimpleNamespace(mesh=m, tensors=rec, options=o, cases=cases))
    res = solve_gstc_sweep(insts, ctx=gpu_ctx)
    assert len(res) == 3
    for inst, r in zip(insts, res):
        ref = sieb200.solve_gstc_dense_batch(inst.mesh, inst.tensors, inst.options, inst.cases, ctx=gpu_ctx)
        assert np.array_equal(r[0].currents, ref[0].currents)
        assert r[0].metrics["relative_residual"] <= 1e-10


def _reciprocal_records(rng, nf, scale=0.5):
    """Random reciprocal maps [[Y, K], [-K^T, Z]] (Y, Z symmetric, complex
    uniform entries) plus their inverses, as (nf, 32) records."""
    recs = np.zeros((nf, 32), np.complex128)
    for f in range(nf):
        def c(*shape):
            return rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)
        Y = c(2, 2); Y = (Y + Y.T) / 2 + 2 * np.eye(2)
        Zm = c(2, 2); Zm = (Zm + Zm.T) / 2 + 2 * np.eye(2)
        K = scale * c(2, 2)
        L = np.block([[Y, K], [-K.T, Zm]])
        recs[f, :16] = L.reshape(-1)
        recs[f, 16:] = np.linalg.inv(L).reshape(-1)
    return recs


@pytest.mark.parametrize("solver,tol", [("lu_cusolver", 1e-12), ("mixed_ir", 1e-9)])
@pytest.mark.parametrize("concurrency", [1, 3])
def test_batched_sweep_matches_individual_solves(solver, tol, concurrency, gpu_ctx):
    """sieb200_solve_gstc_sweep over uneven spheres and frequencies equals
    solve_gstc_dense_batch per instance, in input order, with the metrics
    of each instance."""
    import sieb200
    rng = np.random.default_rng(11)
    insts = []
    for n, ka in [(4, 1.5), (7, 3.0), (5, 2.0), (6, 4.0), (3, 1.0)]:
        m = sieb200.geodesic_sphere(1.0, n)
        t = _reciprocal_records(rng, m.num_faces)
        o = sieb200.GstcSieOptions(frequency_hz=ka * C0 / (2 * np.pi), quadrature_rule=5, solver=solver)
        insts.append(sieb200.SweepInstance(m, t, o, exterior=sieb200.PlaneWaveExcitation()))
    res, secs = sieb200.solve_gstc_sweep_batched(insts, concurrency=concurrency, ctx=gpu_ctx)
    assert secs > 0 and len(res) == len(insts)
    for inst, r in zip(insts, res):
        ref = sieb200.solve_gstc_dense_batch(inst.mesh, inst.tensors, inst.options,
                                             [sieb200.GstcExcitationCase(exterior=inst.exterior)], ctx=gpu_ctx)[0]
        assert np.linalg.norm(r.currents - ref.currents) / np.linalg.norm(ref.currents) < tol
        assert r.metrics["matrix_dimension"] == 4 * inst.mesh.num_edges
        assert r.metrics["relative_residual"] <= 1e-10


def test_batched_sweep_reports_the_failing_instance(gpu_ctx):
    import sieb200
    m = sieb200.geodesic_sphere(1.0, 3)
    t = _reciprocal_records(np.random.default_rng(1), m.num_faces)
    good = sieb200.SweepInstance(m, t, sieb200.GstcSieOptions(frequency_hz=C0, quadrature_rule=5),
                                 exterior=sieb200.PlaneWaveExcitation())
    bad = sieb200.SweepInstance(m, t, sieb200.GstcSieOptions(frequency_hz=C0, quadrature_rule=25),
                                exterior=sieb200.PlaneWaveExcitation())
    with pytest.raises(sieb200.InvalidArgument, match="sweep instance 1"):
        sieb200.solve_gstc_sweep_batched([good, bad], concurrency=2, ctx=gpu_ctx)
