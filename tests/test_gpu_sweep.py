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
