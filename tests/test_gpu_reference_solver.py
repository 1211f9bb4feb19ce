"""GPU: the library against the reference's own GPU dielectric solver
(solve_dielectric_dense with its assembly kernels and cuSOLVER LU, built for
sm_100a from the reference's sources by oracle/Makefile, target ref_gpu), on
the same mesh and inputs: the FP64 currents (cuSOLVER and the own FP64 LU)
within 1e-10 of the reference's, the mixed currents within 1e-9.

The reference returns interior-oriented physical currents [J, M]; the
library returns [J, M] with the same orientation and eta0 scaling."""

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
C0 = 299792458.0


@pytest.fixture(scope="module")
def ref_gpu():
    lib = O.reference_gpu()
    if lib is None:
        pytest.skip("reference GPU solver oracle/_ref/libsieref_gpu.so not built")
    return lib


@pytest.mark.parametrize("solver,tol", [("lu_cusolver", 1e-10), ("lu_fp64", 1e-10), ("mixed_ir", 1e-9)])
def test_dielectric_currents_match_reference_gpu_solver(solver, tol, ref_gpu, gpu_ctx):
    import sieb200
    m = sieb200.icosphere(0.5, 2)
    cur_ref, t = O.reference_gpu_dielectric(ref_gpu, m, C0, 4.0, 7)
    assert t["relative_residual"] < 1e-10
    o = sieb200.DielectricOptions(frequency_hz=C0, quadrature_rule=7, solver=solver,
                                  interior=sieb200.IsotropicMedium(4.0, 1.0))
    r = sieb200.solve_dielectric_dense(m, o, sieb200.PlaneWaveExcitation(), ctx=gpu_ctx)
    assert np.linalg.norm(r.currents - cur_ref) / np.linalg.norm(cur_ref) < tol
