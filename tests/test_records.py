"""Surface-record preparation (sieb200.records) against the reference's own
tensor_io.prepare_tensor_records (golden vectors from
tests/golden/make_records_golden.py) and its error behaviour
(tests/python/test_gstc_tensor_io.py of the reference). Runs on the CPU with
torch; the same code runs on the GPU in tests/test_gpu_records.py."""

from pathlib import Path

import numpy as np
import pytest

RG = Path(__file__).resolve().parent / "golden" / "records_golden.npz"
CASES = {"lossless": ("reciprocal_lossless", "general"), "complex": ("reciprocal_complex", "general"),
         "diagonal": ("reciprocal_lossless", "diagonal")}


def _params(maps):
    m = np.moveaxis(maps, 0, -1)
    return {"Y_ee": m[:2, :2], "Y_em": m[:2, 2:], "Y_me": m[2:, :2], "Y_mm": m[2:, 2:]}


def check_against_golden(device, hermitian_solver="auto"):
    from sieb200.records import prepare_tensor_records
    g = dict(np.load(RG))
    for name, (method, structure) in CASES.items():
        maps = g[f"{name}_maps"]
        rec, diag = prepare_tensor_records(_params(maps), maps.shape[0], reference_impedance=float(g["eta"]),
                                           extraction_method=method, tensor_structure=structure, device=device,
                                           hermitian_solver=hermitian_solver)
        rec = rec.cpu().numpy()
        ref = g[f"{name}_records"]
        assert np.array_equal(rec[:, :16], ref[:, :16]), name  # the map is kept as given
        inv, rinv = rec[:, 16:], ref[:, 16:]
        # per-face relative agreement of the inverses (the maps are ill-scaled by
        # eta^2; LDL^H / LU against scipy's solve: measured <= 3e-15)
        err = np.abs(inv - rinv).max(axis=1) / np.abs(rinv).max(axis=1)
        assert err.max() < 1e-12, name
        assert abs(diag["maximum_map_condition_number"] / float(g[f"{name}_condition"]) - 1) < 1e-8


@pytest.mark.parametrize("solver", ["auto", "lu"])
def test_records_match_reference_on_cpu(solver):
    # "lu" is the branch CUDA takes for lossless maps
    check_against_golden("cpu", solver)


def _one(matrix):
    return {"Y_ee": matrix[:2, :2, None], "Y_em": matrix[:2, 2:, None], "Y_me": matrix[2:, :2, None],
            "Y_mm": matrix[2:, 2:, None]}


def test_record_errors_match_reference():
    from sieb200.records import prepare_tensor_records
    kw = dict(reference_impedance=376.73, extraction_method="reciprocal_lossless", tensor_structure="general",
              device="cpu")
    with pytest.raises(ValueError, match="numerically singular at 1 faces"):
        prepare_tensor_records(_one(1j * np.diag([1, 2, 3, 0])), 1, **kw)
    with pytest.raises(ValueError, match="losslessness"):
        prepare_tensor_records(_one(np.diag([0.1 + 1j, 2j, 3j, 4j])), 1, **dict(kw, reference_impedance=1))
    m = 1j * np.eye(4)
    m[0, 1] = 1j
    with pytest.raises(ValueError, match="reciprocity"):
        prepare_tensor_records(_one(m), 1, **kw)
    m = 1j * np.eye(4)
    m[0, 1] = m[1, 0] = 0.5j
    with pytest.raises(ValueError, match="diagonal structure"):
        prepare_tensor_records(_one(m), 1, **dict(kw, tensor_structure="diagonal"))
    with pytest.raises(ValueError, match="must be finite with shape"):
        prepare_tensor_records(_one(1j * np.eye(4)), 2, **kw)
    with pytest.raises(ValueError, match="reference_impedance must be finite and positive"):
        prepare_tensor_records(_one(1j * np.eye(4)), 1, **dict(kw, reference_impedance=0.0))


def test_complex_map_inverse_is_full_complex_inverse():
    from sieb200.records import prepare_tensor_records
    matrix = np.diag([1 + 2j, 2 - 1j, 3 + 0.5j, 4 - 2j])
    rec, _ = prepare_tensor_records(_one(matrix), 1, reference_impedance=376.7303134118051,
                                    extraction_method="reciprocal_complex", tensor_structure="general", device="cpu")
    rec = rec.numpy()
    assert np.array_equal(rec[0, :16].reshape(4, 4), matrix)
    np.testing.assert_allclose(rec[0, 16:].reshape(4, 4), np.linalg.inv(matrix), rtol=1e-14, atol=0)
