"""GPU: surface-record preparation on the device against the reference's
golden records (same checks as tests/test_records.py)."""

import pytest

from test_records import check_against_golden

pytestmark = pytest.mark.gpu


def test_records_match_reference_on_gpu(gpu_ctx):
    check_against_golden("cuda")


def test_record_errors_on_gpu(gpu_ctx):
    """The kernel path raises the reference's errors (same cases as the CPU test)."""
    import numpy as np
    from sieb200.records import prepare_tensor_records
    from test_records import _one
    kw = dict(reference_impedance=376.73, extraction_method="reciprocal_lossless", tensor_structure="general",
              device="cuda")
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


def test_records_kernel_is_the_cuda_path(gpu_ctx):
    """On CUDA the records come from the library kernel (one launch)."""
    import numpy as np
    from sieb200 import _lib
    from sieb200.records import prepare_tensor_records
    from test_records import _one
    n0 = _lib.lib().sieb200_launch_count()
    prepare_tensor_records(_one(np.diag([1 + 2j, 2 - 1j, 3 + 0.5j, 4 - 2j])), 1, reference_impedance=376.73,
                           extraction_method="reciprocal_complex", tensor_structure="general", device="cuda")
    assert _lib.lib().sieb200_launch_count() - n0 == 1
