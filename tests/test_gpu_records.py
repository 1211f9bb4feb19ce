"""GPU: surface-record preparation on the device against the reference's
golden records (same checks as tests/test_records.py)."""

import pytest

from test_records import check_against_golden

pytestmark = pytest.mark.gpu


def test_records_match_reference_on_gpu(gpu_ctx):
    check_against_golden("cuda")
