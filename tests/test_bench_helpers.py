"""CPU: the benchmark's critical-path summary of the library's per-launch
timeline (bench.timeline_summary), which reads kinds 0 trailing GEMM,
1 triangular solve, 2 FP64 matvec, 3 diagonal block, 4 panels,
6 factorization and 7 refined solve, spans in ms."""

import sys
from pathlib import Path

import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))


def _steps(split: bool):
    """Three block steps: panels, then the GEMM beside the next diagonal
    block. With split panels each step's panels are a head and the rest,
    overlapping in time on two streams."""
    spans = [(6, 0.0, 1.0), (7, 1.0, 1.5)]
    t = 0.0
    for k, (gemm, diag) in enumerate([(0.10, 0.05), (0.04, 0.06), (0.03, 0.02)]):
        if split:
            spans += [(4, t, t + 0.012), (4, t + 0.001, t + 0.015)]
        else:
            spans.append((4, t, t + 0.015))
        t += 0.015
        spans += [(0, t + 0.002, t + 0.002 + gemm), (3, t + 0.001, t + 0.001 + diag)]
        t += 0.002 + max(gemm, diag)
    spans.append((4, t, t + 0.015))
    spans += [(1, 1.1, 1.3), (2, 1.3, 1.4)]
    return spans


@pytest.mark.parametrize("split", [False, True])
def test_timeline_summary_counts_each_step_once(split):
    import bench
    out = bench.timeline_summary(_steps(split))
    assert out["factorization_ms"] == pytest.approx(1.0)
    assert out["refined_solve_ms"] == pytest.approx(0.5)
    # three steps between four panels spans, whether or not the panels split
    assert out["steps_bound_by_gemm"] == 2
    assert out["steps_bound_by_diag"] == 1
    assert out["sum_max_gemm_diag_ms"] == pytest.approx(0.10 + 0.06 + 0.03)
    assert out["gaps_ms"] == pytest.approx(3 * 0.002, abs=1e-9)
    assert out["trsv_us"] == [200.0]
    assert out["matvec_us"] == [100.0]
    # panels time is the sum of the launches' own durations
    per_step = 0.012 + 0.014 if split else 0.015
    assert out["panels_ms"] == pytest.approx(3 * per_step + 0.015)
