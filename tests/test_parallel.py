"""CPU: sharding of independent systems across ranks (world_size 2, gloo).

The multi-GPU path has no data-path collective, so what needs testing is the
host logic: the cost partition, that every item is computed exactly once and
every rank ends with all results in order, and the max-over-ranks timing."""

import os
import socket

import pytest

import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "sie-gstc-2026_b200"))

from sieb200.parallel import dense_solve_cost, max_over_ranks, partition_by_cost, run_sharded  # noqa: E402


def test_partition_by_cost_balances_and_covers():
    rng_costs = [dense_solve_cost(n) for n in (4000, 24000, 8000, 12000, 16000, 4000, 20000, 6000)]
    shares = partition_by_cost(rng_costs, 3)
    flat = sorted(i for s in shares for i in s)
    assert flat == list(range(len(rng_costs)))
    loads = [sum(rng_costs[i] for i in s) for s in shares]
    # LPT bound: the slowest rank is within 4/3 of the ideal share (or the largest item)
    ideal = max(sum(rng_costs) / 3, max(rng_costs))
    assert max(loads) <= 4.0 / 3.0 * ideal
    assert partition_by_cost(rng_costs, 3) == shares  # deterministic
    assert partition_by_cost([1.0, 1.0], 4)[2:] == [[], []]


def test_run_sharded_without_group_is_local():
    assert run_sharded([1, 2, 3], lambda v: v * v) == [1, 4, 9]
    assert max_over_ranks(2.5) == 2.5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        calls = []

        def fn(item):
            calls.append(item["id"])
            return {"id": item["id"], "rank": rank, "value": item["n"] * 2}

        sizes = [6000, 1000, 3000, 5000, 2000, 4000, 1500]
        items = [{"id": i, "n": n} for i, n in enumerate(sizes)]
        res = run_sharded(items, fn, costs=[dense_solve_cost(n) for n in sizes])
        t = max_over_ranks(float(rank + 1))
        with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
            f.write(repr((calls, [(r["id"], r["rank"], r["value"]) for r in res], t)))
    finally:
        dist.destroy_process_group()


def test_run_sharded_two_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    r0 = eval((tmp_path / "r0.txt").read_text())
    r1 = eval((tmp_path / "r1.txt").read_text())
    calls0, res0, t0 = r0
    calls1, res1, t1 = r1
    assert sorted(calls0 + calls1) == list(range(7))  # each item computed once
    assert not set(calls0) & set(calls1)
    assert res0 == res1  # every rank has every result, in item order
    assert [r[0] for r in res0] == list(range(7))
    assert [r[2] for r in res0] == [2 * n for n in (6000, 1000, 3000, 5000, 2000, 4000, 1500)]
    assert t0 == t1 == 2.0
