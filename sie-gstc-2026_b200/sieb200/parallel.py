"""Multi-GPU execution of independent systems (one process per GPU).

The dense MoM path has no data-path collective: a single system is solved
on one GPU, and several GPUs help only by taking different systems — the
instances of a frequency sweep over uneven meshes, the right-hand-side
blocks of a batch, the perturbed objectives of a finite-difference check.
So scaling is sharding plus one gather of the (small) results:

* `partition_by_cost` assigns items to ranks by the longest-processing-time
  rule on an estimated cost (N^3 for a dense factorization), which keeps the
  slowest rank within 4/3 of the optimum;
* `run_sharded` runs a rank's share and gathers every item's result on every
  rank (torch.distributed object all-gather; NCCL on GPUs, gloo on CPU);
* `max_over_ranks` is the timing rule for multi-GPU numbers.

No NCCL collective touches device data on the hot path, and nothing here
uses TMA multicast.
"""

from __future__ import annotations

import heapq
from typing import Callable, Sequence


def partition_by_cost(costs: Sequence[float], world_size: int) -> list[list[int]]:
    """Item indices per rank: largest cost first, each to the least-loaded
    rank (ties to the lower rank), so the result is deterministic."""
    if world_size < 1:
        raise ValueError("world_size must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world_size)]
    heapq.heapify(heap)
    shares: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shares]


def dense_solve_cost(n: int) -> float:
    """Relative cost of one dense factorization + solve of order n."""
    return float(n) ** 3


def _dist():
    import torch.distributed as dist
    return dist


def run_sharded(items: Sequence, fn: Callable, costs: Sequence[float] | None = None, group=None) -> list:
    """fn(item) for every item, each on one rank; returns the list of all
    results (in item order) on every rank. Without an initialized process
    group everything runs locally."""
    dist = _dist()
    if not (dist.is_available() and dist.is_initialized()):
        return [fn(it) for it in items]
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    costs = costs if costs is not None else [1.0] * len(items)
    mine = partition_by_cost(costs, world)[rank]
    local = {i: fn(items[i]) for i in mine}
    gathered: list = [None] * world
    dist.all_gather_object(gathered, local, group=group)
    out: list = [None] * len(items)
    for part in gathered:
        for i, v in part.items():
            out[i] = v
    return out


def max_over_ranks(value: float, group=None) -> float:
    """Largest value over the ranks (the time of a multi-GPU step)."""
    dist = _dist()
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    import torch
    backend = dist.get_backend(group)
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def solve_gstc_sweep(instances: Sequence, ctx=None, group=None) -> list:
    """Sweep of independent SIE-GSTC systems (uneven meshes,
    frequencies, tensor records), each an object with attributes mesh,
    tensors, options and cases (sieb200.GstcExcitationCase list). Instances
    are spread over the ranks by N^3 cost; every rank returns all results
    (per instance, the list of SolveResult of its cases) in input order."""
    from .solvers import solve_gstc_dense_batch

    def one(inst):
        return solve_gstc_dense_batch(inst.mesh, inst.tensors, inst.options, inst.cases, ctx=ctx)

    costs = [dense_solve_cost(4 * inst.mesh.num_edges) for inst in instances]
    return run_sharded(instances, one, costs=costs, group=group)
