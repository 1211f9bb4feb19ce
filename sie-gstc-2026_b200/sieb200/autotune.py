"""Measured choice of the sweep's lane count, cached per GPU and size class.

The batched sweep (sieb200_solve_gstc_sweep) runs its systems on several
concurrent lanes, each with its share of the SMs for the trailing GEMM. How
many lanes pay depends on the sizes: small systems leave most SMs idle in the
latency-bound end of every factorization and gain from sharing the GPU, large
ones lose from the smaller GEMM grids. tune_sweep() times a calibration sweep
at each candidate lane count and stores the fastest in a JSON cache keyed by
the device name and the size class (the largest N, rounded up to a power of
two); sweep_concurrency() reads it, and falls back to a size rule when the
class has not been tuned.

Cache file: $SIEB200_AUTOTUNE_CACHE, else ~/.cache/sieb200/autotune.json.
"""

from __future__ import annotations

import json
import os
from pathlib import Path
from typing import Iterable, Sequence

CANDIDATES = (1, 2, 3, 4)


def cache_path() -> Path:
    p = os.environ.get("SIEB200_AUTOTUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "sieb200" / "autotune.json"


def size_class(sizes: Iterable[int]) -> int:
    """Smallest power of two >= the largest system dimension."""
    n = max(int(x) for x in sizes)
    c = 1
    while c < n:
        c *= 2
    return c


def device_name(ctx=None) -> str:
    try:
        import torch
        dev = ctx.device if ctx is not None else 0
        return torch.cuda.get_device_name(dev)
    except Exception:
        return "unknown"


def _load(path: Path) -> dict:
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def _key(device: str, cls: int) -> str:
    return f"{device}|sweep|{cls}"


def default_concurrency(sizes: Sequence[int]) -> int:
    """Size rule used before tuning: more lanes for smaller systems."""
    n = max(int(x) for x in sizes)
    if n <= 8192:
        return 4
    if n <= 16384:
        return 3
    return 2


def sweep_concurrency(sizes: Sequence[int], ctx=None, path: Path | None = None) -> int:
    entry = _load(path or cache_path()).get(_key(device_name(ctx), size_class(sizes)))
    if isinstance(entry, dict) and int(entry.get("concurrency", 0)) in CANDIDATES:
        return int(entry["concurrency"])
    return default_concurrency(sizes)


def record(sizes: Sequence[int], timings: dict, ctx=None, path: Path | None = None) -> int:
    """Store the fastest of {lane count: seconds} for this size class and
    device; returns the chosen lane count."""
    best = min(timings, key=lambda c: timings[c])
    path = path or cache_path()
    data = _load(path)
    data[_key(device_name(ctx), size_class(sizes))] = {
        "concurrency": int(best), "seconds": {str(k): float(v) for k, v in sorted(timings.items())}}
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_suffix(".tmp")
    tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
    os.replace(tmp, path)
    return int(best)


def tune_sweep(instances, candidates: Sequence[int] = CANDIDATES, ctx=None, path: Path | None = None,
               repeats: int = 1) -> tuple[int, dict]:
    """Time the sweep of `instances` at each lane count (after one warm-up
    run) and cache the fastest. Returns (best, {lane count: seconds})."""
    from .solvers import solve_gstc_sweep_batched
    solve_gstc_sweep_batched(instances, concurrency=max(candidates), ctx=ctx)  # warm-up: workspaces, modules
    timings = {}
    for c in candidates:
        best = None
        for _ in range(repeats):
            _, secs = solve_gstc_sweep_batched(instances, concurrency=c, ctx=ctx)
            best = secs if best is None else min(best, secs)
        timings[c] = best
    sizes = [4 * inst.mesh.num_edges for inst in instances]
    return record(sizes, timings, ctx=ctx, path=path), timings
