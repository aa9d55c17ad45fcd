"""Launch-shape autotuner: times the LW chunk size of the two-kernel LW on this device and remembers the
fastest per (device, layers, route, column-count bucket).

The chunk size is the column tile of the LW gas-optics / sweep kernel pair: how many columns share one
scratch pass (95 KB per column) before the sweeps read it back.  Small chunks keep more of the scratch in
L2 but launch more often and leave the GPU idle at each chunk's tail; large chunks do the opposite.  Every
candidate gives the same bits (each column's arithmetic is independent of the chunking), so the tuner
changes speed only.

    from woof_nam_b200.tune import tuned_config
    cfg = tuned_config(ncol=796590)          # SolverConfig with the fastest lw_chunk for this GPU
"""
from __future__ import annotations

import json
import os
from dataclasses import replace
from pathlib import Path

from .solver import SolverConfig

CANDIDATES = (4096, 8192, 16384, 32768, 65536, 131072)
CACHE = Path(os.environ.get("WOOF_NAM_B200_TUNE", Path.home() / ".cache" / "woof_nam_b200" / "tune.json"))


def bucket(ncol: int) -> int:
    """Power-of-two ceiling of the column count (the cache key's size class), at least 1024."""
    b = 1024
    while b < ncol:
        b *= 2
    return b


def key(device: str, nlay: int, route: str, ncol: int) -> str:
    return f"{device}|nlay={nlay}|route={route}|cols<={bucket(ncol)}"


def load_cache(path: Path = CACHE) -> dict:
    try:
        return json.loads(Path(path).read_text())
    except (OSError, ValueError):
        return {}


def save_cache(cache: dict, path: Path = CACHE) -> None:
    p = Path(path)
    p.parent.mkdir(parents=True, exist_ok=True)
    tmp = p.with_suffix(".tmp")
    tmp.write_text(json.dumps(cache, indent=1, sort_keys=True))
    tmp.replace(p)


def choose(times: dict) -> int:
    """The fastest candidate; ties go to the larger chunk (fewer launches)."""
    return min(times, key=lambda c: (times[c], -c))


def time_candidates(base: SolverConfig, ncol: int, candidates=CANDIDATES, reps: int = 2, seed: int = 2002) -> dict:
    """Device time (ms) of the LW of one solve of min(ncol, 131072) synthetic columns per candidate chunk
    size, CUDA events on the current stream, after one warm-up solve."""
    import torch
    from .columns import make_columns
    from .solver import RadSolver
    n = min(ncol, max(CANDIDATES))
    cols = make_columns(n, seed)
    times = {}
    dev = None
    for c in candidates:
        if c > n and c != candidates[0]:
            continue
        s = RadSolver(replace(base, lw_chunk=c, parts="lw"))
        if dev is None:
            dev = s.to_device(cols)
        out = s.alloc_outputs(n)
        s.solve(dev, cols.solcon, out)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            s.solve(dev, cols.solcon, out)
        e1.record()
        torch.cuda.synchronize()
        times[c] = e0.elapsed_time(e1) / reps
        s.close()
    return times


def tuned_config(ncol: int, base: SolverConfig | None = None, cache_path: Path = CACHE, timer=None,
                 device: str | None = None, max_chunk: int | None = None) -> SolverConfig:
    """base (default SolverConfig()) with lw_chunk set to the fastest measured chunk for a request of ncol
    columns on this device; measured once per cache key and remembered in cache_path.  max_chunk bounds the
    choice (and so the scratch a handle holds: 95 KB per column of a chunk).  timer(base, ncol) ->
    {chunk: ms} replaces the device measurement (tests)."""
    base = base or SolverConfig()
    if base.precision != "mixed" or base.parts == "sw":
        return base
    if device is None:
        import torch
        device = torch.cuda.get_device_name()
    k = key(device, base.nlay, base.route, ncol)
    cache = load_cache(cache_path)
    if k not in cache:
        times = (timer or time_candidates)(base, ncol)
        cache[k] = {"lw_chunk": choose(times), "ms": {str(c): t for c, t in times.items()}}
        save_cache(cache, cache_path)
    if max_chunk is not None:
        times = {int(c): t for c, t in cache[k]["ms"].items() if int(c) <= max_chunk}
        if times:
            return replace(base, lw_chunk=choose(times))
        return replace(base, lw_chunk=max_chunk)
    return replace(base, lw_chunk=int(cache[k]["lw_chunk"]))
