"""Launch-shape autotuner: times the column tiles of the LW and the SW on this device and remembers the
fastest per (device, layers, route, column-count bucket).

* lw_chunk: the column tile of the LW gas-optics / sweep kernel pair -- how many columns share one scratch
  pass (95 KB per column) before the sweeps read it back.
* sw_sweep_chunk: the tile of sunlit columns of the SW's three kernels (gas optics into the image, layer R/T
  into the blocks, adding sweeps; ~330 KB per column).

Small tiles keep more of the scratch in L2 but launch more often and leave the GPU idle at each tile's tail;
large tiles do the opposite and hold more HBM.  Every candidate gives the same bits (each column's arithmetic
is independent of the tiling; tests/test_tune.py checks it on the device), so the tuner changes speed only.
The split of g-points over lanes is fixed by the kernels (five per lane in the LW sweeps, one per thread of
the SW's R/T and sweeps) and is not a runtime choice.

    from woof_nam_b200.tune import tuned_config
    cfg = tuned_config(ncol=796590)          # SolverConfig with the fastest lw_chunk / sw_sweep_chunk here
"""
from __future__ import annotations

import json
import os
from dataclasses import replace
from pathlib import Path

from .solver import SolverConfig

CANDIDATES = (4096, 8192, 16384, 32768, 65536, 131072)
SW_CANDIDATES = (8192, 16384, 32768, 65536)
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


def time_candidates_sw(base: SolverConfig, ncol: int, candidates=SW_CANDIDATES, reps: int = 2,
                       seed: int = 2002) -> dict:
    """Device time (ms) of the SW of one solve of min(ncol, 262144) synthetic columns per candidate tile of
    sunlit columns, CUDA events on the current stream, after one warm-up solve."""
    import torch
    from .columns import make_columns
    from .solver import RadSolver
    n = min(ncol, 262144)
    cols = make_columns(n, seed)
    nday = int((cols.coszen >= 1e-4).sum())
    times = {}
    dev = None
    for c in candidates:
        if c > 2 * nday and c != candidates[0]:
            continue
        s = RadSolver(replace(base, sw_sweep_chunk=c, parts="sw"))
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


def _bounded(ms: dict, bound: int | None):
    times = {int(c): t for c, t in ms.items() if bound is None or int(c) <= bound}
    return choose(times) if times else bound


def tuned_config(ncol: int, base: SolverConfig | None = None, cache_path: Path = CACHE, timer=None,
                 device: str | None = None, max_chunk: int | None = None, sw_timer=None,
                 max_sw_chunk: int | None = None) -> SolverConfig:
    """base (default SolverConfig()) with lw_chunk and sw_sweep_chunk set to the fastest measured tiles for a
    request of ncol columns on this device; measured once per cache key and remembered in cache_path.  The SW
    tile is tuned only where base leaves it at its default (sw_sweep_chunk 0).  max_chunk / max_sw_chunk bound
    the choices (and so the scratch a handle holds).  timer(base, ncol) / sw_timer(base, ncol) -> {tile: ms}
    replace the device measurements (tests)."""
    base = base or SolverConfig()
    if base.precision != "mixed":
        return base
    tune_lw = base.parts != "sw"
    tune_sw = base.parts != "lw" and base.sw_sweep_chunk == 0
    if not (tune_lw or tune_sw):
        return base
    if device is None:
        import torch
        device = torch.cuda.get_device_name()
    k = key(device, base.nlay, base.route, ncol)
    cache = load_cache(cache_path)
    entry = cache.get(k, {})
    changed = False
    if tune_lw and "ms" not in entry:
        times = (timer or time_candidates)(base, ncol)
        entry.update(lw_chunk=choose(times), ms={str(c): t for c, t in times.items()})
        changed = True
    if tune_sw and "ms_sw" not in entry:
        times = (sw_timer or time_candidates_sw)(base, ncol)
        entry.update(sw_sweep_chunk=choose(times), ms_sw={str(c): t for c, t in times.items()})
        changed = True
    if changed:
        cache[k] = entry
        save_cache(cache, cache_path)
    cfg = base
    if tune_lw:
        cfg = replace(cfg, lw_chunk=int(_bounded(entry["ms"], max_chunk) if max_chunk is not None
                                        else entry["lw_chunk"]))
    if tune_sw:
        cfg = replace(cfg, sw_sweep_chunk=int(_bounded(entry["ms_sw"], max_sw_chunk) if max_sw_chunk is not None
                                              else entry["sw_sweep_chunk"]))
    return cfg
