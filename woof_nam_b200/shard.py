"""Column radiation over several GPUs of one node: one process per GPU, no collective in the compute.

Columns are independent except through the SW MINVAL(laytrop) groups (8 consecutive day columns for
taumol19/23, the window for taumol25/28; namgpu/kernels/phys_rrtm_sw_taumol19.cu:33-42,
rrtm_sw_kmin_windows.cu:1-28), which are defined per window of ``window_cols`` columns (the reference's
row windows, namgpu/physics/rrtm/rrtm_call.py:108-134).  So one request splits across ranks into
contiguous, window-aligned column ranges: each rank solves its range as a request of its own with the
same windows, and the results equal the single-GPU solve to the bit.  A request solved as one window
(window_cols = 0) does not split; it runs whole on one rank (serving places whole requests per GPU).

After the solves, ``gather`` assembles the outputs on every rank with one all-gather per output
(torch.distributed: NCCL over NVLink on the GPUs, gloo on the host); ranks that only need their own
columns skip it.
"""
from __future__ import annotations

import numpy as np


def plan(ncol: int, world: int, window_cols: int) -> list:
    """[(c0, c1)] per rank: contiguous column ranges, each starting on a window boundary, windows split as
    evenly as whole windows allow.  window_cols = 0 (one window) puts every column on rank 0."""
    if world < 1 or ncol < 0:
        raise ValueError("world must be >= 1 and ncol >= 0")
    if window_cols <= 0:
        return [(0, ncol)] + [(ncol, ncol)] * (world - 1)
    nwin = (ncol + window_cols - 1) // window_cols
    base, extra = divmod(nwin, world)
    out, w = [], 0
    for r in range(world):
        w1 = w + base + (1 if r < extra else 0)
        out.append((min(w * window_cols, ncol), min(w1 * window_cols, ncol)))
        w = w1
    return out


def local_range(ncol: int, window_cols: int, rank: int, world: int) -> tuple:
    return plan(ncol, world, window_cols)[rank]


def gather(local: dict, ranges: list, group=None) -> dict:
    """All-gather each output array ([..., ncol_local], column last) from every rank into the full
    request ([..., ncol]) on every rank.  Arrays are torch tensors on the backend's device."""
    import torch
    import torch.distributed as dist
    width = max(c1 - c0 for c0, c1 in ranges)
    out = {}
    for k in sorted(local):
        t = local[k]
        pad = torch.zeros(*t.shape[:-1], width, dtype=t.dtype, device=t.device)
        pad[..., :t.shape[-1]] = t
        parts = [torch.empty_like(pad) for _ in ranges]
        dist.all_gather(parts, pad, group=group)
        out[k] = torch.cat([p[..., :c1 - c0] for p, (c0, c1) in zip(parts, ranges)], dim=-1)
    return out


def shard_solve(columns, solve_fn, window_cols: int, rank: int, world: int, group=None,
                gather_outputs: bool = True) -> dict:
    """Solve this rank's window-aligned share of a request with solve_fn(columns_slice) -> {name: tensor}
    and, with gather_outputs, assemble the whole request's outputs on every rank."""
    ranges = plan(columns.ncol, world, window_cols)
    c0, c1 = ranges[rank]
    local = solve_fn(columns.slice(c0, c1))
    if not gather_outputs:
        return local
    return gather(local, ranges, group=group)


def gpu_solver_fn(solver, device=None):
    """solve_fn for shard_solve on this rank's GPU through the library (host columns in, device outputs)."""
    import torch

    def fn(cols):
        if cols.ncol == 0:
            nlay = solver.cfg.nlay
            from .solver import output_shapes
            return {k: torch.zeros(s, dtype=torch.float32, device=device or "cuda")
                    for k, s in output_shapes(nlay, 0, solver.cfg.route).items()}
        d = solver.to_device(cols, device=device or "cuda")
        return solver.solve(d, cols.solcon)
    return fn


def window_aligned(ranges: list, window_cols: int) -> bool:
    return all(c0 % window_cols == 0 for c0, c1 in ranges if c1 > c0) if window_cols > 0 else True


def balance(ranges: list) -> float:
    """Largest share over the mean share (1.0 = perfectly even)."""
    sizes = np.array([c1 - c0 for c0, c1 in ranges], dtype=np.float64)
    return float(sizes.max() / max(sizes.mean(), 1e-30))
