"""Several GPUs, one process each: the window-aligned column split and the output all-gather, run as two
gloo ranks on the host with the oracle standing in for each rank's GPU solve.  The split request equals
the unsplit one to the bit; a split off the window boundaries does not (the SW group minima move)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from woof_nam_b200 import shard

W = 48          # columns per SW MINVAL(laytrop) window
NCOL = 250


def _columns():
    """Seeded columns with the pressure of every third column scaled by 0.8 (high terrain), so laytrop
    differs between neighbouring columns and the SW group minima depend on the grouping."""
    from woof_nam_b200.columns import make_columns
    c = make_columns(NCOL, 4242)
    c.plyr[:, ::3] *= np.float32(0.8)
    c.plvl[:, ::3] *= np.float32(0.8)
    return c


def test_plan_covers_aligned_and_balanced():
    for ncol, world, w in [(250, 2, 48), (1000, 3, 64), (5, 4, 2), (796590, 8, 30528), (0, 2, 16), (17, 8, 100)]:
        r = shard.plan(ncol, world, w)
        assert len(r) == world
        assert r[0][0] == 0 and r[-1][1] == ncol
        assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
        assert shard.window_aligned(r, w)
        nwin = -(-ncol // w)
        counts = [-(-(c1 - c0) // w) if c1 > c0 else 0 for c0, c1 in r]
        assert max(counts) - min(counts) <= 1 or nwin < world
    assert shard.plan(100, 3, 0) == [(0, 100), (100, 100), (100, 100)]
    with pytest.raises(ValueError):
        shard.plan(10, 0, 4)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path, split_at):
    import torch
    import torch.distributed as dist
    from oracle import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        cols = _columns()

        def solve_fn(c):
            r = oracle.solve(c, precision="double", window_cols=W)
            return {k: torch.from_numpy(v) for k, v in r.items()}

        if split_at is None:
            full = shard.shard_solve(cols, solve_fn, W, rank, world)
        else:                                   # a split off the window grid, for the negative check
            ranges = [(0, split_at), (split_at, NCOL)]
            c0, c1 = ranges[rank]
            full = shard.gather(solve_fn(cols.slice(c0, c1)), ranges)
        if rank == 0:
            np.savez(out_path, **{k: v.numpy() for k, v in full.items()})
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run(tmp_path, split_at=None):
    import torch.multiprocessing as mp
    out = tmp_path / f"r{split_at}.npz"
    mp.start_processes(_rank_main, args=(2, _free_port(), str(out), split_at), nprocs=2, join=True,
                       start_method="spawn")
    return dict(np.load(out))


def test_two_gloo_ranks_equal_single(tmp_path):
    from oracle import oracle
    got = _run(tmp_path)
    ref = oracle.solve(_columns(), precision="double", window_cols=W)
    for k, v in ref.items():
        assert np.array_equal(v, got[k]), k


def test_split_off_window_grid_differs(tmp_path):
    """The alignment rule is load-bearing: splitting mid-window regroups the SW minima (bands 19/23/25/28)."""
    from oracle import oracle
    cols = _columns()
    lt = (np.log(cols.plyr) > 4.56).sum(axis=0)[cols.coszen >= np.float32(1e-4)]
    assert len(np.unique(lt)) > 1
    ref = oracle.solve(cols, precision="double", window_cols=W)
    got = _run(tmp_path, split_at=W + W // 2 + 3)
    assert np.array_equal(ref["htlw"], got["htlw"])          # LW has no cross-column coupling
    assert not np.array_equal(ref["htsw"], got["htsw"])
