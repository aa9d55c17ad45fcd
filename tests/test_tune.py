"""The launch-shape autotuner: cache keys, the choice rule, measure-once-then-remember, and (GPU) that every
candidate chunk size gives the same bits."""
from __future__ import annotations

import pytest

from woof_nam_b200 import tune
from woof_nam_b200.solver import SolverConfig


def test_bucket_and_key():
    assert tune.bucket(1) == 1024 and tune.bucket(1024) == 1024 and tune.bucket(1025) == 2048
    assert tune.bucket(796590) == 1048576
    assert tune.key("B200", 61, "nam", 796590) == "B200|nlay=61|route=nam|cols<=1048576"


def test_choose_prefers_fastest_then_larger():
    assert tune.choose({4096: 3.0, 32768: 2.0, 65536: 2.5}) == 32768
    assert tune.choose({16384: 2.0, 32768: 2.0}) == 32768


def test_measures_once_then_remembers(tmp_path):
    calls = []

    def timer(base, ncol):
        calls.append(ncol)
        return {8192: 5.0, 32768: 4.0, 65536: 4.5}

    sw_calls = []

    def sw_timer(base, ncol):
        sw_calls.append(ncol)
        return {8192: 3.0, 16384: 2.5, 65536: 2.6}

    cache = tmp_path / "tune.json"
    kw = dict(cache_path=cache, timer=timer, sw_timer=sw_timer, device="gpu-x")
    c1 = tune.tuned_config(300000, **kw)
    c2 = tune.tuned_config(290000, **kw)                                            # same bucket
    assert c1.lw_chunk == c2.lw_chunk == 32768 and calls == [300000]
    assert c1.sw_sweep_chunk == c2.sw_sweep_chunk == 16384 and sw_calls == [300000]
    tune.tuned_config(1000, **kw)                                                    # new bucket
    assert len(calls) == 2 and len(sw_calls) == 2
    assert tune.tuned_config(300000, max_chunk=16384, **kw).lw_chunk == 8192
    assert tune.tuned_config(300000, max_sw_chunk=12000, **kw).sw_sweep_chunk == 8192
    assert tune.tuned_config(300000, base=SolverConfig(precision="fp64"), **kw).lw_chunk == 0   # FP64: nothing to tune
    # a tile set by the caller is kept; an LW-only or SW-only solver tunes only its part
    assert tune.tuned_config(300000, base=SolverConfig(sw_sweep_chunk=4096), **kw).sw_sweep_chunk == 4096
    assert tune.tuned_config(300000, base=SolverConfig(parts="sw"), **kw).lw_chunk == SolverConfig().lw_chunk
    assert tune.tuned_config(300000, base=SolverConfig(parts="lw"), **kw).sw_sweep_chunk == 0
    assert len(calls) == 2 and len(sw_calls) == 2


def test_old_cache_entries_gain_the_sw_tile(tmp_path):
    import json
    cache = tmp_path / "tune.json"
    cache.write_text(json.dumps({tune.key("gpu-x", 61, "nam", 5000): {"lw_chunk": 65536, "ms": {"65536": 1.0}}}))
    c = tune.tuned_config(5000, cache_path=cache, timer=lambda b, n: 1 / 0, sw_timer=lambda b, n: {32768: 1.0},
                          device="gpu-x")
    assert c.lw_chunk == 65536 and c.sw_sweep_chunk == 32768


@pytest.mark.gpu
def test_candidates_give_identical_bits(tmp_path):
    import torch
    from woof_nam_b200.columns import make_columns
    from woof_nam_b200.solver import RadSolver
    cfg = tune.tuned_config(20000, cache_path=tmp_path / "t.json")
    assert cfg.lw_chunk in tune.CANDIDATES and cfg.sw_sweep_chunk in tune.SW_CANDIDATES
    cols = make_columns(9000, 31)
    outs = []
    for chunk, swc in ((4096, 8192), (32768, 0), (cfg.lw_chunk, cfg.sw_sweep_chunk), (8192, 1000)):
        s = RadSolver(lw_chunk=chunk, sw_sweep_chunk=swc)
        outs.append(s.solve(s.to_device(cols), cols.solcon))
    torch.cuda.synchronize()
    for o in outs[1:]:
        for k, v in outs[0].items():
            assert torch.equal(v, o[k]), k
