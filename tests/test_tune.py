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

    cache = tmp_path / "tune.json"
    c1 = tune.tuned_config(300000, cache_path=cache, timer=timer, device="gpu-x")
    c2 = tune.tuned_config(290000, cache_path=cache, timer=timer, device="gpu-x")   # same bucket
    assert c1.lw_chunk == c2.lw_chunk == 32768 and calls == [300000]
    tune.tuned_config(1000, cache_path=cache, timer=timer, device="gpu-x")          # new bucket
    assert len(calls) == 2
    assert tune.tuned_config(300000, cache_path=cache, timer=timer, device="gpu-x", max_chunk=16384).lw_chunk == 8192
    assert tune.tuned_config(300000, base=SolverConfig(precision="fp64"), cache_path=cache, timer=timer,
                             device="gpu-x").lw_chunk == 0                           # FP64: nothing to tune


@pytest.mark.gpu
def test_candidates_give_identical_bits(tmp_path):
    import torch
    from woof_nam_b200.columns import make_columns
    from woof_nam_b200.solver import RadSolver
    cfg = tune.tuned_config(20000, cache_path=tmp_path / "t.json")
    assert cfg.lw_chunk in tune.CANDIDATES
    cols = make_columns(9000, 31)
    outs = []
    for chunk in (4096, 32768, cfg.lw_chunk):
        s = RadSolver(lw_chunk=chunk)
        outs.append(s.solve(s.to_device(cols), cols.solcon))
    torch.cuda.synchronize()
    for o in outs[1:]:
        for k, v in outs[0].items():
            assert torch.equal(v, o[k]), k
