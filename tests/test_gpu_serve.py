"""Serving: requests arriving over time on concurrent streams give the same bits as the same requests
solved alone, and the server's accounting (admission under the HBM budget, latency, columns/s) holds."""
from __future__ import annotations

import numpy as np
import pytest

from woof_nam_b200.serve import Request, poisson_requests

SIZES = {"a": 300, "b": 1000, "c": 4096}


def test_poisson_requests_shape():
    rs = poisson_requests(400, 40.0, 10, seed=1)
    t = np.array([r.arrival for r in rs])
    assert (np.diff(t) >= 0).all()
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert abs(gaps.mean() - 1 / 40.0) < 0.25 / 40.0
    assert {r.member for r in rs} <= set(range(10))
    assert len({r.domain for r in rs}) == 4


@pytest.mark.gpu
def test_serve_alone_equals_mix():
    import torch
    from woof_nam_b200.columns import SOLCON
    from woof_nam_b200.serve import RadServer, member_states
    from woof_nam_b200.solver import RadSolver
    states = member_states(3, sizes=SIZES)
    torch.cuda.synchronize()
    srv = RadServer(states, SOLCON, slots=3, keep_outputs=True)
    rng = np.random.default_rng(5)
    reqs = [Request(i, list(SIZES)[rng.integers(3)], int(rng.integers(3)), 0.002 * i) for i in range(12)]
    res = srv.run(reqs)
    assert res["requests"] == 12 and res["columns"] == sum(SIZES[r.domain] for r in reqs)
    assert res["p99_ms"] >= res["p50_ms"] > 0 and res["columns_per_s"] > 0
    assert srv.in_use == 0
    alone = RadSolver(precision="mixed")
    for r in reqs:
        assert r.done >= r.start >= r.arrival
        ref = alone.solve(states[r.domain][r.member], SOLCON)
        torch.cuda.synchronize()
        for k, v in ref.items():
            assert torch.equal(v, r.out[k]), (r.rid, k)
    # members differ: the perturbation reaches the outputs
    a = alone.solve(states["a"][0], SOLCON)["htlw"]
    b = alone.solve(states["a"][1], SOLCON)["htlw"]
    assert not torch.equal(a, b)


@pytest.mark.gpu
def test_serve_budget_admission():
    """A budget that holds the resident state and one request at a time serialises the requests."""
    import torch
    from woof_nam_b200.columns import SOLCON
    from woof_nam_b200.serve import RadServer, member_states
    states = member_states(1, sizes={"c": 4096})
    torch.cuda.synchronize()
    probe = RadServer(states, SOLCON, slots=1)
    one = probe.request_bytes(4096, probe.slots[0].solver)
    budget = (probe.resident + 3 * probe.held + one * 1.5) / 1e9     # three slots' scratch, 1.5 requests
    srv = RadServer(states, SOLCON, slots=3, hbm_budget_gb=budget)
    reqs = [Request(i, "c", 0, 0.0) for i in range(4)]
    srv.run(reqs)
    spans = sorted((r.start, r.done) for r in reqs)
    for (s0, d0), (s1, _) in zip(spans, spans[1:]):
        assert s1 >= d0 - 1e-3           # admitted only after the previous one completed
    with pytest.raises(MemoryError):
        RadServer(states, SOLCON, hbm_budget_gb=probe.resident / 2e9)
