"""HostPipeline (double-buffered host->device copies, solves and device->host copies on three streams): five
host-resident requests through two buffer sets give, each in its own host outputs, the same bits as solving that
request alone, and the pipeline's streams order the buffer reuse (no request reads another's inputs)."""
from __future__ import annotations

import numpy as np
import pytest

from woof_nam_b200.columns import make_columns

pytestmark = pytest.mark.gpu


def test_pipelined_requests_equal_solve():
    import torch
    from woof_nam_b200.pipeline import HostPipeline
    from woof_nam_b200.solver import INPUT_FIELDS, RadSolver
    n = 6000
    s = RadSolver(precision="mixed")
    reqs = [make_columns(n, 700 + i) for i in range(5)]
    hins = [{k: torch.from_numpy(np.ascontiguousarray(getattr(c, k), dtype=np.float32)).pin_memory()
             for k in INPUT_FIELDS} for c in reqs]
    shapes = {k: v.shape for k, v in s.alloc_outputs(n).items()}
    houts = [{k: torch.empty(sh, dtype=torch.float32, pin_memory=True) for k, sh in shapes.items()} for _ in reqs]
    pipe = HostPipeline(s, n, depth=2)
    for c, hi, ho in zip(reqs, hins, houts):
        pipe.submit(hi, c.solcon, ho)
    pipe.synchronize()
    assert all(pipe.done(i) for i in range(len(reqs)))
    for c, ho in zip(reqs, houts):
        ref = s.solve_host(c)
        for k, v in ref.items():
            assert np.array_equal(ho[k].numpy(), v), k


def test_depth_must_overlap():
    from woof_nam_b200.pipeline import HostPipeline
    from woof_nam_b200.solver import RadSolver
    with pytest.raises(ValueError):
        HostPipeline(RadSolver(), 100, depth=1)
