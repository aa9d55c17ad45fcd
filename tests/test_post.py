"""The radiation call's post step (rrtm_post_outputs): the oracle against the reference kernel's golden
vectors, then the CUDA kernel through the C ABI against the oracle, bit for bit (copies, float adds and a
left-to-right product: no rounding freedom)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import ROOT
from oracle import post

GOLD = ROOT / "tests" / "golden" / "post_golden.npz"
LM = 60


def _golden():
    g = np.load(GOLD)
    inp = {k[3:]: g[k] for k in g.files if k.startswith("in_")}
    state = {k[6:]: g[k] for k in g.files if k.startswith("state_")}
    return g, inp, state


@pytest.mark.parametrize("tag,lw", [("lw", True), ("sw", False)])
def test_oracle_matches_reference_kernel(tag, lw):
    g, inp, state = _golden()
    r = post.post_outputs(inp, state, LM, lw_step=lw)
    for k, v in r.items():
        assert np.array_equal(v, g[f"{tag}_{k}"]), k
    dry = inp["cw"].max(axis=0) < post.EPSQ2
    assert dry.any() and (~dry).any()
    assert (r["cldfra"][:, dry] == 0).all() and (r["ncfrst"] == state["ncfrst"] + 1).all()


def test_oracle_known_answers():
    """Hand-set columns: a dry column loses its cloud, a cloudy CU column accumulates both counters."""
    inp, state = post.make_case(2, 3, 1)
    inp["cw"][:] = [[0.0, 1e-3], [5e-9, 0.0], [0.0, 0.0]]
    inp["cu_cloud"][:] = [1, 1]
    inp["cldsa"][3] = [0.5, 0.25]
    state["acfrst"][:] = 1.0
    state["acfrcv"][:] = 2.0
    inp["t"][2] = [300.0, 250.0]
    r = post.post_outputs(inp, state, 3)
    assert (r["cldfra"][:, 0] == 0).all() and (r["cldsa"][:, 0] == 0).all()
    assert r["acfrst"].tolist() == [1.0, 1.25] and r["acfrcv"].tolist() == [2.0, 2.25]
    t = np.float32(300.0)
    assert r["sigt4"][0] == (((np.float32(5.67051e-8) * t) * t) * t) * t


def _dev(d):
    import torch
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in d.items()}


def _run(s, inp, state, lm, kd, cloud_block, lw_step):
    import torch
    n = inp["coszen_v"].shape[-1]
    din = _dev(inp)
    out = {k: torch.zeros((lm, n), dtype=torch.float32, device="cuda") for k in post.OUT_3D}
    out.update({k: torch.zeros(n, dtype=torch.float32, device="cuda") for k in post.OUT_2D})
    out["ncfrst"] = torch.zeros(n, dtype=torch.int32, device="cuda")
    out["ncfrcv"] = torch.zeros(n, dtype=torch.int32, device="cuda")
    for k in post.ACCUM:
        out[k].copy_(torch.from_numpy(state[k]))
    s.post_outputs(din, out, lm, kd=kd, cloud_block=cloud_block, lw_step=lw_step)
    torch.cuda.synchronize()
    r = {k: v.cpu().numpy() for k, v in out.items()}
    r["cldcov"], r["cldsa"] = din["cldcov"].cpu().numpy(), din["cldsa"].cpu().numpy()
    return r


@pytest.mark.gpu
@pytest.mark.parametrize("tag,lw", [("lw", True), ("sw", False)])
def test_kernel_matches_golden(tag, lw):
    from woof_nam_b200.solver import RadSolver
    g, inp, state = _golden()
    r = _run(RadSolver(), inp, state, LM, 0, True, lw)
    for k, v in r.items():
        assert np.array_equal(v, g[f"{tag}_{k}"]), k


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 255, 4097, 70001])
def test_kernel_fused_from_solve_layout(n):
    """kd = 1: heating rates read from [LM + 1] arrays (the solve's htlw / htsw), ragged column counts."""
    from woof_nam_b200.solver import RadSolver
    inp, state = post.make_case(n, LM, 100 + n, kd=1)
    ref = post.post_outputs(inp, state, LM, kd=1)
    r = _run(RadSolver(), inp, state, LM, 1, True, True)
    for k, v in ref.items():
        assert np.array_equal(v, r[k]), k


@pytest.mark.gpu
def test_kernel_without_cloud_block():
    from woof_nam_b200.solver import RadSolver
    inp, state = post.make_case(1000, LM, 7)
    ref = post.post_outputs(inp, state, LM, cloud_block=False, lw_step=False)
    r = _run(RadSolver(), inp, state, LM, 0, False, False)
    for k in ("rlwtt", "rswtt", "rlwin", "rswin", "rswinc", "rswout", "rlwtoa", "rswtoa", "czmean", "coszdg",
              "sigt4", "acfrst", "ncfrst", "cldcov"):
        assert np.array_equal(ref[k], r[k]), k
