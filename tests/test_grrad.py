"""grrad's radiation-layer set-up of the model state in the oracle, pinned to the reference's kernels
(rrtm_grrad_setup + phys_rrtm_grrad_gases): the restatement reproduces the golden vectors bit for bit."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import oracle

GOLDEN = Path(__file__).resolve().parent / "golden" / "grrad_golden.npz"
MODEL = ("pint", "pmid", "prslk", "t", "q", "tsfc")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN)


@pytest.mark.parametrize("case", ["plain", "stress"])
def test_bit_exact(gold, case):
    r = oracle.grrad_setup({k: gold[f"{case}_in_{k}"] for k in MODEL})
    for k in oracle.GRRAD_FIELDS:
        assert np.array_equal(r[k], gold[f"{case}_{k}"]), k


@pytest.mark.parametrize("case", ["plain", "stress"])
def test_layout(gold, case):
    lm, n = gold[f"{case}_in_pmid"].shape
    assert gold[f"{case}_plvl"].shape == (lm + 2, n) and gold[f"{case}_plyr"].shape == (lm + 1, n)
    assert (gold[f"{case}_plvl"][0] == np.float32(1e-6)).all()                 # the extra top interface
    assert np.array_equal(gold[f"{case}_plyr"][0], np.float32(0.5) * gold[f"{case}_plvl"][1])
    assert (np.diff(gold[f"{case}_plvl"], axis=0) > 0).all()
    r = gold[f"{case}_rhly"]
    assert ((r >= 0) & (r <= 1)).all() and np.array_equal(gold[f"{case}_tsfg"], gold[f"{case}_in_tsfc"])
