"""coszmn on the GPU (rad_coszmn through the C-ABI) against the golden vectors of the reference's kernel and
against the oracle on 100,000 columns.  CUDA's cosf / sinf differ from the host's in the last bit, so the
means agree to 2e-6."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from woof_nam_b200 import solar

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden" / "solar_golden.npz"


def _gpu(sun, lon, lat, solhr, dtswav, nrads=48):
    import torch
    from woof_nam_b200.solver import RadSolver
    s = RadSolver()
    a, b = solar.coszmn(s, sun, torch.as_tensor(lon, device="cuda"), torch.as_tensor(lat, device="cuda"), solhr,
                        dtswav, nrads)
    torch.cuda.synchronize()
    return a.cpu().numpy(), b.cpu().numpy()


def test_golden():
    z = np.load(GOLDEN)
    for i in range(z["date"].shape[0]):
        sun = solar.sol_update(z["date"][i], float(z["deltsw"][i]), float(z["deltim"][i]))
        cz, cd = _gpu(sun, z["glon"][i], z["glat"][i], float(z["solhr"][i]), float(z["dtswav"][i]))
        assert np.abs(cz - z["coszen"][i]).max() < 2e-6 and np.abs(cd - z["coszdg"][i]).max() < 2e-6, i


def test_against_oracle_large():
    rng = np.random.default_rng(5)
    n = 100_000
    lon = rng.uniform(-np.pi, np.pi, n).astype(np.float32)
    lat = rng.uniform(-1.5, 1.5, n).astype(np.float32)
    date, dsw = (2026, 12, 3, 18, 30, 0), 1200.0
    ref = oracle.solar(date, dsw, 25.0, 1366.0, lon, lat, 18.5, dsw / 3600.0, 48)
    sun = solar.sol_update(date, dsw, 25.0)
    cz, cd = _gpu(sun, lon, lat, 18.5, dsw / 3600.0)
    assert np.abs(cz - ref["coszen"]).max() < 2e-6 and np.abs(cd - ref["coszdg"]).max() < 2e-6
    day = ref["coszen"] >= 1e-4
    assert 0.3 < day.mean() < 0.7 and (np.asarray(cz >= 1e-4) != day).sum() <= 2   # the SW day predicate
