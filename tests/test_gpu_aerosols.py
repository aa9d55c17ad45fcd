"""The aerosol optics on the GPU (rad_load_aerosols + rad_setaer through the C-ABI) against the oracle: the
golden requests of the reference's kernels and 8,192-column requests over the NAM domain and the globe, and
a radiation solve fed with the GPU's aerosol optics against the float64 oracle solve fed with the oracle's.

The kernel contracts multiply-adds and takes CUDA's expf / logf, so values agree to float rounding, not to
the bit: relative 1e-4, set by the reference's own formula for a layer's effective thickness near the
surface, h (exp(-z_top / h) - exp(-z_bottom / h)), whose float cancellation turns the exponentials' last-bit
differences into ~3e-5.  The reference's smoothing of optical depth at domain boundaries is a threshold on
the ratio of adjacent layers (30 and 1 / 30): where that ratio lies within rounding of a threshold the two
sides may choose differently, moving 20 % of the pair's optical depth between its two layers.  Such pairs
are accepted when the pair's sum agrees and they are rare (at most 1 in 10^5 values).

The volcanic term (rad_setaer_volc) is built with IEEE arithmetic and its spectral factors come from the
host's powf, so it matches the oracle bit for bit: on the golden cases of phys_rrtm_setaer_volc and on 8,192
columns over the globe in both level orders."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import assert_within
from oracle import oracle
from woof_nam_b200 import aerosols
from woof_nam_b200.columns import make_columns

pytestmark = pytest.mark.gpu
RTOL = 1.0e-4


def _gpu(month, cols, ai, solver=None):
    import torch
    from woof_nam_b200.solver import RadSolver
    s = solver or RadSolver()
    aer = aerosols.Aerosols(s, month)
    dev = s.to_device(cols)
    t = {k: torch.as_tensor(np.ascontiguousarray(v), device="cuda") for k, v in ai.items()}
    fsw, flw = aer.optics(dev, t["rhly"], t["xlon"], t["xlat"], t["slmsk"])
    torch.cuda.synchronize()
    return s, dev, fsw, flw


def _rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1.0e-6)


def _close(got, ref, what):
    """[3][band][nlay][ncol]: albedo and asymmetry within RTOL; optical depth within RTOL except smoothing
    pairs decided differently at a threshold (adjacent layers, pair sums within RTOL, rare)."""
    got = got.detach().cpu().numpy() if hasattr(got, "detach") else got
    assert got.shape == ref.shape, what
    assert np.isfinite(got).all(), what
    g, r = got.astype(np.float64), ref.astype(np.float64)
    for f in (1, 2):
        e = _rel(g[f], r[f])
        assert e.max() <= RTOL, f"{what} field {f}: relative error {e.max():.3e} at {np.unravel_index(e.argmax(), e.shape)}"
    bad = _rel(g[0], r[0]) > RTOL
    nb, nl, nc = np.nonzero(bad)
    for b, k, c in zip(nb, nl, nc):
        pair = [k - 1, k] if k > 0 and bad[b, k - 1, c] else [k, k + 1]
        assert pair[0] >= 0 and pair[1] < g.shape[2] and bad[b, pair[1], c] and bad[b, pair[0], c], \
            f"{what}: optical depth off at band {b} layer {k} column {c} outside a smoothing pair"
        sg, sr = g[0, b, pair, c].sum(), r[0, b, pair, c].sum()
        assert abs(sg - sr) <= RTOL * max(abs(sr), 1.0e-6), f"{what}: smoothing pair sum differs at {b, k, c}"
    assert bad.sum() <= max(2, 1.0e-5 * bad.size), f"{what}: {bad.sum()} optical depths differ"


@pytest.mark.parametrize("case", ["jan_nam", "jul_globe"])
def test_golden(case):
    from test_aerosols import golden_request
    z = np.load(Path(__file__).resolve().parent / "golden" / "aer_golden.npz")
    month, cols, ai = golden_request(z, case)
    _, _, fsw, flw = _gpu(month, cols, ai)
    _close(fsw, z[f"{case}_faersw"], f"{case} faersw")
    _close(flw, z[f"{case}_faerlw"], f"{case} faerlw")


@pytest.mark.parametrize("month,region", [(4, "nam"), (10, "globe")])
def test_against_oracle(month, region):
    cols = make_columns(8192, 40 + month)
    ai = aerosols.make_inputs(cols, month, region)
    ref = oracle.aerosols(aerosols.climatology(month), cols, ai)
    _, _, fsw, flw = _gpu(month, cols, ai)
    _close(fsw, ref["faersw"], f"{region} faersw")
    _close(flw, ref["faerlw"], f"{region} faerlw")


def test_month_reload_and_repeat():
    """A second month on the same handle replaces the tables; two calls in a row give the same bits."""
    import torch
    cols = make_columns(1024, 77)
    ai = aerosols.make_inputs(cols, 3, "globe")
    s, dev, a1, b1 = _gpu(1, cols, ai)
    aer = aerosols.Aerosols(s, 8)
    t = {k: torch.as_tensor(np.ascontiguousarray(v), device="cuda") for k, v in ai.items()}
    a8, b8 = aer.optics(dev, t["rhly"], t["xlon"], t["xlat"], t["slmsk"])
    a8b, b8b = aer.optics(dev, t["rhly"], t["xlon"], t["xlat"], t["slmsk"])
    torch.cuda.synchronize()
    assert torch.equal(a8, a8b) and torch.equal(b8, b8b)
    ref8 = oracle.aerosols(aerosols.climatology(8), cols, ai)
    _close(a8, ref8["faersw"], "august faersw")
    assert not torch.equal(a1, a8)


def test_solve_with_aerosols():
    """The radiation with the GPU's aerosol optics against the float64 oracle with the oracle's optics."""
    cols = make_columns(2048, 91)
    ai = aerosols.make_inputs(cols, 2, "nam")
    ref_aer = oracle.aerosols(aerosols.climatology(6), cols, ai)
    ref = oracle.solve(cols, precision="double", faerlw=ref_aer["faerlw"], faersw=ref_aer["faersw"])
    s, dev, fsw, flw = _gpu(6, cols, ai)
    dev["faersw"], dev["faerlw"] = fsw, flw
    out = s.solve(dev, cols.solcon)
    host = {k: v.cpu().numpy().astype(np.float64) for k, v in out.items()}
    assert_within(host, ref, what="mixed solve with aerosols")
    plain = oracle.solve(cols, precision="double")
    assert np.abs(plain["sfcfsw"] - ref["sfcfsw"]).max() > 1.0    # the aerosols matter at the surface


VOLC_CASES = {"top_first": (0, 0, 2026, 7), "surface_first": (1, 0, 1991, 6), "one_lw_band": (0, 1, 7, 12)}


@pytest.mark.parametrize("case", list(VOLC_CASES))
def test_volcanic_golden(case):
    import torch
    from woof_nam_b200.solver import RadSolver
    z = np.load(Path(__file__).resolve().parent / "golden" / "aer_golden.npz")
    ivflip, lw1bd, kyrsav, kmonsav = VOLC_CASES[case]
    pl = z["jul_globe_in_plvl"]
    pl = pl if ivflip == 0 else np.ascontiguousarray(pl[::-1])
    s = RadSolver(nlay=pl.shape[0] - 1)
    cu = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    faer = (cu(z["jul_globe_faersw"]), cu(z["jul_globe_faerlw"]))
    aerosols.volcanic(s, cu(pl), cu(z["volc_in_xlat"]), z["volc_in_ivolae"], kyrsav, kmonsav, faer, ivflip=ivflip,
                      lw1bd=bool(lw1bd))
    torch.cuda.synchronize()
    assert s.device_error() == 0
    assert np.array_equal(faer[0][0].cpu().numpy(), z[f"volc_{case}_extsw"])
    assert np.array_equal(faer[1][0].cpu().numpy(), z[f"volc_{case}_extlw"])
    assert np.array_equal(faer[0][1:].cpu().numpy(), z["jul_globe_faersw"][1:])


@pytest.mark.parametrize("ivflip", [0, 1])
def test_volcanic_against_oracle(ivflip):
    import torch
    cols = make_columns(8192, 97)
    ai = aerosols.make_inputs(cols, 98, "globe")
    s, dev, fsw, flw = _gpu(4, cols, ai)
    iv = np.random.default_rng(5).integers(0, 800, (10, 4, 12)).astype(np.int32)
    sw0, lw0 = fsw.cpu().numpy(), flw.cpu().numpy()
    pl = cols.plvl if ivflip == 0 else np.ascontiguousarray(cols.plvl[::-1])
    ref = oracle.setaer_volc(pl, ai["xlat"], iv, 2031, 4, sw0, lw0, ivflip=ivflip)
    aerosols.volcanic(s, torch.as_tensor(np.ascontiguousarray(pl), device="cuda"),
                      torch.as_tensor(ai["xlat"], device="cuda"), iv, 2031, 4, (fsw, flw), ivflip=ivflip)
    torch.cuda.synchronize()
    assert np.array_equal(fsw.cpu().numpy(), ref["faersw"])
    assert np.array_equal(flw.cpu().numpy(), ref["faerlw"])
    with pytest.raises(Exception, match="kmonsav"):
        aerosols.volcanic(s, dev["plvl"], torch.as_tensor(ai["xlat"], device="cuda"), iv, 2031, 13, (fsw, flw))


def test_shapes_checked_before_launch():
    """Inputs or outputs whose shapes disagree with the solver's layer count are refused on the host (the kernels
    index by the handle's nlay)."""
    import torch
    from woof_nam_b200.solver import RadSolver
    cols = make_columns(64, 11)
    ai = aerosols.make_inputs(cols, 12, "nam")
    s = RadSolver()
    dev = s.to_device(cols)
    t = {k: torch.as_tensor(np.ascontiguousarray(v), device="cuda") for k, v in ai.items()}
    aer = aerosols.Aerosols(s, 3)
    with pytest.raises(ValueError):
        aer.optics(dev, t["rhly"][:-1].contiguous(), t["xlon"], t["xlat"], t["slmsk"])
    with pytest.raises(ValueError):
        aer.optics(dev, t["rhly"], t["xlon"], t["xlat"], t["slmsk"],
                   out=(torch.empty((3, 14, cols.nlay - 1, 64), device="cuda"),
                        torch.empty((3, 16, cols.nlay - 1, 64), device="cuda")))
    fsw, flw = aer.optics(dev, t["rhly"], t["xlon"], t["xlat"], t["slmsk"])
    iv = np.zeros((10, 4, 12), np.int32)
    with pytest.raises(ValueError):
        aerosols.volcanic(s, dev["plvl"][1:].contiguous(), t["xlat"], iv, 1, 1, (fsw, flw))
    with pytest.raises(ValueError):
        aerosols.volcanic(RadSolver(nlay=40), dev["plvl"], t["xlat"], iv, 1, 1, (fsw, flw))
    torch.cuda.synchronize()


def test_surface_first():
    """ivflip 1: a surface-first request (the golden "jul_globe" request with its layers reversed) against the
    reference's own ivflip = 1 output, and bit for bit the top-first optics reversed."""
    import torch
    from test_aerosols import golden_request
    z = np.load(Path(__file__).resolve().parent / "golden" / "aer_golden.npz")
    month, cols, ai = golden_request(z, "jul_globe")
    s, dev, fsw, flw = _gpu(month, cols, ai)
    aer = aerosols.Aerosols(s, month)
    rev = {k: torch.flip(dev[k], dims=[0]).contiguous() for k in ("plvl", "plyr", "tlyr", "qlyr")}
    t = {k: torch.as_tensor(np.ascontiguousarray(v), device="cuda") for k, v in ai.items()}
    gsw, glw = aer.optics(rev, torch.flip(t["rhly"], dims=[0]).contiguous(), t["xlon"], t["xlat"], t["slmsk"],
                          ivflip=1)
    torch.cuda.synchronize()
    _close(gsw, z["flip_faersw"], "surface-first faersw")
    _close(glw, z["flip_faerlw"], "surface-first faerlw")
    assert torch.equal(gsw, torch.flip(fsw, dims=[2])) and torch.equal(glw, torch.flip(flw, dims=[2]))
