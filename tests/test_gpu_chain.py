"""A whole domain's radiation call on the GPU without row windows (chain.radiation_call: grrad's set-up, DAYPARTS,
getozn, getgases, progcld2, setalb, setemis, then the LW and SW solve, one stream) against the same chain in
the oracle -- the restatement's front end feeding the float64 solve -- within the mixed-precision tolerances
(0.05 W/m^2, 0.01 K/day).  A second call on the work tensors of the first gives the same bits, and so does
a CUDA graph of the whole call.  With the climatological aerosol optics in the call (setaer, January) the same
holds against the oracle's chain with its aerosol restatement."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import assert_within
from oracle import oracle
from woof_nam_b200.columns import Columns, cloud_state, front_tables, make_columns, model_state, surface_state

pytestmark = pytest.mark.gpu
IM, JM = 128, 48
CALL = dict(solhr=14.5, dtswav=1200.0 / 3600.0, nrads=48, kmonsav=7, k1oz=6, k2oz=7, facoz=0.4, ico2flg=2,
            ialbflg=1, iemslw=1)


def _domain(seed=31):
    n = IM * JM
    cols = make_columns(n, seed)
    model = model_state(cols)
    lay = oracle.grrad_setup(model)
    cld = cloud_state(lay, seed + 1)
    sfc = surface_state(n, seed + 2)
    lon = np.linspace(-2.4, -0.9, IM, dtype=np.float32)[None, :].repeat(JM, 0).ravel()
    lat = np.linspace(0.2, 1.1, JM, dtype=np.float32)[:, None].repeat(IM, 1).ravel()
    sfc.update(glon=lon, glat=lat, sinlat=np.sin(lat).astype(np.float32), coslat=np.cos(lat).astype(np.float32))
    state = dict(model)
    state.update({k: cld[k] for k in ("clw", "f_ice", "f_rain", "r_rime", "cldfk1")})
    state.update(sfc)
    return state, front_tables(seed + 3), lay


def _sun():
    from woof_nam_b200 import solar
    return solar.sol_update((2026, 7, 1, 14, 30, 0), deltsw=1200.0, deltim=25.0)


def _oracle_chain(state, tab, lay, sun, month=None, ntcw=None):
    n = IM * JM
    dp = oracle.dayparts(state["glon"], state["sinlat"], state["coslat"], IM, CALL["solhr"], CALL["dtswav"],
                         CALL["nrads"], [sun["sollag"], sun["sindec"], sun["cosdec"]])
    olyr = oracle.getozn(lay["prslk1"], state["glat"], tab["o3r"], tab["pkstr"], CALL["k1oz"], CALL["k2oz"],
                         CALL["facoz"], tab["blte"], tab["dlte"], 0, init=np.zeros_like(lay["prslk1"]))
    gas = oracle.getgases(lay["plvl"], state["glon"], state["glat"], tab["co2_glb"], tab["gco2cyc"],
                          tab["co2vmr_sav"], CALL["ico2flg"], CALL["kmonsav"], 0)
    cin = {k: lay[k] for k in ("plyr", "plvl", "tlyr", "tvly", "qlyr", "qstl", "rhly")}
    cin.update({k: state[k] for k in ("clw", "f_ice", "f_rain", "r_rime", "cldfk1")}, xlat=state["glat"])
    if ntcw is not None:
        cin["clw"] = oracle.grrad_clw(state["tracer1"], ntcw, 1)
    cld = oracle.progcld2(cin, dict(ivflip=0, llyr=2, iovr=1, lcrick=0, lcnorm=0, lnoprec=0, lsashal=0,
                                    cld_fraction=0))
    sfc = dict(state, coszf=dp["coszen"])
    if CALL["ialbflg"] == 2 and "sfcalbedo" in state:
        from woof_nam_b200 import front
        pa = oracle.payne_albedo(state["sfcalbedo"], state["sm"], dp["coszen"], front.payne_tables())
        sfc.update({k: pa[k] for k in ("alvsf", "alnsf", "alvwf", "alnwf", "facsf", "facwf")})
    alb = oracle.setalb(sfc, CALL["ialbflg"])
    ems = oracle.setemis(state, tab["idxems"], CALL["ialbflg"], CALL["iemslw"])
    cols = Columns(plyr=lay["plyr"], plvl=lay["plvl"], tlyr=lay["tlyr"], tlvl=lay["tlvl"], qlyr=lay["qlyr"],
                   olyr=olyr, gasvmr=gas, clouds=cld["clouds"], sfcemis=ems, tsfg=lay["tsfg"], sfcalb=alb,
                   coszen=dp["coszen"], solcon=float(sun["solcon"]))
    assert 0 < (dp["coszen"] >= 1e-4).sum() < n          # day and night in the domain
    if month is None:
        return oracle.solve(cols, precision="double")
    aer = oracle.aerosols(oracle.aer_climatology(month), cols,
                          {"rhly": lay["rhly"], "xlon": state["glon"], "xlat": state["glat"], "slmsk": state["slmsk"]})
    return oracle.solve(cols, precision="double", faersw=aer["faersw"], faerlw=aer["faerlw"])


def _dev(state, tab):
    import torch
    d = {k: torch.as_tensor(np.ascontiguousarray(v), device="cuda") for k, v in state.items()}
    c = {k: (torch.as_tensor(np.ascontiguousarray(v), device="cuda") if isinstance(v, np.ndarray) else v)
         for k, v in tab.items()}
    c["co2_glb"] = torch.as_tensor(np.atleast_1d(np.float32(tab["co2_glb"])), device="cuda")
    return d, c


def test_chain_against_oracle_and_graph():
    import torch
    from woof_nam_b200.chain import radiation_call
    from woof_nam_b200.solver import RadSolver
    state, tab, lay = _domain()
    sun = _sun()
    s = RadSolver(precision="mixed", nlay=lay["plyr"].shape[0])
    d, c = _dev(state, tab)
    out = radiation_call(s, d, c, sun=sun, im=IM, **CALL)
    torch.cuda.synchronize()
    first = {k: v.cpu().numpy() for k, v in out.items() if k != "work"}
    ref = _oracle_chain(state, tab, lay, sun)
    assert_within(first, {k: ref[k] for k in first}, what="radiation call of the whole domain")
    # again on the same work tensors, and captured in one CUDA graph
    work = out["work"]
    outs = {k: v for k, v in out.items() if k != "work"}
    again = radiation_call(s, d, c, sun=sun, im=IM, work=work, out=outs, **CALL)
    torch.cuda.synchronize()
    for k in first:
        assert np.array_equal(again[k].cpu().numpy(), first[k]), k
    for v in outs.values():
        v.zero_()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        radiation_call(s, d, c, sun=sun, im=IM, work=work, out=outs, **CALL)
    g.replay()
    torch.cuda.synchronize()
    for k in first:
        assert np.array_equal(outs[k].cpu().numpy(), first[k]), k


def test_chain_with_aerosols():
    import torch
    from woof_nam_b200 import aerosols
    from woof_nam_b200.chain import radiation_call
    from woof_nam_b200.solver import RadSolver
    state, tab, lay = _domain(57)
    sun = _sun()
    s = RadSolver(precision="mixed", nlay=lay["plyr"].shape[0])
    d, c = _dev(state, tab)
    out = radiation_call(s, d, c, sun=sun, im=IM, aerosols=aerosols.Aerosols(s, 1), **CALL)
    torch.cuda.synchronize()
    got = {k: v.cpu().numpy() for k, v in out.items() if k != "work"}
    assert out["work"]["faer"][0].abs().sum().item() > 0
    ref = _oracle_chain(state, tab, lay, sun, month=1)
    assert_within(got, {k: ref[k] for k in got}, what="radiation call with aerosol")


def test_chain_from_tracers_and_ialb2_albedo():
    """The call started from the cloud tracers (clw = tracer ntcw, grrad's condensate) and, with ialbflg 2, from
    the surface albedo and land mask through grrad's IALB = 2 block, against the oracle's chain doing the same."""
    import torch
    from woof_nam_b200.chain import radiation_call
    from woof_nam_b200.solver import RadSolver
    state, tab, lay = _domain(63)
    r = np.random.default_rng(64)
    n = IM * JM
    tracer = r.random((3, lay["plyr"].shape[0], n)).astype(np.float32) * 1e-3
    tracer[1] = state["clw"]
    state.update(tracer1=tracer, sfcalbedo=r.uniform(0.05, 0.6, n).astype(np.float32),
                 clw=np.zeros_like(state["clw"]))
    sun = _sun()
    call = dict(CALL, ialbflg=2)
    s = RadSolver(precision="mixed", nlay=lay["plyr"].shape[0])
    d, c = _dev(state, tab)
    out = radiation_call(s, d, c, sun=sun, im=IM, ntcw=2, **call)
    torch.cuda.synchronize()
    got = {k: v.cpu().numpy() for k, v in out.items() if k != "work"}
    saved = dict(CALL)
    CALL.update(ialbflg=2)
    try:
        ref = _oracle_chain(state, tab, lay, sun, ntcw=2)
    finally:
        CALL.clear()
        CALL.update(saved)
    assert_within(got, {k: ref[k] for k in got}, what="radiation call from tracers, IALB 2")
    assert out["work"]["clw"].abs().sum().item() > 0 and "albedo" in out["work"]
