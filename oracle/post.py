"""CPU restatement of the radiation call's post step (test infrastructure only).

Restates rrtm_post_outputs, namgpu/kernels/phys_rrtm_driver_post.cu:71-145 (module_RA_RRTM.F90:1142-1240,
ICWP /= -1, LSSAV true), in numpy float32 over columns: every array is [level or component][ncol].
``reference_post`` runs the reference kernel itself, compiled for the host into ``_ref/libref_rrtm.so``
(``ref_post_outputs`` in ``ref_driver.cpp``), where the reference tree was available to build it.

Only the tests and the fixture script import this module.
"""
from __future__ import annotations

import ctypes

import numpy as np

EPSQ2 = np.float32(1.0e-8)        # module_RA_RRTM.F90:286 (phys_rrtm_driver_post.cu RRTM_EPSQ2)
STBOLT = np.float32(5.67051e-8)   # nmmb_common NMMB_STBOLT

IN_2D = ("coszdg_v", "coszen_v", "sfcflw_dnfxc", "sfcfsw_dnfxc", "sfcfsw_upfxc", "sfcfsw_dnfx0", "topflw_upfxc",
         "topfsw_upfxc")
OUT_3D = ("rlwtt", "rswtt", "cldfra", "csmid")
OUT_2D = ("rlwin", "rswin", "rswinc", "rswout", "rlwtoa", "rswtoa", "czmean", "sigt4", "coszdg", "cfracl",
          "cfracm", "cfrach", "acfrst", "acfrcv")
ACCUM = ("acfrst", "acfrcv", "ncfrst", "ncfrcv", "sigt4")    # outputs read before they are written


def post_outputs(inp: dict, state: dict, lm: int, kd: int = 0, cloud_block: bool = True,
                 lw_step: bool = True) -> dict:
    """inp: hlw, swh [lm + kd][n]; the IN_2D rows [n]; cldcov [lm][n], cldsa [5][n] (returned zeroed on dry
    columns); cw, t [lm][n]; cu_cloud int32 [n].  state: the accumulators acfrst, acfrcv (float32), ncfrst,
    ncfrcv (int32) and sigt4 before the call.  Returns every output plus the updated cldcov / cldsa."""
    f32 = np.float32
    o = {}
    # 2-D copies (1142-1143, 1164-1170)
    o["coszdg"] = inp["coszdg_v"].astype(f32, copy=True)
    o["czmean"] = inp["coszen_v"].astype(f32, copy=True)
    o["rlwin"] = inp["sfcflw_dnfxc"].astype(f32, copy=True)
    o["rswin"] = inp["sfcfsw_dnfxc"].astype(f32, copy=True)
    o["rswout"] = inp["sfcfsw_upfxc"].astype(f32, copy=True)
    o["rswinc"] = inp["sfcfsw_dnfx0"].astype(f32, copy=True)
    o["rlwtoa"] = inp["topflw_upfxc"].astype(f32, copy=True)
    o["rswtoa"] = inp["topfsw_upfxc"].astype(f32, copy=True)
    # heating-rate copies, DO L = 1, LM (1145-1148); kd skips the solve's extra top layer
    o["rlwtt"] = inp["hlw"][kd:kd + lm].astype(f32, copy=True)
    o["rswtt"] = inp["swh"][kd:kd + lm].astype(f32, copy=True)
    cldcov = inp["cldcov"].astype(f32, copy=True)
    cldsa = inp["cldsa"].astype(f32, copy=True)
    o["acfrst"] = state["acfrst"].astype(f32, copy=True)
    o["acfrcv"] = state["acfrcv"].astype(f32, copy=True)
    o["ncfrst"] = state["ncfrst"].astype(np.int32, copy=True)
    o["ncfrcv"] = state["ncfrcv"].astype(np.int32, copy=True)
    if cloud_block:
        # ARG_CW = MAXVAL(CW(IDEX, J, 1:LM)); cloud fields zeroed where ARG_CW < EPSQ2 (1180-1194)
        dry = inp["cw"][:lm].max(axis=0) < EPSQ2
        cldcov[:, dry] = 0.0
        cldsa[:, dry] = 0.0
        o["cldfra"] = cldcov.copy()                     # 1197-1200
        o["csmid"] = cldcov.copy()
        o["cfracl"], o["cfracm"], o["cfrach"] = cldsa[0].copy(), cldsa[1].copy(), cldsa[2].copy()   # 1202-1204
        o["acfrst"] = (o["acfrst"] + cldsa[3]).astype(f32)                                         # 1210-1211
        o["ncfrst"] = o["ncfrst"] + 1
        cu = inp["cu_cloud"] != 0                                                                  # 1213-1214
        o["acfrcv"] = np.where(cu, (o["acfrcv"] + cldsa[3]).astype(f32), o["acfrcv"])
        o["ncfrcv"] = o["ncfrcv"] + 1
    o["sigt4"] = state["sigt4"].astype(f32, copy=True)
    if lw_step:
        # SIGT4 = STBOLT * TDUM * TDUM * TDUM * TDUM, TDUM = T(I, J, LM)   (1232-1240), left to right in float
        td = inp["t"][lm - 1].astype(f32)
        o["sigt4"] = (((STBOLT * td) * td) * td) * td
    o["cldcov"], o["cldsa"] = cldcov, cldsa
    return o


def reference_post(inp: dict, state: dict, lm: int, lw_step: bool = True) -> dict:
    """The reference kernel rrtm_post_outputs on the host (oracle/_ref), kd = 0 interface, ICWP = 1."""
    from . import oracle
    lib = ctypes.CDLL(str(oracle.REF_LIB))
    n = inp["coszen_v"].shape[-1]
    c = lambda a, dt=np.float32: np.ascontiguousarray(a, dtype=dt)  # noqa: E731
    ins = {k: c(inp[k]) for k in ("hlw", "swh", *IN_2D, "cw", "t")}
    cldcov, cldsa = c(inp["cldcov"]).copy(), c(inp["cldsa"]).copy()
    cu = c(inp["cu_cloud"], np.int32)
    out = {k: np.zeros((lm, n), np.float32) for k in OUT_3D}
    out.update({k: np.zeros(n, np.float32) for k in OUT_2D})
    out["ncfrst"] = np.zeros(n, np.int32)
    out["ncfrcv"] = np.zeros(n, np.int32)
    for k in ACCUM:
        out[k][...] = state[k]
    fp = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    rc = lib.ref_post_outputs(
        ctypes.c_int(n), ctypes.c_int(lm), ctypes.c_int(1), ctypes.c_int(int(lw_step)), fp(ins["hlw"]),
        fp(ins["swh"]), fp(ins["coszdg_v"]), fp(ins["coszen_v"]), fp(ins["sfcflw_dnfxc"]), fp(ins["sfcfsw_dnfxc"]),
        fp(ins["sfcfsw_upfxc"]), fp(ins["sfcfsw_dnfx0"]), fp(ins["topflw_upfxc"]), fp(ins["topfsw_upfxc"]),
        fp(cldcov), fp(cldsa), fp(ins["cw"]), fp(ins["t"]), fp(cu),
        *[fp(out[k]) for k in ("rlwtt", "rswtt", "cldfra", "csmid", "rlwin", "rswin", "rswinc", "rswout", "rlwtoa",
                               "rswtoa", "czmean", "sigt4", "coszdg", "cfracl", "cfracm", "cfrach", "acfrst",
                               "acfrcv", "ncfrst", "ncfrcv")])
    if rc != 0:
        raise RuntimeError("ref_post_outputs failed")
    out["cldcov"], out["cldsa"] = cldcov, cldsa
    return out


def make_case(n: int, lm: int, seed: int, kd: int = 0) -> tuple:
    """Seeded post-step inputs: heating rates, fluxes, cloud cover / amounts, condensate with a quarter of
    the columns dry (max CW below 1e-8), temperatures, CU_cloud flags, and non-zero accumulators."""
    rng = np.random.default_rng(seed)
    f = lambda *s: rng.standard_normal(s).astype(np.float32)  # noqa: E731
    u = lambda lo, hi, *s: rng.uniform(lo, hi, s).astype(np.float32)  # noqa: E731
    cw = u(0.0, 1e-3, lm, n)
    dry = rng.random(n) < 0.25
    cw[:, dry] = u(0.0, 9.9e-9, lm, int(dry.sum()))
    inp = {"hlw": f(lm + kd, n) * np.float32(3e-5), "swh": f(lm + kd, n) * np.float32(3e-5),
           "coszdg_v": u(0, 1, n), "coszen_v": u(0, 1, n), "sfcflw_dnfxc": u(150, 450, n),
           "sfcfsw_dnfxc": u(0, 1000, n), "sfcfsw_upfxc": u(0, 300, n), "sfcfsw_dnfx0": u(0, 1100, n),
           "topflw_upfxc": u(150, 320, n), "topfsw_upfxc": u(0, 600, n), "cldcov": u(0, 1, lm, n),
           "cldsa": u(0, 1, 5, n), "cw": cw, "t": u(190, 310, lm, n),
           "cu_cloud": (rng.random(n) < 0.3).astype(np.int32)}
    state = {"acfrst": u(0, 20, n), "acfrcv": u(0, 20, n), "ncfrst": rng.integers(0, 40, n).astype(np.int32),
             "ncfrcv": rng.integers(0, 40, n).astype(np.int32), "sigt4": u(0, 500, n)}
    return inp, state
