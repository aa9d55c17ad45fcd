"""ctypes binding of libradb200.so (include/radb200.h).

The product path is this library: if it is missing or fails to load, every solve raises -- there is no
CPU or PyTorch fallback.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libradb200.so"

RAD_OK, RAD_E_INVALID, RAD_E_TABLES, RAD_E_CUDA, RAD_E_NOMEM, RAD_E_BUDGET, RAD_E_TIMEOUT, RAD_E_BUSY = \
    0, -1, -2, -3, -4, -5, -6, -7
PREC = {"fp64": 0, "mixed": 1}
ROUTE = {"nam": 0, "mcica": 1}
PARTS = {"lw": 1, "sw": 2, "both": 3}

_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int32)
_up = ctypes.POINTER(ctypes.c_uint32)


class RadConfig(ctypes.Structure):
    _fields_ = [("nlay", ctypes.c_int32), ("precision", ctypes.c_int32), ("route", ctypes.c_int32),
                ("iswmode", ctypes.c_int32), ("diagnostic", ctypes.c_int32), ("window_cols", ctypes.c_int32),
                ("sw_chunk", ctypes.c_int32), ("iovrlw", ctypes.c_int32), ("iovrsw", ctypes.c_int32),
                ("lw_seed0", ctypes.c_int32), ("sw_seed0", ctypes.c_int32), ("cpathfac", ctypes.c_float),
                ("parts", ctypes.c_int32), ("lw_chunk", ctypes.c_int32),
                ("sw_sweep_chunk", ctypes.c_int32)]


class RadColumns(ctypes.Structure):
    _fields_ = [("plyr", ctypes.c_void_p), ("plvl", ctypes.c_void_p), ("tlyr", ctypes.c_void_p),
                ("tlvl", ctypes.c_void_p), ("qlyr", ctypes.c_void_p), ("olyr", ctypes.c_void_p),
                ("gasvmr", ctypes.c_void_p), ("clouds", ctypes.c_void_p), ("faerlw", ctypes.c_void_p),
                ("faersw", ctypes.c_void_p), ("sfcemis", ctypes.c_void_p), ("tsfg", ctypes.c_void_p),
                ("sfcalb", ctypes.c_void_p), ("coszen", ctypes.c_void_p), ("icseed", ctypes.c_void_p),
                ("solcon", ctypes.c_float)]


class RadOutputs(ctypes.Structure):
    _fields_ = [("htlw", ctypes.c_void_p), ("htsw", ctypes.c_void_p), ("topflw", ctypes.c_void_p),
                ("sfcflw", ctypes.c_void_p), ("topfsw", ctypes.c_void_p), ("sfcfsw", ctypes.c_void_p),
                ("fdncmp", ctypes.c_void_p), ("lw_mask", ctypes.c_void_p), ("sw_mask", ctypes.c_void_p),
                ("hsw0", ctypes.c_void_p), ("htswb", ctypes.c_void_p), ("swflxprf", ctypes.c_void_p),
                ("hlw0", ctypes.c_void_p), ("hlwb", ctypes.c_void_p), ("lwflxprf", ctypes.c_void_p)]


class RadProfile(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_int64), ("solves", ctypes.c_int64), ("columns", ctypes.c_int64),
                ("lw_ms", ctypes.c_double), ("prep_ms", ctypes.c_double), ("sw_ms", ctypes.c_double)]


POST_IN_FIELDS = ("hlw", "swh", "coszdg_v", "coszen_v", "sfcflw_dnfxc", "topflw_upfxc", "sfcfsw_upfxc",
                  "sfcfsw_dnfxc", "sfcfsw_dnfx0", "topfsw_upfxc", "cldcov", "cldsa", "cw", "t", "cu_cloud")
POST_OUT_FIELDS = ("rlwtt", "rswtt", "cldfra", "csmid", "rlwin", "rswin", "rswinc", "rswout", "rlwtoa", "rswtoa",
                   "czmean", "sigt4", "coszdg", "cfracl", "cfracm", "cfrach", "acfrst", "acfrcv", "ncfrst", "ncfrcv")


class RadPostIn(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in POST_IN_FIELDS]


class RadPostOut(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in POST_OUT_FIELDS]


class RadRdtemp(ctypes.Structure):
    _fields_ = [("ntsd", ctypes.c_int32), ("dt", ctypes.c_float), ("julday", ctypes.c_int32),
                ("julyr", ctypes.c_int32), ("ihrst", ctypes.c_int32), ("leap_seen", ctypes.c_int32),
                ("glat", ctypes.c_void_p), ("glon", ctypes.c_void_p), ("czmean", ctypes.c_void_p),
                ("rswtt", ctypes.c_void_p), ("rlwtt", ctypes.c_void_p), ("czen", ctypes.c_void_p),
                ("t", ctypes.c_void_p), ("im", ctypes.c_int32), ("jm", ctypes.c_int32), ("lm", ctypes.c_int32),
                ("its", ctypes.c_int32), ("ite", ctypes.c_int32), ("jts", ctypes.c_int32), ("jte", ctypes.c_int32),
                ("its_b1", ctypes.c_int32), ("ite_b1", ctypes.c_int32), ("jts_b1", ctypes.c_int32),
                ("jte_b1", ctypes.c_int32)]


# Every symbol include/radb200.h declares, with its ctypes signature.
AER_CLIM_FIELDS = ("iendwv", "haer", "prsref", "rhid", "rhdp", "straext0", "nwvns0", "s0intv", "month_idx",
                   "month_cmix", "month_kprf", "month_denn")
AER_COL_FIELDS = ("plvl", "plyr", "tlyr", "qlyr", "rhly", "xlon", "xlat", "slmsk")


class RadAerClim(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in AER_CLIM_FIELDS]


class RadAerColumns(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in AER_COL_FIELDS]


MODEL_FIELDS = ("pint", "pmid", "prslk", "t", "q", "tsfc")
LAYER_FIELDS = ("plvl", "plyr", "tlyr", "tlvl", "qlyr", "rhly", "qstl", "prslk1", "tvly", "tsfg")


class RadModelColumns(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in MODEL_FIELDS]


class RadLayerFields(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in LAYER_FIELDS]


class RadSolarIn(ctypes.Structure):
    _fields_ = [("year", ctypes.c_int32), ("month", ctypes.c_int32), ("day", ctypes.c_int32),
                ("hour", ctypes.c_int32), ("minute", ctypes.c_int32), ("second", ctypes.c_int32),
                ("deltsw", ctypes.c_float), ("deltim", ctypes.c_float), ("solc0", ctypes.c_double)]


class RadSolarState(ctypes.Structure):
    _fields_ = [("sollag", ctypes.c_float), ("sindec", ctypes.c_float), ("cosdec", ctypes.c_float),
                ("anginc", ctypes.c_float), ("solcon", ctypes.c_float), ("nstp", ctypes.c_int32)]


DAYPARTS_FIELDS = ("coszen", "coszdg", "dp_start", "dp_len", "dp_day", "ndayparts")
ALBEDO_FIELDS = ("slmsk", "snowf", "sncovr", "snoalb", "zorlf", "coszf", "tsknf", "hprif", "alvsf", "alnsf", "alvwf",
                 "alnwf", "facsf", "facwf", "fice", "tisfc")
EMIS_FIELDS = ("glon", "glat", "sm", "sice", "si", "sncovr", "z0", "stdh", "tskin", "idxems")
CLOUD_IN_FIELDS = ("plyr", "plvl", "tlyr", "tvly", "qlyr", "qstl", "rhly", "clw", "f_ice", "f_rain", "r_rime", "cldfk1",
                   "xlat")
CLOUD_CFG_FIELDS = ("ivflip", "llyr", "iovr", "lcrick", "lcnorm", "lnoprec", "lsashal", "cld_fraction")
CLOUD_OUT_FIELDS = ("clouds", "clds", "mtop", "mbot")


class RadDayparts(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in DAYPARTS_FIELDS]


class RadGasSetup(ctypes.Structure):
    _fields_ = [("co2_glb", ctypes.c_void_p), ("gco2cyc", ctypes.c_void_p), ("co2vmr_sav", ctypes.c_void_p),
                ("ico2flg", ctypes.c_int32), ("kmonsav", ctypes.c_int32), ("ivflip", ctypes.c_int32)]


class RadOzoneClim(ctypes.Structure):
    _fields_ = [("o3r", ctypes.c_void_p), ("pkstr", ctypes.c_void_p), ("jmr", ctypes.c_int32), ("loz", ctypes.c_int32),
                ("k1oz", ctypes.c_int32), ("k2oz", ctypes.c_int32), ("facoz", ctypes.c_float),
                ("blte", ctypes.c_float), ("dlte", ctypes.c_float), ("ivflip", ctypes.c_int32)]


class RadAlbedoIn(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in ALBEDO_FIELDS]


class RadEmisIn(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in EMIS_FIELDS]


class RadPayneTables(ctypes.Structure):
    _fields_ = [(k, ctypes.POINTER(ctypes.c_float)) for k in ("trn", "za", "dza", "albd")]


class RadCloudIn(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in CLOUD_IN_FIELDS]


class RadCloudCfg(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int32) for k in CLOUD_CFG_FIELDS]


class RadCloudOut(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in CLOUD_OUT_FIELDS]


SIGNATURES = {
    "rad_version": ([], ctypes.c_int),
    "rad_config_default": ([ctypes.POINTER(RadConfig), ctypes.c_int32], None),
    "rad_create": ([ctypes.POINTER(RadConfig), ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "rad_load_tables": ([ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int),
    "rad_solve": ([ctypes.c_void_p, ctypes.POINTER(RadColumns), ctypes.POINTER(RadOutputs), ctypes.c_int64,
                   ctypes.c_void_p], ctypes.c_int),
    "rad_workspace_bytes": ([ctypes.c_void_p, ctypes.c_int64], ctypes.c_int64),
    "rad_solve_batch": ([ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(RadColumns), ctypes.POINTER(RadOutputs),
                         ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p], ctypes.c_int),
    "rad_graph_create": ([ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(RadColumns), ctypes.POINTER(RadOutputs),
                          ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "rad_graph_launch": ([ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rad_graph_destroy": ([ctypes.c_void_p], None),
    "rad_solve_noalloc": ([ctypes.c_void_p, ctypes.POINTER(RadColumns), ctypes.POINTER(RadOutputs), ctypes.c_int64,
                           ctypes.c_void_p], ctypes.c_int),
    "rad_post_outputs": ([ctypes.c_void_p, ctypes.POINTER(RadPostIn), ctypes.POINTER(RadPostOut), ctypes.c_int64,
                          ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p], ctypes.c_int),
    "rad_rdtemp": ([ctypes.c_void_p, ctypes.POINTER(RadRdtemp), ctypes.c_void_p], ctypes.c_int),
    "rad_load_aerosols": ([ctypes.c_void_p, ctypes.POINTER(RadAerClim)], ctypes.c_int),
    "rad_sol_update": ([ctypes.POINTER(RadSolarIn), ctypes.POINTER(RadSolarState)], ctypes.c_int),
    "rad_grrad_setup": ([ctypes.c_void_p, ctypes.POINTER(RadModelColumns), ctypes.c_int64, ctypes.c_int32,
                         ctypes.POINTER(RadLayerFields), ctypes.c_void_p], ctypes.c_int),
    "rad_coszmn": ([ctypes.c_void_p, ctypes.POINTER(RadSolarState), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                    ctypes.c_float, ctypes.c_float, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
                   ctypes.c_int),
    "rad_dayparts": ([ctypes.c_void_p, ctypes.POINTER(RadSolarState), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                      ctypes.c_int32, ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_int32,
                      ctypes.POINTER(RadDayparts), ctypes.c_void_p], ctypes.c_int),
    "rad_getgases": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                      ctypes.POINTER(RadGasSetup), ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rad_getozn": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                    ctypes.POINTER(RadOzoneClim), ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rad_setalb": ([ctypes.c_void_p, ctypes.POINTER(RadAlbedoIn), ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p,
                    ctypes.c_void_p], ctypes.c_int),
    "rad_setemis": ([ctypes.c_void_p, ctypes.POINTER(RadEmisIn), ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                     ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rad_progcld2": ([ctypes.c_void_p, ctypes.POINTER(RadCloudIn), ctypes.c_int64, ctypes.c_int32,
                      ctypes.POINTER(RadCloudCfg), ctypes.POINTER(RadCloudOut), ctypes.c_void_p], ctypes.c_int),
    "rad_setaer": ([ctypes.c_void_p, ctypes.POINTER(RadAerColumns), ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                    ctypes.c_void_p], ctypes.c_int),
    "rad_grrad_clw": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32,
                       ctypes.c_int32, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rad_payne_albedo": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                          ctypes.POINTER(RadPayneTables), ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p],
                         ctypes.c_int),
    "rad_setaer_volc": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                         ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                         ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "rad_queue_create": ([ctypes.POINTER(ctypes.c_void_p), ctypes.c_int32, ctypes.c_int64,
                          ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "rad_submit": ([ctypes.c_void_p, ctypes.POINTER(RadColumns), ctypes.POINTER(RadOutputs), ctypes.c_int64,
                    ctypes.POINTER(ctypes.c_int64)], ctypes.c_int),
    "rad_poll": ([ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int32)], ctypes.c_int),
    "rad_wait": ([ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32], ctypes.c_int),
    "rad_queue_destroy": ([ctypes.c_void_p], None),
    "rad_device_error": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)], ctypes.c_int),
    "rad_profile_enable": ([ctypes.c_void_p, ctypes.c_int], ctypes.c_int),
    "rad_profile_read": ([ctypes.c_void_p, ctypes.POINTER(RadProfile)], ctypes.c_int),
    "rad_last_error": ([ctypes.c_void_p], ctypes.c_char_p),
    "rad_destroy": ([ctypes.c_void_p], None),
}

_LIB = None


class RadError(RuntimeError):
    """A failing library call: carries the RAD_E_* code."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (code {code})")
        self.code = code


def load(path: Path | None = None):
    """Load libradb200.so and bind every declared symbol; raises if the library is missing."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is not built: run woof_nam_b200.build.build() (nvcc, sm_100a)")
    lib = ctypes.CDLL(str(p))
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if path is None:
        _LIB = lib
    return lib


def check(lib, handle, rc: int, what: str):
    if rc != RAD_OK:
        msg = lib.rad_last_error(handle)
        raise RadError(rc, f"{what}: {msg.decode() if msg else 'error'}")
