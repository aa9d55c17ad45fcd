"""Pack the RRTM LW/SW k-distribution and cloud-optics tables into one normalised npz.

Runs where the reference tree is available (it reads the reference's extracted table files under
``namgpu/data/``) and writes ``rrtm_tables.npz`` next to this script.  The packed file is what the
library, the oracle and the tests load; nothing at run time reads the reference tree.

Normalisation rules (one per table family, so every consumer indexes the same way):

* every k-table is float32 with the g-point axis LAST (``[..., g]``).  The reference stores most LW/SW
  tables that way already; the band-5 LW tables (float64, ``[g, ...]``, ``data/rrtm_lw_kgb05.npz``) and
  the SW band 16/20/24/25/28 tables (``[g, ind]``) are transposed here.  Band 5 is rounded to float32
  exactly as the reference's loader does (``physics/rrtm/phys_rrtm_lw_taugb05.py:87-94``).
* names are ``lw{BB}_{name}`` for LW band BB (01..16) and ``sw{BB}_{name}`` for SW band BB (16..29).
* scalar per-band constants (rayl, strrat, givfac, ...) are stored as 0-d float32 arrays.
* the LW Planck table ``totplnk[16, 181]``, reference profiles ``preflog/tref/chi_mls`` and the cloud
  optics tables keep the reference's C order.

Which file each table comes from follows the reference's own loaders:
``physics/rrtm/phys_rrtm_lw_setcoef.py:160-169`` (totplnk, preflog, tref, chi_mls, delwave),
``physics/rrtm/phys_rrtm_lw_cldprop.py:57`` (``data/rrtm_lw_cldprlw.npz``),
``physics/rrtm/phys_rrtm_sw_cldprop.py:58`` (``data/rrtm_sw_cldprtb.npz``),
``physics/rrtm/phys_rrtm_sw_table_sflux.py:31`` (``data/rrtm_sw/sflux.npz``).

Usage:  python woof_nam_b200/data/pack_tables.py [REFERENCE_ROOT]
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

LW_NG = (10, 12, 16, 14, 16, 8, 12, 8, 12, 6, 8, 8, 4, 2, 2, 2)
SW_NG = {16: 6, 17: 12, 18: 8, 19: 8, 20: 10, 21: 10, 22: 2, 23: 10, 24: 8, 25: 6, 26: 6, 27: 8,
         28: 6, 29: 12}
# SW bands whose k-tables the reference stores g-first ([g, ind]); the rest are [ind, g].
SW_G_FIRST = {16, 20, 24, 25, 28}
# LW delwave (radlw_param.f:133), restated by the reference at physics/rrtm/phys_rrtm_lw_setcoef.py:64.
DELWAVE = np.array([340., 150., 130., 70., 120., 160., 100., 100., 210., 90., 320., 280., 170., 130.,
                    220., 650.], dtype=np.float32)


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def pack(ref_root: Path) -> dict:
    d = ref_root / "namgpu" / "data"
    out: dict[str, np.ndarray] = {}

    # ---- LW k-tables -------------------------------------------------------------------------------
    for b in range(1, 17):
        ng = LW_NG[b - 1]
        if b == 5:
            z = np.load(d / "rrtm_lw_kgb05.npz")
            for name in ("absa", "absb", "selfref", "forref", "fracrefa", "fracrefb"):
                out[f"lw05_{name}"] = _f32(z[name].T)
            out["lw05_ka_mo3"] = _f32(z["ka_mo3"].transpose(2, 1, 0))      # [19, 9, 16]
            out["lw05_ccl4"] = _f32(z["ccl4"])
            out["lw05_chi_mls_f64"] = np.ascontiguousarray(z["chi_mls"].T, dtype=np.float64)  # [59, 7]
            continue
        z = np.load(d / "rrtm_lw" / f"kgb{b:02d}.npz")
        for name in z.files:
            a = z[name]
            if a.dtype.kind in "US":
                continue
            if name == "chi_mls" or name.startswith("nmmb_") or name == "chi_mls_co2":
                continue                      # chi_mls is packed once below; nmmb_* tables are unused by NAM
            a = _f32(a)
            if a.ndim >= 1 and a.shape[-1] != ng:
                raise ValueError(f"lw{b:02d}_{name}: g axis is not last: {a.shape}")
            out[f"lw{b:02d}_{name}"] = a

    # ---- LW setcoef / Planck / reference profiles ----------------------------------------------------
    out["lw_totplnk"] = _f32(np.load(d / "rrtm_lw_avplank.npz")["totplnk"])     # [16, 181]
    ref = np.load(d / "rrtm_lw" / "ref.npz")
    out["lw_preflog"] = _f32(ref["preflog"])
    out["lw_tref"] = _f32(ref["tref"])
    out["lw_chi_mls"] = _f32(ref["chi_mls"])                                     # [59, 7] = chi(gas, lev)
    chi2 = np.load(d / "rrtm_lw" / "ref_chi_mls.npz")["chi_mls"]
    if not np.array_equal(chi2, ref["chi_mls"]):
        raise ValueError("ref.npz and ref_chi_mls.npz chi_mls differ")
    out["lw_delwave"] = DELWAVE.copy()

    # ---- LW cloud optics (radlw_datatb.f module_radlw_cldprlw) ---------------------------------------
    c = np.load(d / "rrtm_lw_cldprlw.npz")
    for name in ("absliq1", "absice1", "absice2", "absice3"):
        out[f"lw_{name}"] = _f32(c[name])
    out["lw_ipat"] = np.ascontiguousarray(c["ipat"], dtype=np.int32)

    # ---- SW k-tables ---------------------------------------------------------------------------------
    for b in range(16, 30):
        ng = SW_NG[b]
        z = np.load(d / "rrtm_sw" / f"kgb{b}.npz")
        for name in z.files:
            a = z[name]
            if a.dtype.kind in "US":
                continue
            a = np.asarray(a, dtype=np.float32)
            if a.ndim == 2 and b in SW_G_FIRST and name != "rayla":
                if a.shape[0] != ng:
                    raise ValueError(f"sw{b}_{name}: expected g-first {a.shape}")
                a = a.T
            if a.ndim >= 1 and a.shape[-1] != ng:
                raise ValueError(f"sw{b}_{name}: g axis is not last: {a.shape}")
            key = name
            if name.startswith("strrat"):
                key = "strrat"
            out[f"sw{b}_{key}"] = _f32(a)

    # ---- SW reference profiles, solar source, cloud optics -------------------------------------------
    sref = np.load(d / "rrtm_sw" / "ref.npz")
    out["sw_preflog"] = _f32(sref["preflog"])
    out["sw_tref"] = _f32(sref["tref"])
    s = np.load(d / "rrtm_sw" / "sflux.npz")
    for name in ("sfluxref01", "sfluxref02", "sfluxref03", "strrat", "specwt"):
        out[f"sw_{name}"] = _f32(s[name])
    for name in ("layreffr", "ix1", "ix2", "ibx"):
        out[f"sw_{name}"] = np.ascontiguousarray(s[name], dtype=np.int32)
    out["sw_scalekur"] = _f32(s["scalekur"])
    cp = np.load(d / "rrtm_sw_cldprtb.npz")
    for name in ("extliq1", "ssaliq1", "asyliq1", "extice2", "ssaice2", "asyice2", "extice3", "ssaice3",
                 "asyice3"):
        out[f"sw_{name}"] = _f32(cp[name])
    return out


def main(argv):
    if len(argv) < 2:
        raise SystemExit("usage: python pack_tables.py <reference tree>")
    ref_root = Path(argv[1])
    out = pack(ref_root)
    dst = Path(__file__).resolve().parent / "rrtm_tables.npz"
    np.savez_compressed(dst, **out)
    n = sum(a.size for a in out.values())
    print(f"wrote {dst} ({len(out)} arrays, {n} values)")


if __name__ == "__main__":
    main(sys.argv)
