// rad_sw.cuh -- RRTM shortwave column kernel for sm_100a: one CTA per sunlit column, fused prep, cloud
// optics, setcoef, solar source, gas optics (14 bands, 112 g-points) and the two-stream solver (spcvrtc +
// swflux adding method).
//
// Reference path: namgpu/kernels/phys_rrtm_sw_swrad.cu:127-418 (prep/post), phys_rrtm_sw_cldprop.cu,
// phys_rrtm_sw_setcoef.cu, phys_rrtm_sw_taumol.cu, phys_rrtm_sw_taumol16..29.cu, phys_rrtm_sw_spcvrtc.cu,
// driven as namgpu/physics/rrtm/sw_seam.py does (the reference launches spcvrtc once per g-point, 112
// launches per chunk, read-modify-writing [14, nlp1] band accumulators in HBM on every one).
// Phases as in rad_lw.cuh; the MINVAL(laytrop) group minima of bands 19/23 (8 day columns) and 25/28
// (the chunk) arrive precomputed per day column (sw_groups_kernel), so every column's result depends only
// on its own request.
//
// Precision.  R = double runs the reference statements in FP64 (the plain kernel).  R = float (mixed):
// optics, Rayleigh and gas optics in float; the layer reflectance/transmittance uses an algebraically
// equal form without 1/exp(-x) (the reference's float form overflows to inf/NaN once k*tau exceeds ~100 and
// returns NaN fluxes), and switches the layer to float64 where the delta-scaled single-scattering albedo is
// within 1e-4 of 1 (near-conservative scattering, where sqrt((g1-g2)(g1+g2)) cancels in float) or where the
// direct beam sits within 1% of the two-stream resonance k*mu0 = 1 (1 - (k mu0)^2 divides the beam terms);
// flux sums and the heating-rate differences are float64.
#pragma once
#include "rad_common.cuh"

namespace rad {

constexpr int SW_THREADS = 128;   // 4 warps, lanes 0..111 carry g-points
constexpr int SW_WARPS = SW_THREADS / 32;

template <class R>
struct SwShared {
    static constexpr bool kRatio64 = false;
    R pavel[NLAY_MAX], tavel[NLAY_MAX], delp[NLAY_MAX], coldry[NLAY_MAX], colmol[NLAY_MAX], h2ovmr[NLAY_MAX];
    R colamt[6][NLAY_MAX];
    R fac00[NLAY_MAX], fac01[NLAY_MAX], fac10[NLAY_MAX], fac11[NLAY_MAX];
    R selffac[NLAY_MAX], selffrac[NLAY_MAX], forfac[NLAY_MAX], forfrac[NLAY_MAX];
    int jp[NLAY_MAX], jt[NLAY_MAX], jt1[NLAY_MAX], indself[NLAY_MAX], indfor[NLAY_MAX];
    R cfrac[NLAY_MAX], cldfrc[NLAY_MAX];
    R taucw[14][NLAY_MAX], ssacw[14][NLAY_MAX], asycw[14][NLAY_MAX];
    R tauae[14][NLAY_MAX], ssaae[14][NLAY_MAX], asyae[14][NLAY_MAX];
    R taug[SW_NGPT][NLAY_MAX], taur[SW_NGPT][NLAY_MAX];
    R sfluxzen[SW_NGPT];
    double fn0[SW_WARPS][NLAY_MAX + 2], fnc[SW_WARPS][NLAY_MAX + 2];   // per-warp net-flux partials, clear/cloudy
    double sc[SW_WARPS][18];               // per-warp scalar partials, clear (0..8) and cloudy (9..17)
    R cosz, sntz, ssolar, albbm[2], albdf[2], zcf0, zcf1;
    int laytrop, kmin8, kminw;
};

struct SwIn {
    const float *plyr, *plvl, *tlyr, *qlyr, *olyr, *gasvmr, *clouds, *faersw, *sfcalb, *coszen;
    const int* daycol;        // [nday] column of each day index in the launch's concatenated column space
    const int* nday;          // device count of day columns
    const int* kmin8;         // [nday] MINVAL(laytrop) of the column's 8-day-column group
    const int* kminw;         // [nday] MINVAL(laytrop) of the column's chunk
    float *htsw, *topfsw, *sfcfsw, *fdncmp;
    int64_t ncol;
    int nlay, diagnostic, iswmode;
    float solcon;
    const uint32_t* mask;     // McICA route: sub-column cloud words [4][nlay][ncol] (null: NAM route)
    int iovr;                 // overlap of the clear-sky view fraction: 0 random, 1 maximum-random, 2 maximum
};

// Clear-sky view fraction zcf0 of swrad_prep (phys_rrtm_sw_swrad.cu:251-279) from the layer cloud fractions
// (surface first): the product of clear fractions (random overlap), of the clear fractions of contiguous
// cloud blocks (maximum-random) or the smallest clear fraction (maximum), then the ftiny / oneminus snaps.
template <class R, class T>
__device__ __forceinline__ R sw_zcf0(const T* cfrac, int nlay, int iovr)
{
    const R ftiny = (R)1.0e-12f, oneminus = (R)1.0f - (R)1.0e-6f;
    R z0 = 1, z1 = 1;
    if (iovr == 0) {
        for (int k0 = 0; k0 < nlay; ++k0) z0 = z0 * ((R)1 - (R)cfrac[k0]);
    } else if (iovr == 1) {
        for (int k0 = 0; k0 < nlay; ++k0) {
            const R cf = (R)cfrac[k0];
            if (cf > ftiny) z1 = fminR(z1, (R)1 - cf);
            else if (z1 < (R)1) { z0 = z0 * z1; z1 = 1; }
        }
        z0 = z0 * z1;
    } else if (iovr == 2) {
        for (int k0 = 0; k0 < nlay; ++k0) z0 = fminR(z0, (R)1 - (R)cfrac[k0]);
    }
    if (z0 <= ftiny) z0 = 0;
    if (z0 > oneminus) z0 = 1;
    return z0;
}

template <class R>
struct SwLut {
    const R* ex;             // exp_tbl(0:10000) of rswinit
};

// Key-species counts of the lower / upper atmosphere k-tables per SW band (taumol16..29: nspa, nspb).
__constant__ int c_sw_nspa[14] = {9, 9, 9, 9, 1, 9, 9, 1, 9, 1, 0, 1, 9, 1};
__constant__ int c_sw_nspb[14] = {1, 5, 1, 1, 1, 5, 1, 0, 1, 0, 0, 1, 5, 1};

// ------------------------------------------------------------------------------------------------------
// Key-species parameter of the SW bands that interpolate their k-tables in a species ratio (taumol16..19, 21,
// 22, 24, 28: slots 0..7): sm = mult * min(om, x1 / sc) with sc = x1 + strrat x2, entry js = 1 + int(sm), fraction
// fs = sm - int(sm) (guard: ratio 0 when sc <= 0, as bands 18 and 22 write it).  The entries of neighbouring js
// may differ by an order of magnitude, so fs carries the float division's error into the optical depth almost
// tenfold; a layout that holds the ratio of each slot and layer in float64 (kRatio64: `spr`, formed from the
// float64 column amounts) takes it from there and rounds fs once.
template <class R, class S>
__device__ __forceinline__ void sw_species(const S& s, int slot, int k0, R x1, R sc, R mult, R om, bool guard, int& js,
                                           R& fs)
{
    if constexpr (S::kRatio64) {
        const double sm = (double)mult * fmin((double)om, s.spr[slot][k0]);
        const int j = (int)sm;
        js = 1 + j;
        fs = (R)(sm - (double)j);
    } else {
        const R ratio = guard ? (sc > 0 ? x1 / sc : (R)0) : x1 / sc;
        const R sm = mult * fminR(om, ratio);
        js = 1 + (int)sm;
        fs = guard ? sm - (R)(int)sm : rfmod1(sm);
    }
}

// ------------------------------------------------------------------------------------------------------
// Gas and Rayleigh optical depths of SW g-point g (0..111) at layer k0 (phys_rrtm_sw_taumol16..29.cu with
// the reference's handling of the layer k = laytrop).
template <class R, class S>
__device__ void sw_gas(const S& s, int g, int k0, R& tg, R& tr, int band_of_g = -1)
{
    const int k = k0 + 1, lt = s.laytrop;
    const int jpk = s.jp[k0], jtk = s.jt[k0], jt1k = s.jt1[k0];
    const R f00 = s.fac00[k0], f01 = s.fac01[k0], f10 = s.fac10[k0], f11 = s.fac11[k0];
    const R cm = s.colmol[k0];
    const R c1 = s.colamt[0][k0], c2 = s.colamt[1][k0], c3 = s.colamt[2][k0], c5 = s.colamt[4][k0],
            c6 = s.colamt[5][k0];
    const int inds = s.indself[k0], indf = s.indfor[k0];
    const R sfac = s.selffac[k0], sfrac = s.selffrac[k0], ffac = s.forfac[k0], ffrac = s.forfrac[k0];
    const R oneminus = (R)1.0f - (R)1.0e-6f, swom = (R)0.999999f;
    int b = band_of_g;
    if (b < 0) {
        b = 0;
        while (g >= c_sw_ns[b + 1]) ++b;
    }
    const int ig = g - c_sw_ns[b], jb = b + 16;
    auto idx = [&](int jbb, int& id0, int& id1) {
        const int bb = jbb - 16;
        if (k <= lt) { id0 = ((jpk - 1) * 5 + (jtk - 1)) * c_sw_nspa[bb]; id1 = (jpk * 5 + (jt1k - 1)) * c_sw_nspa[bb]; }
        else { id0 = ((jpk - 13) * 5 + (jtk - 1)) * c_sw_nspb[bb]; id1 = ((jpk - 12) * 5 + (jt1k - 1)) * c_sw_nspb[bb]; }
    };
    auto sum8 = [&](const R* A, int ng, int msa, int id0, int id1, int js, R fs, int o1, int o2) {
        const R fs1 = (R)1 - fs;
        const R fac000 = fs1 * f00, fac010 = fs1 * f10, fac100 = fs * f00, fac110 = fs * f10;
        const R fac001 = fs1 * f01, fac011 = fs1 * f11, fac101 = fs * f01, fac111 = fs * f11;
        const int i01 = max(1, min(msa, id0 + js)), i02 = min(msa, i01 + 1), i03 = min(msa, i01 + o1), i04 = min(msa, i01 + o2);
        const int i11 = max(1, min(msa, id1 + js)), i12 = min(msa, i11 + 1), i13 = min(msa, i11 + o1), i14 = min(msa, i11 + o2);
        auto a = [&](int i) { return ldt(A + (size_t)(i - 1) * ng + ig); };
        return fac000 * a(i01) + fac100 * a(i02) + fac010 * a(i03) + fac110 * a(i04) + fac001 * a(i11) +
               fac101 * a(i12) + fac011 * a(i13) + fac111 * a(i14);
    };
    auto sum4 = [&](const R* A, int ng, int ms, int id0, int id1) {
        const int i01 = max(1, min(ms, id0 + 1)), i02 = min(ms, i01 + 1);
        const int i11 = max(1, min(ms, id1 + 1)), i12 = min(ms, i11 + 1);
        auto a = [&](int i) { return ldt(A + (size_t)(i - 1) * ng + ig); };
        return f00 * a(i01) + f10 * a(i02) + f01 * a(i11) + f11 * a(i12);
    };
    // key-species ratio parameter of the band's layer (sw_species); sc = x1 + strr x2 multiplies the sum
    auto jsfs = [&](int slot, R x1, R strr, R x2, R mult, R om, R& sc, int& js, R& fs, bool guard = false) {
        sc = x1 + strr * x2;
        sw_species<R>(s, slot, k0, x1, sc, mult, om, guard, js, fs);
    };
    auto SF = [&](int id, int ng) { return sfac * interp(tab<R>(id), ng, inds, ig, sfrac); };
    auto FF = [&](int id, int ng) { return ffac * interp(tab<R>(id), ng, indf, ig, ffrac); };
    int id0, id1;
    switch (jb) {
    case 16: {
        const int NG = 6;
        idx(16, id0, id1);
        tr = cm * ldt(tab<R>(T_SW16_RAYL));
        tg = 0;
        if (k <= lt) {
            R sc, fs; int js;
            jsfs(0, c1, ldt(tab<R>(T_SW16_STRRAT)), c5, (R)8, oneminus, sc, js, fs);
            tg = sc * sum8(tab<R>(T_SW16_ABSA), NG, 585, id0, id1, js, fs, 9, 10) +
                 c1 * (SF(T_SW16_SELFREF, NG) + FF(T_SW16_FORREF, NG));
        }
        if (k >= lt) tg = c5 * sum4(tab<R>(T_SW16_ABSB), NG, 235, id0, id1);
        break;
    }
    case 17: {
        const int NG = 12;
        const R strr = (R)ldt(tab<R>(T_SW_STRRAT) + 1);
        tr = cm * (R)6.86e-10f;
        R sc, fs; int js;
        if (k0 < lt) {
            jsfs(1, c1, strr, c2, (R)8, oneminus, sc, js, fs);
            const int i0 = ((jpk - 1) * 5 + (jtk - 1)) * 9, i1 = (jpk * 5 + (jt1k - 1)) * 9;
            const R selfpart = inds > 0 ? SF(T_SW17_SELFREF, NG) : (R)0;
            tg = sc * sum8(tab<R>(T_SW17_ABSA), NG, 585, i0, i1, js, fs, 9, 10) + c1 * (selfpart + FF(T_SW17_FORREF, NG));
        } else {
            jsfs(1, c1, strr, c2, (R)4, oneminus, sc, js, fs);
            const int i0 = ((jpk - 13) * 5 + (jtk - 1)) * 5, i1 = ((jpk - 12) * 5 + (jt1k - 1)) * 5;
            tg = sc * sum8(tab<R>(T_SW17_ABSB), NG, 1175, i0, i1, js, fs, 5, 6) + (c1 * ffac) * interp(tab<R>(T_SW17_FORREF), NG, indf, ig, ffrac);
        }
        break;
    }
    case 18: {
        const int NG = 8;
        tr = cm * ldt(tab<R>(T_SW18_RAYL));
        idx(18, id0, id1);
        if (k <= lt) {
            R sc, fs; int js;
            jsfs(2, c1, (R)ldt(tab<R>(T_SW_STRRAT) + 2), c5, (R)8, swom, sc, js, fs, true);
            tg = sc * sum8(tab<R>(T_SW18_ABSA), NG, 585, id0, id1, js, fs, 9, 10) +
                 c1 * (SF(T_SW18_SELFREF, NG) + FF(T_SW18_FORREF, NG));
        } else {
            tg = c5 * sum4(tab<R>(T_SW18_ABSB), NG, 235, id0, id1);
        }
        break;
    }
    case 19: {
        const int NG = 8;
        tr = cm * (R)2.29e-09f;
        idx(19, id0, id1);
        tg = 0;
        if (k <= lt) {
            R sc, fs; int js;
            jsfs(3, c1, (R)5.49281e+0f, c2, (R)8, swom, sc, js, fs);
            tg = sc * sum8(tab<R>(T_SW19_ABSA), NG, 585, id0, id1, js, fs, 9, 10) +
                 c1 * (SF(T_SW19_SELFREF, NG) + FF(T_SW19_FORREF, NG));
        }
        if (k >= lt && k >= s.kmin8 + 1) tg = c2 * sum4(tab<R>(T_SW19_ABSB), NG, 235, id0, id1);
        break;
    }
    case 20: {
        const int NG = 10;
        tr = cm * ldt(tab<R>(T_SW20_RAYL));
        const R ch4 = ldt(tab<R>(T_SW20_ABSCH4) + ig);
        if (k <= lt) {
            const int i0 = (jpk - 1) * 5 + (jtk - 1), i1 = jpk * 5 + (jt1k - 1);
            tg = c1 * ((sum4(tab<R>(T_SW20_ABSA), NG, 65, i0, i1)) + sfac * interp(tab<R>(T_SW20_SELFREF), NG, inds, ig, sfrac) +
                       ffac * interp(tab<R>(T_SW20_FORREF), NG, indf, ig, ffrac)) + c5 * ch4;
        } else {
            const int i0 = (jpk - 13) * 5 + (jtk - 1), i1 = (jpk - 12) * 5 + (jt1k - 1);
            tg = c1 * ((sum4(tab<R>(T_SW20_ABSB), NG, 235, i0, i1)) + ffac * interp(tab<R>(T_SW20_FORREF), NG, indf, ig, ffrac)) + c5 * ch4;
        }
        break;
    }
    case 21: {
        const int NG = 10;
        tr = cm * (R)9.41e-09f;
        const R strr = (R)4.53210e-03f;
        if (k <= lt) { id0 = ((jpk - 1) * 5 + (jtk - 1)) * 9; id1 = (jpk * 5 + (jt1k - 1)) * 9; }
        else { id0 = ((jpk - 13) * 5 + (jtk - 1)) * 5; id1 = ((jpk - 12) * 5 + (jt1k - 1)) * 5; }
        tg = 0;
        R sc, fs; int js;
        if (k < lt) {
            jsfs(4, c1, strr, c2, (R)8, oneminus, sc, js, fs);
            tg = sc * sum8(tab<R>(T_SW21_ABSA), NG, 585, id0, id1, js, fs, 9, 10) +
                 c1 * (SF(T_SW21_SELFREF, NG) + FF(T_SW21_FORREF, NG));
        }
        if (k >= lt) {
            jsfs(4, c1, strr, c2, (R)4, oneminus, sc, js, fs);
            tg = sc * sum8(tab<R>(T_SW21_ABSB), NG, 1175, id0, id1, js, fs, 5, 6) +
                 c1 * ffac * interp(tab<R>(T_SW21_FORREF), NG, indf, ig, ffrac);
        }
        break;
    }
    case 22: {
        const int NG = 2;
        idx(22, id0, id1);
        tr = cm * (R)1.54e-08f;
        const R o2cont = (R)4.35e-4f / ((R)350.0f * (R)2.0f) * c6;
        if (k <= lt) {
            R sc, fs; int js;
            jsfs(5, c1, (R)3.63328e-02f, c6, (R)8, oneminus, sc, js, fs, true);
            tg = sc * (sum8(tab<R>(T_SW22_ABSA), NG, 585, id0, id1, js, fs, 9, 10)) +
                 c1 * (SF(T_SW22_SELFREF, NG) + FF(T_SW22_FORREF, NG)) + o2cont;
        } else {
            tg = c6 * (R)1.6f * (sum4(tab<R>(T_SW22_ABSB), NG, 235, id0, id1)) + o2cont;
        }
        break;
    }
    case 23: {
        const int NG = 10;
        tr = cm * ldt(tab<R>(T_SW23_RAYL) + ig);
        const bool zero_cond = (k >= s.kmin8 + 1) && (k >= lt);
        if ((k <= lt) && !zero_cond) {
            const int i0 = (jpk - 1) * 5 + (jtk - 1), i1 = jpk * 5 + (jt1k - 1);
            tg = c1 * ((R)1.029f * sum4(tab<R>(T_SW23_ABSA), NG, 65, i0, i1) + SF(T_SW23_SELFREF, NG) + FF(T_SW23_FORREF, NG));
        } else {
            tg = 0;
        }
        break;
    }
    case 24: {
        const int NG = 8;
        idx(24, id0, id1);
        if (k <= lt) {
            R sc, fs; int js;
            jsfs(6, c1, (R)1.24692e-1f, c6, (R)8, swom, sc, js, fs);
            tg = sc * sum8(tab<R>(T_SW24_ABSA), NG, 585, id0, id1, js, fs, 9, 10) + c3 * ldt(tab<R>(T_SW24_ABSO3A) + ig) +
                 c1 * (SF(T_SW24_SELFREF, NG) + FF(T_SW24_FORREF, NG));
            const R r0 = ldt(tab<R>(T_SW24_RAYLA) + (size_t)(js - 1) * NG + ig), r1 = ldt(tab<R>(T_SW24_RAYLA) + (size_t)js * NG + ig);
            tr = cm * (r0 + fs * (r1 - r0));
        } else {
            tg = c6 * sum4(tab<R>(T_SW24_ABSB), NG, 235, id0, id1) + c3 * ldt(tab<R>(T_SW24_ABSO3B) + ig);
            tr = cm * ldt(tab<R>(T_SW24_RAYLB) + ig);
        }
        break;
    }
    case 25: {
        const int NG = 6;
        tr = cm * ldt(tab<R>(T_SW25_RAYL) + ig);
        tg = 0;
        if (k <= lt) {
            idx(25, id0, id1);
            tg = c1 * sum4(tab<R>(T_SW25_ABSA), NG, 65, id0, id1) + c3 * ldt(tab<R>(T_SW25_ABSO3A) + ig);
        }
        if (k >= s.kminw + 1 && k >= lt) tg = c3 * ldt(tab<R>(T_SW25_ABSO3B) + ig);
        break;
    }
    case 26:
        tg = 0;
        tr = cm * ldt(tab<R>(T_SW26_RAYL) + ig);
        break;
    case 27: {
        const int NG = 8;
        tr = cm * ldt(tab<R>(T_SW27_RAYL) + ig);
        if (k <= lt) { id0 = (jpk - 1) * 5 + (jtk - 1); id1 = jpk * 5 + (jt1k - 1); }
        else { id0 = (jpk - 13) * 5 + (jtk - 1); id1 = (jpk - 12) * 5 + (jt1k - 1); }
        tg = 0;
        if (k < lt) tg = c3 * sum4(tab<R>(T_SW27_ABSA), NG, 65, id0, id1);
        if (k >= lt) tg = c3 * sum4(tab<R>(T_SW27_ABSB), NG, 235, id0, id1);
        break;
    }
    case 28: {
        const int NG = 6;
        idx(28, id0, id1);
        tr = cm * ldt(tab<R>(T_SW28_RAYL));
        const R strr = ldt(tab<R>(T_SW28_STRRAT));
        tg = 0;
        if (k <= lt) {
            R sc, fs; int js;
            jsfs(7, c3, strr, c6, (R)8, swom, sc, js, fs);
            tg = sc * sum8(tab<R>(T_SW28_ABSA), NG, 585, id0, id1, js, fs, 9, 10);
        }
        if (k >= s.kminw + 1 && k >= lt) {
            R sc, fs; int js;
            jsfs(7, c3, strr, c6, (R)4, swom, sc, js, fs);
            tg = sc * sum8(tab<R>(T_SW28_ABSB), NG, 1175, id0, id1, js, fs, 5, 6);
        }
        break;
    }
    default: {   // 29
        const int NG = 12;
        tr = cm * (R)9.30e-11f;
        const bool low = k <= lt;
        const int i0 = low ? (jpk - 1) * 5 + (jtk - 1) : (jpk - 13) * 5 + (jtk - 1);
        const int i1 = low ? jpk * 5 + (jt1k - 1) : (jpk - 12) * 5 + (jt1k - 1);
        if (low) {
            const int indsp = min(inds + 1, 10), indfp = min(indf + 1, 4);
            const R* Sref = tab<R>(T_SW29_SELFREF);
            const R* Fref = tab<R>(T_SW29_FORREF);
            auto Sv = [&](int i) { return ldt(Sref + (size_t)(i - 1) * NG + ig); };
            auto Fv = [&](int i) { return ldt(Fref + (size_t)(i - 1) * NG + ig); };
            tg = c1 * ((sum4(tab<R>(T_SW29_ABSA), NG, 65, i0, i1)) + sfac * (Sv(inds) + sfrac * (Sv(indsp) - Sv(inds))) +
                       ffac * (Fv(indf) + ffrac * (Fv(indfp) - Fv(indf)))) + c2 * ldt(tab<R>(T_SW29_ABSCO2) + ig);
        } else {
            tg = c2 * (sum4(tab<R>(T_SW29_ABSB), NG, 235, i0, i1)) + c1 * ldt(tab<R>(T_SW29_ABSH2O) + ig);
        }
        break;
    }
    }
}

// Solar source of band b (taumol.cu:59-120): sfluxzen of the band's g-points from the reference solar
// source at the layer the band's interpolation uses.
template <class R, class S>
__device__ void sw_sfluxzen(S& s, int b, int nlay)
{
    const int jb = b + 16, lt = s.laytrop;
    const int ibd = (int)ldt(tab<R>(T_SW_IBX) + b), njb = c_sw_ns[b + 1] - c_sw_ns[b], ns = c_sw_ns[b];
    const int lr = (int)ldt(tab<R>(T_SW_LAYREFFR) + b);
    const R* sf01 = tab<R>(T_SW_SFLUXREF01);
    if (jb == 16 || jb == 20 || jb == 23 || jb == 25 || jb == 26 || jb == 29 || jb == 27) {
        const R scl = jb == 27 ? ldt(tab<R>(T_SW_SCALEKUR)) : (R)1;
        for (int j = 0; j < njb; ++j) {
            const R v = ldt(sf01 + (ibd - 1) * 16 + j);
            s.sfluxzen[ns + j] = jb == 27 ? scl * v : v;
        }
    } else {
        int ks;
        const bool two = (jb == 17 || jb == 28);
        if (two) {
            ks = nlay;
            for (int k = lt; k <= nlay - 1; ++k)
                if (s.jp[k - 1] < lr && s.jp[k] >= lr) { ks = k + 1; break; }
        } else {
            ks = lt;
            for (int k = 1; k <= lt - 1; ++k)
                if (s.jp[k - 1] < lr && s.jp[k] >= lr) { ks = k + 1; break; }
        }
        const int ix1 = (int)ldt(tab<R>(T_SW_IX1) + b), ix2 = (int)ldt(tab<R>(T_SW_IX2) + b);
        const R colm1 = s.colamt[ix1 - 1][ks - 1], colm2 = s.colamt[ix2 - 1][ks - 1];
        const R sc = colm1 + ldt(tab<R>(T_SW_STRRAT) + b) * colm2;
        const R sm = ldt(tab<R>(T_SW_SPECWT) + b) * fminR((R)0.999999f, colm1 / sc);
        const int jsi = (int)sm;
        const int js = 1 + jsi;
        const R fs = sm - (R)jsi;
        const R* sf = tab<R>(two ? T_SW_SFLUXREF02 : T_SW_SFLUXREF03);
        const int base = ((ibd - 1) * (two ? 5 : 9)) * 16;
        for (int j = 0; j < njb; ++j) {
            const R x0 = ldt(sf + base + (js - 1) * 16 + j), x1 = ldt(sf + base + js * 16 + j);
            s.sfluxzen[ns + j] = x0 + fs * (x1 - x0);
        }
    }
}

// ------------------------------------------------------------------------------------------------------
// exp(-zb) as spcvrtc evaluates it (spcvrtc.cu:20-43): expansion below 0.06, else the table; `clamped`
// selects the direct-beam index form.
template <class R>
__device__ __forceinline__ R sw_expm(R zb, const R* ex, bool clamped)
{
    if (zb <= (R)0.06f) return (R)1 - zb + (R)0.5f * zb * zb;
    const R ftind = zb / ((R)1.0f / (R)0.278f + zb);
    int it = clamped ? (int)((R)0.5f + (R)10000 * ftind) : (int)(ftind * (R)10000 + (R)0.5f);
    if (clamped) it = max(0, min(10000, it));
    return ldt(ex + it);
}

template <class R>
__device__ __forceinline__ void sw_gam(int mode, R zssa1, R zasy1, R zasy3, R cz, R& g1, R& g2, R& g3)
{
    if (mode == 1) {
        g1 = (R)1.75f - zssa1 * ((R)1 + zasy3);
        g2 = (R)-0.25f - zssa1 * ((R)1 - zasy3);
        g3 = (R)0.5f - zasy3 * cz;
    } else if (mode == 2) {
        g1 = (R)2 - zssa1 * ((R)1.25f + zasy3);
        g2 = (R)0.75f * zssa1 * ((R)1 - zasy1);
        g3 = (R)0.5f - zasy3 * cz;
    } else {
        const R zsr3 = (R)1.7320508f;
        g1 = zsr3 * ((R)2 - zssa1 * ((R)1 + zasy1)) * (R)0.5f;
        g2 = zsr3 * zssa1 * ((R)1 - zasy1) * (R)0.5f;
        g3 = ((R)1 - zsr3 * zasy1 * cz) * (R)0.5f;
    }
}

// Layer R/T (spcvrtc.cu:112-173).  The reference form (kRefForm = true) divides by exp(-k tau); the
// rescaled form multiplies numerator and denominator by exp(-k tau) and is finite for any depth.
template <class T, bool kRefForm>
__device__ __forceinline__ void sw_rt(T ztau1, T zssaw, T zssa1, T g1, T g2, T g3, T g4, T cz, T snt, const T* ex,
                                      T& rb, T& rd, T& tb, T& td)
{
    const T eps1 = (T)1.0e-8f;
    if (zssaw >= (T)0.9999995f) {
        const T za1 = g1 * cz - g3, za2 = g1 * ztau1;
        const T zb2 = sw_expm(fminR(ztau1 * snt, (T)500), ex, false);
        rb = fmaxR((T)0, fminR((T)1, (za2 - za1 * ((T)1 - zb2)) / ((T)1 + za2)));
        tb = fmaxR((T)0, fminR((T)1, (T)1 - rb));
        rd = fmaxR((T)0, fminR((T)1, za2 / ((T)1 + za2)));
        td = fmaxR((T)0, fminR((T)1, (T)1 - rd));
        return;
    }
    const T za1 = g1 * g4 + g2 * g3, za2 = g1 * g3 + g2 * g4;
    const T zrk = sqrtR((g1 - g2) * (g1 + g2));
    const T zrk2 = (T)2 * zrk, zrp = zrk * cz, zrp1 = (T)1 + zrp, zrm1 = (T)1 - zrp;
    T zrpp = (T)1 - zrp * zrp;
    if (fabs(zrpp) < eps1) zrpp = zrpp < 0 ? -eps1 : eps1;
    const T zrkg1 = zrk + g1, zrkg3 = zrk * g3, zrkg4 = zrk * g4;
    const T zr1 = zrm1 * (za2 + zrkg3), zr2 = zrp1 * (za2 - zrkg3), zr3 = zrk2 * (g3 - za2 * cz);
    const T zr4 = zrpp * zrkg1, zr5 = zrpp * (zrk - g1);
    const T zt1 = zrp1 * (za1 + zrkg4), zt2 = zrm1 * (za1 - zrkg4), zt3 = zrk2 * (g4 + za1 * cz);
    const T e1 = sw_expm(fminR(zrk * ztau1, (T)500), ex, false);
    const T e2 = sw_expm(fminR(ztau1 * snt, (T)500), ex, false);
    if (kRefForm) {
        const T zexp1 = (T)1 / e1, zexp2 = (T)1 / e2;
        const T ze1r45 = zr4 * zexp1 + zr5 * e1;
        if (ze1r45 >= -eps1 && ze1r45 <= eps1) {
            rb = eps1;
            tb = e2;
        } else {
            const T zden1 = zssa1 / ze1r45;
            rb = fmaxR((T)0, fminR((T)1, (zr1 * zexp1 - zr2 * e1 - zr3 * e2) * zden1));
            tb = fmaxR((T)0, fminR((T)1, e2 * ((T)1 - (zt1 * zexp1 - zt2 * e1 - zt3 * zexp2) * zden1)));
        }
        const T zden1d = zr4 / (ze1r45 * zrkg1);
        rd = fmaxR((T)0, fminR((T)1, g2 * (zexp1 - e1) * zden1d));
        td = fmaxR((T)0, fminR((T)1, zrk2 * zden1d));
    } else {
        const T e11 = e1 * e1;
        const T D = zr4 + zr5 * e11;                       // ze1r45 * e1
        if (D >= -eps1 * e1 && D <= eps1 * e1) {
            rb = eps1;
            tb = e2;
        } else {
            const T q = zssa1 / D;
            rb = fmaxR((T)0, fminR((T)1, (zr1 - zr2 * e11 - zr3 * e2 * e1) * q));
            tb = fmaxR((T)0, fminR((T)1, e2 - e2 * (zt1 - zt2 * e11) * q + zt3 * e1 * q));
        }
        const T dd = zr4 / (D * zrkg1);
        rd = fmaxR((T)0, fminR((T)1, g2 * ((T)1 - e11) * dd));
        td = fmaxR((T)0, fminR((T)1, zrk2 * e1 * dd));
    }
}

// Layer optics -> R/T for the kernel precision R (exd = the float64 table for the mixed fallback).
template <class R>
__device__ __forceinline__ void sw_layer(R ztau0, R zssa0, R zasy0, int mode, R cz, R snt, const R* ex,
                                         const double* exd, R& rb, R& rd, R& tb, R& td, R& ztau1)
{
    const R oneminus = (R)1.0f - (R)1.0e-6f, ftiny = (R)1.0e-12f;
    const R zssaw = fminR(oneminus, zssa0 / ztau0);
    const R zasyw = zasy0 / fmaxR(ftiny, zssa0);
    const R za1s = zasyw * zasyw, za2s = zssaw * za1s;
    ztau1 = ((R)1 - za2s) * ztau0;
    const R zssa1 = (zssaw - za2s) / ((R)1 - za2s);
    const R zasy1 = zasyw / ((R)1 + zasyw), zasy3 = (R)0.75f * zasy1;
    R g1, g2, g3;
    sw_gam<R>(mode, zssa1, zasy1, zasy3, cz, g1, g2, g3);
    bool fp64_layer = false;
    if (sizeof(R) == 4) {
        // float64 where float loses the result: near-conservative scattering (SSA within 1e-4 of 1, where
        // (g1-g2) cancels) and the direct-beam resonance k*mu0 ~ 1 (1 - (k mu0)^2 divides the beam terms)
        const R zrp = sqrtR((g1 - g2) * (g1 + g2)) * cz;
        fp64_layer = zssaw > (R)(1.0f - 1.0e-4f) || fabs((R)1 - zrp * zrp) < (R)0.01f;
    }
    if (fp64_layer) {
        const double t0 = ztau0, s0 = zssa0, y0 = zasy0;
        const double zsw = fmin((double)(1.0f - 1.0e-6f), s0 / t0);
        const double zaw = y0 / fmax(1.0e-12, s0);
        const double a1 = zaw * zaw, a2 = zsw * a1;
        const double zt1 = (1 - a2) * t0;
        const double zs1 = (zsw - a2) / (1 - a2);
        const double zy1 = zaw / (1 + zaw), zy3 = 0.75 * zy1;
        double g1, g2, g3;
        sw_gam<double>(mode, zs1, zy1, zy3, (double)cz, g1, g2, g3);
        double drb, drd, dtb, dtd;
        sw_rt<double, false>(zt1, zsw, zs1, g1, g2, g3, 1.0 - g3, (double)cz, (double)snt, exd, drb, drd, dtb, dtd);
        rb = (R)drb; rd = (R)drd; tb = (R)dtb; td = (R)dtd;
        return;
    }
    sw_rt<R, (sizeof(R) == 8)>(ztau1, zssaw, zssa1, g1, g2, g3, (R)1 - g3, cz, snt, ex, rb, rd, tb, td);
}

// swflux (spcvrtc.cu:178-215): level fluxes from the layer R/T; arrays 1-based, 1 = surface.
template <class R>
__device__ __forceinline__ void sw_swflux(const R* zrefb, const R* zrefd, const R* ztrab, const R* ztrad,
                                          const R* zldbt, const R* ztdbt, int nlay, R* zfu, R* zfd)
{
    const int nlp1 = nlay + 1;
    R zrupb[NLAY_MAX + 3], zrupd[NLAY_MAX + 3], zrdnd[NLAY_MAX + 3], ztdn[NLAY_MAX + 3];
    zrupb[1] = zrefb[1];
    zrupd[1] = zrefd[1];
    for (int k = 1; k <= nlay; ++k) {
        const int kp = k + 1;
        const R zden1 = (R)1 / ((R)1 - zrupd[k] * zrefd[kp]);
        zrupb[kp] = zrefb[kp] + (ztrad[kp] * ((ztrab[kp] - zldbt[kp]) * zrupd[k] + zldbt[kp] * zrupb[k])) * zden1;
        zrupd[kp] = zrefd[kp] + ztrad[kp] * ztrad[kp] * zrupd[k] * zden1;
    }
    ztdn[nlp1] = 1;
    zrdnd[nlp1] = 0;
    ztdn[nlay] = ztrab[nlp1];
    zrdnd[nlay] = zrefd[nlp1];
    for (int k = nlay; k >= 2; --k) {
        const R zden1 = (R)1 / ((R)1 - zrefd[k] * zrdnd[k]);
        ztdn[k - 1] = ztdbt[k] * ztrab[k] + (ztrad[k] * ((ztdn[k] - ztdbt[k]) + ztdbt[k] * zrefb[k] * zrdnd[k])) * zden1;
        zrdnd[k - 1] = zrefd[k] + ztrad[k] * ztrad[k] * zrdnd[k] * zden1;
    }
    for (int k = 1; k <= nlp1; ++k) {
        const R zden1 = (R)1 / ((R)1 - zrdnd[k] * zrupd[k]);
        zfu[k] = (ztdbt[k] * zrupb[k] + (ztdn[k] - ztdbt[k]) * zrupd[k]) * zden1;
        zfd[k] = ztdbt[k] + (ztdn[k] - ztdbt[k] + ztdbt[k] * zrupb[k] * zrdnd[k]) * zden1;
    }
}

// ------------------------------------------------------------------------------------------------------
using SwBatch = ReqBatch<SwIn>;

template <class R>
__global__ void __launch_bounds__(SW_THREADS) sw_column_kernel(const __grid_constant__ SwBatch bt, SwLut<R> lut,
                                                               const double* exd, int* err)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SwShared<R>& s = *reinterpret_cast<SwShared<R>*>(smem_raw);
    const int d = blockIdx.x;
    if (d >= *bt.req[0].nday) return;
    const int64_t gcol = bt.req[0].daycol[d];
    const int rq = bt.find(gcol);
    const SwIn& a = bt.req[rq];
    const int nlay = a.nlay, nlp1 = nlay + 1;
    if (nlay > NLAY_MAX) {
        if (threadIdx.x == 0) atomicExch(err, RAD_DEV_NLAY);
        return;
    }
    const int64_t N = a.ncol;
    const int64_t col = gcol - bt.off[rq];
    const int tid = threadIdx.x;
    const int iswcliq = a.diagnostic ? 0 : 1;
    auto IN = [&](const float* p, int lev) { return (R)__ldg(p + (size_t)lev * N + col); };
    // ---- phase A1: swrad_prep per layer (swrad.cu:166-240)
    for (int k0 = tid; k0 < nlay; k0 += SW_THREADS) {
        const int kk0 = nlay - 1 - k0;
        const R amdw = (R)28.9644f / (R)18.0154f, amdo3 = (R)28.9644f / (R)47.9982f;
        const R tem1 = (R)100.0f * (R)9.80665f, tem2 = (R)1.0e-20f * (R)1.0e3f * (R)6.0221415e23f;
        s.pavel[k0] = IN(a.plyr, kk0);
        s.tavel[k0] = IN(a.tlyr, kk0);
        const R dl = IN(a.plvl, kk0 + 1) - IN(a.plvl, kk0);
        s.delp[k0] = dl;
        const R qv = IN(a.qlyr, kk0), ov = IN(a.olyr, kk0);
        const R h2o = fmaxR((R)0, qv * amdw / ((R)1 - qv));
        const R o3 = fmaxR((R)0, ov * amdo3);
        s.h2ovmr[k0] = h2o;
        const R tem0 = ((R)1 - h2o) * (R)28.9644f + h2o * (R)18.0154f;
        const R cd = tem2 * dl / (tem1 * tem0 * ((R)1 + h2o));
        s.coldry[k0] = cd;
        const R tc = (R)1.0e-12f * cd;
        auto G = [&](int n) { return (R)__ldg(a.gasvmr + ((size_t)n * nlay + kk0) * N + col); };
        s.colamt[0][k0] = fmaxR((R)0, cd * h2o);
        s.colamt[1][k0] = fmaxR(tc, cd * G(0));
        s.colamt[2][k0] = fmaxR((R)0, cd * o3);
        s.colmol[k0] = cd + s.colamt[0][k0];
        s.colamt[3][k0] = fmaxR(tc, cd * G(1));
        s.colamt[4][k0] = fmaxR(tc, cd * G(2));
        s.colamt[5][k0] = fmaxR(tc, cd * G(3));
        for (int ib = 0; ib < 14; ++ib) {
            R ta = 0, sa = 0, ya = 0;
            if (a.faersw) {
                ta = (R)__ldg(a.faersw + (((size_t)ib) * nlay + kk0) * N + col);
                sa = (R)__ldg(a.faersw + (((size_t)(14 + ib)) * nlay + kk0) * N + col);
                ya = (R)__ldg(a.faersw + (((size_t)(28 + ib)) * nlay + kk0) * N + col);
            }
            s.tauae[ib][k0] = ta; s.ssaae[ib][k0] = sa; s.asyae[ib][k0] = ya;
        }
        s.cfrac[k0] = (R)__ldg(a.clouds + (size_t)kk0 * N + col);
        // setcoef (setcoef.cu:17-97)
        const R pav = s.pavel[k0], tav = s.tavel[k0];
        const R forf = pav * ((R)296.0f / (R)1013.0f) / (tav * ((R)1 + h2o));
        s.forfac[k0] = forf;
        const R plog = rlog(pav);
        const int jpk = max(1, min(58, (int)((R)36 - (R)5 * (plog + (R)0.04f))));
        const int jp1 = jpk + 1;
        const R* preflog = tab<R>(T_SW_PREFLOG);
        const R* tref = tab<R>(T_SW_TREF);
        const R fp = (R)5 * (ldt(preflog + jpk - 1) - plog);
        const R t1 = (tav - ldt(tref + jpk - 1)) / (R)15, t2 = (tav - ldt(tref + jp1 - 1)) / (R)15;
        const int jtk = max(1, min(4, (int)((R)3 + t1))), jt1k = max(1, min(4, (int)((R)3 + t2)));
        const R ft = t1 - (R)(jtk - 3), ft1 = t2 - (R)(jt1k - 3);
        s.jp[k0] = jpk; s.jt[k0] = jtk; s.jt1[k0] = jt1k;
        const R fp1 = (R)1 - fp;
        s.fac10[k0] = fp1 * ft;
        s.fac00[k0] = fp1 * ((R)1 - ft);
        s.fac11[k0] = fp * ft1;
        s.fac01[k0] = fp * ((R)1 - ft1);
        if (plog > (R)4.56f) {
            const R tem1f = ((R)332 - tav) / (R)36;
            const int indf = min(2, max(1, (int)tem1f));
            s.indfor[k0] = indf;
            s.forfrac[k0] = tem1f - (R)indf;
            const R tem2s = (tav - (R)188) / (R)7.2f;
            const int inds = min(9, max(1, (int)tem2s - 7));
            s.indself[k0] = inds;
            s.selffrac[k0] = tem2s - (R)(inds + 7);
            s.selffac[k0] = h2o * forf;
        } else {
            const R tem1f = (tav - (R)188) / (R)36;
            s.indfor[k0] = 3;
            s.forfrac[k0] = tem1f - (R)1;
            s.indself[k0] = 0;
            s.selffrac[k0] = 0;
            s.selffac[k0] = 0;
        }
    }
    __syncthreads();
    // ---- column scalars (thread 0): sun, albedo, overlap fractions, laytrop
    if (tid == 0) {
        const R cz = (R)__ldg(a.coszen + col);
        s.cosz = cz;
        s.sntz = (R)1 / cz;
        s.ssolar = ((R)a.solcon / (R)1368.22f) * cz;
        s.albbm[0] = (R)__ldg(a.sfcalb + col);
        s.albdf[0] = (R)__ldg(a.sfcalb + N + col);
        s.albbm[1] = (R)__ldg(a.sfcalb + 2 * N + col);
        s.albdf[1] = (R)__ldg(a.sfcalb + 3 * N + col);
        const R z0 = sw_zcf0<R>(s.cfrac, nlay, a.iovr);
        s.zcf0 = z0;
        s.zcf1 = (R)1 - z0;
        int lt = nlay;
        for (int k0 = 0; k0 < nlay; ++k0)
            if (rlog(s.pavel[k0]) > (R)4.56f) lt = k0 + 1;
        s.laytrop = lt;
        s.kmin8 = a.kmin8[d];
        s.kminw = a.kminw[d];
    }
    __syncthreads();
    // ---- phase A2: cloud optics per (band, layer) (sw_cldprop.cu), solar source per band
    for (int p = tid; p < 14 * nlay; p += SW_THREADS) {
        const int ib = p / nlay, k0 = p - ib * nlay;
        const int kk0 = nlay - 1 - k0;
        auto CLD = [&](int n) { return (R)__ldg(a.clouds + ((size_t)n * nlay + kk0) * N + col); };
        R tcw = 0, scw = 0, acw = 0;
        const R ftiny = (R)1.0e-12f;
        if (s.zcf1 > 0) {
            scw = 1;
            const R cf = s.cfrac[k0];
            if (iswcliq > 0) {
                if (cf > ftiny) {
                    const float b0r[14] = {0.466f, 0.437f, 0.416f, 0.391f, 0.374f, 0.352f, 0.183f, 0.048f, 0.012f, 0.000f, 0.000f, 0.000f, 0.000f, 0.496f};
                    const float c0r[14] = {0.975f, 0.965f, 0.960f, 0.955f, 0.952f, 0.950f, 0.944f, 0.894f, 0.884f, 0.883f, 0.883f, 0.883f, 0.883f, 0.980f};
                    const float b0s[14] = {0.460f, 0.460f, 0.460f, 0.460f, 0.460f, 0.460f, 0.460f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.460f};
                    const float b1s[14] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.62e-5f, 1.62e-5f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
                    const float c0s[14] = {0.970f, 0.970f, 0.970f, 0.970f, 0.970f, 0.970f, 0.970f, 0.970f, 0.970f, 0.700f, 0.700f, 0.700f, 0.700f, 0.970f};
                    const R cldran = CLD(5), cldsnw = CLD(7), refsnw = CLD(8);
                    const R dgesnw = (R)1.0315f * refsnw;
                    const R tauran = cldran * (R)3.07e-3f;
                    const R tausnw = (cldsnw > 0 && refsnw > (R)10) ? cldsnw * (R)1.09087f * ((R)0 + (R)1.5f / dgesnw) : (R)0;
                    const R ssaran = tauran * ((R)1 - (R)b0r[ib]);
                    const R ssasnw = tausnw * ((R)1 - ((R)b0s[ib] + (R)b1s[ib] * dgesnw));
                    const R asyran = ssaran * (R)c0r[ib], asysnw = ssasnw * (R)c0s[ib];
                    const R cldliq = CLD(1), refliq = CLD(2), cldice = CLD(3), refice = CLD(4);
                    R tl = 0, sl = 0, al = 0, ti = 0, si = 0, ai = 0;
                    if (!(cldliq <= 0)) {
                        const R factor = refliq - (R)1.5f;
                        const int index = max(1, min(57, (int)factor));
                        const R fint = factor - (R)index;
                        const R *e = tab<R>(T_SW_EXTLIQ1) + ib * 58, *sv = tab<R>(T_SW_SSALIQ1) + ib * 58, *av = tab<R>(T_SW_ASYLIQ1) + ib * 58;
                        const R ext = fmaxR((R)0, ldt(e + index - 1) + fint * (ldt(e + index) - ldt(e + index - 1)));
                        const R ssa = fmaxR((R)0, fminR((R)1, ldt(sv + index - 1) + fint * (ldt(sv + index) - ldt(sv + index - 1))));
                        const R asy = fmaxR((R)0, fminR((R)1, ldt(av + index - 1) + fint * (ldt(av + index) - ldt(av + index - 1))));
                        tl = cldliq * ext; sl = tl * ssa; al = sl * asy;
                    }
                    if (!(cldice <= 0)) {
                        const R dge = fmaxR((R)5, fminR((R)140, (R)1.0315f * refice));
                        const R factor = (dge - (R)2) / (R)3;
                        const int index = max(1, min(45, (int)factor));
                        const R fint = factor - (R)index;
                        const R *e = tab<R>(T_SW_EXTICE3) + ib * 46, *sv = tab<R>(T_SW_SSAICE3) + ib * 46, *av = tab<R>(T_SW_ASYICE3) + ib * 46;
                        const R ext = fmaxR((R)0, ldt(e + index - 1) + fint * (ldt(e + index) - ldt(e + index - 1)));
                        const R ssa = fmaxR((R)0, fminR((R)1, ldt(sv + index - 1) + fint * (ldt(sv + index) - ldt(sv + index - 1))));
                        const R asy = fmaxR((R)0, fminR((R)1, ldt(av + index - 1) + fint * (ldt(av + index) - ldt(av + index - 1))));
                        ti = cldice * ext; si = ti * ssa; ai = si * asy;
                    }
                    tcw = tl + ti + tauran + tausnw;
                    scw = sl + si + ssaran + ssasnw;
                    acw = al + ai + asyran + asysnw;
                }
            } else if (cf > ftiny) {
                tcw = CLD(1);
                scw = CLD(1) * CLD(2);
                acw = scw * CLD(3);
            }
        }
        s.taucw[ib][k0] = tcw; s.ssacw[ib][k0] = scw; s.asycw[ib][k0] = acw;
        if (ib == 0) s.cldfrc[k0] = s.zcf1 > 0 ? s.cfrac[k0] / s.zcf1 : (R)0;
    }
    if (tid < 14) sw_sfluxzen<R>(s, tid, nlay);
    __syncthreads();
    // ---- phase B: gas and Rayleigh optical depths per (g, layer), g-major
    for (int p = tid; p < SW_NGPT * nlay; p += SW_THREADS) {
        const int g = p / nlay, k0 = p - g * nlay;
        R tg, tr;
        sw_gas(s, g, k0, tg, tr);
        s.taug[g][k0] = tg;
        s.taur[g][k0] = tr;
    }
    __syncthreads();
    // ---- phase C: spcvrtc per g-point (one lane each), clear and cloudy passes
    const int warp = tid >> 5, lane = tid & 31;
    const int g = tid;
    const bool act = g < SW_NGPT;
    int ib0 = 0;
    if (act)
        while (g >= c_sw_ns[ib0 + 1]) ++ib0;
    const int IDXSFC[14] = {1, 1, 1, 1, 1, 1, 1, 1, 0, 2, 2, 2, 2, 1};
    const int ibd = IDXSFC[ib0];
    const R eps = (R)1.0e-6f, ftiny = (R)1.0e-12f;
    const R cz = s.cosz, snt = s.sntz, cf1v = s.zcf1;
    const bool cloudy = cf1v > eps;
    R zrefb[NLAY_MAX + 3], zrefd[NLAY_MAX + 3], ztrab[NLAY_MAX + 3], ztrad[NLAY_MAX + 3], ztdbt[NLAY_MAX + 3],
        zldbt[NLAY_MAX + 3], zfu[NLAY_MAX + 3], zfd[NLAY_MAX + 3], zldbt0[NLAY_MAX + 3];
    const R zsolar = act ? s.ssolar * s.sfluxzen[g] : (R)0;
    for (int pass = 0; pass < (cloudy ? 2 : 1); ++pass) {
        R ztdbt0 = 1;
        if (act) {
            ztdbt[nlp1] = 1;
            zldbt[1] = 0;
            if (ibd != 0) { zrefb[1] = s.albbm[ibd - 1]; zrefd[1] = s.albdf[ibd - 1]; }
            else { zrefb[1] = (R)0.5f * (s.albbm[0] + s.albbm[1]); zrefd[1] = (R)0.5f * (s.albdf[0] + s.albdf[1]); }
            ztrab[1] = 0;
            ztrad[1] = 0;
            for (int k = nlay; k >= 1; --k) {
                const int kp = k + 1, q = k - 1;
                const R ta = s.tauae[ib0][q], sa = s.ssaae[ib0][q], ya = s.asyae[ib0][q];
                const R ct0 = fmaxR(ftiny, s.taur[g][q] + s.taug[g][q] + ta);
                const R cs0 = s.taur[g][q] + ta * sa;
                const R cy0 = ya * sa * ta;
                R rb, rd, tb, td, ztau1;
                sw_layer(ct0, cs0, cy0, a.iswmode, cz, snt, lut.ex, exd, rb, rd, tb, td, ztau1);
                R e3 = sw_expm(ztau1 * snt, lut.ex, true);
                R e4 = sw_expm(ct0 * snt, lut.ex, true);
                const R zc1 = s.cldfrc[q];
                if (pass == 1 && zc1 > ftiny) {
                    const R zc0 = (R)1 - zc1;
                    const R ot0 = ct0 + s.taucw[ib0][q], os0 = cs0 + s.ssacw[ib0][q], oy0 = cy0 + s.asycw[ib0][q];
                    R rb2, rd2, tb2, td2, ztau1c;
                    sw_layer(ot0, os0, oy0, a.iswmode, cz, snt, lut.ex, exd, rb2, rd2, tb2, td2, ztau1c);
                    rb = zc0 * rb + zc1 * rb2;
                    rd = zc0 * rd + zc1 * rd2;
                    tb = zc0 * tb + zc1 * tb2;
                    td = zc0 * td + zc1 * td2;
                    e3 = zc0 * e3 + zc1 * sw_expm(ztau1c * snt, lut.ex, true);
                    e4 = zc0 * e4 + zc1 * sw_expm(ot0 * snt, lut.ex, true);
                }
                zrefb[kp] = rb; zrefd[kp] = rd; ztrab[kp] = tb; ztrad[kp] = td;
                zldbt[kp] = e3;
                ztdbt[k] = e3 * ztdbt[kp];
                zldbt0[k] = e4;
                ztdbt0 = e4 * ztdbt0;
            }
            sw_swflux(zrefb, zrefd, ztrab, ztrad, zldbt, ztdbt, nlay, zfu, zfd);
        }
        // per-level net flux (down - up) summed over the warp's g-points
        for (int k = 1; k <= nlp1; ++k) {
            double f = act ? (double)(zsolar * zfd[k]) - (double)(zsolar * zfu[k]) : 0.0;
            f = warp_sum(f);
            if (lane == 0) (pass == 0 ? s.fn0 : s.fnc)[warp][k - 1] = f;
        }
        // scalars: toa up, toa down, sfc up, sfc down, uv-b, nir beam, nir diffuse, uv-vis beam, uv-vis diffuse
        double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (act) {
            v[0] = (double)(zsolar * zfu[nlp1]);
            v[1] = (double)(zsolar * zfd[nlp1]);
            v[2] = (double)(zsolar * zfu[1]);
            v[3] = (double)(zsolar * zfd[1]);
            v[4] = ib0 == 11 ? (double)(zsolar * zfd[1]) : 0.0;
            const double zb1 = (double)(zsolar * ztdbt0), zb2 = (double)(zsolar * (zfd[1] - ztdbt0));
            if (ibd == 1) { v[5] = zb1; v[6] = zb2; }
            else if (ibd == 2) { v[7] = zb1; v[8] = zb2; }
            else { v[5] = 0.5 * zb1; v[6] = 0.5 * zb2; v[7] = 0.5 * zb1; v[8] = 0.5 * zb2; }
        }
        for (int i = 0; i < 9; ++i) v[i] = warp_sum(v[i]);
        if (lane == 0)
            for (int i = 0; i < 9; ++i) s.sc[warp][pass * 9 + i] = v[i];
        __syncwarp();
    }
    __syncthreads();
    // ---- column end (spcvrtc.cu:493-545) and swrad_post (swrad.cu:365-403)
    const double heatfac = sizeof(R) == 4 ? (double)(float)(9.80665 * 1.0e-2 / 1.0046e3) : 9.80665 * 1.0e-2 / 1.0046e3;
    const double c1d = (double)s.zcf1, c0d = (double)s.zcf0;
    auto tot = [&](double clr, double cld) { return cloudy ? c1d * cld + c0d * clr : clr; };
    for (int k = tid; k < nlay; k += SW_THREADS) {
        double a0 = 0, a1 = 0, b0 = 0, b1 = 0;
        for (int w = 0; w < SW_WARPS; ++w) {
            a0 += s.fn0[w][k]; a1 += s.fn0[w][k + 1];
            if (cloudy) { b0 += s.fnc[w][k]; b1 += s.fnc[w][k + 1]; }
        }
        const double fk = tot(a0, b0), fk1 = tot(a1, b1);
        a.htsw[(size_t)(nlay - 1 - k) * N + col] = (float)((fk1 - fk) * (heatfac / (double)s.delp[k]));
    }
    if (tid == 0) {
        double c[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, t[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int w = 0; w < SW_WARPS; ++w)
            for (int i = 0; i < 9; ++i) {
                c[i] += s.sc[w][i];
                t[i] += cloudy ? s.sc[w][9 + i] : 0.0;
            }
        // slots: 0 toa up, 1 toa dn, 2 sfc up, 3 sfc dn, 4 uv-b, 5 nir beam, 6 nir diffuse, 7 vis beam, 8 vis diffuse
        a.topfsw[col] = (float)tot(c[0], t[0]);
        a.topfsw[N + col] = (float)c[1];
        a.topfsw[2 * N + col] = (float)c[0];
        a.sfcfsw[col] = (float)tot(c[2], t[2]);
        a.sfcfsw[N + col] = (float)tot(c[3], t[3]);
        a.sfcfsw[2 * N + col] = (float)c[2];
        a.sfcfsw[3 * N + col] = (float)c[3];
        if (a.fdncmp) {
            a.fdncmp[col] = (float)c[4];
            a.fdncmp[N + col] = (float)tot(c[4], t[4]);
            a.fdncmp[2 * N + col] = (float)tot(c[5], t[5]);
            a.fdncmp[3 * N + col] = (float)tot(c[6], t[6]);
            a.fdncmp[4 * N + col] = (float)tot(c[7], t[7]);
            a.fdncmp[5 * N + col] = (float)tot(c[8], t[8]);
        }
    }
}

}  // namespace rad
