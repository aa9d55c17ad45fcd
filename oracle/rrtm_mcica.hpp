// rrtm_mcica.hpp -- CPU oracle: the McICA route (test infrastructure only).
//
//   sub-column generators  namgpu/kernels/phys_rrtm_lw_mcica_subcol.cu:48-191 (radlw mcica_subcol)
//                          namgpu/kernels/phys_rrtm_sw_mcica_subcol.cu:63-203 (radsw mcica_subcol)
//   LW transfer            namgpu/kernels/phys_rrtm_lw_rtrnmc.cu:85-310 (rtrnmc)
//   SW transfer            spcvrtc's layer solver and adding method with the per-g-point binary cloud of
//                          the SW masks in place of the cloud-fraction blend (the reference has no spcvmc).
//
// The random stream is MT19937 (Matsumoto and Nishimura, ACM TOMACS 8, 3-30, 1998) with the seeding,
// tempering and float conversion the reference applies: mt[0] = seed (0 -> 4357), mt[i] = 69069 mt[i-1]
// mod 2^32; a draw is the tempered word over 2^32 in float (words read as negative int32 get 2^32 added in
// float first).  Masks are bit-packed [word][layer][column], bit g & 31 of word g >> 5, layers surface first.
#pragma once
#include "rrtm_lw.hpp"
#include "rrtm_sw.hpp"

namespace orc {

struct Mt19937 {
    uint32_t mt[624];
    int mti = 624;
    explicit Mt19937(int seed)
    {
        mt[0] = seed == 0 ? 4357u : (uint32_t)seed;
        for (int i = 1; i < 624; ++i) mt[i] = 69069u * mt[i - 1];
        mti = 624;
    }
    void twist()
    {
        const uint32_t upper = 0x80000000u, lower = 0x7fffffffu, a = 0x9908b0dfu;
        for (int k = 0; k < 624; ++k) {
            const uint32_t y = (mt[k] & upper) | (mt[(k + 1) % 624] & lower);
            mt[k] = mt[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? a : 0u);
        }
        mti = 0;
    }
    float next()
    {
        if (mti >= 624) twist();
        uint32_t y = mt[mti++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        y ^= y >> 18;
        const int32_t ys = (int32_t)y;
        const float two32 = 4294967296.0f;
        if (ys < 0) return ((float)ys + two32) / two32;
        return (float)ys / two32;
    }
};

// Sub-column cloud bits of one column: words[w * nlay + k0], cf[k0] the layer cloud fraction (surface
// first), iovr 0 random, 1 maximum-random, 2 maximum overlap.
inline void mcica_bits(const std::vector<float>& cf, int nlay, int ngpt, int iovr, int seed, std::vector<uint32_t>& words)
{
    const int nword = (ngpt + 31) / 32;
    words.assign((size_t)nword * nlay, 0u);
    Mt19937 r(seed);
    auto set = [&](int g, int k0) { words[(size_t)(g >> 5) * nlay + k0] |= 1u << (g & 31); };
    if (iovr == 0) {
        for (int g = 0; g < ngpt; ++g)
            for (int k0 = 0; k0 < nlay; ++k0)
                if (r.next() >= 1.0f - cf[k0]) set(g, k0);
    } else if (iovr == 1) {
        for (int g = 0; g < ngpt; ++g) {
            float prev = 0;
            for (int k0 = 0; k0 < nlay; ++k0) {
                const float x = r.next();
                float cd;
                if (k0 == 0) cd = x;
                else {
                    const float tem1 = 1.0f - cf[k0 - 1];
                    cd = prev > tem1 ? prev : x * tem1;
                }
                prev = cd;
                if (cd >= 1.0f - cf[k0]) set(g, k0);
            }
        }
    } else if (iovr == 2) {
        for (int g = 0; g < ngpt; ++g) {
            const float x = r.next();
            for (int k0 = 0; k0 < nlay; ++k0)
                if (x >= 1.0f - cf[k0]) set(g, k0);
        }
    }
}

inline bool mask_bit(const std::vector<uint32_t>& words, int nlay, int g, int k0)
{
    return (words[(size_t)(g >> 5) * nlay + k0] >> (g & 31)) & 1u;
}

// LW generator of column col: cldf = the input cloud fraction in internal order, zero for a column whose
// layers all have cloud fraction <= 1e-6 (the lcf1 gate of cldprop); seed icseed[col] or lw_seed0 + col + 1.
// Fills c.cldfmc [140][nlay] with 1/0 and writes the packed words to out (may be null) [5][nlay][ncol].
template <class R>
void lw_mcica(LwColumn<R>& c, const float*, int, const Config& cfg, const Inputs& in, int col, unsigned int* out)
{
    const int nlay = c.nlay;
    std::vector<float> cf(nlay, 0.0f);
    if (c.lcf1)
        for (int k0 = 0; k0 < nlay; ++k0) cf[k0] = in.clouds[(size_t)(nlay - 1 - k0) * in.ncol + col];
    const int seed = in.icseed ? in.icseed[col] : cfg.lw_seed0 + col + 1;
    std::vector<uint32_t> w;
    mcica_bits(cf, nlay, 140, cfg.iovrlw, seed, w);
    c.cldfmc.assign((size_t)140 * nlay, 0);
    for (int g = 0; g < 140; ++g)
        for (int k0 = 0; k0 < nlay; ++k0) c.cldfmc[(size_t)g * nlay + k0] = mask_bit(w, nlay, g, k0) ? (R)1 : (R)0;
    if (out)
        for (int ww = 0; ww < 5; ++ww)
            for (int k0 = 0; k0 < nlay; ++k0) out[((size_t)ww * nlay + k0) * in.ncol + col] = w[(size_t)ww * nlay + k0];
}

// rtrnmc (phys_rrtm_lw_rtrnmc.cu:85-310): per band, per g-point, the down/up sweeps with the binary
// sub-column cloud and effective clear fraction efclrfr = 1 - (1 - exp(-odcld)) cldfmc.
template <class R>
void lw_rtrnmc(LwColumn<R>& c, const LwTables<R>& tb, R heatfac, R fluxfac)
{
    const int nlay = c.nlay, nlp1 = nlay + 1;
    const R eps = (R)1.0e-6f, bpade = (R)1.0f / (R)0.278f, tblint = (R)10000, rec_6 = (R)0.166667f,
            c06 = (R)0.06f;
    const R flxfac = (R)0.5f * fluxfac;
    std::vector<R> gassrcu(nlay), totsrcu(nlay), trngas(nlay), efclrfr(nlay);
    std::vector<R> tur(nlp1), tdr(nlp1), cur(nlp1), cdr(nlp1), tuf(nlp1, 0), tdf(nlp1, 0), tuc(nlp1, 0), tdc(nlp1, 0);
    auto PKL = [&](int ib, int s) { return c.pklay[(size_t)s * 16 + ib]; };
    auto PKV = [&](int ib, int s) { return c.pklev[(size_t)s * 16 + ib]; };
    for (int ib = 0; ib < 16; ++ib) {
        const R semi = c.semiss[ib], sdif = c.secdiff[ib];
        for (int k = 0; k <= nlay; ++k) { tur[k] = 0; tdr[k] = 0; cur[k] = 0; cdr[k] = 0; }
        for (int g = LW_NS[ib]; g < LW_NS[ib] + LW_NG[ib]; ++g) {
            R radtotd = 0, radclrd = 0;
            for (int k = nlay; k >= 1; --k) {
                R odepth = fmaxR((R)0, sdif * c.TG(g, k - 1));
                R atrgas, trng, gasfac;
                if (odepth <= c06) {
                    atrgas = odepth - (R)0.5f * odepth * odepth;
                    trng = (R)1 - atrgas;
                    gasfac = rec_6 * odepth;
                } else {
                    const R tblind = odepth / (bpade + odepth);
                    const int it = (int)(tblint * tblind + (R)0.5f);
                    trng = tb.ex[it]; atrgas = (R)1 - trng; gasfac = tb.tfn[it]; odepth = tb.tau[it];
                }
                const R plfrac = c.FR(g, k - 1);
                const R blay = PKL(ib, k);
                const R dplnku = PKV(ib, k) - blay, dplnkd = PKV(ib, k - 1) - blay;
                const R bbdgas = plfrac * (blay + dplnkd * gasfac), bbugas = plfrac * (blay + dplnku * gasfac);
                const R gassrcd = bbdgas * atrgas;
                gassrcu[k - 1] = bbugas * atrgas;
                trngas[k - 1] = trng;
                const R clfm = c.cldfmc[(size_t)g * nlay + (k - 1)];
                if (clfm >= eps) {
                    const R odcld = sdif * c.taucld[(size_t)ib * nlay + (k - 1)];
                    efclrfr[k - 1] = (R)1 - ((R)1 - mexp(-odcld)) * clfm;
                    const R odtot = odepth + odcld;
                    R totfac, atrtot;
                    if (odtot < c06) {
                        totfac = rec_6 * odtot;
                        atrtot = odtot - (R)0.5f * odtot * odtot;
                    } else {
                        const R tblind = odtot / (bpade + odtot);
                        const int it = (int)(tblint * tblind + (R)0.5f);
                        totfac = tb.tfn[it];
                        atrtot = (R)1 - tb.ex[it];
                    }
                    const R bbdtot = plfrac * (blay + dplnkd * totfac), bbutot = plfrac * (blay + dplnku * totfac);
                    const R totsrcd = bbdtot * atrtot;
                    totsrcu[k - 1] = bbutot * atrtot;
                    radtotd = radtotd * trng * efclrfr[k - 1] + gassrcd + clfm * (totsrcd - gassrcd);
                    tdr[k - 1] = tdr[k - 1] + radtotd;
                    radclrd = radclrd * trng + gassrcd;
                    cdr[k - 1] = cdr[k - 1] + radclrd;
                } else {
                    radtotd = radtotd * trng + gassrcd;
                    tdr[k - 1] = tdr[k - 1] + radtotd;
                    radclrd = radclrd * trng + gassrcd;
                    cdr[k - 1] = cdr[k - 1] + radclrd;
                }
            }
            const R reflct = (R)1 - semi;
            const R rad0 = semi * c.FR(g, 0) * PKL(ib, 0);
            R radtotu = rad0 + reflct * radtotd;
            tur[0] = tur[0] + radtotu;
            R radclru = rad0 + reflct * radclrd;
            cur[0] = cur[0] + radclru;
            for (int k = 1; k <= nlay; ++k) {
                const R clfm = c.cldfmc[(size_t)g * nlay + (k - 1)];
                const R trng = trngas[k - 1], gasu = gassrcu[k - 1];
                if (clfm > eps) {
                    radtotu = radtotu * trng * efclrfr[k - 1] + gasu + clfm * (totsrcu[k - 1] - gasu);
                    tur[k] = tur[k] + radtotu;
                    radclru = radclru * trng + gasu;
                    cur[k] = cur[k] + radclru;
                } else {
                    radtotu = radtotu * trng + gasu;
                    tur[k] = tur[k] + radtotu;
                    radclru = radclru * trng + gasu;
                    cur[k] = cur[k] + radclru;
                }
            }
        }
        for (int k = 0; k <= nlay; ++k) {
            tuf[k] = tuf[k] + tur[k]; tdf[k] = tdf[k] + tdr[k];
            tuc[k] = tuc[k] + cur[k]; tdc[k] = tdc[k] + cdr[k];
            c.fnetb[(size_t)ib * (nlay + 1) + k] = (tur[k] - tdr[k]) * flxfac;
        }
    }
    for (int k = 0; k <= nlay; ++k) {
        c.totuflux[k] = tuf[k] * flxfac; c.totdflux[k] = tdf[k] * flxfac;
        c.totuclfl[k] = tuc[k] * flxfac; c.totdclfl[k] = tdc[k] * flxfac;
    }
    R fprev = c.totuflux[0] - c.totdflux[0];
    for (int k = 1; k <= nlay; ++k) {
        const R fk = c.totuflux[k] - c.totdflux[k];
        c.htr[k - 1] = (fprev - fk) * (heatfac / c.delp[k - 1]);
        fprev = fk;
    }
    (void)nlp1;
}

// SW generator of column col: cldf = the input cloud fraction in internal order with values below 1e-12
// set to 0; seed icseed[ncol + col] or sw_seed0 + col + 1.  Writes packed words [4][nlay][ncol] to out.
inline void sw_mcica_words(const Config& cfg, const Inputs& in, int col, std::vector<uint32_t>& w)
{
    const int nlay = in.nlay;
    std::vector<float> cf(nlay);
    for (int k0 = 0; k0 < nlay; ++k0) {
        const float x = in.clouds[(size_t)(nlay - 1 - k0) * in.ncol + col];
        cf[k0] = x < 1.0e-12f ? 0.0f : x;
    }
    const int seed = in.icseed ? in.icseed[(size_t)in.ncol + col] : cfg.sw_seed0 + col + 1;
    mcica_bits(cf, nlay, 112, cfg.iovrsw, seed, w);
}

template <class R>
void sw_mcica(SwColumn<R>& c, const Config& cfg, const Inputs& in, int col, unsigned int*)
{
    std::vector<uint32_t> w;
    sw_mcica_words(cfg, in, col, w);
    const int nlay = c.nlay;
    c.cldfmc.assign((size_t)112 * nlay, 0);
    for (int g = 0; g < 112; ++g)
        for (int k0 = 0; k0 < nlay; ++k0) c.cldfmc[(size_t)g * nlay + k0] = mask_bit(w, nlay, g, k0) ? (R)1 : (R)0;
}

// spcvrtc with the McICA cloud: the clear pass as spcvrtc; the total-sky pass takes, per g-point, the
// cloud-mixture optics in the cloudy layers (cloud fraction above 1e-12) whose sub-column bit is set and the
// clear optics elsewhere, with no cloud-fraction blend; total-sky outputs come from that pass alone.
template <class R>
void sw_spcvrtm(SwColumn<R>& c, const SwExpTable<R>& tb, int iswmode)
{
    // Run spcvrtc with the cloud fractions of the layers replaced per g-point: reuse sw_spcvrtc on a
    // column copy per g-point would cost 112 full solves, so the loop is restated here.
    static const int IDXSFC[14] = {1, 1, 1, 1, 1, 1, 1, 1, 0, 2, 2, 2, 2, 1};
    const int nlay = c.nlay, nlp1 = nlay + 1;
    const R oneminus = (R)1.0f - (R)1.0e-6f, ftiny = (R)1.0e-12f;
    const int LP = nlp1 + 2;
    std::vector<R> zrefb(LP), zrefd(LP), ztrab(LP), ztrad(LP), ztdbt(LP), zldbt(LP), zfu(LP), zfd(LP);
    for (auto* v : {&c.fxupc, &c.fxdnc, &c.fxup0, &c.fxdn0})
        for (auto& x : *v) x = 0;
    for (int n = 0; n < 2; ++n) { c.sfbmc[n] = c.sfdfc[n] = c.sfbm0[n] = c.sfdf0[n] = 0; }
    const R cz = c.cosz, snt = c.sntz;
    auto FX = [&](std::vector<R>& v, int ib, int k) -> R& { return v[(size_t)ib * nlp1 + k]; };
    auto layer = [&](R ztau0, R zssa0, R zasy0, int kp, R& e3, R& e4) {
        const R zssaw = fminR(oneminus, zssa0 / ztau0);
        const R zasyw = zasy0 / fmaxR(ftiny, zssa0);
        const R za1s = zasyw * zasyw, za2s = zssaw * za1s;
        const R ztau1 = ((R)1 - za2s) * ztau0;
        const R zssa1 = (zssaw - za2s) / ((R)1 - za2s);
        const R zasy1 = zasyw / ((R)1 + zasyw), zasy3 = (R)0.75f * zasy1;
        R g1, g2, g3;
        sw_gam(iswmode, zssa1, zasy1, zasy3, cz, g1, g2, g3);
        sw_layer_rt(ztau1, zssaw, zssa1, g1, g2, g3, (R)1 - g3, cz, snt, tb, zrefb[kp], zrefd[kp], ztrab[kp], ztrad[kp]);
        e3 = sw_expm(ztau1 * snt, tb, true);
        e4 = sw_expm(ztau0 * snt, tb, true);
    };
    for (int jg = 0; jg < 112; ++jg) {
        int ib0 = 0;
        while (!(jg >= SW_NS[ib0] && jg < SW_NS[ib0] + SW_NG[ib0])) ++ib0;
        const int ibd = IDXSFC[ib0];
        const R zsolar = c.ssolar * c.sfluxzen[jg];
        for (int pass = 0; pass < 2; ++pass) {
            R ztdbt0 = 1;
            ztdbt[nlp1] = 1;
            zldbt[1] = 0;
            if (ibd != 0) { zrefb[1] = c.albbm[ibd - 1]; zrefd[1] = c.albdf[ibd - 1]; }
            else { zrefb[1] = (R)0.5f * (c.albbm[0] + c.albbm[1]); zrefd[1] = (R)0.5f * (c.albdf[0] + c.albdf[1]); }
            ztrab[1] = 0;
            ztrad[1] = 0;
            for (int k = nlay; k >= 1; --k) {
                const int kp = k + 1, q = k - 1;
                const R ta = c.tauae[(size_t)ib0 * nlay + q], sa = c.ssaae[(size_t)ib0 * nlay + q],
                        ya = c.asyae[(size_t)ib0 * nlay + q];
                R t0 = fmaxR(ftiny, c.TR(jg, q) + c.TG(jg, q) + ta), s0 = c.TR(jg, q) + ta * sa, y0 = ya * sa * ta;
                if (pass == 1 && c.cldfmc[(size_t)jg * nlay + q] > ftiny && c.cldfrc[q] > ftiny) {
                    t0 = t0 + c.taucw[(size_t)ib0 * nlay + q];
                    s0 = s0 + c.ssacw[(size_t)ib0 * nlay + q];
                    y0 = y0 + c.asycw[(size_t)ib0 * nlay + q];
                }
                R e3, e4;
                layer(t0, s0, y0, kp, e3, e4);
                ztdbt[k] = e3 * ztdbt[kp];
                zldbt[kp] = e3;
                ztdbt0 = e4 * ztdbt0;
            }
            sw_swflux(zrefb.data(), zrefd.data(), ztrab.data(), ztrad.data(), zldbt.data(), ztdbt.data(), nlay, nlp1,
                      zfu.data(), zfd.data());
            std::vector<R>& fu = pass ? c.fxupc : c.fxup0;
            std::vector<R>& fd = pass ? c.fxdnc : c.fxdn0;
            for (int k = 1; k <= nlp1; ++k) {
                FX(fu, ib0, k - 1) = FX(fu, ib0, k - 1) + zsolar * zfu[k];
                FX(fd, ib0, k - 1) = FX(fd, ib0, k - 1) + zsolar * zfd[k];
            }
            R* sfbm = pass ? c.sfbmc : c.sfbm0;
            R* sfdf = pass ? c.sfdfc : c.sfdf0;
            const R zb1 = zsolar * ztdbt0, zb2 = zsolar * (zfd[1] - ztdbt0);
            if (ibd != 0) { sfbm[ibd - 1] = sfbm[ibd - 1] + zb1; sfdf[ibd - 1] = sfdf[ibd - 1] + zb2; }
            else {
                const R zf1 = (R)0.5f * zb1, zf2 = (R)0.5f * zb2;
                sfbm[0] = sfbm[0] + zf1; sfdf[0] = sfdf[0] + zf2;
                sfbm[1] = sfbm[1] + zf1; sfdf[1] = sfdf[1] + zf2;
            }
        }
    }
    R s_adc = 0, s_au0 = 0, s_su0 = 0, s_sd0 = 0, t_au = 0, t_su = 0, t_sd = 0;
    for (int ib = 0; ib < 14; ++ib) {
        s_adc = s_adc + FX(c.fxdn0, ib, nlp1 - 1);
        s_au0 = s_au0 + FX(c.fxup0, ib, nlp1 - 1);
        s_su0 = s_su0 + FX(c.fxup0, ib, 0);
        s_sd0 = s_sd0 + FX(c.fxdn0, ib, 0);
        t_au = t_au + FX(c.fxupc, ib, nlp1 - 1);
        t_su = t_su + FX(c.fxupc, ib, 0);
        t_sd = t_sd + FX(c.fxdnc, ib, 0);
    }
    c.ftoadc = s_adc; c.ftoau0 = s_au0; c.fsfcu0 = s_su0; c.fsfcd0 = s_sd0;
    c.ftoauc = t_au; c.fsfcuc = t_su; c.fsfcdc = t_sd;
    c.suvbf0 = FX(c.fxdn0, 11, 0);
    c.suvbfc = FX(c.fxdnc, 11, 0);
}

}  // namespace orc
