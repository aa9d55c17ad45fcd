// rrtm_sw.hpp -- CPU oracle: RRTM shortwave column solve (NAM route: spcvrtc, iswmode 2), serial.
//
// Restates the reference's SW chain for one day column:
//   swrad_prep          namgpu/kernels/phys_rrtm_sw_swrad.cu:127-279 (ivflip 0, iovrsw 0 / 1 / 2)
//   cldprop             namgpu/kernels/phys_rrtm_sw_cldprop.cu:76 (iswcliq 1, iswcice 3; or iswcliq 0)
//   setcoef             namgpu/kernels/phys_rrtm_sw_setcoef.cu:131-191
//   taumol (sfluxzen)   namgpu/kernels/phys_rrtm_sw_taumol.cu:59-120
//   taumol16..29        namgpu/kernels/phys_rrtm_sw_taumol16.cu .. taumol29.cu, with the reference's
//                       MINVAL(laytrop) rules (8-column day groups for bands 19 and 23, the chunk
//                       minimum for bands 25 and 28; physics/rrtm/sw_seam.py:23-37)
//   spcvrtc + swflux    namgpu/kernels/phys_rrtm_sw_spcvrtc.cu:65-547
//   swrad_post          namgpu/kernels/phys_rrtm_sw_swrad.cu:289-418
// Test infrastructure only: never linked into the product.
#pragma once
#include "rrtm_common.hpp"

namespace orc {

template <class R>
struct SwColumn {
    int nlay = 0;
    std::vector<R> pavel, tavel, delp, coldry, colmol, h2ovmr, colamt;   // colamt [6][nlay]
    std::vector<R> cfrac, cliqp, reliq, cicep, reice, cdat1, cdat2, cdat3, cdat4;
    std::vector<R> tauae, ssaae, asyae;                                 // [14][nlay]
    std::vector<R> taucw, ssacw, asycw, cldfrc;                         // [14][nlay], [nlay]
    R zcf0 = 1, zcf1 = 0, cosz = 0, sntz = 0, ssolar = 0;
    R albbm[2] = {0, 0}, albdf[2] = {0, 0};
    int laytrop = 0;
    std::vector<int> jp, jt, jt1, indself, indfor;
    std::vector<R> fac00, fac01, fac10, fac11, selffac, selffrac, forfac, forfrac;
    std::vector<R> taug, taur;         // [112][nlay]
    std::vector<R> sfluxzen;           // [112]
    // spcvrtc outputs: [14][nlp1] band fluxes (level 0 = surface), scalars
    std::vector<R> fxupc, fxdnc, fxup0, fxdn0;
    R ftoadc = 0, ftoauc = 0, ftoau0 = 0, fsfcuc = 0, fsfcu0 = 0, fsfcdc = 0, fsfcd0 = 0, suvbfc = 0, suvbf0 = 0;
    R sfbmc[2] = {0, 0}, sfdfc[2] = {0, 0}, sfbm0[2] = {0, 0}, sfdf0[2] = {0, 0};
    std::vector<R> cldfmc;             // McICA route: [112][nlay]

    explicit SwColumn(int n) : nlay(n) {
        for (auto* v : {&pavel, &tavel, &delp, &coldry, &colmol, &h2ovmr, &cfrac, &cliqp, &reliq, &cicep, &reice,
                        &cdat1, &cdat2, &cdat3, &cdat4, &cldfrc, &fac00, &fac01, &fac10, &fac11, &selffac,
                        &selffrac, &forfac, &forfrac})
            v->assign(n, 0);
        colamt.assign(6 * n, 0);
        for (auto* v : {&tauae, &ssaae, &asyae, &taucw, &ssacw, &asycw}) v->assign(14 * n, 0);
        for (auto* v : {&jp, &jt, &jt1, &indself, &indfor}) v->assign(n, 0);
        taug.assign(112 * n, 0); taur.assign(112 * n, 0); sfluxzen.assign(112, 0);
        for (auto* v : {&fxupc, &fxdnc, &fxup0, &fxdn0}) v->assign(14 * (n + 1), 0);
    }
    R& CA(int m, int k0) { return colamt[(size_t)m * nlay + k0]; }
    R& TG(int g, int k0) { return taug[(size_t)g * nlay + k0]; }
    R& TR(int g, int k0) { return taur[(size_t)g * nlay + k0]; }
};

// ---------------------------------------------------------------------------------------------------
// swrad_prep (phys_rrtm_sw_swrad.cu:127-279) for one day column.
template <class R>
void sw_prep(SwColumn<R>& c, const Inputs& in, int col, int iswcliq, int iovrsw = 1)
{
    const int nlay = c.nlay, N = in.ncol;
    auto IN = [&](const float* a, int lev) { return (R)a[(size_t)lev * N + col]; };
    const R amdw = (R)CON_AMD / (R)CON_AMW, amdo3 = (R)CON_AMD / (R)CON_AMO3;
    const R s0fac = (R)(float)in.solcon / (R)1368.22f;
    const R cz = (R)in.coszen[col];
    c.cosz = cz;
    c.sntz = (R)1 / cz;
    c.ssolar = s0fac * cz;
    c.albbm[0] = (R)in.sfcalb[0 * (size_t)N + col];
    c.albdf[0] = (R)in.sfcalb[1 * (size_t)N + col];
    c.albbm[1] = (R)in.sfcalb[2 * (size_t)N + col];
    c.albdf[1] = (R)in.sfcalb[3 * (size_t)N + col];
    const R tem1 = (R)100.0f * (R)CON_G, tem2 = (R)1.0e-20f * (R)1.0e3f * (R)CON_AVGD;
    for (int k0 = 0; k0 < nlay; ++k0) {
        const int kk0 = nlay - 1 - k0;
        c.pavel[k0] = IN(in.plyr, kk0);
        c.tavel[k0] = IN(in.tlyr, kk0);
        const R dl = IN(in.plvl, kk0 + 1) - IN(in.plvl, kk0);
        c.delp[k0] = dl;
        const R qv = IN(in.qlyr, kk0), ov = IN(in.olyr, kk0);
        const R h2o = fmaxR((R)0, qv * amdw / ((R)1 - qv));
        const R o3 = fmaxR((R)0, ov * amdo3);
        c.h2ovmr[k0] = h2o;
        const R tem0 = ((R)1 - h2o) * (R)CON_AMD + h2o * (R)CON_AMW;
        const R cd = tem2 * dl / (tem1 * tem0 * ((R)1 + h2o));
        c.coldry[k0] = cd;
        const R tc = (R)1.0e-12f * cd;
        auto G = [&](int n) { return (R)in.gasvmr[((size_t)n * nlay + kk0) * N + col]; };
        c.CA(0, k0) = fmaxR((R)0, cd * h2o);
        c.CA(1, k0) = fmaxR(tc, cd * G(0));
        c.CA(2, k0) = fmaxR((R)0, cd * o3);
        c.colmol[k0] = cd + c.CA(0, k0);
        c.CA(3, k0) = fmaxR(tc, cd * G(1));
        c.CA(4, k0) = fmaxR(tc, cd * G(2));
        c.CA(5, k0) = fmaxR(tc, cd * G(3));
        for (int ib = 0; ib < 14; ++ib) {
            R ta = 0, sa = 0, ya = 0;
            if (in.faersw) {
                ta = (R)in.faersw[(((size_t)(0 * 14 + ib)) * nlay + kk0) * N + col];
                sa = (R)in.faersw[(((size_t)(1 * 14 + ib)) * nlay + kk0) * N + col];
                ya = (R)in.faersw[(((size_t)(2 * 14 + ib)) * nlay + kk0) * N + col];
            }
            c.tauae[(size_t)ib * nlay + k0] = ta;
            c.ssaae[(size_t)ib * nlay + k0] = sa;
            c.asyae[(size_t)ib * nlay + k0] = ya;
        }
        auto CLD = [&](int n) { return (R)in.clouds[((size_t)n * nlay + kk0) * N + col]; };
        if (iswcliq > 0) {
            c.cfrac[k0] = CLD(0); c.cliqp[k0] = CLD(1); c.reliq[k0] = CLD(2); c.cicep[k0] = CLD(3);
            c.reice[k0] = CLD(4); c.cdat1[k0] = CLD(5); c.cdat2[k0] = CLD(6); c.cdat3[k0] = CLD(7); c.cdat4[k0] = CLD(8);
        } else {
            c.cfrac[k0] = CLD(0); c.cdat1[k0] = CLD(1); c.cdat2[k0] = CLD(2); c.cdat3[k0] = CLD(3);
        }
    }
    // clear-sky view fraction (phys_rrtm_sw_swrad.cu:251-279): iovrsw 0 random, 1 maximum-random,
    // 2 maximum overlap of the layer cloud fractions
    const R ftiny = (R)1.0e-12f, oneminus = (R)1.0f - (R)1.0e-6f;
    R z0 = 1, z1 = 1;
    if (iovrsw == 0) {
        for (int k0 = 0; k0 < nlay; ++k0) z0 = z0 * ((R)1 - c.cfrac[k0]);
    } else if (iovrsw == 1) {
        for (int k0 = 0; k0 < nlay; ++k0) {
            const R cf = c.cfrac[k0];
            if (cf > ftiny) z1 = fminR(z1, (R)1 - cf);
            else if (z1 < (R)1) { z0 = z0 * z1; z1 = 1; }
        }
        z0 = z0 * z1;
    } else if (iovrsw == 2) {
        for (int k0 = 0; k0 < nlay; ++k0) z0 = fminR(z0, (R)1 - c.cfrac[k0]);
    }
    if (z0 <= ftiny) z0 = 0;
    if (z0 > oneminus) z0 = 1;
    c.zcf0 = z0;
    c.zcf1 = (R)1 - z0;
}

// ---------------------------------------------------------------------------------------------------
// cldprop (phys_rrtm_sw_cldprop.cu:76-351), iswcliq 1 / iswcice 3, or iswcliq 0; isubcsw = 0.
template <class R>
void sw_cldprop(SwColumn<R>& c, int iswcliq)
{
    const int nlay = c.nlay;
    const TableStore& T = tables();
    const R ftiny = (R)1.0e-12f;
    for (int i = 0; i < 14 * nlay; ++i) { c.taucw[i] = 0; c.ssacw[i] = 0; c.asycw[i] = 0; }
    if (!(c.zcf1 > 0)) {
        for (int k0 = 0; k0 < nlay; ++k0) c.cldfrc[k0] = 0;
        return;
    }
    for (int i = 0; i < 14 * nlay; ++i) { c.taucw[i] = 0; c.ssacw[i] = 1; c.asycw[i] = 0; }
    static const float b0r[14] = {0.466f, 0.437f, 0.416f, 0.391f, 0.374f, 0.352f, 0.183f, 0.048f, 0.012f,
                                  0.000f, 0.000f, 0.000f, 0.000f, 0.496f};
    static const float c0r[14] = {0.975f, 0.965f, 0.960f, 0.955f, 0.952f, 0.950f, 0.944f, 0.894f, 0.884f,
                                  0.883f, 0.883f, 0.883f, 0.883f, 0.980f};
    static const float b0s[14] = {0.460f, 0.460f, 0.460f, 0.460f, 0.460f, 0.460f, 0.460f, 0.000f, 0.000f,
                                  0.000f, 0.000f, 0.000f, 0.000f, 0.460f};
    static const float b1s[14] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.62e-5f, 1.62e-5f, 0.0f, 0.0f,
                                  0.0f, 0.0f, 0.0f};
    static const float c0s[14] = {0.970f, 0.970f, 0.970f, 0.970f, 0.970f, 0.970f, 0.970f, 0.970f, 0.970f,
                                  0.700f, 0.700f, 0.700f, 0.700f, 0.970f};
    const R a0r = (R)3.07e-3f, a0s = 0, a1s = (R)1.5f;
    const double *extliq1 = T.f("sw_extliq1"), *ssaliq1 = T.f("sw_ssaliq1"), *asyliq1 = T.f("sw_asyliq1");
    const double *extice3 = T.f("sw_extice3"), *ssaice3 = T.f("sw_ssaice3"), *asyice3 = T.f("sw_asyice3");
    auto OUT = [&](std::vector<R>& v, int ib, int k0) -> R& { return v[(size_t)ib * nlay + k0]; };
    if (iswcliq > 0) {
        for (int k0 = 0; k0 < nlay; ++k0) {
            const R cf = c.cfrac[k0];
            if (!(cf > ftiny)) continue;
            R tauran = 0, tausnw = 0, ssaran[14], asyran[14], ssasnw[14], asysnw[14];
            R tauliq[14], ssaliq[14], asyliq[14], tauice[14], ssaice[14], asyice[14];
            for (int ib = 0; ib < 14; ++ib) {
                ssaran[ib] = asyran[ib] = ssasnw[ib] = asysnw[ib] = 0;
                tauliq[ib] = ssaliq[ib] = asyliq[ib] = tauice[ib] = ssaice[ib] = asyice[ib] = 0;
            }
            const R cldran = c.cdat1[k0], cldsnw = c.cdat3[k0], refsnw = c.cdat4[k0];
            const R dgesnw_fu = (R)1.0315f * refsnw;
            tauran = cldran * a0r;
            if (cldsnw > 0 && refsnw > (R)10) tausnw = cldsnw * (R)1.09087f * (a0s + a1s / dgesnw_fu);
            else tausnw = 0;
            for (int ib = 0; ib < 14; ++ib) {
                ssaran[ib] = tauran * ((R)1 - (R)b0r[ib]);
                ssasnw[ib] = tausnw * ((R)1 - ((R)b0s[ib] + (R)b1s[ib] * dgesnw_fu));
                asyran[ib] = ssaran[ib] * (R)c0r[ib];
                asysnw[ib] = ssasnw[ib] * (R)c0s[ib];
            }
            const R cldliq = c.cliqp[k0], refliq = c.reliq[k0], cldice = c.cicep[k0], refice = c.reice[k0];
            if (!(cldliq <= 0)) {
                const R factor = refliq - (R)1.5f;
                const int index = imax(1, imin(57, (int)factor));
                const R fint = factor - (R)index;
                for (int ib = 0; ib < 14; ++ib) {
                    const double *e = extliq1 + ib * 58, *s = ssaliq1 + ib * 58, *a = asyliq1 + ib * 58;
                    const R ext = fmaxR((R)0, (R)e[index - 1] + fint * ((R)e[index] - (R)e[index - 1]));
                    const R ssa = fmaxR((R)0, fminR((R)1, (R)s[index - 1] + fint * ((R)s[index] - (R)s[index - 1])));
                    const R asy = fmaxR((R)0, fminR((R)1, (R)a[index - 1] + fint * ((R)a[index] - (R)a[index - 1])));
                    tauliq[ib] = cldliq * ext;
                    ssaliq[ib] = tauliq[ib] * ssa;
                    asyliq[ib] = ssaliq[ib] * asy;
                }
            }
            if (!(cldice <= 0)) {
                const R dgeice = fmaxR((R)5, fminR((R)140, (R)1.0315f * refice));
                const R factor = (dgeice - (R)2) / (R)3;
                const int index = imax(1, imin(45, (int)factor));
                const R fint = factor - (R)index;
                for (int ib = 0; ib < 14; ++ib) {
                    const double *e = extice3 + ib * 46, *s = ssaice3 + ib * 46, *a = asyice3 + ib * 46;
                    const R ext = fmaxR((R)0, (R)e[index - 1] + fint * ((R)e[index] - (R)e[index - 1]));
                    const R ssa = fmaxR((R)0, fminR((R)1, (R)s[index - 1] + fint * ((R)s[index] - (R)s[index - 1])));
                    const R asy = fmaxR((R)0, fminR((R)1, (R)a[index - 1] + fint * ((R)a[index] - (R)a[index - 1])));
                    tauice[ib] = cldice * ext;
                    ssaice[ib] = tauice[ib] * ssa;
                    asyice[ib] = ssaice[ib] * asy;
                }
            }
            for (int ib = 0; ib < 14; ++ib) {
                OUT(c.taucw, ib, k0) = tauliq[ib] + tauice[ib] + tauran + tausnw;
                OUT(c.ssacw, ib, k0) = ssaliq[ib] + ssaice[ib] + ssaran[ib] + ssasnw[ib];
                OUT(c.asycw, ib, k0) = asyliq[ib] + asyice[ib] + asyran[ib] + asysnw[ib];
            }
        }
    } else {
        for (int k0 = 0; k0 < nlay; ++k0)
            if (c.cfrac[k0] > ftiny)
                for (int ib = 0; ib < 14; ++ib) {
                    OUT(c.taucw, ib, k0) = c.cdat1[k0];
                    OUT(c.ssacw, ib, k0) = c.cdat1[k0] * c.cdat2[k0];
                    OUT(c.asycw, ib, k0) = OUT(c.ssacw, ib, k0) * c.cdat3[k0];
                }
    }
    for (int k0 = 0; k0 < nlay; ++k0) c.cldfrc[k0] = c.cfrac[k0] / c.zcf1;
}

// ---------------------------------------------------------------------------------------------------
// setcoef (phys_rrtm_sw_setcoef.cu:17-97)
template <class R>
void sw_setcoef(SwColumn<R>& c)
{
    const TableStore& T = tables();
    const double *preflog = T.f("sw_preflog"), *tref = T.f("sw_tref");
    const R stpfac = (R)296.0f / (R)1013.0f;
    int lt = c.nlay;
    for (int k = 1; k <= c.nlay; ++k) {
        const int k0 = k - 1;
        const R pav = c.pavel[k0], tav = c.tavel[k0], h2o = c.h2ovmr[k0];
        const R forf = pav * stpfac / (tav * ((R)1 + h2o));
        c.forfac[k0] = forf;
        const R plog = mlog(pav);
        const int jpk = imax(1, imin(58, (int)((R)36 - (R)5 * (plog + (R)0.04f))));
        const int jp1 = jpk + 1;
        const R fp = (R)5 * ((R)preflog[jpk - 1] - plog);
        const R tem1 = (tav - (R)tref[jpk - 1]) / (R)15;
        const R tem2 = (tav - (R)tref[jp1 - 1]) / (R)15;
        const int jtk = imax(1, imin(4, (int)((R)3 + tem1)));
        const int jt1k = imax(1, imin(4, (int)((R)3 + tem2)));
        const R ft = tem1 - (R)(jtk - 3), ft1 = tem2 - (R)(jt1k - 3);
        c.jp[k0] = jpk; c.jt[k0] = jtk; c.jt1[k0] = jt1k;
        const R fp1 = (R)1 - fp;
        c.fac10[k0] = fp1 * ft;
        c.fac00[k0] = fp1 * ((R)1 - ft);
        c.fac11[k0] = fp * ft1;
        c.fac01[k0] = fp * ((R)1 - ft1);
        if (plog > (R)4.56f) {
            lt = k;
            const R tem1f = ((R)332 - tav) / (R)36;
            const int indf = imin(2, imax(1, (int)tem1f));
            c.indfor[k0] = indf;
            c.forfrac[k0] = tem1f - (R)indf;
            const R tem2s = (tav - (R)188) / (R)7.2f;
            const int inds = imin(9, imax(1, (int)tem2s - 7));
            c.indself[k0] = inds;
            c.selffrac[k0] = tem2s - (R)(inds + 7);
            c.selffac[k0] = h2o * forf;
        } else {
            const R tem1f = (tav - (R)188) / (R)36;
            c.indfor[k0] = 3;
            c.forfrac[k0] = tem1f - (R)1;
            c.indself[k0] = 0;
            c.selffrac[k0] = 0;
            c.selffac[k0] = 0;
        }
    }
    c.laytrop = lt;
}

// SW band constants (rrtm_sw_bands.cuh): nspa/nspb per band 16..29.
static const int SW_NSPA[14] = {9, 9, 9, 9, 1, 9, 9, 1, 9, 1, 0, 1, 9, 1};
static const int SW_NSPB[14] = {1, 5, 1, 1, 1, 5, 1, 0, 1, 0, 0, 1, 5, 1};

inline void sw_index(int jb, int k1, int lt, int jp, int jt, int jt1, int& id0, int& id1)
{
    const int b = jb - 16;
    if (k1 <= lt) { id0 = ((jp - 1) * 5 + (jt - 1)) * SW_NSPA[b]; id1 = (jp * 5 + (jt1 - 1)) * SW_NSPA[b]; }
    else { id0 = ((jp - 13) * 5 + (jt - 1)) * SW_NSPB[b]; id1 = ((jp - 12) * 5 + (jt1 - 1)) * SW_NSPB[b]; }
}

// ---------------------------------------------------------------------------------------------------
// taumol: sfluxzen (phys_rrtm_sw_taumol.cu:59-120) and bands 16..29.  kmin8 is MINVAL(laytrop) over the
// column's 8-day-column group, kminw over its day-column chunk (see the file header).
template <class R>
void sw_taumol(SwColumn<R>& c, int kmin8, int kminw)
{
    const TableStore& T = tables();
    const int nlay = c.nlay, lt = c.laytrop;
    const R oneminus = (R)1.0f - (R)1.0e-6f;
    const R swoneminus = (R)0.999999f;
    auto t = [&](const char* n) { return T.f(n); };
    // ---- sfluxzen
    {
        const double *sf01 = t("sw_sfluxref01"), *sf02 = t("sw_sfluxref02"), *sf03 = t("sw_sfluxref03");
        const double *strrat = t("sw_strrat"), *specwt = t("sw_specwt");
        const int *layreffr = T.i("sw_layreffr"), *ix1 = T.i("sw_ix1"), *ix2 = T.i("sw_ix2"), *ibx = T.i("sw_ibx");
        const R scalekur = (R)t("sw_scalekur")[0];
        for (int b = 0; b < 14; ++b) {
            const int jb = b + 16, ibd = ibx[b], njb = SW_NG[b], ns = SW_NS[b], lr = layreffr[b];
            if (jb == 16 || jb == 20 || jb == 23 || jb == 25 || jb == 26 || jb == 29) {
                for (int j = 0; j < njb; ++j) c.sfluxzen[ns + j] = (R)sf01[((ibd - 1) * 1 + 0) * 16 + j];
            } else if (jb == 27) {
                for (int j = 0; j < njb; ++j) c.sfluxzen[ns + j] = scalekur * (R)sf01[((ibd - 1) * 1 + 0) * 16 + j];
            } else {
                int ks;
                if (jb == 17 || jb == 28) {
                    ks = nlay;
                    for (int k = lt; k <= nlay - 1; ++k)
                        if (c.jp[k - 1] < lr && c.jp[k] >= lr) { ks = k + 1; break; }
                } else {
                    ks = lt;
                    for (int k = 1; k <= lt - 1; ++k)
                        if (c.jp[k - 1] < lr && c.jp[k] >= lr) { ks = k + 1; break; }
                }
                const R colm1 = c.CA(ix1[b] - 1, ks - 1), colm2 = c.CA(ix2[b] - 1, ks - 1);
                const R speccomb = colm1 + (R)strrat[b] * colm2;
                const R specmult = (R)specwt[b] * fminR(swoneminus, colm1 / speccomb);
                const int jsi = (int)specmult;
                const int js = 1 + jsi;
                const R fs = specmult - (R)jsi;
                const bool two = (jb == 17 || jb == 28);
                const double* sf = two ? sf02 : sf03;
                const int mfs = two ? 5 : 9;
                const int base = ((ibd - 1) * mfs) * 16;
                for (int j = 0; j < njb; ++j) {
                    const R a = (R)sf[base + (js - 1) * 16 + j], cc = (R)sf[base + js * 16 + j];
                    c.sfluxzen[ns + j] = a + fs * (cc - a);
                }
            }
        }
    }
    // Shared 8-point lower-atmosphere form of the SW binary bands: returns the absa sum with the
    // reference's MAX/MIN clamps of the table rows (e.g. phys_rrtm_sw_taumol16.cu:143-170).
    auto sum8 = [&](const double* A, int ng, int ig, int msa, int id0, int id1, int js, R fs,
                    R f00, R f01, R f10, R f11, int o1, int o2) {
        const R fs1 = (R)1 - fs;
        const R fac000 = fs1 * f00, fac010 = fs1 * f10, fac100 = fs * f00, fac110 = fs * f10;
        const R fac001 = fs1 * f01, fac011 = fs1 * f11, fac101 = fs * f01, fac111 = fs * f11;
        const int i01 = imax(1, imin(msa, id0 + js)), i02 = imin(msa, i01 + 1), i03 = imin(msa, i01 + o1),
                  i04 = imin(msa, i01 + o2);
        const int i11 = imax(1, imin(msa, id1 + js)), i12 = imin(msa, i11 + 1), i13 = imin(msa, i11 + o1),
                  i14 = imin(msa, i11 + o2);
        auto a = [&](int i) { return (R)A[(size_t)(i - 1) * ng + ig]; };
        return fac000 * a(i01) + fac100 * a(i02) + fac010 * a(i03) + fac110 * a(i04) + fac001 * a(i11) +
               fac101 * a(i12) + fac011 * a(i13) + fac111 * a(i14);
    };
    auto sum4 = [&](const double* A, int ng, int ig, int ms, int id0, int id1, R f00, R f01, R f10, R f11) {
        const int i01 = imax(1, imin(ms, id0 + 1)), i02 = imin(ms, i01 + 1);
        const int i11 = imax(1, imin(ms, id1 + 1)), i12 = imin(ms, i11 + 1);
        auto a = [&](int i) { return (R)A[(size_t)(i - 1) * ng + ig]; };
        return f00 * a(i01) + f10 * a(i02) + f01 * a(i11) + f11 * a(i12);
    };
    auto js_fs = [&](R c1, R strr, R c2, R mult, R& speccomb, int& js, R& fs) {
        speccomb = c1 + strr * c2;
        const R specmult = mult * fminR(oneminus, c1 / speccomb);
        js = 1 + (int)specmult;
        fs = fmod1(specmult);
    };
    const double* strrat = t("sw_strrat");

    for (int k0 = 0; k0 < nlay; ++k0) {
        const int k = k0 + 1;
        const int jpk = c.jp[k0], jtk = c.jt[k0], jt1k = c.jt1[k0];
        const R f00 = c.fac00[k0], f01 = c.fac01[k0], f10 = c.fac10[k0], f11 = c.fac11[k0];
        const R cm = c.colmol[k0];
        const R c1 = c.CA(0, k0), c2 = c.CA(1, k0), c3 = c.CA(2, k0), c5 = c.CA(4, k0), c6 = c.CA(5, k0);
        const int inds = c.indself[k0], indf = c.indfor[k0];
        const R sfac = c.selffac[k0], sfrac = c.selffrac[k0], ffac = c.forfac[k0], ffrac = c.forfrac[k0];
        auto self_t = [&](const double* S, int ng, int ig) { return interp(S, ng, inds, ig, sfrac); };
        auto for_t = [&](const double* F, int ng, int ig) { return interp(F, ng, indf, ig, ffrac); };
        int id0, id1;

        // ---- band 16 (taumol16.cu:75-212): lower k <= laytrop, upper k >= laytrop (upper wins at laytrop)
        {
            const int NG = 6, NS = 0;
            const double *A = t("sw16_absa"), *B = t("sw16_absb"), *S = t("sw16_selfref"), *F = t("sw16_forref");
            const R rayl = (R)t("sw16_rayl")[0], strr = (R)t("sw16_strrat")[0];
            sw_index(16, k, lt, jpk, jtk, jt1k, id0, id1);
            for (int g = 0; g < NG; ++g) c.TR(NS + g, k0) = cm * rayl;
            if (k <= lt) {
                R sc, fs; int js;
                js_fs(c1, strr, c5, (R)8, sc, js, fs);
                for (int g = 0; g < NG; ++g)
                    c.TG(NS + g, k0) = sc * sum8(A, NG, g, 585, id0, id1, js, fs, f00, f01, f10, f11, 9, 10) +
                                       c1 * (sfac * self_t(S, NG, g) + ffac * for_t(F, NG, g));
            }
            if (k >= lt)
                for (int g = 0; g < NG; ++g) c.TG(NS + g, k0) = c5 * sum4(B, NG, g, 235, id0, id1, f00, f01, f10, f11);
        }
        // ---- band 17 (taumol17.cu:26-239): no overlap; self term skipped where indself == 0
        {
            const int NG = 12, NS = 6;
            const double *A = t("sw17_absa"), *B = t("sw17_absb"), *S = t("sw17_selfref"), *F = t("sw17_forref");
            const R strr = (R)strrat[1], rayl = (R)6.86e-10f;
            for (int g = 0; g < NG; ++g) c.TR(NS + g, k0) = cm * rayl;
            if (k0 < lt) {
                R sc, fs; int js;
                js_fs(c1, strr, c2, (R)8, sc, js, fs);
                const int i0 = ((jpk - 1) * 5 + (jtk - 1)) * 9, i1 = (jpk * 5 + (jt1k - 1)) * 9;
                for (int g = 0; g < NG; ++g) {
                    const R selfpart = inds > 0 ? sfac * self_t(S, NG, g) : (R)0;
                    c.TG(NS + g, k0) = sc * sum8(A, NG, g, 585, i0, i1, js, fs, f00, f01, f10, f11, 9, 10) +
                                       c1 * (selfpart + ffac * for_t(F, NG, g));
                }
            } else {
                R sc, fs; int js;
                js_fs(c1, strr, c2, (R)4, sc, js, fs);
                const int i0 = ((jpk - 13) * 5 + (jtk - 1)) * 5, i1 = ((jpk - 12) * 5 + (jt1k - 1)) * 5;
                for (int g = 0; g < NG; ++g)
                    c.TG(NS + g, k0) = sc * sum8(B, NG, g, 1175, i0, i1, js, fs, f00, f01, f10, f11, 5, 6) +
                                       (c1 * ffac) * for_t(F, NG, g);
            }
        }
        // ---- band 18 (taumol18.cu): no overlap; H2O/CH4 lower, CH4 upper
        {
            const int NG = 8, NS = 18;
            const double *A = t("sw18_absa"), *B = t("sw18_absb"), *S = t("sw18_selfref"), *F = t("sw18_forref");
            const R rayl = (R)t("sw18_rayl")[0], strr = (R)strrat[2];
            for (int g = 0; g < NG; ++g) c.TR(NS + g, k0) = cm * rayl;
            sw_index(18, k, lt, jpk, jtk, jt1k, id0, id1);
            if (k <= lt) {
                const R sc = c1 + strr * c5;
                const R ratio = sc > 0 ? c1 / sc : (R)0;
                const R specmult = (R)8 * fminR(swoneminus, ratio);
                const int jsi = (int)specmult;
                const int js = 1 + jsi;
                const R fs = specmult - (R)jsi;
                for (int g = 0; g < NG; ++g)
                    c.TG(NS + g, k0) = sc * sum8(A, NG, g, 585, id0, id1, js, fs, f00, f01, f10, f11, 9, 10) +
                                       c1 * (sfac * self_t(S, NG, g) + ffac * for_t(F, NG, g));
            } else {
                for (int g = 0; g < NG; ++g) c.TG(NS + g, k0) = c5 * sum4(B, NG, g, 235, id0, id1, f00, f01, f10, f11);
            }
        }
        // ---- band 19 (taumol19.cu): upper form where k >= laytrop and k >= MINVAL(8-group) + 1
        {
            const int NG = 8, NS = 26;
            const double *A = t("sw19_absa"), *B = t("sw19_absb"), *S = t("sw19_selfref"), *F = t("sw19_forref");
            const R rayl = (R)2.29e-09f, strr = (R)5.49281e+0f;
            for (int g = 0; g < NG; ++g) c.TR(NS + g, k0) = cm * rayl;
            sw_index(19, k, lt, jpk, jtk, jt1k, id0, id1);
            if (k <= lt) {
                R sc, fs; int js;
                sc = c1 + strr * c2;
                const R specmult = (R)8 * fminR(swoneminus, c1 / sc);
                js = 1 + (int)specmult;
                fs = fmod1(specmult);
                for (int g = 0; g < NG; ++g)
                    c.TG(NS + g, k0) = sc * sum8(A, NG, g, 585, id0, id1, js, fs, f00, f01, f10, f11, 9, 10) +
                                       c1 * (sfac * self_t(S, NG, g) + ffac * for_t(F, NG, g));
            }
            if (k >= lt && k >= kmin8 + 1)
                for (int g = 0; g < NG; ++g) c.TG(NS + g, k0) = c2 * sum4(B, NG, g, 235, id0, id1, f00, f01, f10, f11);
        }
        // ---- band 20 (taumol20.cu): no overlap; H2O with CH4 continuum term
        {
            const int NG = 10, NS = 34;
            const double *A = t("sw20_absa"), *B = t("sw20_absb"), *S = t("sw20_selfref"), *F = t("sw20_forref"),
                         *ch4 = t("sw20_absch4");
            const R rayl = (R)t("sw20_rayl")[0];
            for (int g = 0; g < NG; ++g) c.TR(NS + g, k0) = cm * rayl;
            if (k <= lt) {
                const int i0 = ((jpk - 1) * 5 + (jtk - 1)) * 1, i1 = (jpk * 5 + (jt1k - 1)) * 1;
                for (int g = 0; g < NG; ++g)
                    c.TG(NS + g, k0) = c1 * ((sum4(A, NG, g, 65, i0, i1, f00, f01, f10, f11)) + sfac * (self_t(S, NG, g)) +
                                             ffac * (for_t(F, NG, g))) + c5 * (R)ch4[g];
            } else {
                const int i0 = ((jpk - 13) * 5 + (jtk - 1)) * 1, i1 = ((jpk - 12) * 5 + (jt1k - 1)) * 1;
                for (int g = 0; g < NG; ++g)
                    c.TG(NS + g, k0) = c1 * ((sum4(B, NG, g, 235, i0, i1, f00, f01, f10, f11)) + ffac * (for_t(F, NG, g))) +
                                       c5 * (R)ch4[g];
            }
        }
        // ---- band 21 (taumol21.cu): lower where k < laytrop, upper where k >= laytrop
        {
            const int NG = 10, NS = 44;
            const double *A = t("sw21_absa"), *B = t("sw21_absb"), *S = t("sw21_selfref"), *F = t("sw21_forref");
            const R rayl = (R)9.41e-09f, strr = (R)4.53210e-03f;
            for (int g = 0; g < NG; ++g) c.TR(NS + g, k0) = cm * rayl;
            if (k <= lt) { id0 = ((jpk - 1) * 5 + (jtk - 1)) * 9; id1 = (jpk * 5 + (jt1k - 1)) * 9; }
            else { id0 = ((jpk - 13) * 5 + (jtk - 1)) * 5; id1 = ((jpk - 12) * 5 + (jt1k - 1)) * 5; }
            if (k < lt) {
                R sc, fs; int js;
                js_fs(c1, strr, c2, (R)8, sc, js, fs);
                for (int g = 0; g < NG; ++g)
                    c.TG(NS + g, k0) = sc * sum8(A, NG, g, 585, id0, id1, js, fs, f00, f01, f10, f11, 9, 10) +
                                       c1 * (sfac * self_t(S, NG, g) + ffac * for_t(F, NG, g));
            }
            if (k >= lt) {
                R sc, fs; int js;
                js_fs(c1, strr, c2, (R)4, sc, js, fs);
                for (int g = 0; g < NG; ++g)
                    c.TG(NS + g, k0) = sc * sum8(B, NG, g, 1175, id0, id1, js, fs, f00, f01, f10, f11, 5, 6) +
                                       c1 * ffac * for_t(F, NG, g);
            }
        }
        // ---- band 22 (taumol22.cu): no overlap; H2O/O2 lower, O2 upper, O2 continuum
        {
            const int NG = 2, NS = 54;
            const double *A = t("sw22_absa"), *B = t("sw22_absb"), *S = t("sw22_selfref"), *F = t("sw22_forref");
            const R rayl = (R)1.54e-08f, strr = (R)3.63328e-02f, o2adj = (R)1.6f;
            const R o2tem = (R)4.35e-4f / ((R)350.0f * (R)2.0f);
            sw_index(22, k, lt, jpk, jtk, jt1k, id0, id1);
            for (int g = 0; g < NG; ++g) c.TR(NS + g, k0) = cm * rayl;
            const R o2cont = o2tem * c6;
            if (k <= lt) {
                const R sc = c1 + strr * c6;
                const R ratio = sc > 0 ? c1 / sc : (R)0;
                const R specmult = (R)8 * fminR(oneminus, ratio);
                const int js = 1 + (int)specmult;
                const R fs = fmod1(specmult);
                for (int g = 0; g < NG; ++g)
                    c.TG(NS + g, k0) = sc * (sum8(A, NG, g, 585, id0, id1, js, fs, f00, f01, f10, f11, 9, 10)) +
                                       c1 * (sfac * (self_t(S, NG, g)) + ffac * (for_t(F, NG, g))) + o2cont;
            } else {
                for (int g = 0; g < NG; ++g)
                    c.TG(NS + g, k0) = c6 * o2adj * (sum4(B, NG, g, 235, id0, id1, f00, f01, f10, f11)) + o2cont;
            }
        }
        // ---- band 23 (taumol23.cu): lower layers; at k = laytrop only where laytrop is the group minimum
        {
            const int NG = 10, NS = 56;
            const double *A = t("sw23_absa"), *S = t("sw23_selfref"), *F = t("sw23_forref"), *ray = t("sw23_rayl");
            const R givfac = (R)1.029f;
            for (int g = 0; g < NG; ++g) c.TR(NS + g, k0) = cm * (R)ray[g];
            const bool zero_cond = (k >= kmin8 + 1) && (k >= lt);
            const bool compute = (k <= lt) && !zero_cond;
            if (!compute) {
                for (int g = 0; g < NG; ++g) c.TG(NS + g, k0) = 0;
            } else {
                const int i0 = ((jpk - 1) * 5 + (jtk - 1)) * 1, i1 = (jpk * 5 + (jt1k - 1)) * 1;
                for (int g = 0; g < NG; ++g)
                    c.TG(NS + g, k0) = c1 * (givfac * sum4(A, NG, g, 65, i0, i1, f00, f01, f10, f11) +
                                             sfac * self_t(S, NG, g) + ffac * for_t(F, NG, g));
            }
        }
        // ---- band 24 (taumol24.cu): no overlap; H2O/O2 lower with O3 and js-dependent Rayleigh
        {
            const int NG = 8, NS = 66;
            const double *A = t("sw24_absa"), *B = t("sw24_absb"), *S = t("sw24_selfref"), *F = t("sw24_forref"),
                         *o3a = t("sw24_abso3a"), *o3b = t("sw24_abso3b"), *rla = t("sw24_rayla"), *rlb = t("sw24_raylb");
            const R strr = (R)1.24692e-1f;
            sw_index(24, k, lt, jpk, jtk, jt1k, id0, id1);
            if (k <= lt) {
                const R sc = c1 + strr * c6;
                const R specmult = (R)8 * fminR(swoneminus, c1 / sc);
                const int jsi = (int)specmult;
                const int js = 1 + jsi;
                const R fs = specmult - (R)jsi;
                for (int g = 0; g < NG; ++g) {
                    c.TG(NS + g, k0) = sc * sum8(A, NG, g, 585, id0, id1, js, fs, f00, f01, f10, f11, 9, 10) +
                                       c3 * (R)o3a[g] + c1 * (sfac * self_t(S, NG, g) + ffac * for_t(F, NG, g));
                    const R r0 = (R)rla[(size_t)(js - 1) * NG + g], r1 = (R)rla[(size_t)js * NG + g];
                    c.TR(NS + g, k0) = cm * (r0 + fs * (r1 - r0));
                }
            } else {
                for (int g = 0; g < NG; ++g) {
                    c.TG(NS + g, k0) = c6 * sum4(B, NG, g, 235, id0, id1, f00, f01, f10, f11) + c3 * (R)o3b[g];
                    c.TR(NS + g, k0) = cm * (R)rlb[g];
                }
            }
        }
        // ---- band 25 (taumol25.cu): upper O3 form where k >= laytrop and k >= MINVAL(chunk) + 1
        {
            const int NG = 6, NS = 74;
            const double *A = t("sw25_absa"), *o3a = t("sw25_abso3a"), *o3b = t("sw25_abso3b"), *ray = t("sw25_rayl");
            for (int g = 0; g < NG; ++g) c.TR(NS + g, k0) = cm * (R)ray[g];
            if (k <= lt) {
                sw_index(25, k, lt, jpk, jtk, jt1k, id0, id1);
                for (int g = 0; g < NG; ++g)
                    c.TG(NS + g, k0) = c1 * sum4(A, NG, g, 65, id0, id1, f00, f01, f10, f11) + c3 * (R)o3a[g];
            }
            if (k >= kminw + 1 && k >= lt)
                for (int g = 0; g < NG; ++g) c.TG(NS + g, k0) = c3 * (R)o3b[g];
        }
        // ---- band 26 (taumol26.cu): Rayleigh only
        {
            const int NG = 6, NS = 80;
            const double* ray = t("sw26_rayl");
            for (int g = 0; g < NG; ++g) { c.TG(NS + g, k0) = 0; c.TR(NS + g, k0) = cm * (R)ray[g]; }
        }
        // ---- band 27 (taumol27.cu): O3 lower where k < laytrop, upper where k >= laytrop
        {
            const int NG = 8, NS = 86;
            const double *A = t("sw27_absa"), *B = t("sw27_absb"), *ray = t("sw27_rayl");
            for (int g = 0; g < NG; ++g) c.TR(NS + g, k0) = cm * (R)ray[g];
            if (k <= lt) { id0 = ((jpk - 1) * 5 + (jtk - 1)) * 1; id1 = (jpk * 5 + (jt1k - 1)) * 1; }
            else { id0 = ((jpk - 13) * 5 + (jtk - 1)) * 1; id1 = ((jpk - 12) * 5 + (jt1k - 1)) * 1; }
            if (k < lt)
                for (int g = 0; g < NG; ++g) c.TG(NS + g, k0) = c3 * sum4(A, NG, g, 65, id0, id1, f00, f01, f10, f11);
            if (k >= lt)
                for (int g = 0; g < NG; ++g) c.TG(NS + g, k0) = c3 * sum4(B, NG, g, 235, id0, id1, f00, f01, f10, f11);
        }
        // ---- band 28 (taumol28.cu): O3/O2; upper where k >= laytrop and k >= MINVAL(chunk) + 1
        {
            const int NG = 6, NS = 94;
            const double *A = t("sw28_absa"), *B = t("sw28_absb");
            const R rayl = (R)t("sw28_rayl")[0], strr = (R)t("sw28_strrat")[0];
            sw_index(28, k, lt, jpk, jtk, jt1k, id0, id1);
            for (int g = 0; g < NG; ++g) c.TR(NS + g, k0) = cm * rayl;
            if (k <= lt) {
                R sc, fs; int js;
                sc = c3 + strr * c6;
                const R specmult = (R)8 * fminR(swoneminus, c3 / sc);
                js = 1 + (int)specmult;
                fs = fmod1(specmult);
                for (int g = 0; g < NG; ++g)
                    c.TG(NS + g, k0) = sc * sum8(A, NG, g, 585, id0, id1, js, fs, f00, f01, f10, f11, 9, 10);
            }
            if (k >= kminw + 1 && k >= lt) {
                R sc, fs; int js;
                sc = c3 + strr * c6;
                const R specmult = (R)4 * fminR(swoneminus, c3 / sc);
                js = 1 + (int)specmult;
                fs = fmod1(specmult);
                for (int g = 0; g < NG; ++g)
                    c.TG(NS + g, k0) = sc * sum8(B, NG, g, 1175, id0, id1, js, fs, f00, f01, f10, f11, 5, 6);
            }
        }
        // ---- band 29 (taumol29.cu + sw_seam.py:293-310 index dispatcher): no overlap
        {
            const int NG = 12, NS = 100;
            const double *A = t("sw29_absa"), *B = t("sw29_absb"), *S = t("sw29_selfref"), *F = t("sw29_forref"),
                         *h2o = t("sw29_absh2o"), *co2 = t("sw29_absco2");
            const R rayl = (R)9.30e-11f;
            for (int g = 0; g < NG; ++g) c.TR(NS + g, k0) = cm * rayl;
            const bool low = k <= lt;
            const int i0 = low ? (jpk - 1) * 5 + (jtk - 1) : (jpk - 13) * 5 + (jtk - 1);
            const int i1 = low ? jpk * 5 + (jt1k - 1) : (jpk - 12) * 5 + (jt1k - 1);
            if (low) {
                const int indsp = imin(inds + 1, 10), indfp = imin(indf + 1, 4);
                for (int g = 0; g < NG; ++g) {
                    auto Sv = [&](int i) { return (R)S[(size_t)(i - 1) * NG + g]; };
                    auto Fv = [&](int i) { return (R)F[(size_t)(i - 1) * NG + g]; };
                    c.TG(NS + g, k0) = c1 * ((sum4(A, NG, g, 65, i0, i1, f00, f01, f10, f11)) +
                                             sfac * (Sv(inds) + sfrac * (Sv(indsp) - Sv(inds))) +
                                             ffac * (Fv(indf) + ffrac * (Fv(indfp) - Fv(indf)))) + c2 * (R)co2[g];
                }
            } else {
                for (int g = 0; g < NG; ++g)
                    c.TG(NS + g, k0) = c2 * (sum4(B, NG, g, 235, i0, i1, f00, f01, f10, f11)) + c1 * (R)h2o[g];
            }
        }
    }
    (void)strrat;
}

// ---------------------------------------------------------------------------------------------------
// spcvrtc (phys_rrtm_sw_spcvrtc.cu:65-547) for one day column, all 112 g-points in order.
template <class R>
struct SwExpTable {
    std::vector<R> t;
    SwExpTable()
    {
        const int n = 10000;
        t.assign(n + 1, 0);
        t[0] = 1;
        const double bpade = 1.0 / 0.278;
        for (int i = 1; i < n; ++i) {
            const double tfn = (double)i / ((double)n - i);
            t[i] = (R)std::exp(-bpade * tfn);
        }
        t[n] = (R)1.0e-20f;
    }
};

template <class R>
inline R sw_expm(R zb, const SwExpTable<R>& tb, bool clamped)
{
    const R bpade = (R)1.0f / (R)0.278f;
    if (zb <= (R)0.06f) return (R)1 - zb + (R)0.5f * zb * zb;
    const R ftind = zb / (bpade + zb);
    int it = clamped ? (int)((R)0.5f + (R)10000 * ftind) : (int)(ftind * (R)10000 + (R)0.5f);
    if (clamped) it = imax(0, imin(10000, it));
    return tb.t[it];
}

template <class R>
inline void sw_gam(int iswmode, R zssa1, R zasy1, R zasy3, R cz, R& g1, R& g2, R& g3)
{
    if (iswmode == 1) {
        g1 = (R)1.75f - zssa1 * ((R)1 + zasy3);
        g2 = (R)-0.25f - zssa1 * ((R)1 - zasy3);
        g3 = (R)0.5f - zasy3 * cz;
    } else if (iswmode == 2) {
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

template <class R>
inline void sw_layer_rt(R ztau1, R zssaw, R zssa1, R g1, R g2, R g3, R g4, R cz, R snt, const SwExpTable<R>& tb,
                        R& rb, R& rd, R& tbm, R& td)
{
    const R eps1 = (R)1.0e-8f;
    if (zssaw >= (R)0.9999995f) {
        const R za1 = g1 * cz - g3, za2 = g1 * ztau1;
        const R zb1 = fminR(ztau1 * snt, (R)500);
        const R zb2 = sw_expm(zb1, tb, false);
        rb = fmaxR((R)0, fminR((R)1, (za2 - za1 * ((R)1 - zb2)) / ((R)1 + za2)));
        tbm = fmaxR((R)0, fminR((R)1, (R)1 - rb));
        rd = fmaxR((R)0, fminR((R)1, za2 / ((R)1 + za2)));
        td = fmaxR((R)0, fminR((R)1, (R)1 - rd));
    } else {
        const R za1 = g1 * g4 + g2 * g3, za2 = g1 * g3 + g2 * g4;
        const R zrk = msqrt((g1 - g2) * (g1 + g2));
        const R zrk2 = (R)2 * zrk, zrp = zrk * cz, zrp1 = (R)1 + zrp, zrm1 = (R)1 - zrp;
        R zrpp = (R)1 - zrp * zrp;
        if (mfabs(zrpp) < eps1) zrpp = zrpp < 0 ? -eps1 : eps1;
        const R zrkg1 = zrk + g1, zrkg3 = zrk * g3, zrkg4 = zrk * g4;
        const R zr1 = zrm1 * (za2 + zrkg3), zr2 = zrp1 * (za2 - zrkg3), zr3 = zrk2 * (g3 - za2 * cz);
        const R zr4 = zrpp * zrkg1, zr5 = zrpp * (zrk - g1);
        const R zt1 = zrp1 * (za1 + zrkg4), zt2 = zrm1 * (za1 - zrkg4), zt3 = zrk2 * (g4 + za1 * cz);
        const R zb1 = fminR(zrk * ztau1, (R)500);
        const R zexm1 = sw_expm(zb1, tb, false);
        const R zexp1 = (R)1 / zexm1;
        const R zb2 = fminR(ztau1 * snt, (R)500);
        const R zexm2 = sw_expm(zb2, tb, false);
        const R zexp2 = (R)1 / zexm2;
        const R ze1r45 = zr4 * zexp1 + zr5 * zexm1;
        if (ze1r45 >= -eps1 && ze1r45 <= eps1) {
            rb = eps1;
            tbm = zexm2;
        } else {
            const R zden1 = zssa1 / ze1r45;
            rb = fmaxR((R)0, fminR((R)1, (zr1 * zexp1 - zr2 * zexm1 - zr3 * zexm2) * zden1));
            tbm = fmaxR((R)0, fminR((R)1, zexm2 * ((R)1 - (zt1 * zexp1 - zt2 * zexm1 - zt3 * zexp2) * zden1)));
        }
        const R zden1d = zr4 / (ze1r45 * zrkg1);
        rd = fmaxR((R)0, fminR((R)1, g2 * (zexp1 - zexm1) * zden1d));
        td = fmaxR((R)0, fminR((R)1, zrk2 * zden1d));
    }
}

template <class R>
inline void sw_swflux(const R* zrefb, const R* zrefd, const R* ztrab, const R* ztrad, const R* zldbt, const R* ztdbt,
                      int nlay, int nlp1, R* zfu, R* zfd)
{
    std::vector<R> zrupb(nlp1 + 2), zrupd(nlp1 + 2), zrdnd(nlp1 + 2), ztdn(nlp1 + 2);
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

template <class R>
void sw_spcvrtc(SwColumn<R>& c, const SwExpTable<R>& tb, int iswmode)
{
    static const int IDXSFC[14] = {1, 1, 1, 1, 1, 1, 1, 1, 0, 2, 2, 2, 2, 1};
    const int nlay = c.nlay, nlp1 = nlay + 1;
    const R eps = (R)1.0e-6f, oneminus = (R)1.0f - (R)1.0e-6f, ftiny = (R)1.0e-12f;
    const int LP = nlp1 + 2;
    std::vector<R> zrefb(LP), zrefd(LP), ztrab(LP), ztrad(LP), ztdbt(LP), zldbt(LP), zfu(LP), zfd(LP), ztaus(LP),
        zssas(LP), zasys(LP), zldbt0(LP);
    for (auto* v : {&c.fxupc, &c.fxdnc, &c.fxup0, &c.fxdn0})
        for (auto& x : *v) x = 0;
    for (int n = 0; n < 2; ++n) { c.sfbmc[n] = c.sfdfc[n] = c.sfbm0[n] = c.sfdf0[n] = 0; }
    const R cz = c.cosz, snt = c.sntz, cf1v = c.zcf1, cf0v = c.zcf0;
    auto FX = [&](std::vector<R>& v, int ib, int k) -> R& { return v[(size_t)ib * nlp1 + k]; };
    for (int jg = 1; jg <= 112; ++jg) {
        int ib0 = 0;
        while (!(jg - 1 >= SW_NS[ib0] && jg - 1 < SW_NS[ib0] + SW_NG[ib0])) ++ib0;
        const int ibd = IDXSFC[ib0];
        if (!(cz >= (R)1.0e-4f)) continue;
        const R zsolar = c.ssolar * c.sfluxzen[jg - 1];
        R ztdbt0 = 1;
        ztdbt[nlp1] = 1;
        zldbt[1] = 0;
        if (ibd != 0) { zrefb[1] = c.albbm[ibd - 1]; zrefd[1] = c.albdf[ibd - 1]; }
        else {
            zrefb[1] = (R)0.5f * (c.albbm[0] + c.albbm[1]);
            zrefd[1] = (R)0.5f * (c.albdf[0] + c.albdf[1]);
        }
        ztrab[1] = 0;
        ztrad[1] = 0;
        for (int k = nlay; k >= 1; --k) {
            const int kp = k + 1, q = k - 1;
            const R tr = c.TR(jg - 1, q), tg = c.TG(jg - 1, q);
            const R ta = c.tauae[(size_t)ib0 * nlay + q], sa = c.ssaae[(size_t)ib0 * nlay + q],
                    ya = c.asyae[(size_t)ib0 * nlay + q];
            const R ztau0 = fmaxR(ftiny, tr + tg + ta);
            const R zssa0 = tr + ta * sa;
            const R zasy0 = ya * sa * ta;
            const R zssaw = fminR(oneminus, zssa0 / ztau0);
            const R zasyw = zasy0 / fmaxR(ftiny, zssa0);
            ztaus[k] = ztau0; zssas[k] = zssa0; zasys[k] = zasy0;
            const R za1s = zasyw * zasyw, za2s = zssaw * za1s;
            const R ztau1 = ((R)1 - za2s) * ztau0;
            const R zssa1 = (zssaw - za2s) / ((R)1 - za2s);
            const R zasy1 = zasyw / ((R)1 + zasyw);
            const R zasy3 = (R)0.75f * zasy1;
            R g1, g2, g3;
            sw_gam(iswmode, zssa1, zasy1, zasy3, cz, g1, g2, g3);
            const R g4 = (R)1 - g3;
            sw_layer_rt(ztau1, zssaw, zssa1, g1, g2, g3, g4, cz, snt, tb, zrefb[kp], zrefd[kp], ztrab[kp], ztrad[kp]);
            R zr1 = ztau1 * snt;
            const R zexp3 = sw_expm(zr1, tb, true);
            ztdbt[k] = zexp3 * ztdbt[kp];
            zldbt[kp] = zexp3;
            zr1 = ztau0 * snt;
            const R zexp4 = sw_expm(zr1, tb, true);
            zldbt0[k] = zexp4;
            ztdbt0 = zexp4 * ztdbt0;
        }
        sw_swflux(zrefb.data(), zrefd.data(), ztrab.data(), ztrad.data(), zldbt.data(), ztdbt.data(), nlay, nlp1,
                  zfu.data(), zfd.data());
        for (int k = 1; k <= nlp1; ++k) {
            FX(c.fxup0, ib0, k - 1) = FX(c.fxup0, ib0, k - 1) + zsolar * zfu[k];
            FX(c.fxdn0, ib0, k - 1) = FX(c.fxdn0, ib0, k - 1) + zsolar * zfd[k];
        }
        {
            const R zb1 = zsolar * ztdbt0, zb2 = zsolar * (zfd[1] - ztdbt0);
            if (ibd != 0) { c.sfbm0[ibd - 1] = c.sfbm0[ibd - 1] + zb1; c.sfdf0[ibd - 1] = c.sfdf0[ibd - 1] + zb2; }
            else {
                const R zf1 = (R)0.5f * zb1, zf2 = (R)0.5f * zb2;
                c.sfbm0[0] = c.sfbm0[0] + zf1; c.sfdf0[0] = c.sfdf0[0] + zf2;
                c.sfbm0[1] = c.sfbm0[1] + zf1; c.sfdf0[1] = c.sfdf0[1] + zf2;
            }
        }
        if (cf1v > eps) {
            ztdbt0 = 1;
            zldbt[1] = 0;
            for (int k = nlay; k >= 1; --k) {
                const int kp = k + 1, q = k - 1;
                const R zc1 = c.cldfrc[q], zc0 = (R)1 - zc1;
                if (zc1 > ftiny) {
                    const R ztau0 = ztaus[k] + c.taucw[(size_t)ib0 * nlay + q];
                    const R zssa0 = zssas[k] + c.ssacw[(size_t)ib0 * nlay + q];
                    const R zasy0 = zasys[k] + c.asycw[(size_t)ib0 * nlay + q];
                    const R zssaw = fminR(oneminus, zssa0 / ztau0);
                    const R zasyw = zasy0 / fmaxR(ftiny, zssa0);
                    const R za1s = zasyw * zasyw, za2s = zssaw * za1s;
                    const R ztau1 = ((R)1 - za2s) * ztau0;
                    const R zssa1 = (zssaw - za2s) / ((R)1 - za2s);
                    const R zasy1 = zasyw / ((R)1 + zasyw);
                    const R zasy3 = (R)0.75f * zasy1;
                    R g1, g2, g3;
                    sw_gam(iswmode, zssa1, zasy1, zasy3, cz, g1, g2, g3);
                    const R g4 = (R)1 - g3;
                    const R rb1 = zrefb[kp], rd1 = zrefd[kp], tb1 = ztrab[kp], td1 = ztrad[kp];
                    sw_layer_rt(ztau1, zssaw, zssa1, g1, g2, g3, g4, cz, snt, tb, zrefb[kp], zrefd[kp], ztrab[kp],
                                ztrad[kp]);
                    zrefb[kp] = zc0 * rb1 + zc1 * zrefb[kp];
                    zrefd[kp] = zc0 * rd1 + zc1 * zrefd[kp];
                    ztrab[kp] = zc0 * tb1 + zc1 * ztrab[kp];
                    ztrad[kp] = zc0 * td1 + zc1 * ztrad[kp];
                    R zr1 = ztau1 * snt;
                    const R zexp3 = sw_expm(zr1, tb, true);
                    zldbt[kp] = zc0 * zldbt[kp] + zc1 * zexp3;
                    ztdbt[k] = zldbt[kp] * ztdbt[kp];
                    zr1 = ztau0 * snt;
                    const R zexp4 = sw_expm(zr1, tb, true);
                    ztdbt0 = (zc0 * zldbt0[k] + zc1 * zexp4) * ztdbt0;
                } else {
                    ztdbt[k] = zldbt[kp] * ztdbt[kp];
                    ztdbt0 = zldbt0[k] * ztdbt0;
                }
            }
            sw_swflux(zrefb.data(), zrefd.data(), ztrab.data(), ztrad.data(), zldbt.data(), ztdbt.data(), nlay, nlp1,
                      zfu.data(), zfd.data());
            for (int k = 1; k <= nlp1; ++k) {
                FX(c.fxupc, ib0, k - 1) = FX(c.fxupc, ib0, k - 1) + zsolar * zfu[k];
                FX(c.fxdnc, ib0, k - 1) = FX(c.fxdnc, ib0, k - 1) + zsolar * zfd[k];
            }
            const R zb1 = zsolar * ztdbt0, zb2 = zsolar * (zfd[1] - ztdbt0);
            if (ibd != 0) { c.sfbmc[ibd - 1] = c.sfbmc[ibd - 1] + zb1; c.sfdfc[ibd - 1] = c.sfdfc[ibd - 1] + zb2; }
            else {
                const R zf1 = (R)0.5f * zb1, zf2 = (R)0.5f * zb2;
                c.sfbmc[0] = c.sfbmc[0] + zf1; c.sfdfc[0] = c.sfdfc[0] + zf2;
                c.sfbmc[1] = c.sfbmc[1] + zf1; c.sfdfc[1] = c.sfdfc[1] + zf2;
            }
        }
    }
    // column end section (band sums, cf1 weighting)
    R s_adc = 0, s_au0 = 0, s_su0 = 0, s_sd0 = 0;
    for (int ib = 0; ib < 14; ++ib) {
        s_adc = s_adc + FX(c.fxdn0, ib, nlp1 - 1);
        s_au0 = s_au0 + FX(c.fxup0, ib, nlp1 - 1);
        s_su0 = s_su0 + FX(c.fxup0, ib, 0);
        s_sd0 = s_sd0 + FX(c.fxdn0, ib, 0);
    }
    c.ftoadc = s_adc; c.ftoau0 = s_au0; c.fsfcu0 = s_su0; c.fsfcd0 = s_sd0;
    c.suvbf0 = FX(c.fxdn0, 11, 0);
    c.suvbfc = c.suvbf0;
    if (cf1v <= eps) {
        c.fxupc = c.fxup0; c.fxdnc = c.fxdn0;
        c.ftoauc = c.ftoau0; c.fsfcuc = c.fsfcu0; c.fsfcdc = c.fsfcd0;
        for (int n = 0; n < 2; ++n) { c.sfbmc[n] = c.sfbm0[n]; c.sfdfc[n] = c.sfdf0[n]; }
    } else {
        for (int ib = 0; ib < 14; ++ib)
            for (int k = 0; k < nlp1; ++k) {
                FX(c.fxupc, ib, k) = cf1v * FX(c.fxupc, ib, k) + cf0v * FX(c.fxup0, ib, k);
                FX(c.fxdnc, ib, k) = cf1v * FX(c.fxdnc, ib, k) + cf0v * FX(c.fxdn0, ib, k);
            }
        R t_au = 0, t_su = 0, t_sd = 0;
        for (int ib = 0; ib < 14; ++ib) {
            t_au = t_au + FX(c.fxupc, ib, nlp1 - 1);
            t_su = t_su + FX(c.fxupc, ib, 0);
            t_sd = t_sd + FX(c.fxdnc, ib, 0);
        }
        c.ftoauc = t_au; c.fsfcuc = t_su; c.fsfcdc = t_sd;
        c.suvbfc = FX(c.fxdnc, 11, 0);
        for (int n = 0; n < 2; ++n) {
            c.sfbmc[n] = cf1v * c.sfbmc[n] + cf0v * c.sfbm0[n];
            c.sfdfc[n] = cf1v * c.sfdfc[n] + cf0v * c.sfdf0[n];
        }
    }
}

}  // namespace orc
