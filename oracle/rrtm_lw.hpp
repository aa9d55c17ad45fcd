// rrtm_lw.hpp -- CPU oracle: RRTM longwave column solve (NAM route), one column at a time.
//
// Restates, statement by statement, the reference's LW chain for one column:
//   lwrad_prep        namgpu/kernels/phys_rrtm_lw_lwrad.cu:98-303
//   cldprop           namgpu/kernels/phys_rrtm_lw_cldprop.cu:79-243 (ilwcice = 1)
//   setcoef           namgpu/kernels/phys_rrtm_lw_setcoef.cu:82-244
//   taumol bands      namgpu/kernels/phys_rrtm_lw_taugb01.cu .. taugb16.cu (+ tautot, lw_core.py:83-90)
//   rtrnmr            namgpu/kernels/phys_rrtm_lw_rtrnmr_body.cuh:9-365 (surface-first variant)
//   rtrn              namgpu/kernels/phys_rrtm_lw_rtrn.cu:94-330 (random overlap, iovrlw = 0)
//   lwrad_post        namgpu/kernels/phys_rrtm_lw_lwrad.cu:316-366
// and the grrad glue around it (cloud-path factor, phys_rrtm_grrad_lw.cu:58-80).
// Test infrastructure only: never linked into the product.
#pragma once
#include "rrtm_common.hpp"

namespace orc {

template <class R>
struct LwColumn {
    int nlay = 0;
    // lwrad_prep scratch (internal order: index 0 = surface layer)
    std::vector<R> pavel, tavel, delp, tz, coldry, colbrd, h2ovmr, cldfrc, taucld, tauaer, secdiff, semiss;
    std::vector<R> colamt;   // [7][nlay]
    std::vector<R> wx;       // [4][nlay]
    std::vector<R> cldin;    // [8][nlay]
    R pwvcm = 0, stemp = 0;
    int lcf1 = 0;
    // setcoef outputs
    int laytrop = 0;
    std::vector<int> jp, jt, jt1, indself, indfor, indminor;
    std::vector<R> fac00, fac01, fac10, fac11, selffac, selffrac, forfac, forfrac, minorfrac, scaleminor,
        scaleminorn2;
    std::vector<R> rfrate;   // [2][6][nlay] (side, rate, k)
    std::vector<R> pklay, pklev;  // [nlay+1][16]
    // taumol
    std::vector<R> taug, fracs;   // [140][nlay]
    // rtrnmr outputs (internal order)
    std::vector<R> totuflux, totdflux, totuclfl, totdclfl, htr;
    std::vector<R> fnetb;         // [16][nlay+1] net flux of each band, (up - down) x flxfac (lhlwb's fnet)
    std::vector<R> cldfmc;        // McICA route: [140][nlay]

    explicit LwColumn(int n) : nlay(n) {
        const int L = n, P = n + 1;
        pavel.assign(L, 0); tavel.assign(L, 0); delp.assign(L, 0); tz.assign(P, 0); coldry.assign(L, 0);
        colbrd.assign(L, 0); h2ovmr.assign(L, 0); cldfrc.assign(P + 1, 0); taucld.assign(16 * L, 0);
        tauaer.assign(16 * L, 0); secdiff.assign(16, 0); semiss.assign(16, 0);
        colamt.assign(7 * L, 0); wx.assign(4 * L, 0); cldin.assign(8 * L, 0);
        jp.assign(L, 0); jt.assign(L, 0); jt1.assign(L, 0); indself.assign(L, 0); indfor.assign(L, 0);
        indminor.assign(L, 0);
        for (auto* v : {&fac00, &fac01, &fac10, &fac11, &selffac, &selffrac, &forfac, &forfrac, &minorfrac,
                        &scaleminor, &scaleminorn2})
            v->assign(L, 0);
        rfrate.assign(2 * 6 * L, 0);
        pklay.assign(P * 16, 0); pklev.assign(P * 16, 0);
        taug.assign(140 * L, 0); fracs.assign(140 * L, 0);
        totuflux.assign(P, 0); totdflux.assign(P, 0); totuclfl.assign(P, 0); totdclfl.assign(P, 0);
        htr.assign(L, 0);
        fnetb.assign(16 * P, 0);
    }
    R& CA(int m, int k0) { return colamt[(size_t)m * nlay + k0]; }     // colamt(k, m+1)
    R& WX(int m, int k0) { return wx[(size_t)m * nlay + k0]; }
    R& RF(int side, int rate, int k0) { return rfrate[((size_t)side * 6 + rate) * nlay + k0]; }
    R& TG(int g, int k0) { return taug[(size_t)g * nlay + k0]; }
    R& FR(int g, int k0) { return fracs[(size_t)g * nlay + k0]; }
};

// ---------------------------------------------------------------------------------------------------
// lwrad_prep (phys_rrtm_lw_lwrad.cu:98-303), ivflip = 0, ilwrgas = 1, isubclw as configured.
// clouds9 holds this column's [9][nlay] cloud fields (top first) after the cloud-path factor.
template <class R>
void lw_prep(LwColumn<R>& c, const Inputs& in, int col, const float* clouds9, int ilwcliq)
{
    const int nlay = c.nlay, N = in.ncol;
    auto IN = [&](const float* a, int lev) { return (R)a[(size_t)lev * N + col]; };
    const R amdw = (R)CON_AMD / (R)CON_AMW, amdo3 = (R)CON_AMD / (R)CON_AMO3, eps = (R)1.0e-6;
    const R tem1g = (R)100.0 * (R)CON_G;
    const R tem2c = (R)1.0e-20 * (R)1.0e3 * (R)CON_AVGD;
    c.tz[0] = IN(in.tlvl, nlay);
    for (int k0 = 0; k0 < nlay; ++k0) {
        const int kin = nlay - 1 - k0;
        const R dlp = IN(in.plvl, nlay - k0) - IN(in.plvl, nlay - k0 - 1);
        const R tzk = IN(in.tlvl, nlay - k0 - 1);
        const R qv = IN(in.qlyr, kin), ov = IN(in.olyr, kin);
        c.pavel[k0] = IN(in.plyr, kin);
        c.tavel[k0] = IN(in.tlyr, kin);
        c.delp[k0] = dlp;
        c.tz[k0 + 1] = tzk;
        const R h2ovmr = fmaxR((R)0, qv * amdw / ((R)1 - qv));
        const R o3vmr = fmaxR((R)0, ov * amdo3);
        const R tem0 = ((R)1 - h2ovmr) * (R)CON_AMD + h2ovmr * (R)CON_AMW;
        const R cdry = tem2c * dlp / (tem1g * tem0 * ((R)1 + h2ovmr));
        const R temcol = (R)1.0e-12 * cdry;
        c.coldry[k0] = cdry;
        auto G = [&](int n) { return (R)in.gasvmr[((size_t)n * nlay + kin) * N + col]; };
        c.CA(0, k0) = fmaxR((R)0, cdry * h2ovmr);
        c.CA(1, k0) = fmaxR(temcol, cdry * G(0));
        c.CA(2, k0) = fmaxR(temcol, cdry * o3vmr);
        c.CA(3, k0) = fmaxR(temcol, cdry * G(1));
        c.CA(4, k0) = fmaxR(temcol, cdry * G(2));
        c.CA(5, k0) = fmaxR((R)0, cdry * G(3));
        c.CA(6, k0) = fmaxR((R)0, cdry * G(4));
        c.WX(0, k0) = fmaxR((R)0, cdry * G(8));
        c.WX(1, k0) = fmaxR((R)0, cdry * G(5));
        c.WX(2, k0) = fmaxR((R)0, cdry * G(6));
        c.WX(3, k0) = fmaxR((R)0, cdry * G(7));
        for (int b = 0; b < 16; ++b) {
            R tau = 0, ssa = 0;
            if (in.faerlw) {
                tau = (R)in.faerlw[(((size_t)0 * 16 + b) * nlay + kin) * N + col];
                ssa = (R)in.faerlw[(((size_t)1 * 16 + b) * nlay + kin) * N + col];
            }
            c.tauaer[(size_t)b * nlay + k0] = tau * ((R)1 - ssa);
        }
        if (ilwcliq > 0) {
            c.cldfrc[k0 + 1] = (R)clouds9[0 * nlay + kin];
            for (int s = 0; s < 8; ++s) c.cldin[(size_t)s * nlay + k0] = (R)clouds9[(s + 1) * nlay + kin];
        } else {
            c.cldfrc[k0 + 1] = (R)clouds9[0 * nlay + kin];
            c.cldin[(size_t)4 * nlay + k0] = (R)clouds9[1 * nlay + kin];
        }
    }
    c.cldfrc[0] = 1;
    c.cldfrc[nlay + 1] = 0;
    for (int k0 = 0; k0 < nlay; ++k0) {
        R summol = 0;
        for (int m = 1; m < 7; ++m) summol = summol + c.CA(m, k0);
        c.colbrd[k0] = c.coldry[k0] - summol;
    }
    R tem1 = 0, tem2 = 0;
    for (int k0 = 0; k0 < nlay; ++k0) {
        tem1 = tem1 + c.coldry[k0] + c.CA(0, k0);
        tem2 = tem2 + c.CA(0, k0);
    }
    const R tem0p = (R)10.0 * tem2 / (amdw * tem1 * (R)CON_G);
    const R pwv = tem0p * IN(in.plvl, nlay);
    c.pwvcm = pwv;
    static const float A0[16] = {1.66f, 1.55f, 1.58f, 1.66f, 1.54f, 1.454f, 1.89f, 1.33f, 1.668f, 1.66f,
                                 1.66f, 1.66f, 1.66f, 1.66f, 1.66f, 1.66f};
    static const float A1[16] = {0.00f, 0.25f, 0.22f, 0.00f, 0.13f, 0.446f, -0.10f, 0.40f, -0.006f, 0.00f,
                                 0.00f, 0.00f, 0.00f, 0.00f, 0.00f, 0.00f};
    static const float A2[16] = {0.00f, -12.0f, -11.7f, 0.00f, -0.72f, -0.243f, 0.19f, -0.062f, 0.414f,
                                 0.00f, 0.00f, 0.00f, 0.00f, 0.00f, 0.00f, 0.00f};
    for (int b = 0; b < 16; ++b) {
        const int j1 = b + 1;
        if (j1 == 1 || j1 == 4 || j1 == 10) c.secdiff[b] = (R)1.66f;
        else c.secdiff[b] = fminR((R)1.80f, fmaxR((R)1.50f, (R)A0[b] + (R)A1[b] * mexp((R)A2[b] * pwv)));
    }
    int lcf = 0;
    for (int k = 1; k <= nlay; ++k)
        if (c.cldfrc[k] > eps) { lcf = 1; break; }
    c.lcf1 = lcf;
    const R sfe = (R)in.sfcemis[col];
    for (int b = 0; b < 16; ++b) c.semiss[b] = (sfe > eps && sfe <= (R)1) ? sfe : (R)1;
    c.stemp = (R)in.tsfg[col];
    // lw_core.seam: h2ovmr = colamt(h2o) / max(coldry, 1e-30) (lw_core.py:237-238)
    for (int k0 = 0; k0 < nlay; ++k0) c.h2ovmr[k0] = c.CA(0, k0) / fmaxR(c.coldry[k0], (R)1e-30f);
}

// ---------------------------------------------------------------------------------------------------
// cldprop (phys_rrtm_lw_cldprop.cu:79-243): ilwcliq = 1 with ilwcice = 1 (NAM), or ilwcliq = 0.
template <class R>
void lw_cldprop(LwColumn<R>& c, const float* clouds9, int ilwcliq)
{
    const int nlay = c.nlay;
    const TableStore& T = tables();
    auto CL = [&](int n, int k0) { return (R)clouds9[n * nlay + (nlay - 1 - k0)]; };
    for (auto& v : c.taucld) v = 0;
    int lcf1 = 0;
    for (int k0 = 0; k0 < nlay && !lcf1; ++k0)
        if (CL(0, k0) > (R)1.0e-6f) lcf1 = 1;
    if (!lcf1) return;
    const R absrain = (R)0.33e-3f, abssnow0 = (R)1.5f, cldmin = 0;
    const double* absliq1 = T.f("lw_absliq1");
    const double* absice1 = T.f("lw_absice1");
    const int* ipat = T.i("lw_ipat");
    if (ilwcliq > 0) {
        for (int k0 = 0; k0 < nlay; ++k0) {
            const R cf = CL(0, k0);
            if (!(cf > cldmin)) continue;
            R tauran = absrain * CL(5, k0);
            R tausnw = (CL(7, k0) > 0 && CL(8, k0) > (R)10) ? abssnow0 * (R)1.05756f * CL(7, k0) / CL(8, k0) : (R)0;
            const R cldliq = CL(1, k0), cldice = CL(3, k0), refliq = CL(2, k0);
            R refice = CL(4, k0);
            R tauliq[16], tauice[16];
            for (int b = 0; b < 16; ++b) { tauliq[b] = 0; tauice[b] = 0; }
            if (cldliq > 0) {
                const R factor = refliq - (R)1.5f;
                const int index = imax(1, imin(57, (int)factor));
                const R fint = factor - (R)index;
                for (int b = 0; b < 16; ++b) {
                    const R a1 = (R)absliq1[b * 58 + index - 1], a2 = (R)absliq1[b * 58 + index];
                    tauliq[b] = fmaxR((R)0, cldliq * (a1 + fint * (a2 - a1)));
                }
            }
            if (cldice > 0) {
                refice = fminR((R)130, fmaxR((R)13, refice));
                for (int b = 0; b < 16; ++b) {
                    const int ia0 = ipat[b] - 1;
                    tauice[b] = fmaxR((R)0, cldice * ((R)absice1[ia0 * 2 + 0] + (R)absice1[ia0 * 2 + 1] / refice));
                }
            }
            for (int b = 0; b < 16; ++b)
                c.taucld[(size_t)b * nlay + k0] = tauice[b] + tauliq[b] + tauran + tausnw;
        }
    } else {
        for (int k0 = 0; k0 < nlay; ++k0)
            if (CL(0, k0) > cldmin) {
                const R v = CL(1, k0);
                for (int b = 0; b < 16; ++b) c.taucld[(size_t)b * nlay + k0] = v;
            }
    }
}

// ---------------------------------------------------------------------------------------------------
// setcoef (phys_rrtm_lw_setcoef.cu:82-244)
template <class R>
void lw_setcoef(LwColumn<R>& c)
{
    const TableStore& T = tables();
    const double* totplnk = T.f("lw_totplnk");
    const double* delwave = T.f("lw_delwave");
    const double* preflog = T.f("lw_preflog");
    const double* tref = T.f("lw_tref");
    const double* chi = T.f("lw_chi_mls");   // [59][7]
    auto TOT = [&](int k, int b) { return (R)totplnk[(size_t)(b - 1) * 181 + (k - 1)]; };
    auto CHI = [&](int g, int lev) { return (R)chi[(size_t)(lev - 1) * 7 + (g - 1)]; };
    const int nlay = c.nlay;
    const R stpfac = (R)296.0f / (R)1013.0f;
    {
        const R stemp_v = c.stemp, tz0 = c.tz[0];
        const int indlay0 = imin(180, imax(1, (int)(stemp_v - (R)159)));
        const int indlev0 = imin(180, imax(1, (int)(tz0 - (R)159)));
        const R tlyrfr0 = stemp_v - (R)((int)stemp_v);
        const R tlvlfr0 = tz0 - (R)((int)tz0);
        for (int i = 1; i <= 16; ++i) {
            const R tem1 = TOT(indlay0 + 1, i) - TOT(indlay0, i);
            const R tem2 = TOT(indlev0 + 1, i) - TOT(indlev0, i);
            c.pklay[0 * 16 + i - 1] = (R)delwave[i - 1] * (TOT(indlay0, i) + tlyrfr0 * tem1);
            c.pklev[0 * 16 + i - 1] = (R)delwave[i - 1] * (TOT(indlev0, i) + tlvlfr0 * tem2);
        }
    }
    int laytrop = 0;
    for (int k = 1; k <= nlay; ++k) {
        const int k0 = k - 1;
        const R pav = c.pavel[k0], tav = c.tavel[k0], tzk = c.tz[k];
        const int indlay = imin(180, imax(1, (int)(tav - (R)159)));
        const R tlyrfr = tav - (R)((int)tav);
        const int indlev = imin(180, imax(1, (int)(tzk - (R)159)));
        const R tlvlfr = tzk - (R)((int)tzk);
        for (int i = 1; i <= 16; ++i) {
            c.pklay[k * 16 + i - 1] = (R)delwave[i - 1] * (TOT(indlay, i) + tlyrfr * (TOT(indlay + 1, i) - TOT(indlay, i)));
            c.pklev[k * 16 + i - 1] = (R)delwave[i - 1] * (TOT(indlev, i) + tlvlfr * (TOT(indlev + 1, i) - TOT(indlev, i)));
        }
        const R plog = mlog(pav);
        const int jpk = imax(1, imin(58, (int)((R)36 - (R)5 * (plog + (R)0.04f))));
        const int jp1 = jpk + 1;
        const R fp = fmaxR((R)0, fminR((R)1, (R)5 * ((R)preflog[jpk - 1] - plog)));
        const R tem1t = (tav - (R)tref[jpk - 1]) / (R)15;
        const R tem2t = (tav - (R)tref[jp1 - 1]) / (R)15;
        const int jtk = imax(1, imin(4, (int)((R)3 + tem1t)));
        const int jt1k = imax(1, imin(4, (int)((R)3 + tem2t)));
        const R ft = fmaxR((R)-0.5f, fminR((R)1.5f, tem1t - (R)(jtk - 3)));
        const R ft1 = fmaxR((R)-0.5f, fminR((R)1.5f, tem2t - (R)(jt1k - 3)));
        c.jp[k0] = jpk; c.jt[k0] = jtk; c.jt1[k0] = jt1k;
        const R tem1 = (R)1 - fp;
        c.fac10[k0] = tem1 * ft;
        c.fac00[k0] = tem1 * ((R)1 - ft);
        c.fac11[k0] = fp * ft1;
        c.fac01[k0] = fp * ((R)1 - ft1);
        const R h2o = c.h2ovmr[k0];
        const R forf = pav * stpfac / (tav * ((R)1 + h2o));
        const R selff = h2o * forf;
        c.scaleminor[k0] = pav / tav;
        c.scaleminorn2[k0] = (pav / tav) * (c.colbrd[k0] / (c.coldry[k0] + c.CA(0, k0)));
        const R tem1m = (tav - (R)180.8f) / (R)7.2f;
        const int indmin = imin(18, imax(1, (int)tem1m));
        c.indminor[k0] = indmin;
        c.minorfrac[k0] = tem1m - (R)indmin;
        if (plog > (R)4.56f) {
            laytrop += 1;
            const R tem1f = ((R)332 - tav) / (R)36;
            const int indf = imin(2, imax(1, (int)tem1f));
            c.indfor[k0] = indf;
            c.forfrac[k0] = tem1f - (R)indf;
            const R tem1s = (tav - (R)188) / (R)7.2f;
            const int inds = imin(9, imax(1, (int)tem1s - 7));
            c.indself[k0] = inds;
            c.selffrac[k0] = tem1s - (R)(inds + 7);
            c.RF(0, 0, k0) = CHI(1, jpk) / CHI(2, jpk);  c.RF(1, 0, k0) = CHI(1, jp1) / CHI(2, jp1);
            c.RF(0, 1, k0) = CHI(1, jpk) / CHI(3, jpk);  c.RF(1, 1, k0) = CHI(1, jp1) / CHI(3, jp1);
            c.RF(0, 2, k0) = CHI(1, jpk) / CHI(4, jpk);  c.RF(1, 2, k0) = CHI(1, jp1) / CHI(4, jp1);
            c.RF(0, 3, k0) = CHI(1, jpk) / CHI(6, jpk);  c.RF(1, 3, k0) = CHI(1, jp1) / CHI(6, jp1);
            c.RF(0, 4, k0) = CHI(4, jpk) / CHI(2, jpk);  c.RF(1, 4, k0) = CHI(4, jp1) / CHI(2, jp1);
        } else {
            const R tem1f = (tav - (R)188) / (R)36;
            c.indfor[k0] = 3;
            c.forfrac[k0] = tem1f - (R)1;
            c.indself[k0] = 0;
            c.selffrac[k0] = 0;
            c.RF(0, 0, k0) = CHI(1, jpk) / CHI(2, jpk);  c.RF(1, 0, k0) = CHI(1, jp1) / CHI(2, jp1);
            c.RF(0, 5, k0) = CHI(3, jpk) / CHI(2, jpk);  c.RF(1, 5, k0) = CHI(3, jp1) / CHI(2, jp1);
        }
        c.selffac[k0] = c.CA(0, k0) * selff;
        c.forfac[k0] = c.CA(0, k0) * forf;
    }
    c.laytrop = laytrop;
}

// Lower-atmosphere interpolation weights of the binary-species bands: the three-branch fk/id selection
// (e.g. phys_rrtm_lw_taugb03.cu:158-199).  `joint` selects the bands that test specparm and specparm1
// together (bands 5, 7, 9, 12, 13, 15, 16) rather than each on its own (bands 3, 4).
template <class R>
struct Sel { R fk0, fk1, fk2; int id[6]; };

template <class R>
inline Sel<R> sel_branch(int branch, R fs, int ind)
{
    Sel<R> s;
    if (branch == 0) {           // specparm < 0.125
        const R p = fs - (R)1, p2 = p * p, p4 = p2 * p2;
        s.fk0 = p4; s.fk1 = (R)1 - p - (R)2 * p4; s.fk2 = p + p4;
        s.id[0] = ind; s.id[1] = ind + 9; s.id[2] = ind + 1; s.id[3] = ind + 10; s.id[4] = ind + 2; s.id[5] = ind + 11;
    } else if (branch == 1) {    // specparm > 0.875
        const R p = -fs, p2 = p * p, p4 = p2 * p2;
        s.fk0 = p4; s.fk1 = (R)1 - p - (R)2 * p4; s.fk2 = p + p4;
        s.id[0] = ind + 1; s.id[1] = ind + 10; s.id[2] = ind; s.id[3] = ind + 9; s.id[4] = ind - 1; s.id[5] = ind + 8;
    } else {
        s.fk0 = (R)1 - fs; s.fk1 = fs; s.fk2 = 0;
        s.id[0] = ind; s.id[1] = ind + 9; s.id[2] = ind + 1; s.id[3] = ind + 10; s.id[4] = ind; s.id[5] = ind;
    }
    return s;
}

// specparm/specmult/js/fs of a binary-species key (e.g. phys_rrtm_lw_taugb03.cu:123-128).
template <class R>
inline void spec(R c1, R rat, R c2, R mult, R& speccomb, R& specparm, int& js, R& fs)
{
    const R oneminus = (R)1.0f - (R)1.0e-6f;
    speccomb = c1 + rat * c2;
    specparm = c1 / speccomb;
    const R specmult = mult * fminR(specparm, oneminus);
    js = 1 + (int)specmult;
    fs = fmod1(specmult);
}

// 12-point major-species sum of the lower atmosphere (speccomb * sum + speccomb1 * sum).
template <class R>
inline R major12(const double* absa, int ng, int ig0, R speccomb, const Sel<R>& s0, R f00, R f10,
                 R speccomb1, const Sel<R>& s1, R f01, R f11)
{
    auto A = [&](int id) { return (R)absa[(size_t)(id - 1) * ng + ig0]; };
    const R fac000 = s0.fk0 * f00, fac100 = s0.fk1 * f00, fac200 = s0.fk2 * f00;
    const R fac010 = s0.fk0 * f10, fac110 = s0.fk1 * f10, fac210 = s0.fk2 * f10;
    const R fac001 = s1.fk0 * f01, fac101 = s1.fk1 * f01, fac201 = s1.fk2 * f01;
    const R fac011 = s1.fk0 * f11, fac111 = s1.fk1 * f11, fac211 = s1.fk2 * f11;
    const R t0 = speccomb * (fac000 * A(s0.id[0]) + fac010 * A(s0.id[1]) + fac100 * A(s0.id[2]) +
                             fac110 * A(s0.id[3]) + fac200 * A(s0.id[4]) + fac210 * A(s0.id[5]));
    const R t1 = speccomb1 * (fac001 * A(s1.id[0]) + fac011 * A(s1.id[1]) + fac101 * A(s1.id[2]) +
                              fac111 * A(s1.id[3]) + fac201 * A(s1.id[4]) + fac211 * A(s1.id[5]));
    return t0 + t1;
}

template <class R>
inline int branch_of(R specparm) { return specparm < (R)0.125f ? 0 : (specparm > (R)0.875f ? 1 : 2); }
template <class R>
inline int branch_joint(R sp, R sp1)
{
    if (sp < (R)0.125f && sp1 < (R)0.125f) return 0;
    if (sp > (R)0.875f && sp1 > (R)0.875f) return 1;
    return 2;
}

template <class R>
inline R interp(const double* t, int ng, int ind, int ig0, R frac)   // t(ig, ind) + frac*(t(ig, ind+1) - t(ig, ind))
{
    const R a = (R)t[(size_t)(ind - 1) * ng + ig0], b = (R)t[(size_t)ind * ng + ig0];
    return a + frac * (b - a);
}

// ---------------------------------------------------------------------------------------------------
// taumol: the sixteen LW bands.  Each block below restates one reference kernel; the lower loop runs
// k = 1..laytrop and the upper loop k = laytrop+1..nlay exactly as there.
template <class R>
void lw_taumol(LwColumn<R>& c)
{
    const TableStore& T = tables();
    const int nlay = c.nlay, lt = c.laytrop;
    const double* chi = T.f("lw_chi_mls");
    auto CHI = [&](int g, int lev) { return (R)chi[(size_t)(lev - 1) * 7 + (g - 1)]; };
    auto t = [&](const char* n) { return T.f(n); };

    // ---- band 1 (phys_rrtm_lw_taugb01.cu:62-172)
    {
        const int NG = 10, NS = 0;
        const double *absa = t("lw01_absa"), *absb = t("lw01_absb"), *selfref = t("lw01_selfref"),
                     *forref = t("lw01_forref"), *ka = t("lw01_ka_mn2"), *kb = t("lw01_kb_mn2"),
                     *fa = t("lw01_fracrefa"), *fb = t("lw01_fracrefb");
        for (int k0 = 0; k0 < nlay; ++k0) {
            const R pp = c.pavel[k0];
            const R scalen2 = c.colbrd[k0] * c.scaleminorn2[k0];
            const R col = c.CA(0, k0);
            const int indf = c.indfor[k0], indm = c.indminor[k0];
            if (k0 + 1 <= lt) {
                const int ind0 = ((c.jp[k0] - 1) * 5 + (c.jt[k0] - 1)) * 1 + 1;
                const int ind1 = (c.jp[k0] * 5 + (c.jt1[k0] - 1)) * 1 + 1;
                const int inds = c.indself[k0];
                const R corradj = (pp < (R)250) ? ((R)1 - (R)0.15f * ((R)250 - pp) / (R)154.4f) : (R)1;
                for (int ig = 0; ig < NG; ++ig) {
                    const R tauself = c.selffac[k0] * interp(selfref, NG, inds, ig, c.selffrac[k0]);
                    const R taufor = c.forfac[k0] * interp(forref, NG, indf, ig, c.forfrac[k0]);
                    const R taun2 = scalen2 * interp(ka, NG, indm, ig, c.minorfrac[k0]);
                    auto A = [&](int id) { return (R)absa[(size_t)(id - 1) * NG + ig]; };
                    c.TG(NS + ig, k0) = corradj * (col * (c.fac00[k0] * A(ind0) + c.fac10[k0] * A(ind0 + 1) +
                                                          c.fac01[k0] * A(ind1) + c.fac11[k0] * A(ind1 + 1)) +
                                                   tauself + taufor + taun2);
                    c.FR(NS + ig, k0) = (R)fa[ig];
                }
            } else {
                const int ind0 = ((c.jp[k0] - 13) * 5 + (c.jt[k0] - 1)) * 1 + 1;
                const int ind1 = ((c.jp[k0] - 12) * 5 + (c.jt1[k0] - 1)) * 1 + 1;
                const R corradj = (R)1 - (R)0.15f * (pp / (R)95.6f);
                for (int ig = 0; ig < NG; ++ig) {
                    const R taufor = c.forfac[k0] * interp(forref, NG, indf, ig, c.forfrac[k0]);
                    const R taun2 = scalen2 * interp(kb, NG, indm, ig, c.minorfrac[k0]);
                    auto B = [&](int id) { return (R)absb[(size_t)(id - 1) * NG + ig]; };
                    c.TG(NS + ig, k0) = corradj * (col * (c.fac00[k0] * B(ind0) + c.fac10[k0] * B(ind0 + 1) +
                                                          c.fac01[k0] * B(ind1) + c.fac11[k0] * B(ind1 + 1)) +
                                                   taufor + taun2);
                    c.FR(NS + ig, k0) = (R)fb[ig];
                }
            }
        }
    }
    // ---- band 2 (phys_rrtm_lw_taugb02.cu:283-395)
    {
        const int NG = 12, NS = 10;
        const double *absa = t("lw02_absa"), *absb = t("lw02_absb"), *selfref = t("lw02_selfref"),
                     *forref = t("lw02_forref"), *fa = t("lw02_fracrefa"), *fb = t("lw02_fracrefb");
        for (int k0 = 0; k0 < nlay; ++k0) {
            const R col = c.CA(0, k0);
            const int indf = c.indfor[k0];
            if (k0 < lt) {
                const int ind0 = (c.jp[k0] - 1) * 5 + (c.jt[k0] - 1) + 1;
                const int ind1 = c.jp[k0] * 5 + (c.jt1[k0] - 1) + 1;
                const R corradj = (R)1 - (R)0.05f * (c.pavel[k0] - (R)100) / (R)900;
                for (int ig = 0; ig < NG; ++ig) {
                    const R tauself = c.selffac[k0] * interp(selfref, NG, c.indself[k0], ig, c.selffrac[k0]);
                    const R taufor = c.forfac[k0] * interp(forref, NG, indf, ig, c.forfrac[k0]);
                    auto A = [&](int id) { return (R)absa[(size_t)(id - 1) * NG + ig]; };
                    c.TG(NS + ig, k0) = corradj * (col * (c.fac00[k0] * A(ind0) + c.fac10[k0] * A(ind0 + 1) +
                                                          c.fac01[k0] * A(ind1) + c.fac11[k0] * A(ind1 + 1)) +
                                                   tauself + taufor);
                    c.FR(NS + ig, k0) = (R)fa[ig];
                }
            } else {
                const int ind0 = (c.jp[k0] - 13) * 5 + (c.jt[k0] - 1) + 1;
                const int ind1 = (c.jp[k0] - 12) * 5 + (c.jt1[k0] - 1) + 1;
                for (int ig = 0; ig < NG; ++ig) {
                    const R taufor = c.forfac[k0] * interp(forref, NG, indf, ig, c.forfrac[k0]);
                    auto B = [&](int id) { return (R)absb[(size_t)(id - 1) * NG + ig]; };
                    c.TG(NS + ig, k0) = col * (c.fac00[k0] * B(ind0) + c.fac10[k0] * B(ind0 + 1) +
                                               c.fac01[k0] * B(ind1) + c.fac11[k0] * B(ind1 + 1)) + taufor;
                    c.FR(NS + ig, k0) = (R)fb[ig];
                }
            }
        }
    }
    // ---- bands 3 and 4 (phys_rrtm_lw_taugb03.cu:82-340, phys_rrtm_lw_taugb04.cu:330-494): H2O/CO2 lower,
    //      band 3 CO2(upper via rate 1)/band 4 O3-CO2 upper; each specparm tested on its own.
    for (int band = 3; band <= 4; ++band) {
        const int NG = band == 3 ? 16 : 14, NS = band == 3 ? 22 : 38;
        const char* p = band == 3 ? "lw03_" : "lw04_";
        const double *absa = t((std::string(p) + "absa").c_str()), *absb = t((std::string(p) + "absb").c_str()),
                     *selfref = t((std::string(p) + "selfref").c_str()), *forref = t((std::string(p) + "forref").c_str()),
                     *fa = t((std::string(p) + "fracrefa").c_str()), *fb = t((std::string(p) + "fracrefb").c_str());
        const double* kan = band == 3 ? t("lw03_ka_mn2o") : nullptr;
        const double* kbn = band == 3 ? t("lw03_kb_mn2o") : nullptr;
        R rpa, rpb, rma = 0, rmb = 0;
        if (band == 3) {
            rpa = CHI(1, 9) / CHI(2, 9); rpb = CHI(1, 13) / CHI(2, 13);
            rma = CHI(1, 3) / CHI(2, 3); rmb = CHI(1, 13) / CHI(2, 13);
        } else {   // the band-4 wrapper computes these on the host in float32 (phys_rrtm_lw_taugb04.py:87-99)
            rpa = (R)((float)chi[10 * 7 + 0] / (float)chi[10 * 7 + 1]);
            rpb = (R)((float)chi[12 * 7 + 2] / (float)chi[12 * 7 + 1]);
        }
        for (int k0 = 0; k0 < nlay; ++k0) {
            const int jpk = c.jp[k0], jtk = c.jt[k0], jt1k = c.jt1[k0];
            const R f00 = c.fac00[k0], f01 = c.fac01[k0], f10 = c.fac10[k0], f11 = c.fac11[k0];
            if (k0 < lt) {
                R sc, sp, sc1, sp1, scm, spm, scp, spp, fs, fs1, fmn, fpl;
                int js, js1, jmn, jpl;
                spec(c.CA(0, k0), c.RF(0, 0, k0), c.CA(1, k0), (R)8, sc, sp, js, fs);
                const int ind0 = ((jpk - 1) * 5 + (jtk - 1)) * 9 + js;
                spec(c.CA(0, k0), c.RF(1, 0, k0), c.CA(1, k0), (R)8, sc1, sp1, js1, fs1);
                const int ind1 = (jpk * 5 + (jt1k - 1)) * 9 + js1;
                if (band == 3) spec(c.CA(0, k0), rma, c.CA(1, k0), (R)8, scm, spm, jmn, fmn);
                spec(c.CA(0, k0), rpa, c.CA(1, k0), (R)8, scp, spp, jpl, fpl);
                R adjcoln2o = 0;
                if (band == 3) {
                    const R pn = c.coldry[k0] * CHI(4, jpk + 1);
                    const R ratn2o = c.CA(3, k0) / pn;
                    if (ratn2o > (R)1.5f) adjcoln2o = ((R)0.5f + mpow(ratn2o - (R)0.5f, (R)0.65f)) * pn;
                    else adjcoln2o = c.CA(3, k0);
                }
                const Sel<R> s0 = sel_branch(branch_of(sp), fs, ind0);
                const Sel<R> s1 = sel_branch(branch_of(sp1), fs1, ind1);
                const int inds = c.indself[k0], indf = c.indfor[k0], indm = c.indminor[k0];
                for (int ig = 0; ig < NG; ++ig) {
                    const R tauself = c.selffac[k0] * interp(selfref, NG, inds, ig, c.selffrac[k0]);
                    const R taufor = c.forfac[k0] * interp(forref, NG, indf, ig, c.forfrac[k0]);
                    const R major = major12(absa, NG, ig, sc, s0, f00, f10, sc1, s1, f01, f11);
                    R tg;
                    if (band == 3) {
                        auto KA = [&](int j, int m) { return (R)kan[((size_t)(m - 1) * 9 + (j - 1)) * NG + ig]; };
                        const R n2om1 = KA(jmn, indm) + fmn * (KA(jmn + 1, indm) - KA(jmn, indm));
                        const R n2om2 = KA(jmn, indm + 1) + fmn * (KA(jmn + 1, indm + 1) - KA(jmn, indm + 1));
                        const R absn2o = n2om1 + c.minorfrac[k0] * (n2om2 - n2om1);
                        tg = major + tauself + taufor + adjcoln2o * absn2o;
                    } else {
                        tg = major + tauself + taufor;
                    }
                    c.TG(NS + ig, k0) = tg;
                    c.FR(NS + ig, k0) = (R)fa[(size_t)(jpl - 1) * NG + ig] +
                                        fpl * ((R)fa[(size_t)jpl * NG + ig] - (R)fa[(size_t)(jpl - 1) * NG + ig]);
                }
            } else {
                // band 3 keys H2O/CO2 with rate 1; band 4 keys O3/CO2 with rate 6 (upper atmosphere)
                const R ka1 = band == 3 ? c.CA(0, k0) : c.CA(2, k0);
                const R r0 = band == 3 ? c.RF(0, 0, k0) : c.RF(0, 5, k0);
                const R r1 = band == 3 ? c.RF(1, 0, k0) : c.RF(1, 5, k0);
                R sc, sp, sc1, sp1, scm, spm, scp, spp, fs, fs1, fmn, fpl;
                int js, js1, jmn, jpl;
                spec(ka1, r0, c.CA(1, k0), (R)4, sc, sp, js, fs);
                const int ind0 = ((jpk - 13) * 5 + (jtk - 1)) * 5 + js;
                spec(ka1, r1, c.CA(1, k0), (R)4, sc1, sp1, js1, fs1);
                const int ind1 = ((jpk - 12) * 5 + (jt1k - 1)) * 5 + js1;
                if (band == 3) spec(ka1, rmb, c.CA(1, k0), (R)4, scm, spm, jmn, fmn);
                spec(ka1, rpb, c.CA(1, k0), (R)4, scp, spp, jpl, fpl);
                R adjcoln2o = 0;
                if (band == 3) {
                    const R pn = c.coldry[k0] * CHI(4, jpk + 1);
                    const R ratn2o = c.CA(3, k0) / pn;
                    if (ratn2o > (R)1.5f) adjcoln2o = ((R)0.5f + mpow(ratn2o - (R)0.5f, (R)0.65f)) * pn;
                    else adjcoln2o = c.CA(3, k0);
                }
                const R fac000 = ((R)1 - fs) * f00, fac010 = ((R)1 - fs) * f10, fac100 = fs * f00, fac110 = fs * f10;
                const R fac001 = ((R)1 - fs1) * f01, fac011 = ((R)1 - fs1) * f11, fac101 = fs1 * f01, fac111 = fs1 * f11;
                const int indm = c.indminor[k0];
                for (int ig = 0; ig < NG; ++ig) {
                    auto B = [&](int id) { return (R)absb[(size_t)(id - 1) * NG + ig]; };
                    const R t0 = sc * (fac000 * B(ind0) + fac010 * B(ind0 + 5) + fac100 * B(ind0 + 1) + fac110 * B(ind0 + 6));
                    const R t1 = sc1 * (fac001 * B(ind1) + fac011 * B(ind1 + 5) + fac101 * B(ind1 + 1) + fac111 * B(ind1 + 6));
                    R tg;
                    if (band == 3) {
                        const R taufor = c.forfac[k0] * interp(forref, NG, c.indfor[k0], ig, c.forfrac[k0]);
                        auto KB = [&](int j, int m) { return (R)kbn[((size_t)(m - 1) * 5 + (j - 1)) * NG + ig]; };
                        const R n2om1 = KB(jmn, indm) + fmn * (KB(jmn + 1, indm) - KB(jmn, indm));
                        const R n2om2 = KB(jmn, indm + 1) + fmn * (KB(jmn + 1, indm + 1) - KB(jmn, indm + 1));
                        const R absn2o = n2om1 + c.minorfrac[k0] * (n2om2 - n2om1);
                        tg = t0 + t1 + taufor + adjcoln2o * absn2o;
                    } else {
                        tg = t0 + t1;
                        static const float adj[14] = {1, 1, 1, 1, 1, 1, 1, 0.92f, 0.88f, 1.07f, 1.1f, 0.99f, 0.88f, 0.943f};
                        if (ig >= 7) tg = tg * (R)adj[ig];
                    }
                    c.TG(NS + ig, k0) = tg;
                    c.FR(NS + ig, k0) = (R)fb[(size_t)(jpl - 1) * NG + ig] +
                                        fpl * ((R)fb[(size_t)jpl * NG + ig] - (R)fb[(size_t)(jpl - 1) * NG + ig]);
                }
            }
        }
    }
    // ---- band 5 (phys_rrtm_lw_taugb05.cu:89-435): H2O/CO2 lower (joint test), O3/CO2 upper; minor O3,
    //      CCl4.  Reference ratios from the band's float64 chi_mls, rounded once to float32
    //      (phys_rrtm_lw_taugb05.py:81-85).
    {
        const int NG = 16, NS = 52;
        const double *absa = t("lw05_absa"), *absb = t("lw05_absb"), *selfref = t("lw05_selfref"),
                     *forref = t("lw05_forref"), *fa = t("lw05_fracrefa"), *fb = t("lw05_fracrefb"),
                     *kamo3 = t("lw05_ka_mo3"), *ccl4 = t("lw05_ccl4"), *chi64 = t("lw05_chi_mls_f64");
        auto CH64 = [&](int g, int lev) { return chi64[(size_t)(lev - 1) * 7 + (g - 1)]; };
        const R rpa = (R)(float)(CH64(1, 5) / CH64(2, 5));
        const R rpb = (R)(float)(CH64(3, 43) / CH64(2, 43));
        const R rma = (R)(float)(CH64(1, 7) / CH64(2, 7));
        for (int k0 = 0; k0 < nlay; ++k0) {
            const int jpk = c.jp[k0], jtk = c.jt[k0], jt1k = c.jt1[k0];
            const R f00 = c.fac00[k0], f01 = c.fac01[k0], f10 = c.fac10[k0], f11 = c.fac11[k0];
            const R wxk = c.WX(0, k0);
            if (k0 < lt) {
                R sc, sp, sc1, sp1, scm, spm, scp, spp, fs, fs1, fmo3, fpl;
                int js, js1, jmo3, jpl;
                // band 5 takes fs as specmult - int(specmult): the same value as mod(specmult, 1) for >= 0
                spec(c.CA(0, k0), c.RF(0, 0, k0), c.CA(1, k0), (R)8, sc, sp, js, fs);
                const int ind0 = ((jpk - 1) * 5 + (jtk - 1)) * 9 + js;
                spec(c.CA(0, k0), c.RF(1, 0, k0), c.CA(1, k0), (R)8, sc1, sp1, js1, fs1);
                const int ind1 = (jpk * 5 + (jt1k - 1)) * 9 + js1;
                spec(c.CA(0, k0), rma, c.CA(1, k0), (R)8, scm, spm, jmo3, fmo3);
                spec(c.CA(0, k0), rpa, c.CA(1, k0), (R)8, scp, spp, jpl, fpl);
                const int br = branch_joint(sp, sp1);
                const Sel<R> s0 = sel_branch(br, fs, ind0), s1 = sel_branch(br, fs1, ind1);
                const int inds = c.indself[k0], indf = c.indfor[k0], indm = c.indminor[k0];
                for (int ig = 0; ig < NG; ++ig) {
                    const R tauself = c.selffac[k0] * interp(selfref, NG, inds, ig, c.selffrac[k0]);
                    const R taufor = c.forfac[k0] * interp(forref, NG, indf, ig, c.forfrac[k0]);
                    auto KM = [&](int m, int j) { return (R)kamo3[((size_t)(m - 1) * 9 + (j - 1)) * NG + ig]; };
                    const R o3m1 = KM(indm, jmo3) + fmo3 * (KM(indm, jmo3 + 1) - KM(indm, jmo3));
                    const R o3m2 = KM(indm + 1, jmo3) + fmo3 * (KM(indm + 1, jmo3 + 1) - KM(indm + 1, jmo3));
                    const R abso3 = o3m1 + c.minorfrac[k0] * (o3m2 - o3m1);
                    c.TG(NS + ig, k0) = major12(absa, NG, ig, sc, s0, f00, f10, sc1, s1, f01, f11) + tauself +
                                        taufor + abso3 * c.CA(2, k0) + wxk * (R)ccl4[ig];
                    c.FR(NS + ig, k0) = interp(fa, NG, jpl, ig, fpl);
                }
            } else {
                R sc, sp, sc1, sp1, scp, spp, fs, fs1, fpl;
                int js, js1, jpl;
                spec(c.CA(2, k0), c.RF(0, 5, k0), c.CA(1, k0), (R)4, sc, sp, js, fs);
                const int ind0 = ((jpk - 13) * 5 + (jtk - 1)) * 5 + js;
                spec(c.CA(2, k0), c.RF(1, 5, k0), c.CA(1, k0), (R)4, sc1, sp1, js1, fs1);
                const int ind1 = ((jpk - 12) * 5 + (jt1k - 1)) * 5 + js1;
                spec(c.CA(2, k0), rpb, c.CA(1, k0), (R)4, scp, spp, jpl, fpl);
                const R fac000 = ((R)1 - fs) * f00, fac010 = ((R)1 - fs) * f10, fac100 = fs * f00, fac110 = fs * f10;
                const R fac001 = ((R)1 - fs1) * f01, fac011 = ((R)1 - fs1) * f11, fac101 = fs1 * f01, fac111 = fs1 * f11;
                for (int ig = 0; ig < NG; ++ig) {
                    auto B = [&](int id) { return (R)absb[(size_t)(id - 1) * NG + ig]; };
                    c.TG(NS + ig, k0) = sc * (fac000 * B(ind0) + fac010 * B(ind0 + 5) + fac100 * B(ind0 + 1) + fac110 * B(ind0 + 6)) +
                                        sc1 * (fac001 * B(ind1) + fac011 * B(ind1 + 5) + fac101 * B(ind1 + 1) + fac111 * B(ind1 + 6)) +
                                        wxk * (R)ccl4[ig];
                    c.FR(NS + ig, k0) = interp(fb, NG, jpl, ig, fpl);
                }
            }
        }
    }
    // ---- band 6 (phys_rrtm_lw_taugb06.cu:48-169): H2O lower, minor CO2 (adjusted), CFC-11 and CFC-12
    {
        const int NG = 8, NS = 68;
        const double *absa = t("lw06_absa"), *selfref = t("lw06_selfref"), *forref = t("lw06_forref"),
                     *ka = t("lw06_ka_mco2"), *fa = t("lw06_fracrefa"), *cfc11 = t("lw06_cfc11adj"),
                     *cfc12 = t("lw06_cfc12");
        for (int k0 = 0; k0 < nlay; ++k0) {
            const R wx2 = c.WX(1, k0), wx3 = c.WX(2, k0);
            if (k0 < lt) {
                const int jpk = c.jp[k0];
                const int ind0 = (jpk - 1) * 5 + (c.jt[k0] - 1) + 1, ind1 = jpk * 5 + (c.jt1[k0] - 1) + 1;
                const R temp = c.coldry[k0] * CHI(2, jpk + 1);
                const R ratco2 = c.CA(1, k0) / temp;
                const R adj = ratco2 > (R)3 ? ((R)2 + mpow(ratco2 - (R)2, (R)0.77f)) * temp : c.CA(1, k0);
                for (int ig = 0; ig < NG; ++ig) {
                    const R tauself = c.selffac[k0] * interp(selfref, NG, c.indself[k0], ig, c.selffrac[k0]);
                    const R taufor = c.forfac[k0] * interp(forref, NG, c.indfor[k0], ig, c.forfrac[k0]);
                    const R absco2 = interp(ka, NG, c.indminor[k0], ig, c.minorfrac[k0]);
                    auto A = [&](int id) { return (R)absa[(size_t)(id - 1) * NG + ig]; };
                    c.TG(NS + ig, k0) = c.CA(0, k0) * (c.fac00[k0] * A(ind0) + c.fac10[k0] * A(ind0 + 1) +
                                                       c.fac01[k0] * A(ind1) + c.fac11[k0] * A(ind1 + 1)) +
                                        tauself + taufor + adj * absco2 + wx2 * (R)cfc11[ig] + wx3 * (R)cfc12[ig];
                    c.FR(NS + ig, k0) = (R)fa[ig];
                }
            } else {
                for (int ig = 0; ig < NG; ++ig) {
                    c.TG(NS + ig, k0) = wx2 * (R)cfc11[ig] + wx3 * (R)cfc12[ig];
                    c.FR(NS + ig, k0) = (R)fa[ig];
                }
            }
        }
    }
    // ---- band 7 (phys_rrtm_lw_taugb07.cu:88-390): H2O/O3 lower (joint test), O3 upper, minor CO2
    {
        const int NG = 12, NS = 76;
        const double *absa = t("lw07_absa"), *absb = t("lw07_absb"), *selfref = t("lw07_selfref"),
                     *forref = t("lw07_forref"), *fa = t("lw07_fracrefa"), *fb = t("lw07_fracrefb"),
                     *ka = t("lw07_ka_mco2"), *kb = t("lw07_kb_mco2");
        const R rpa = CHI(1, 3) / CHI(3, 3), rma = CHI(1, 3) / CHI(3, 3);
        for (int k0 = 0; k0 < nlay; ++k0) {
            const int jpk = c.jp[k0], jtk = c.jt[k0], jt1k = c.jt1[k0];
            const R c1 = c.CA(0, k0), c2 = c.CA(1, k0), c3 = c.CA(2, k0);
            const R f00 = c.fac00[k0], f01 = c.fac01[k0], f10 = c.fac10[k0], f11 = c.fac11[k0];
            const R temp = c.coldry[k0] * CHI(2, jpk + 1);
            const R ratco2 = c2 / temp;
            if (k0 < lt) {
                R sc, sp, sc1, sp1, scm, spm, scp, spp, fs, fs1, fm, fpl;
                int js, js1, jm, jpl;
                spec(c1, c.RF(0, 1, k0), c3, (R)8, sc, sp, js, fs);
                const int ind0 = ((jpk - 1) * 5 + (jtk - 1)) * 9 + js;
                spec(c1, c.RF(1, 1, k0), c3, (R)8, sc1, sp1, js1, fs1);
                const int ind1 = (jpk * 5 + (jt1k - 1)) * 9 + js1;
                spec(c1, rma, c3, (R)8, scm, spm, jm, fm);
                spec(c1, rpa, c3, (R)8, scp, spp, jpl, fpl);
                const R adj = ratco2 > (R)3 ? ((R)3 + mpow(ratco2 - (R)3, (R)0.79f)) * temp : c2;
                const int br = branch_joint(sp, sp1);
                const Sel<R> s0 = sel_branch(br, fs, ind0), s1 = sel_branch(br, fs1, ind1);
                const int indm = c.indminor[k0];
                for (int ig = 0; ig < NG; ++ig) {
                    const R tauself = c.selffac[k0] * interp(selfref, NG, c.indself[k0], ig, c.selffrac[k0]);
                    const R taufor = c.forfac[k0] * interp(forref, NG, c.indfor[k0], ig, c.forfrac[k0]);
                    auto KA = [&](int j, int m) { return (R)ka[((size_t)(m - 1) * 9 + (j - 1)) * NG + ig]; };
                    const R m1 = KA(jm, indm) + fm * (KA(jm + 1, indm) - KA(jm, indm));
                    const R m2 = KA(jm, indm + 1) + fm * (KA(jm + 1, indm + 1) - KA(jm, indm + 1));
                    const R absco2 = m1 + c.minorfrac[k0] * (m2 - m1);
                    c.TG(NS + ig, k0) = major12(absa, NG, ig, sc, s0, f00, f10, sc1, s1, f01, f11) + tauself +
                                        taufor + adj * absco2;
                    c.FR(NS + ig, k0) = interp(fa, NG, jpl, ig, fpl);
                }
            } else {
                const R adj = ratco2 > (R)3 ? ((R)2 + mpow(ratco2 - (R)2, (R)0.79f)) * temp : c2;
                const int ind0 = (jpk - 13) * 5 + (jtk - 1) + 1, ind1 = (jpk - 12) * 5 + (jt1k - 1) + 1;
                static const float scl[12] = {1, 1, 1, 1, 1, 0.92f, 0.88f, 1.07f, 1.1f, 0.99f, 0.855f, 1};
                for (int ig = 0; ig < NG; ++ig) {
                    const R absco2 = interp(kb, NG, c.indminor[k0], ig, c.minorfrac[k0]);
                    auto B = [&](int id) { return (R)absb[(size_t)(id - 1) * NG + ig]; };
                    R tg = c3 * (f00 * B(ind0) + f10 * B(ind0 + 1) + f01 * B(ind1) + f11 * B(ind1 + 1)) + adj * absco2;
                    if (ig >= 5 && ig <= 10) tg = tg * (R)scl[ig];
                    c.TG(NS + ig, k0) = tg;
                    c.FR(NS + ig, k0) = (R)fb[ig];
                }
            }
        }
    }
    // ---- band 8 (phys_rrtm_lw_taugb08.cu:54-258): H2O lower, O3 upper; minor CO2, O3, N2O, CFC-12, CFC-22
    {
        const int NG = 8, NS = 88;
        const double *absa = t("lw08_absa"), *absb = t("lw08_absb"), *selfref = t("lw08_selfref"),
                     *forref = t("lw08_forref"), *kaco2 = t("lw08_ka_mco2"), *kbco2 = t("lw08_kb_mco2"),
                     *kao3 = t("lw08_ka_mo3"), *kan2o = t("lw08_ka_mn2o"), *kbn2o = t("lw08_kb_mn2o"),
                     *fa = t("lw08_fracrefa"), *fb = t("lw08_fracrefb"), *cfc12 = t("lw08_cfc12"),
                     *cfc22 = t("lw08_cfc22adj");
        for (int k0 = 0; k0 < nlay; ++k0) {
            const int jpk = c.jp[k0], jtk = c.jt[k0], jt1k = c.jt1[k0];
            const R temp = c.coldry[k0] * CHI(2, jpk + 1);
            const R ratco2 = c.CA(1, k0) / temp;
            const R adj = ratco2 > (R)3 ? ((R)2 + mpow(ratco2 - (R)2, (R)0.65f)) * temp : c.CA(1, k0);
            const R f00 = c.fac00[k0], f01 = c.fac01[k0], f10 = c.fac10[k0], f11 = c.fac11[k0];
            const R w3 = c.WX(2, k0), w4 = c.WX(3, k0);
            if (k0 < lt) {
                const int r0 = (jpk - 1) * 5 + (jtk - 1), r1 = jpk * 5 + (jt1k - 1);
                const int indm = c.indminor[k0];
                for (int ig = 0; ig < NG; ++ig) {
                    const R tauself = c.selffac[k0] * interp(selfref, NG, c.indself[k0], ig, c.selffrac[k0]);
                    const R taufor = c.forfac[k0] * interp(forref, NG, c.indfor[k0], ig, c.forfrac[k0]);
                    const R absco2 = interp(kaco2, NG, indm, ig, c.minorfrac[k0]);
                    const R abso3 = interp(kao3, NG, indm, ig, c.minorfrac[k0]);
                    const R absn2o = interp(kan2o, NG, indm, ig, c.minorfrac[k0]);
                    auto A = [&](int r) { return (R)absa[(size_t)r * NG + ig]; };
                    c.TG(NS + ig, k0) = c.CA(0, k0) * (f00 * A(r0) + f10 * A(r0 + 1) + f01 * A(r1) + f11 * A(r1 + 1)) +
                                        tauself + taufor + adj * absco2 + c.CA(2, k0) * abso3 + c.CA(3, k0) * absn2o +
                                        w3 * (R)cfc12[ig] + w4 * (R)cfc22[ig];
                    c.FR(NS + ig, k0) = (R)fa[ig];
                }
            } else {
                const int r0 = (jpk - 13) * 5 + (jtk - 1), r1 = (jpk - 12) * 5 + (jt1k - 1);
                const int indm = c.indminor[k0];
                for (int ig = 0; ig < NG; ++ig) {
                    const R absco2 = interp(kbco2, NG, indm, ig, c.minorfrac[k0]);
                    const R absn2o = interp(kbn2o, NG, indm, ig, c.minorfrac[k0]);
                    auto B = [&](int r) { return (R)absb[(size_t)r * NG + ig]; };
                    c.TG(NS + ig, k0) = c.CA(2, k0) * (f00 * B(r0) + f10 * B(r0 + 1) + f01 * B(r1) + f11 * B(r1 + 1)) +
                                        adj * absco2 + c.CA(3, k0) * absn2o + w3 * (R)cfc12[ig] + w4 * (R)cfc22[ig];
                    c.FR(NS + ig, k0) = (R)fb[ig];
                }
            }
        }
    }
    // ---- band 9 (phys_rrtm_lw_taugb09.cu:66-378): H2O/CH4 lower (joint test), CH4 upper, minor N2O
    {
        const int NG = 12, NS = 96;
        const double *absa = t("lw09_absa"), *absb = t("lw09_absb"), *selfref = t("lw09_selfref"),
                     *forref = t("lw09_forref"), *ka = t("lw09_ka_mn2o"), *kb = t("lw09_kb_mn2o"),
                     *fa = t("lw09_fracrefa"), *fb = t("lw09_fracrefb");
        const R rpa = CHI(1, 9) / CHI(6, 9), rma = CHI(1, 3) / CHI(6, 3);
        for (int k0 = 0; k0 < nlay; ++k0) {
            const int jpk = c.jp[k0], jtk = c.jt[k0], jt1k = c.jt1[k0];
            const R c1 = c.CA(0, k0), c4 = c.CA(3, k0), c5 = c.CA(4, k0);
            const R f00 = c.fac00[k0], f01 = c.fac01[k0], f10 = c.fac10[k0], f11 = c.fac11[k0];
            const R temp = c.coldry[k0] * CHI(4, jpk + 1);
            const R ratn2o = c4 / temp;
            const R adj = ratn2o > (R)1.5f ? ((R)0.5f + mpow(ratn2o - (R)0.5f, (R)0.65f)) * temp : c4;
            if (k0 < lt) {
                R sc, sp, sc1, sp1, scm, spm, scp, spp, fs, fs1, fm, fpl;
                int js, js1, jm, jpl;
                spec(c1, c.RF(0, 3, k0), c5, (R)8, sc, sp, js, fs);
                const int ind0 = ((jpk - 1) * 5 + (jtk - 1)) * 9 + js;
                spec(c1, c.RF(1, 3, k0), c5, (R)8, sc1, sp1, js1, fs1);
                const int ind1 = (jpk * 5 + (jt1k - 1)) * 9 + js1;
                spec(c1, rma, c5, (R)8, scm, spm, jm, fm);
                spec(c1, rpa, c5, (R)8, scp, spp, jpl, fpl);
                const int br = branch_joint(sp, sp1);
                const Sel<R> s0 = sel_branch(br, fs, ind0), s1 = sel_branch(br, fs1, ind1);
                const int indm = c.indminor[k0];
                for (int ig = 0; ig < NG; ++ig) {
                    const R tauself = c.selffac[k0] * interp(selfref, NG, c.indself[k0], ig, c.selffrac[k0]);
                    const R taufor = c.forfac[k0] * interp(forref, NG, c.indfor[k0], ig, c.forfrac[k0]);
                    auto KA = [&](int j, int m) { return (R)ka[((size_t)(m - 1) * 9 + (j - 1)) * NG + ig]; };
                    const R m1 = KA(jm, indm) + fm * (KA(jm + 1, indm) - KA(jm, indm));
                    const R m2 = KA(jm, indm + 1) + fm * (KA(jm + 1, indm + 1) - KA(jm, indm + 1));
                    const R absn2o = m1 + c.minorfrac[k0] * (m2 - m1);
                    c.TG(NS + ig, k0) = major12(absa, NG, ig, sc, s0, f00, f10, sc1, s1, f01, f11) + tauself +
                                        taufor + adj * absn2o;
                    c.FR(NS + ig, k0) = interp(fa, NG, jpl, ig, fpl);
                }
            } else {
                const int ind0 = (jpk - 13) * 5 + (jtk - 1) + 1, ind1 = (jpk - 12) * 5 + (jt1k - 1) + 1;
                for (int ig = 0; ig < NG; ++ig) {
                    const R absn2o = interp(kb, NG, c.indminor[k0], ig, c.minorfrac[k0]);
                    auto B = [&](int id) { return (R)absb[(size_t)(id - 1) * NG + ig]; };
                    c.TG(NS + ig, k0) = c5 * (f00 * B(ind0) + f10 * B(ind0 + 1) + f01 * B(ind1) + f11 * B(ind1 + 1)) +
                                        adj * absn2o;
                    c.FR(NS + ig, k0) = (R)fb[ig];
                }
            }
        }
    }
    // ---- bands 10, 11, 14 (taugb10.cu:71-199, taugb11.cu:51-166, taugb14.cu:53-161): single key species
    //      (H2O, H2O, CO2), band 11 with minor O2 scaled by scaleminor.
    for (int band : {10, 11, 14}) {
        const int NG = band == 10 ? 6 : (band == 11 ? 8 : 2);
        const int NS = band == 10 ? 108 : (band == 11 ? 114 : 134);
        char p[8];
        std::snprintf(p, sizeof p, "lw%02d_", band);
        auto tb = [&](const char* n) { return t((std::string(p) + n).c_str()); };
        const double *absa = tb("absa"), *absb = tb("absb"), *selfref = tb("selfref"), *forref = tb("forref"),
                     *fa = tb("fracrefa"), *fb = tb("fracrefb");
        const double* ka = band == 11 ? t("lw11_ka_mo2") : nullptr;
        const double* kb = band == 11 ? t("lw11_kb_mo2") : nullptr;
        for (int k0 = 0; k0 < nlay; ++k0) {
            const int jpk = c.jp[k0], jtk = c.jt[k0], jt1k = c.jt1[k0];
            const R col = band == 14 ? c.CA(1, k0) : c.CA(0, k0);
            const R f00 = c.fac00[k0], f01 = c.fac01[k0], f10 = c.fac10[k0], f11 = c.fac11[k0];
            const R scaleo2 = c.CA(5, k0) * c.scaleminor[k0];
            if (k0 < lt) {
                const int ind0 = (jpk - 1) * 5 + (jtk - 1) + 1, ind1 = jpk * 5 + (jt1k - 1) + 1;
                for (int ig = 0; ig < NG; ++ig) {
                    const R tauself = c.selffac[k0] * interp(selfref, NG, c.indself[k0], ig, c.selffrac[k0]);
                    const R taufor = c.forfac[k0] * interp(forref, NG, c.indfor[k0], ig, c.forfrac[k0]);
                    auto A = [&](int id) { return (R)absa[(size_t)(id - 1) * NG + ig]; };
                    R tg = col * (f00 * A(ind0) + f10 * A(ind0 + 1) + f01 * A(ind1) + f11 * A(ind1 + 1)) + tauself + taufor;
                    if (band == 11) tg = tg + scaleo2 * interp(ka, NG, c.indminor[k0], ig, c.minorfrac[k0]);
                    c.TG(NS + ig, k0) = tg;
                    c.FR(NS + ig, k0) = (R)fa[ig];
                }
            } else {
                const int ind0 = (jpk - 13) * 5 + (jtk - 1) + 1, ind1 = (jpk - 12) * 5 + (jt1k - 1) + 1;
                for (int ig = 0; ig < NG; ++ig) {
                    auto B = [&](int id) { return (R)absb[(size_t)(id - 1) * NG + ig]; };
                    R tg = col * (f00 * B(ind0) + f10 * B(ind0 + 1) + f01 * B(ind1) + f11 * B(ind1 + 1));
                    if (band != 14) tg = tg + c.forfac[k0] * interp(forref, NG, c.indfor[k0], ig, c.forfrac[k0]);
                    if (band == 11) tg = tg + scaleo2 * interp(kb, NG, c.indminor[k0], ig, c.minorfrac[k0]);
                    c.TG(NS + ig, k0) = tg;
                    c.FR(NS + ig, k0) = (R)fb[ig];
                }
            }
        }
    }
    // ---- bands 12 and 16 (taugb12.cu:72-264, taugb16.cu:84-289): H2O/CO2 resp. H2O/CH4 lower (joint
    //      test); band 12 upper is zero, band 16 upper uses absb with nspb(16) = 0.
    for (int band : {12, 16}) {
        const int NG = band == 12 ? 8 : 2, NS = band == 12 ? 122 : 138;
        const char* p = band == 12 ? "lw12_" : "lw16_";
        auto tb = [&](const char* n) { return t((std::string(p) + n).c_str()); };
        const double *absa = tb("absa"), *selfref = tb("selfref"), *forref = tb("forref"), *fa = tb("fracrefa");
        const int rate = band == 12 ? 0 : 3;
        const int gas2 = band == 12 ? 1 : 4;
        const R rpa = band == 12 ? CHI(1, 10) / CHI(2, 10) : CHI(1, 6) / CHI(6, 6);
        for (int k0 = 0; k0 < nlay; ++k0) {
            const int jpk = c.jp[k0], jtk = c.jt[k0], jt1k = c.jt1[k0];
            const R f00 = c.fac00[k0], f01 = c.fac01[k0], f10 = c.fac10[k0], f11 = c.fac11[k0];
            if (k0 < lt) {
                const R c1 = c.CA(0, k0), c2 = c.CA(gas2, k0);
                R sc, sp, sc1, sp1, fs, fs1, fpl;
                int js, js1, jpl;
                spec(c1, c.RF(0, rate, k0), c2, (R)8, sc, sp, js, fs);
                const int ind0 = ((jpk - 1) * 5 + (jtk - 1)) * 9 + js;
                spec(c1, c.RF(1, rate, k0), c2, (R)8, sc1, sp1, js1, fs1);
                const int ind1 = (jpk * 5 + (jt1k - 1)) * 9 + js1;
                {
                    // Planck key: band 12 clamps specparm_planck before scaling (taugb12.cu:127-130);
                    // band 16 takes min(specparm, oneminus) as the others (same value)
                    const R oneminus = (R)1.0f - (R)1.0e-6f;
                    const R scp = c1 + rpa * c2;
                    R spp = c1 / scp;
                    if (spp >= oneminus) spp = oneminus;
                    const R smp = (R)8 * spp;
                    jpl = 1 + (int)smp;
                    fpl = fmod1(smp);
                }
                const int br = branch_joint(sp, sp1);
                const Sel<R> s0 = sel_branch(br, fs, ind0), s1 = sel_branch(br, fs1, ind1);
                for (int ig = 0; ig < NG; ++ig) {
                    const R tauself = c.selffac[k0] * interp(selfref, NG, c.indself[k0], ig, c.selffrac[k0]);
                    const R taufor = c.forfac[k0] * interp(forref, NG, c.indfor[k0], ig, c.forfrac[k0]);
                    c.TG(NS + ig, k0) = major12(absa, NG, ig, sc, s0, f00, f10, sc1, s1, f01, f11) + tauself + taufor;
                    c.FR(NS + ig, k0) = interp(fa, NG, jpl, ig, fpl);
                }
            } else if (band == 12) {
                for (int ig = 0; ig < NG; ++ig) { c.TG(NS + ig, k0) = 0; c.FR(NS + ig, k0) = 0; }
            } else {
                const double *absb = t("lw16_absb"), *fb = t("lw16_fracrefb");
                const int ind0 = ((jpk - 13) * 5 + (jtk - 1)) * 0 + 1, ind1 = ((jpk - 12) * 5 + (jt1k - 1)) * 0 + 1;
                for (int ig = 0; ig < NG; ++ig) {
                    auto B = [&](int id) { return (R)absb[(size_t)(id - 1) * NG + ig]; };
                    c.TG(NS + ig, k0) = c.CA(4, k0) * (f00 * B(ind0) + f10 * B(ind0 + 1) + f01 * B(ind1) + f11 * B(ind1 + 1));
                    c.FR(NS + ig, k0) = (R)fb[ig];
                }
            }
        }
    }
    // ---- band 13 (taugb13.cu:51-318): H2O/N2O lower (joint test), minor CO2 and CO; upper minor O3
    {
        const int NG = 4, NS = 130;
        const double *absa = t("lw13_absa"), *selfref = t("lw13_selfref"), *forref = t("lw13_forref"),
                     *fa = t("lw13_fracrefa"), *fb = t("lw13_fracrefb"), *kaco2 = t("lw13_ka_mco2"),
                     *kaco = t("lw13_ka_mco"), *kbo3 = t("lw13_kb_mo3");
        const R rpa = CHI(1, 5) / CHI(4, 5), rma = CHI(1, 1) / CHI(4, 1), rma3 = CHI(1, 3) / CHI(4, 3);
        for (int k0 = 0; k0 < nlay; ++k0) {
            const int jpk = c.jp[k0], jtk = c.jt[k0], jt1k = c.jt1[k0];
            const int indm = c.indminor[k0];
            if (k0 < lt) {
                const R c1 = c.CA(0, k0), c2 = c.CA(1, k0), c4 = c.CA(3, k0), c7 = c.CA(6, k0);
                R sc, sp, sc1, sp1, scm, spm, scmc, spmc, scp, spp, fs, fs1, fm, fmc, fpl;
                int js, js1, jm, jmc, jpl;
                spec(c1, c.RF(0, 2, k0), c4, (R)8, sc, sp, js, fs);
                const int ind0 = ((jpk - 1) * 5 + (jtk - 1)) * 9 + js;
                spec(c1, c.RF(1, 2, k0), c4, (R)8, sc1, sp1, js1, fs1);
                const int ind1 = (jpk * 5 + (jt1k - 1)) * 9 + js1;
                spec(c1, rma, c4, (R)8, scm, spm, jm, fm);
                spec(c1, rma3, c4, (R)8, scmc, spmc, jmc, fmc);
                spec(c1, rpa, c4, (R)8, scp, spp, jpl, fpl);
                const R temp = c.coldry[k0] * (R)3.55e-4f;
                const R ratco2 = c2 / temp;
                const R adj = ratco2 > (R)3 ? ((R)2 + mpow(ratco2 - (R)2, (R)0.68f)) * temp : c2;
                const int br = branch_joint(sp, sp1);
                const Sel<R> s0 = sel_branch(br, fs, ind0), s1 = sel_branch(br, fs1, ind1);
                const R f00 = c.fac00[k0], f01 = c.fac01[k0], f10 = c.fac10[k0], f11 = c.fac11[k0];
                for (int ig = 0; ig < NG; ++ig) {
                    const R tauself = c.selffac[k0] * interp(selfref, NG, c.indself[k0], ig, c.selffrac[k0]);
                    const R taufor = c.forfac[k0] * interp(forref, NG, c.indfor[k0], ig, c.forfrac[k0]);
                    auto K2 = [&](const double* tt, int j, int m) { return (R)tt[((size_t)(m - 1) * 9 + (j - 1)) * NG + ig]; };
                    const R co2m1 = K2(kaco2, jm, indm) + fm * (K2(kaco2, jm + 1, indm) - K2(kaco2, jm, indm));
                    const R co2m2 = K2(kaco2, jm, indm + 1) + fm * (K2(kaco2, jm + 1, indm + 1) - K2(kaco2, jm, indm + 1));
                    const R absco2 = co2m1 + c.minorfrac[k0] * (co2m2 - co2m1);
                    const R com1 = K2(kaco, jmc, indm) + fmc * (K2(kaco, jmc + 1, indm) - K2(kaco, jmc, indm));
                    const R com2 = K2(kaco, jmc, indm + 1) + fmc * (K2(kaco, jmc + 1, indm + 1) - K2(kaco, jmc, indm + 1));
                    const R absco = com1 + c.minorfrac[k0] * (com2 - com1);
                    c.TG(NS + ig, k0) = major12(absa, NG, ig, sc, s0, f00, f10, sc1, s1, f01, f11) + tauself +
                                        taufor + adj * absco2 + c7 * absco;
                    c.FR(NS + ig, k0) = interp(fa, NG, jpl, ig, fpl);
                }
            } else {
                for (int ig = 0; ig < NG; ++ig) {
                    const R abso3 = interp(kbo3, NG, indm, ig, c.minorfrac[k0]);
                    c.TG(NS + ig, k0) = c.CA(2, k0) * abso3;
                    c.FR(NS + ig, k0) = (R)fb[ig];
                }
            }
        }
    }
    // ---- band 15 (taugb15.cu:57-277): N2O/CO2 lower (joint test), minor N2; upper zero.  The wrapper
    //      passes refrat_planck_a = refrat_m_a = chi_mls(4,1)/chi_mls(2,1) as float32.
    {
        const int NG = 2, NS = 136;
        const double *absa = t("lw15_absa"), *selfref = t("lw15_selfref"), *forref = t("lw15_forref"),
                     *ka = t("lw15_ka_mn2"), *fa = t("lw15_fracrefa");
        const R rpa = (R)((float)chi[0 * 7 + 3] / (float)chi[0 * 7 + 1]);
        const R rma = rpa;
        for (int k0 = 0; k0 < nlay; ++k0) {
            if (k0 < lt) {
                const int jpk = c.jp[k0], jtk = c.jt[k0], jt1k = c.jt1[k0];
                const R cn = c.CA(3, k0), cc = c.CA(1, k0);
                R sc, sp, sc1, sp1, scm, spm, scp, spp, fs, fs1, fm, fpl;
                int js, js1, jm, jpl;
                spec(cn, c.RF(0, 4, k0), cc, (R)8, sc, sp, js, fs);
                const int ind0 = ((jpk - 1) * 5 + (jtk - 1)) * 9 + js;
                spec(cn, c.RF(1, 4, k0), cc, (R)8, sc1, sp1, js1, fs1);
                const int ind1 = (jpk * 5 + (jt1k - 1)) * 9 + js1;
                spec(cn, rma, cc, (R)8, scm, spm, jm, fm);
                spec(cn, rpa, cc, (R)8, scp, spp, jpl, fpl);
                const R scalen2 = c.colbrd[k0] * c.scaleminor[k0];
                const int br = branch_joint(sp, sp1);
                Sel<R> s0 = sel_branch(br, fs, ind0), s1 = sel_branch(br, fs1, ind1);
                // band 15 writes fk1 as (1 - p) - 2 p^4: the same rounding as 1 - p - 2 p^4
                const R f00 = c.fac00[k0], f01 = c.fac01[k0], f10 = c.fac10[k0], f11 = c.fac11[k0];
                const int indm = c.indminor[k0];
                for (int ig = 0; ig < NG; ++ig) {
                    const R tauself = c.selffac[k0] * interp(selfref, NG, c.indself[k0], ig, c.selffrac[k0]);
                    const R taufor = c.forfac[k0] * interp(forref, NG, c.indfor[k0], ig, c.forfrac[k0]);
                    auto KA = [&](int j, int m) { return (R)ka[((size_t)(m - 1) * 9 + (j - 1)) * NG + ig]; };
                    const R n2m1 = KA(jm, indm) + fm * (KA(jm + 1, indm) - KA(jm, indm));
                    const R n2m2 = KA(jm, indm + 1) + fm * (KA(jm + 1, indm + 1) - KA(jm, indm + 1));
                    const R taun2 = scalen2 * (n2m1 + c.minorfrac[k0] * (n2m2 - n2m1));
                    auto A = [&](int id) { return (R)absa[(size_t)(id - 1) * NG + ig]; };
                    const R fac000 = s0.fk0 * f00, fac100 = s0.fk1 * f00, fac200 = s0.fk2 * f00;
                    const R fac010 = s0.fk0 * f10, fac110 = s0.fk1 * f10, fac210 = s0.fk2 * f10;
                    const R fac001 = s1.fk0 * f01, fac101 = s1.fk1 * f01, fac201 = s1.fk2 * f01;
                    const R fac011 = s1.fk0 * f11, fac111 = s1.fk1 * f11, fac211 = s1.fk2 * f11;
                    const R sumA = fac000 * A(s0.id[0]) + fac010 * A(s0.id[1]) + fac100 * A(s0.id[2]) +
                                   fac110 * A(s0.id[3]) + fac200 * A(s0.id[4]) + fac210 * A(s0.id[5]);
                    const R sumB = fac001 * A(s1.id[0]) + fac011 * A(s1.id[1]) + fac101 * A(s1.id[2]) +
                                   fac111 * A(s1.id[3]) + fac201 * A(s1.id[4]) + fac211 * A(s1.id[5]);
                    c.TG(NS + ig, k0) = sc * sumA + sc1 * sumB + tauself + taufor + taun2;
                    c.FR(NS + ig, k0) = interp(fa, NG, jpl, ig, fpl);
                }
            } else {
                for (int ig = 0; ig < NG; ++ig) { c.TG(NS + ig, k0) = 0; c.FR(NS + ig, k0) = 0; }
            }
        }
    }
    // ---- tautot = taug + tauaer(ngb(g)) (lw_core.py:83-90)
    for (int b = 0; b < 16; ++b)
        for (int g = LW_NS[b]; g < LW_NS[b] + LW_NG[b]; ++g)
            for (int k0 = 0; k0 < nlay; ++k0) c.TG(g, k0) = c.TG(g, k0) + c.tauaer[(size_t)b * nlay + k0];
}

// ---------------------------------------------------------------------------------------------------
// rlwinit lookup tables (phys_rrtm_lw_rtrnmr.py:108-131): float32 recipe for R = float, the same
// statements in double for R = double.
template <class R>
struct LwTables {
    std::vector<R> tau, ex, tfn;
    LwTables()
    {
        const int ntbl = 10000;
        tau.assign(ntbl + 1, 0); ex.assign(ntbl + 1, 0); tfn.assign(ntbl + 1, 0);
        const R bpade = (R)1.0f / (R)0.278f;
        const R expeps = (R)1.0e-20f;
        const R explimit = (R)std::trunc(-std::log((double)std::numeric_limits<R>::min()));
        ex[0] = 1; tau[0] = 0; tfn[0] = 0;
        for (int i = 1; i < ntbl; ++i) {
            const R tf = (R)i / (R)(ntbl - i);
            const R ta = bpade * tf;
            const R e = ta >= explimit ? expeps : (R)std::exp(-(double)ta);
            tau[i] = ta;
            ex[i] = e;
            tfn[i] = ta < (R)0.06f ? ta / (R)6 : (R)1 - (R)2 * (((R)1 / ta) - (e / ((R)1 - e)));
        }
        ex[ntbl] = expeps; tau[ntbl] = (R)1.0e10f; tfn[ntbl] = 1;
    }
};

// ---------------------------------------------------------------------------------------------------
// rtrnmr (phys_rrtm_lw_rtrnmr_body.cuh:9-365), surface-first slot map; lhlw0 = lhlwb = 0.
template <class R>
void lw_rtrnmr(LwColumn<R>& c, const LwTables<R>& tb, R heatfac, R fluxfac)
{
    const int nlay = c.nlay, nlp1 = nlay + 1;
    const R eps = (R)1.0e-6f, bpade = (R)1.0f / (R)0.278f, wtdiff = (R)0.5f, tblint = (R)10000,
            rec_6 = (R)0.166667f, c06 = (R)0.06f;
    std::vector<R> cf(nlp1 + 1);
    for (int m = 0; m <= nlp1; ++m) cf[m] = c.cldfrc[m];
    std::vector<R> faccld1u(nlp1 + 1, 0), faccld2u(nlp1 + 1, 0), facclr1u(nlp1 + 1, 0), facclr2u(nlp1 + 1, 0),
        faccmb1u(nlp1 + 1, 0), faccmb2u(nlp1 + 1, 0);
    std::vector<int> lstu(nlp1 + 1, 0), lstd(nlp1 + 1, 0);
    lstu[1] = cf[1] > eps ? 1 : 0;
    R rat1 = 0, rat2 = 0;
    for (int k = 1; k <= nlay - 1; ++k) {
        lstu[k + 1] = (cf[k + 1] > eps && cf[k] <= eps) ? 1 : 0;
        if (cf[k] > eps) {
            if (cf[k + 1] >= cf[k]) {
                if (lstu[k]) {
                    if (cf[k] < (R)1) facclr2u[k + 1] = (cf[k + 1] - cf[k]) / ((R)1 - cf[k]);
                    facclr2u[k] = 0; faccld2u[k] = 0;
                } else {
                    const R fmax = fmaxR(cf[k], cf[k - 1]);
                    if (cf[k + 1] > fmax) {
                        facclr1u[k + 1] = rat2;
                        facclr2u[k + 1] = (cf[k + 1] - fmax) / ((R)1 - fmax);
                    } else if (cf[k + 1] < fmax) {
                        facclr1u[k + 1] = (cf[k + 1] - cf[k]) / (cf[k - 1] - cf[k]);
                    } else {
                        facclr1u[k + 1] = rat2;
                    }
                }
                if (facclr1u[k + 1] > 0 || facclr2u[k + 1] > 0) { rat1 = 1; rat2 = 0; }
                else { rat1 = 0; rat2 = 0; }
            } else {
                if (lstu[k]) {
                    faccld2u[k + 1] = (cf[k] - cf[k + 1]) / cf[k];
                    facclr2u[k] = 0; faccld2u[k] = 0;
                } else {
                    const R fmin = fminR(cf[k], cf[k - 1]);
                    if (cf[k + 1] <= fmin) {
                        faccld1u[k + 1] = rat1;
                        faccld2u[k + 1] = (fmin - cf[k + 1]) / fmin;
                    } else {
                        faccld1u[k + 1] = (cf[k] - cf[k + 1]) / (cf[k] - fmin);
                    }
                }
                if (faccld1u[k + 1] > 0 || faccld2u[k + 1] > 0) { rat1 = 0; rat2 = 1; }
                else { rat1 = 0; rat2 = 0; }
            }
            faccmb1u[k + 1] = facclr1u[k + 1] * faccld2u[k] * cf[k - 1];
            faccmb2u[k + 1] = faccld1u[k + 1] * facclr2u[k] * ((R)1 - cf[k - 1]);
        }
    }
    std::vector<R> faccld1d(nlp1 + 1, 0), faccld2d(nlp1 + 1, 0), facclr1d(nlp1 + 1, 0), facclr2d(nlp1 + 1, 0),
        faccmb1d(nlp1 + 1, 0), faccmb2d(nlp1 + 1, 0);
    lstd[nlay] = cf[nlay] > eps ? 1 : 0;
    rat1 = 0; rat2 = 0;
    for (int k = nlay; k >= 2; --k) {
        lstd[k - 1] = (cf[k - 1] > eps && cf[k] <= eps) ? 1 : 0;
        if (cf[k] > eps) {
            if (cf[k - 1] >= cf[k]) {
                if (lstd[k]) {
                    if (cf[k] < (R)1) facclr2d[k - 1] = (cf[k - 1] - cf[k]) / ((R)1 - cf[k]);
                    facclr2d[k] = 0; faccld2d[k] = 0;
                } else {
                    const R fmax = fmaxR(cf[k], cf[k + 1]);
                    if (cf[k - 1] > fmax) {
                        facclr1d[k - 1] = rat2;
                        facclr2d[k - 1] = (cf[k - 1] - fmax) / ((R)1 - fmax);
                    } else if (cf[k - 1] < fmax) {
                        facclr1d[k - 1] = (cf[k - 1] - cf[k]) / (cf[k + 1] - cf[k]);
                    } else {
                        facclr1d[k - 1] = rat2;
                    }
                }
                if (facclr1d[k - 1] > 0 || facclr2d[k - 1] > 0) { rat1 = 1; rat2 = 0; }
                else { rat1 = 0; rat2 = 0; }
            } else {
                if (lstd[k]) {
                    faccld2d[k - 1] = (cf[k] - cf[k - 1]) / cf[k];
                    facclr2d[k] = 0; faccld2d[k] = 0;
                } else {
                    const R fmin = fminR(cf[k], cf[k + 1]);
                    if (cf[k - 1] <= fmin) {
                        faccld1d[k - 1] = rat1;
                        faccld2d[k - 1] = (fmin - cf[k - 1]) / fmin;
                    } else {
                        faccld1d[k - 1] = (cf[k] - cf[k - 1]) / (cf[k] - fmin);
                    }
                }
                if (faccld1d[k - 1] > 0 || faccld2d[k - 1] > 0) { rat1 = 0; rat2 = 1; }
                else { rat1 = 0; rat2 = 0; }
            }
            faccmb1d[k - 1] = facclr1d[k - 1] * faccld2d[k] * cf[k + 1];
            faccmb2d[k - 1] = faccld1d[k - 1] * facclr2d[k] * ((R)1 - cf[k + 1]);
        }
    }
    std::vector<R> tuf(nlp1, 0), tdf(nlp1, 0), tuc(nlp1, 0), tdc(nlp1, 0), rfdelp(nlp1, 0);
    for (int k = 1; k <= nlay; ++k) rfdelp[k] = heatfac / c.delp[k - 1];
    const R flxfac = wtdiff * fluxfac;
    std::vector<R> toturad(nlp1), totdrad(nlp1), clrurad(nlp1), clrdrad(nlp1), totsrcu(nlp1 + 1), trntot(nlp1 + 1),
        gassrcu(nlp1 + 1), trngas(nlp1 + 1);
    R radtotd = 0, radclrd = 0, totradd = 0, clrradd = 0, rad = 0, radtotu = 0, radclru = 0, totradu = 0, clrradu = 0;
    auto PKL = [&](int ib, int s) { return c.pklay[(size_t)s * 16 + ib]; };
    auto PKV = [&](int ib, int s) { return c.pklev[(size_t)s * 16 + ib]; };
    for (int ib = 0; ib < 16; ++ib) {
        for (int k = 0; k <= nlay; ++k) { toturad[k] = 0; totdrad[k] = 0; clrurad[k] = 0; clrdrad[k] = 0; }
        const R semi = c.semiss[ib], sdif = c.secdiff[ib];
        for (int ig = LW_NS[ib]; ig < LW_NS[ib] + LW_NG[ib]; ++ig) {
            radtotd = 0; radclrd = 0;
            for (int k = nlay; k >= 1; --k) {
                R odepth = fmaxR((R)0, sdif * c.TG(ig, k - 1));
                R atrgas, trng, gasfac;
                if (odepth <= c06) {
                    atrgas = odepth - (R)0.5f * odepth * odepth;
                    trng = (R)1 - atrgas;
                    gasfac = rec_6 * odepth;
                } else {
                    const R tblind = odepth / (bpade + odepth);
                    const int itgas = (int)(tblint * tblind + (R)0.5f);
                    trng = tb.ex[itgas]; atrgas = (R)1 - trng; gasfac = tb.tfn[itgas]; odepth = tb.tau[itgas];
                }
                const R plfrac = c.FR(ig, k - 1);
                const R blay = PKL(ib, k);
                const R dplnku = PKV(ib, k) - blay;
                const R dplnkd = PKV(ib, k - 1) - blay;
                const R bbdgas = plfrac * (blay + dplnkd * gasfac);
                const R bbugas = plfrac * (blay + dplnku * gasfac);
                const R gassrcd = bbdgas * atrgas;
                gassrcu[k] = bbugas * atrgas;
                trngas[k] = trng;
                const R clfr = cf[k];
                if (lstd[k]) { totradd = clfr * radtotd; clrradd = radtotd - totradd; rad = 0; }
                if (clfr >= eps) {
                    const R odcld = sdif * c.taucld[(size_t)ib * nlay + (k - 1)];
                    const R odtot = odepth + odcld;
                    R totfac, atrtot, trnt;
                    if (odtot < c06) {
                        totfac = rec_6 * odtot; atrtot = odtot - (R)0.5f * odtot * odtot; trnt = (R)1 - atrtot;
                    } else {
                        const R tblind = odtot / (bpade + odtot);
                        const int ittot = (int)(tblint * tblind + (R)0.5f);
                        totfac = tb.tfn[ittot]; trnt = tb.ex[ittot]; atrtot = (R)1 - trnt;
                    }
                    const R bbdtot = plfrac * (blay + dplnkd * totfac);
                    const R bbutot = plfrac * (blay + dplnku * totfac);
                    const R totsrcd = bbdtot * atrtot;
                    totsrcu[k] = bbutot * atrtot;
                    trntot[k] = trnt;
                    totradd = totradd * trnt + clfr * totsrcd;
                    clrradd = clrradd * trng + ((R)1 - clfr) * gassrcd;
                    radtotd = totradd + clrradd;
                    totdrad[k - 1] = totdrad[k - 1] + radtotd;
                    radclrd = radclrd * trng + gassrcd;
                    clrdrad[k - 1] = clrdrad[k - 1] + radclrd;
                    const R radmod = rad * (facclr1d[k - 1] * trng + faccld1d[k - 1] * trnt) -
                                     faccmb1d[k - 1] * gassrcd + faccmb2d[k - 1] * totsrcd;
                    rad = -radmod + facclr2d[k - 1] * (clrradd + radmod) - faccld2d[k - 1] * (totradd - radmod);
                    totradd = totradd + rad;
                    clrradd = clrradd - rad;
                } else {
                    radtotd = radtotd * trng + gassrcd;
                    totdrad[k - 1] = totdrad[k - 1] + radtotd;
                    radclrd = radclrd * trng + gassrcd;
                    clrdrad[k - 1] = clrdrad[k - 1] + radclrd;
                }
            }
            const R reflct = (R)1 - semi;
            const R rad0 = semi * c.FR(ig, 0) * PKL(ib, 0);
            radtotu = rad0 + reflct * radtotd;
            toturad[0] = toturad[0] + radtotu;
            radclru = rad0 + reflct * radclrd;
            clrurad[0] = clrurad[0] + radclru;
            for (int k = 1; k <= nlay; ++k) {
                const R clfr = cf[k], trng = trngas[k], gasu = gassrcu[k];
                if (lstu[k]) { totradu = clfr * radtotu; clrradu = radtotu - totradu; rad = 0; }
                if (clfr >= eps) {
                    const R trnt = trntot[k], totu = totsrcu[k];
                    totradu = totradu * trnt + clfr * totu;
                    clrradu = clrradu * trng + ((R)1 - clfr) * gasu;
                    radtotu = totradu + clrradu;
                    toturad[k] = toturad[k] + radtotu;
                    radclru = radclru * trng + gasu;
                    clrurad[k] = clrurad[k] + radclru;
                    const R radmod = rad * (facclr1u[k + 1] * trng + faccld1u[k + 1] * trnt) -
                                     faccmb1u[k + 1] * gasu + faccmb2u[k + 1] * totu;
                    rad = -radmod + facclr2u[k + 1] * (clrradu + radmod) - faccld2u[k + 1] * (totradu - radmod);
                    totradu = totradu + rad;
                    clrradu = clrradu - rad;
                } else {
                    radtotu = radtotu * trng + gasu;
                    toturad[k] = toturad[k] + radtotu;
                    radclru = radclru * trng + gasu;
                    clrurad[k] = clrurad[k] + radclru;
                }
            }
        }
        for (int k = 0; k <= nlay; ++k) {
            tuf[k] = tuf[k] + toturad[k]; tdf[k] = tdf[k] + totdrad[k];
            tuc[k] = tuc[k] + clrurad[k]; tdc[k] = tdc[k] + clrdrad[k];
            c.fnetb[(size_t)ib * nlp1 + k] = (toturad[k] - totdrad[k]) * flxfac;   // the lhlwb block's fnet
        }
    }
    for (int k = 0; k <= nlay; ++k) {
        tuf[k] = tuf[k] * flxfac; tdf[k] = tdf[k] * flxfac; tuc[k] = tuc[k] * flxfac; tdc[k] = tdc[k] * flxfac;
        c.totuflux[k] = tuf[k]; c.totdflux[k] = tdf[k]; c.totuclfl[k] = tuc[k]; c.totdclfl[k] = tdc[k];
    }
    std::vector<R> fnet(nlp1);
    fnet[0] = tuf[0] - tdf[0];
    for (int k = 1; k <= nlay; ++k) {
        fnet[k] = tuf[k] - tdf[k];
        c.htr[k - 1] = (fnet[k - 1] - fnet[k]) * rfdelp[k];
    }
}

// ---------------------------------------------------------------------------------------------------
// rtrn, random cloud overlap (phys_rrtm_lw_rtrn.cu:94-330; Fortran radlw_main_nmmb.f:2127-2484), the LW
// transfer of the NAM route when iovrlw = 0; lhlw0 = lhlwb = 0.  Surface-first indices as above (layer k,
// interface m); the kernel's top-first slot map is a storage order only.  A cloudy layer (clfr >= 1e-6)
// blends cloud and gas sources by clfr and scales the gas transmittance by the effective clear fraction
// efclrfr = 1 - (1 - exp(-odcld)) clfr; the clear-sky radiances ignore the cloud.
template <class R>
void lw_rtrn(LwColumn<R>& c, const LwTables<R>& tb, R heatfac, R fluxfac)
{
    const int nlay = c.nlay, nlp1 = nlay + 1;
    const R eps = (R)1.0e-6f, bpade = (R)1.0f / (R)0.278f, wtdiff = (R)0.5f, tblint = (R)10000,
            rec_6 = (R)0.166667f, c06 = (R)0.06f;
    const R flxfac = wtdiff * fluxfac;
    auto PKL = [&](int ib, int s) { return c.pklay[(size_t)s * 16 + ib]; };
    auto PKV = [&](int ib, int s) { return c.pklev[(size_t)s * 16 + ib]; };
    // layer k terms of g-point ig in band ib (rtrn_layer, phys_rrtm_lw_rtrn.cu:94-164)
    struct Lay { R trng, gassrcd, gassrcu, efclrfr, totsrcd, totsrcu, clfr; bool cloudy; };
    auto layer = [&](int k, int ig, int ib) {
        Lay t{};
        const R sdif = c.secdiff[ib];
        R odepth = fmaxR((R)0, sdif * c.TG(ig, k - 1));
        R atrgas, gasfac;
        if (odepth <= c06) {
            atrgas = odepth - (R)0.5f * odepth * odepth;
            t.trng = (R)1 - atrgas;
            gasfac = rec_6 * odepth;
        } else {
            const R tblind = odepth / (bpade + odepth);
            const int itgas = (int)(tblint * tblind + (R)0.5f);
            t.trng = tb.ex[itgas]; atrgas = (R)1 - t.trng; gasfac = tb.tfn[itgas]; odepth = tb.tau[itgas];
        }
        const R plfrac = c.FR(ig, k - 1);
        const R blay = PKL(ib, k);
        const R dplnku = PKV(ib, k) - blay;
        const R dplnkd = PKV(ib, k - 1) - blay;
        t.gassrcd = plfrac * (blay + dplnkd * gasfac) * atrgas;
        t.gassrcu = plfrac * (blay + dplnku * gasfac) * atrgas;
        t.clfr = c.cldfrc[k];
        t.cloudy = t.clfr >= eps;
        t.efclrfr = 1; t.totsrcd = 0; t.totsrcu = 0;
        if (t.cloudy) {
            const R odcld = sdif * c.taucld[(size_t)ib * nlay + (k - 1)];
            t.efclrfr = (R)1 - ((R)1 - mexp(-odcld)) * t.clfr;
            const R odtot = odepth + odcld;
            R totfac, atrtot;
            if (odtot < c06) {
                totfac = rec_6 * odtot; atrtot = odtot - (R)0.5f * odtot * odtot;
            } else {
                const R tblind = odtot / (bpade + odtot);
                const int ittot = (int)(tblint * tblind + (R)0.5f);
                totfac = tb.tfn[ittot]; atrtot = (R)1 - tb.ex[ittot];
            }
            t.totsrcd = plfrac * (blay + dplnkd * totfac) * atrtot;
            t.totsrcu = plfrac * (blay + dplnku * totfac) * atrtot;
        }
        return t;
    };
    std::vector<R> tuf(nlp1, 0), tdf(nlp1, 0), tuc(nlp1, 0), tdc(nlp1, 0);
    std::vector<R> bu(nlp1), bd(nlp1), cu(nlp1), cd(nlp1);
    for (int ib = 0; ib < 16; ++ib) {
        for (int m = 0; m <= nlay; ++m) { bu[m] = 0; bd[m] = 0; cu[m] = 0; cd[m] = 0; }
        const R semi = c.semiss[ib], reflct = (R)1 - semi;
        for (int ig = LW_NS[ib]; ig < LW_NS[ib] + LW_NG[ib]; ++ig) {
            R radtotd = 0, radclrd = 0;
            for (int k = nlay; k >= 1; --k) {
                const Lay t = layer(k, ig, ib);
                if (t.cloudy)
                    radtotd = radtotd * t.trng * t.efclrfr + t.gassrcd + t.clfr * (t.totsrcd - t.gassrcd);
                else
                    radtotd = radtotd * t.trng + t.gassrcd;
                bd[k - 1] = bd[k - 1] + radtotd;
                radclrd = radclrd * t.trng + t.gassrcd;
                cd[k - 1] = cd[k - 1] + radclrd;
            }
            const R rad0 = semi * c.FR(ig, 0) * PKL(ib, 0);
            R radtotu = rad0 + reflct * radtotd;
            bu[0] = bu[0] + radtotu;
            R radclru = rad0 + reflct * radclrd;
            cu[0] = cu[0] + radclru;
            for (int k = 1; k <= nlay; ++k) {
                const Lay t = layer(k, ig, ib);
                if (t.cloudy)
                    radtotu = radtotu * t.trng * t.efclrfr + t.gassrcu + t.clfr * (t.totsrcu - t.gassrcu);
                else
                    radtotu = radtotu * t.trng + t.gassrcu;
                bu[k] = bu[k] + radtotu;
                radclru = radclru * t.trng + t.gassrcu;
                cu[k] = cu[k] + radclru;
            }
        }
        for (int m = 0; m <= nlay; ++m) {
            tuf[m] = tuf[m] + bu[m]; tdf[m] = tdf[m] + bd[m];
            tuc[m] = tuc[m] + cu[m]; tdc[m] = tdc[m] + cd[m];
            c.fnetb[(size_t)ib * nlp1 + m] = (bu[m] - bd[m]) * flxfac;
        }
    }
    for (int m = 0; m <= nlay; ++m) {
        tuf[m] = tuf[m] * flxfac; tdf[m] = tdf[m] * flxfac; tuc[m] = tuc[m] * flxfac; tdc[m] = tdc[m] * flxfac;
        c.totuflux[m] = tuf[m]; c.totdflux[m] = tdf[m]; c.totuclfl[m] = tuc[m]; c.totdclfl[m] = tdc[m];
    }
    R fprev = tuf[0] - tdf[0];
    for (int k = 1; k <= nlay; ++k) {
        const R rfdelp = heatfac / c.delp[k - 1];
        const R fk = tuf[k] - tdf[k];
        c.htr[k - 1] = (fprev - fk) * rfdelp;
        fprev = fk;
    }
}

}  // namespace orc
