// rrtm_aer.hpp -- CPU oracle: the NAM radiation's climatological aerosol optics (test infrastructure only).
//
// Restates, in the reference's float arithmetic, statement by statement:
//   set_spectrum      namgpu/kernels/phys_rrtm_aer_init.cu:145-173   solar / IR flux per wavenumber
//   set_aercoef       namgpu/kernels/phys_rrtm_clim_aerinit.cu:61-160 OPAC band -> SW / LW band weights
//   optavg            namgpu/kernels/phys_rrtm_clim_aerinit.cu:165-284 band-averaged species optics
//   trop_update fill  namgpu/kernels/phys_rrtm_aer_update.cu:40-63    the month's 5-degree climatology
//   setaer prep       namgpu/kernels/phys_rrtm_setaer.cu:80-150       lon / lat in degrees, dz, hz (ivflip 0)
//   aer_property      namgpu/kernels/phys_rrtm_aer_property.cu:117-434 (ivflip 0, NSWBND 14, NLWBND 16)
//   volcanic term     namgpu/kernels/phys_rrtm_setaer.cu:178-330 (lavoflg; ivflip 0 and 1, NLWBND 16 or 1),
//                     year and month from namgpu/physics/rrtm/phys_rrtm_setaer.py:178-192
// Never linked into the product.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace orc {
namespace aer {

constexpr int NAERBND = 61, NRHLEV = 8, NCM1 = 6, NCM2 = 4, NCM = 10, NDM = 5, NAE = 7;
constexpr int IMXAE = 72, JMXAE = 37, NXC = 5, NSW = 14, NLW = 16, NBT = NSW + NLW;
constexpr int NWVSOL = 151, NWVTOT = 57600, NWVTIR = 4000;
// Band limits in cm-1 (radsw_param_nmmb.f wvnum1/wvnum2, radlw_param_nmmb.f wvnlw1/wvnlw2).
constexpr float WSW1[NSW] = {2600, 3251, 4001, 4651, 5151, 6151, 7701, 8051, 12851, 16001, 22651, 29001, 38001, 820};
constexpr float WSW2[NSW] = {3250, 4000, 4650, 5150, 6150, 7700, 8050, 12850, 16000, 22650, 29000, 38000, 50000, 2600};
constexpr float WLW1[NLW] = {10, 251, 501, 631, 701, 821, 981, 1081, 1181, 1391, 1481, 1801, 2081, 2251, 2381, 2601};
constexpr float WLW2[NLW] = {250, 500, 630, 700, 820, 980, 1080, 1180, 1390, 1480, 1800, 2080, 2250, 2380, 2600, 3000};
constexpr float RHLEV[NRHLEV] = {0.0f, 0.5f, 0.7f, 0.8f, 0.9f, 0.95f, 0.98f, 0.99f};

// The climatology as packed (aer_tables.npz): optical tables and one month.
struct Clim {
    const int32_t* iendwv;        // [61]
    const float *haer, *prsref;   // [NAE][NDM]
    const float* rhid;            // [4][NCM1][61]         ext, sca, ssa, asy
    const float* rhdp;            // [4][NCM2][NRHLEV][61] ext, sca, ssa, asy
    const float* straext0;        // [61]
    const int32_t* nwvns0;        // [151]
    const float* s0intv;          // [151]
    const int32_t* midx;          // [JMXAE][IMXAE][NXC]
    const double* mcmix;          // [JMXAE][IMXAE][NXC]
    const int32_t* mkprf;         // [JMXAE][IMXAE]
    const double* mdenn;          // [JMXAE][IMXAE]
};

// Derived tables, in the index order of aer_property.
struct Tables {
    float sigref[NAE * NDM];
    float extrhi[NBT * NCM1], scarhi[NBT * NCM1], ssarhi[NBT * NCM1], asyrhi[NBT * NCM1];
    float extrhd[NBT * NCM2 * NRHLEV], scarhd[NBT * NCM2 * NRHLEV], ssarhd[NBT * NCM2 * NRHLEV],
        asyrhd[NBT * NCM2 * NRHLEV];
    float extstra[NBT];
    float solbnd[NSW], eirbnd[NLW];
    std::vector<float> cmixg, denng;      // [JMXAE][IMXAE][NXC], [JMXAE][IMXAE][2]
    std::vector<int32_t> idxcg, kprfg;    // [JMXAE][IMXAE][NXC], [JMXAE][IMXAE]
};

// set_spectrum: solar flux per wavenumber (the 151 intervals' constants), black-body flux at 273.15 K.
inline void spectrum(const Clim& c, std::vector<float>& sol, std::vector<float>& eir)
{
    sol.assign(NWVTOT, 0.0f);
    int nw1 = 0;
    for (int nb = 0; nb < NWVSOL; ++nb) {
        for (int j = 0; j < c.nwvns0[nb]; ++j) sol[nw1 + j] = c.s0intv[nb];
        nw1 += c.nwvns0[nb];
    }
    const float pi = 3.1415926535897931f, cl = 2.99792458e+8f, plnk = 6.6260693e-34f, boltz = 1.3806505e-23f,
                t0c = 2.7315e+2f;
    const float tmp1 = 2.0f * pi * plnk * (cl * cl);
    const float tmp2 = plnk * cl / (boltz * t0c);
    eir.assign(NWVTIR, 0.0f);
    for (int nw = 1; nw <= NWVTIR; ++nw) {
        const float tmp3 = 100.0f * (float)nw;
        eir[nw - 1] = (tmp1 * (tmp3 * tmp3 * tmp3)) / (std::exp(tmp2 * tmp3) - 1.0f);
    }
}

// set_aercoef for one band: the OPAC bands [lo, hi] it overlaps, the flux of each inside the band, the total.
inline void band_weights(const Clim& c, const std::vector<float>& f, int iw1, int iw2, float* w, int& lo, int& hi,
                         float& total)
{
    for (int ni = 0; ni < NAERBND; ++ni) w[ni] = 0.0f;
    int ii = 1;
    while (ii != NAERBND && iw1 > c.iendwv[ii - 1]) ++ii;
    lo = ii;
    float tb = 0.0f, part = 0.0f;
    for (int iw = iw1; iw <= iw2; ++iw) {
        const float x = f[iw - 1];
        tb = tb + x;
        part = part + x;
        if (iw == c.iendwv[ii - 1]) {
            w[ii - 1] = part;
            if (ii < NAERBND) { part = 0.0f; ++ii; }
        }
    }
    if (iw2 != c.iendwv[ii - 1]) w[ii - 1] = part;
    hi = ii;
    total = tb;
}

// optavg of one species row: the band's flux-weighted extinction, scattering, asymmetry, and the
// single-scattering albedo that reproduces the weighted two-stream reflectance.
inline void optavg(const float* ext, const float* sca, const float* ssa, const float* asy, const float* w, int lo,
                   int hi, float rnorm, float& oe, float& os, float& ow, float& og)
{
    float sk = 0, ss = 0, sok = 0, sokg = 0, sref = 0;
    for (int ni = lo; ni <= hi; ++ni) {
        const float wt = w[ni - 1];
        const float a = ssa[ni - 1], g = asy[ni - 1], e = ext[ni - 1], s = sca[ni - 1];
        const float sp = std::sqrt((1.0f - a) / (1.0f - a * g));
        const float reft = (1.0f - sp) / (1.0f + sp);
        sref = sref + reft * wt;
        sk = sk + e * wt;
        ss = ss + s * wt;
        sok = sok + a * wt * e;
        sokg = sokg + a * wt * e * g;
    }
    const float refb = sref * rnorm;
    const float asyo = sokg / (sok + 1.0e-10f);
    oe = sk * rnorm;
    os = ss * rnorm;
    og = asyo;
    ow = 4.0f * refb / ((1.0f + refb) * (1.0f + refb) - asyo * ((1.0f - refb) * (1.0f - refb)));
}

inline void build(const Clim& c, Tables& t)
{
    std::vector<float> sol, eir;
    spectrum(c, sol, eir);
    for (int i = 0; i < NAE * NDM; ++i) t.sigref[i] = 0.001f * c.prsref[i];
    const size_t R1 = (size_t)NCM1 * NAERBND, R2 = (size_t)NCM2 * NRHLEV * NAERBND;
    for (int ib = 0; ib < NBT; ++ib) {
        const bool sw = ib < NSW;
        float w[NAERBND], total;
        int lo, hi;
        if (sw) band_weights(c, sol, (int)std::lround(WSW1[ib]), (int)std::lround(WSW2[ib]), w, lo, hi, total);
        else band_weights(c, eir, (int)std::lround(WLW1[ib - NSW]), (int)std::lround(WLW2[ib - NSW]), w, lo, hi, total);
        if (sw) t.solbnd[ib] = total; else t.eirbnd[ib - NSW] = total;
        const float rnorm = 1.0f / total;
        for (int nc = 0; nc < NCM1; ++nc) {
            const size_t o = (size_t)nc * NAERBND;
            optavg(c.rhid + o, c.rhid + R1 + o, c.rhid + 2 * R1 + o, c.rhid + 3 * R1 + o, w, lo, hi, rnorm,
                   t.extrhi[ib * NCM1 + nc], t.scarhi[ib * NCM1 + nc], t.ssarhi[ib * NCM1 + nc],
                   t.asyrhi[ib * NCM1 + nc]);
        }
        for (int nc = 0; nc < NCM2; ++nc)
            for (int nh = 0; nh < NRHLEV; ++nh) {
                const size_t o = ((size_t)nc * NRHLEV + nh) * NAERBND;
                const int q = (ib * NCM2 + nc) * NRHLEV + nh;
                optavg(c.rhdp + o, c.rhdp + R2 + o, c.rhdp + 2 * R2 + o, c.rhdp + 3 * R2 + o, w, lo, hi, rnorm,
                       t.extrhd[q], t.scarhd[q], t.ssarhd[q], t.asyrhd[q]);
            }
        float sk = 0;
        for (int ni = lo; ni <= hi; ++ni) sk = sk + c.straext0[ni - 1] * w[ni - 1];
        t.extstra[ib] = sk * rnorm;
    }
    const int ncell = IMXAE * JMXAE;
    t.cmixg.assign((size_t)ncell * NXC, 0.0f);
    t.denng.assign((size_t)ncell * 2, 0.0f);
    t.idxcg.assign((size_t)ncell * NXC, 0);
    t.kprfg.assign(ncell, 0);
    for (int cell = 0; cell < ncell; ++cell) {
        const int kp = c.mkprf[cell];
        t.kprfg[cell] = kp;
        double tem = 1.0;
        for (int k = 0; k < NXC; ++k) t.idxcg[(size_t)cell * NXC + k] = c.midx[(size_t)cell * NXC + k];
        for (int k = 0; k < NXC - 1; ++k) {
            t.cmixg[(size_t)cell * NXC + k] = (float)c.mcmix[(size_t)cell * NXC + k];
            tem = tem - c.mcmix[(size_t)cell * NXC + k];
        }
        t.cmixg[(size_t)cell * NXC + NXC - 1] = (float)tem;
        t.denng[2 * (size_t)cell] = (float)c.mdenn[cell];
        t.denng[2 * (size_t)cell + 1] = kp >= 6 ? (float)c.mcmix[(size_t)cell * NXC + NXC - 1] : 0.0f;
    }
}

// One column: setaer's prep and aer_property.  Inputs top first (ivflip 0): prsi [nlp1], prsl, tlay, qlay,
// rhlay [nlay]; outputs sw [3][NSW][nlay], lw [3][NLW][nlay] at stride n (column-major over columns).
inline void column(const Tables& t, const Clim& c, int nlay, const float* prsi, const float* prsl, const float* tlay,
                   const float* qlay, const float* rhlay, float xlon, float xlat, float slmsk, float* sw, float* lw,
                   size_t n)
{
    const int nlp1 = nlay + 1;
    const float pi = 3.1415926535897931f, rd = 2.8705e+2f, g0 = 9.80665e+0f, rv = 4.6150e+2f;
    const float rdg = 180.0f / pi, rovg = 0.001f * rd / g0, fvirt = rv / rd - 1.0f;
    float alon = xlon * rdg;
    if (alon < 0.0f) alon = alon + 360.0f;
    float alat = xlat * rdg;
    if (alat < -90.0f) alat = -90.0f;
    if (alat > 90.0f) alat = 90.0f;
    std::vector<float> dz(nlay + 2), hz(nlp1 + 2);
    for (int k = 1; k <= nlay; ++k) {
        const float a = k == 1 ? std::log(prsl[0]) : std::log(prsi[k - 1]);
        const float b = std::log(prsi[k]);
        dz[k] = rovg * (b - a) * tlay[k - 1] * (1.0f + fvirt * qlay[k - 1]);
    }
    dz[1] = 2.0f * dz[1];
    hz[nlp1] = 0.0f;
    for (int k = nlay; k >= 1; --k) hz[k] = hz[k + 1] + dz[k];

    // the 5-degree cell bracket: longitude cells from 0 east, latitude rows from 90 N south
    const float dltg = 360.0f / (float)IMXAE, hdlt = 0.5f * dltg, rdlt = 1.0f / dltg;
    int i3 = 1;
    float dtmp = alon < 0.0f ? 0.0f : alon;
    while (dtmp > dltg && i3 < IMXAE) { ++i3; dtmp = alon - dltg * (float)(i3 - 1); }
    const int i1 = i3, i2 = i3 % IMXAE + 1;
    const float wi = dtmp * rdlt;
    const int kpi = dtmp <= hdlt ? i3 : i2;
    int j3 = 1;
    float dtl = 90.0f - alat;
    while (dtl > dltg && j3 < JMXAE) { ++j3; dtl = (90.0f - dltg * (float)(j3 - 1)) - alat; }
    const int j1 = j3, j2 = j3 + 1 > JMXAE ? JMXAE : j3 + 1;
    const float wj = dtl * rdlt;
    const int kpj = dtl <= hdlt ? j3 : j2;
    auto KP = [&](int i, int j) { return t.kprfg[(size_t)(j - 1) * IMXAE + (i - 1)]; };
    auto HA = [&](int idm, int kp) { return c.haer[(kp - 1) * NDM + (idm - 1)]; };
    auto PR = [&](int idm, int kp) { return c.prsref[(kp - 1) * NDM + (idm - 1)]; };
    auto SG = [&](int idm, int kp) { return t.sigref[(kp - 1) * NDM + (idm - 1)]; };
    int kp = KP(kpi, kpj);
    const int kpa = std::max(std::max(KP(i1, j1), KP(i1, j2)), std::max(KP(i2, j1), KP(i2, j2)));
    float h1 = HA(1, kp);
    int ii = 1;
    if (kp != kpa) {
        if (kpa == 6) {
            ii = 2;
            if (slmsk > 0.0f) { kp = 7; h1 = 0.5f * (HA(1, 6) + HA(1, 7)); }
            else { kp = kpa; h1 = HA(1, 6); }
        } else if (kpa == 7) {
            ii = 2;
            if (slmsk <= 0.0f) { kp = 6; h1 = 0.5f * (HA(1, 6) + HA(1, 7)); }
            else { kp = kpa; h1 = HA(1, 7); }
        } else {
            h1 = HA(1, kpa);
            kp = kpa;
        }
    }
    const float w11 = (1.0f - wi) * (1.0f - wj), w12 = (1.0f - wi) * wj, w21 = wi * (1.0f - wj), w22 = wi * wj;
    auto DN = [&](int m, int i, int j) { return t.denng[((size_t)(j - 1) * IMXAE + (i - 1)) * 2 + (m - 1)]; };
    auto CM = [&](int m, int i, int j) { return t.cmixg[((size_t)(j - 1) * IMXAE + (i - 1)) * NXC + (m - 1)]; };
    auto IX = [&](int m, int i, int j) { return t.idxcg[((size_t)(j - 1) * IMXAE + (i - 1)) * NXC + (m - 1)]; };
    float denn[3] = {0, 0, 0};
    for (int m = 1; m <= ii; ++m)
        denn[m] = w11 * DN(m, i1, j1) + w12 * DN(m, i1, j2) + w21 * DN(m, i2, j1) + w22 * DN(m, i2, j2);
    float cmix[NCM + 1];
    for (int q = 0; q <= NCM; ++q) cmix[q] = 0.0f;
    for (int m = 1; m <= NXC; ++m) {
        int ic = IX(m, i1, j1);
        if (ic > 0) cmix[ic] = cmix[ic] + w11 * CM(m, i1, j1);
        ic = IX(m, i1, j2);
        if (ic > 0) cmix[ic] = cmix[ic] + w12 * CM(m, i1, j2);
        ic = IX(m, i2, j1);
        if (ic > 0) cmix[ic] = cmix[ic] + w21 * CM(m, i2, j1);
        ic = IX(m, i2, j2);
        if (ic > 0) cmix[ic] = cmix[ic] + w22 * CM(m, i2, j2);
    }
    // domain of each layer, walking up from the surface (top-first storage), and its effective thickness
    std::vector<float> delz(nlay + 2), rdrh(nlay + 2), tau(nlay + 2), ssa(nlay + 2), asy(nlay + 2);
    std::vector<int> idm(nlay + 2), ih1v(nlay + 2), ih2v(nlay + 2);
    const float rps = 1.0f / prsi[nlay];
    ii = 1;
    for (int k = nlay; k >= 1; --k) {
        if (ii <= NDM && prsi[k - 1] * rps < SG(ii, kp)) {
            ii = ii + 1;
            if (ii == 2 && PR(2, kp) == PR(3, kp)) ii = 3;
        }
        idm[k] = ii;
        const float h = ii > 1 ? (ii <= NDM ? HA(ii, kp) : 0.0f) : h1;
        if (h > 0.0f) {
            const float r = 1.0f / h;
            delz[k] = h * (std::exp(-hz[k + 1] * r) - std::exp(-hz[k] * r));
        } else {
            delz[k] = dz[k];
        }
    }
    for (int k = 1; k <= nlay; ++k) {
        const float rh = rhlay[k - 1];
        int b = 1;
        while (b <= NRHLEV && rh > RHLEV[b - 1]) ++b;
        const int a = std::max(1, b - 1);
        b = std::min(NRHLEV, b);
        rdrh[k] = a == b ? 0.0f : (rh - RHLEV[a - 1]) / (RHLEV[b - 1] - RHLEV[a - 1]);
        ih1v[k] = a;
        ih2v[k] = b;
    }
    auto EI = [&](const float* x, int ic, int ib) { return x[(ib - 1) * NCM1 + (ic - 1)]; };
    auto ED = [&](const float* x, int ir, int ic, int ib) { return x[((ib - 1) * NCM2 + (ic - 1)) * NRHLEV + (ir - 1)]; };
    for (int ib = 1; ib <= NBT; ++ib) {
        const bool isw = ib <= NSW;
        for (int k = 1; k <= nlay; ++k) {
            const int d = idm[k], a = ih1v[k], b = ih2v[k];
            const float r = rdrh[k], z = delz[k];
            auto RD = [&](const float* x, int ic) { return ED(x, a, ic, ib) + r * (ED(x, b, ic, ib) - ED(x, a, ic, ib)); };
            if (d == 5 || d == 4) {
                tau[k] = d == 5 ? 0.0f : t.extstra[ib - 1] * z;
                ssa[k] = isw ? 0.99f : 0.5f;
                asy[k] = isw ? 0.696f : 0.3f;
            } else if (d == 3) {
                const float e1 = EI(t.extrhi, 1, ib), s1 = EI(t.scarhi, 1, ib), w1 = EI(t.ssarhi, 1, ib), g1 = EI(t.asyrhi, 1, ib);
                const float e2 = EI(t.extrhi, 2, ib), s2 = EI(t.scarhi, 2, ib), w2 = EI(t.ssarhi, 2, ib), g2 = EI(t.asyrhi, 2, ib);
                const float e3 = RD(t.extrhd, 1), s3 = RD(t.scarhd, 1), w3 = RD(t.ssarhd, 1), g3 = RD(t.asyrhd, 1);
                const float ext1 = 0.17e-3f * e1 + 0.4f * e2 + 0.59983f * e3;
                const float sca1 = 0.17e-3f * s1 + 0.4f * s2 + 0.59983f * s3;
                const float ssa1 = 0.17e-3f * w1 * e1 + 0.4f * w2 * e2 + 0.59983f * w3 * e3;
                const float asy1 = 0.17e-3f * g1 * s1 + 0.4f * g2 * s2 + 0.59983f * g3 * s3;
                tau[k] = ext1 * 730.0f * z;
                ssa[k] = ext1 > 0.0f ? std::min(1.0f, ssa1 / ext1) : 1.0f;
                asy[k] = sca1 > 0.0f ? std::min(1.0f, asy1 / sca1) : 0.0f;
            } else if (d == 1) {
                float ext1 = 0, sca1 = 0, ssa1 = 0, asy1 = 0;
                for (int ic = 1; ic <= NCM; ++ic) {
                    const float cm = cmix[ic];
                    if (!(cm > 0.0f)) continue;
                    if (ic <= NCM1) {
                        ext1 = ext1 + cm * EI(t.extrhi, ic, ib);
                        sca1 = sca1 + cm * EI(t.scarhi, ic, ib);
                        ssa1 = ssa1 + cm * EI(t.ssarhi, ic, ib) * EI(t.extrhi, ic, ib);
                        asy1 = asy1 + cm * EI(t.asyrhi, ic, ib) * EI(t.scarhi, ic, ib);
                    } else {
                        const int q = ic - NCM1;
                        const float e0 = RD(t.extrhd, q), s0 = RD(t.scarhd, q), w0 = RD(t.ssarhd, q), g0 = RD(t.asyrhd, q);
                        ext1 = ext1 + cm * e0;
                        sca1 = sca1 + cm * s0;
                        ssa1 = ssa1 + cm * w0 * e0;
                        asy1 = asy1 + cm * g0 * s0;
                    }
                }
                tau[k] = ext1 * denn[1] * z;
                ssa[k] = ext1 > 0.0f ? std::min(1.0f, ssa1 / ext1) : 1.0f;
                asy[k] = sca1 > 0.0f ? std::min(1.0f, asy1 / sca1) : 0.0f;
            } else if (d == 2) {
                tau[k] = EI(t.extrhi, 6, ib) * denn[2] * z;
                ssa[k] = EI(t.ssarhi, 6, ib);
                asy[k] = EI(t.asyrhi, 6, ib);
            } else {
                tau[k] = 0.0f; ssa[k] = 1.0f; asy[k] = 0.0f;
            }
        }
        // smoothing across domain boundaries, top to surface
        for (int k = 2; k <= nlay; ++k) {
            const float ratio = tau[k] > 0.0f ? tau[k - 1] / tau[k] : 1.0f;
            const float s = tau[k] + tau[k - 1], lo = 0.2f * s, hi = s - lo;
            if (ratio > 30.0f) { tau[k] = lo; tau[k - 1] = hi; }
            if (ratio < 0.03333f) { tau[k] = hi; tau[k - 1] = lo; }
        }
        float* o = isw ? sw : lw;
        const int nb = isw ? NSW : NLW, m = isw ? ib - 1 : ib - NSW - 1;
        for (int k = 1; k <= nlay; ++k) {
            o[(((size_t)0 * nb + m) * nlay + (k - 1)) * n] = tau[k];
            o[(((size_t)1 * nb + m) * nlay + (k - 1)) * n] = ssa[k];
            o[(((size_t)2 * nb + m) * nlay + (k - 1)) * n] = asy[k];
        }
    }
}

// The volcanic stratospheric term of one column, added to the extinction (component 0) of sw [3][NSW][nlay]
// and lw [3][NLW][nlay] at stride n.  prsi [nlay + 1] in mb in the order of ivflip; xlat in radians; iv[4]
// the table's values of the four latitude zones (90N-45N, 45N-0, 0-45S, 45S-90S) for the year and month.
// Levels and layers are 0-based here: the reference's level k is prsi[k - 1], its layer k is index k - 1.
inline void volcanic(int nlay, int ivflip, const float* prsi, float xlat, const int32_t iv[4], bool add_sw,
                     bool add_lw, bool lw1bd, float* sw, float* lw, size_t n)
{
    const float pi = 3.1415926535897931f, rdg = 180.0f / pi, psrfh = 5.0f;
    float lat = xlat * rdg;
    if (lat < -90.0f) lat = -90.0f;
    if (lat > 90.0f) lat = 90.0f;
    // zone value, halved sums of two zones within a degree of 45N, the equator and 45S
    float volcae;
    if (lat > 46.0f)       volcae = 1.0e-4f * (float)iv[0];
    else if (lat > 44.0f)  volcae = 5.0e-5f * (float)(iv[0] + iv[1]);
    else if (lat > 1.0f)   volcae = 1.0e-4f * (float)iv[1];
    else if (lat > -1.0f)  volcae = 5.0e-5f * (float)(iv[1] + iv[2]);
    else if (lat > -44.0f) volcae = 1.0e-4f * (float)iv[2];
    else if (lat > -46.0f) volcae = 5.0e-5f * (float)(iv[2] + iv[3]);
    else                   volcae = 1.0e-4f * (float)iv[3];
    // lower edge of the layer: 250 mb poleward of 70 degrees, 150 mb within 20, linear between
    const float alat = std::fabs(lat);
    const float psrfl = alat > 70.0f ? 250.0f : (alat < 20.0f ? 150.0f : 110.0f + 2.0f * alat);

    // top layer kh and bottom layer kl of the aerosol (0-based layers), rdelp = 1 / their pressure depth
    int kh, kl;
    float rdelp;
    if (ivflip == 0) {
        kh = nlay - 2; kl = 1; rdelp = 1.0f / prsi[1];
        for (int i = 1; i <= nlay - 3; ++i)
            if (prsi[i] >= psrfh) { kh = i - 1; break; }
        for (int i = 1; i <= nlay - 3; ++i)
            if (prsi[i] >= psrfl) { kl = i - 1; rdelp = 1.0f / (prsi[i] - prsi[kh]); break; }
    } else {
        kh = 1; kl = nlay - 2; rdelp = 1.0f / prsi[nlay - 2];
        for (int i = nlay - 2; i >= 1; --i)
            if (prsi[i] >= psrfh) { kh = i; break; }
        for (int i = nlay - 1; i >= 1; --i)
            if (prsi[i] >= psrfl) { kl = i; rdelp = 1.0f / (prsi[i] - prsi[kh + 1]); break; }
    }
    // layer j's share of the column: its pressure depth times rdelp
    auto share = [&](int j) {
        return ivflip == 0 ? (prsi[j + 1] - prsi[j]) * rdelp : (prsi[j] - prsi[j + 1]) * rdelp;
    };
    const int j0 = ivflip == 0 ? kh : kl, j1 = ivflip == 0 ? kl : kh;
    const int below = ivflip == 0 ? kl + 1 : kl - 1;     // the layer under the bottom one
    if (add_sw) {
        for (int b = 0; b < NSW; ++b) {
            // wavelength exponent: 0.74 below 0.5 micron (above 20000 cm-1), 1.14 above it, 0.94 across it
            const float e = WSW1[b] > 20000.0f ? 0.74f : (WSW2[b] < 20000.0f ? 1.14f : 0.94f);
            const float tb = std::pow(0.275e-4f * (WSW2[b] + WSW1[b]), e);
            float* x = sw + (size_t)b * nlay * n;
            for (int j = j0; j <= j1; ++j) {
                const float tmp2 = tb * share(j);
                x[j * n] = x[j * n] + tmp2 * volcae;
            }
            if (x[kl * n] > 10.0f * x[below * n]) {      // spread a sharp bottom edge 80 / 20 over two layers
                const float s2 = x[kl * n] + x[below * n];
                x[kl * n] = 0.8f * s2;
                x[below * n] = 0.2f * s2;
            }
        }
    }
    if (add_lw) {
        for (int b = 0; b < NLW; ++b) {
            const float tb = lw1bd ? std::pow(0.55f / 11.0f, 1.2f) : std::pow(0.275e-4f * (WLW2[b] + WLW1[b]), 1.2f);
            float* x = lw + (size_t)b * nlay * n;
            for (int j = j0; j <= j1; ++j) {
                const float tmp2 = tb * share(j);
                x[j * n] = x[j * n] + tmp2 * volcae;
            }
        }
    }
}

}  // namespace aer
}  // namespace orc
