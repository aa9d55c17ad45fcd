// rrtm_front.hpp -- CPU oracle: grrad's front end ahead of the column solve (test infrastructure only).
//
// Restates, in the reference's single-precision arithmetic and statement order (Fortran semantics of the
// NMMB sources the reference kernels port):
//   dayparts   namgpu/kernels/phys_rrtm_dayparts.cu:50-138 (grrad_nmmb.f:606-656 with coszmn_nmmb): the
//              cosine of the solar zenith angle over the SW interval and the per-row runs of day / night
//              points, computed here as the Fortran does, one row after another
//   getgases   namgpu/kernels/phys_rrtm_getgases.cu:67-130 (radiation_gases_nmmb.f:843-979)
//   getozn     namgpu/kernels/phys_rrtm_getozn.cu:43-111 (radiation_gases_nmmb.f:984-1094)
//   setalb     namgpu/kernels/phys_rrtm_setalb.cu:35-248 (radiation_surface_nmmb.f:407-725), ialbflg 0, 1, 2
//   setemis    namgpu/kernels/phys_rrtm_setemis.cu:40-133 (radiation_surface_nmmb.f:730-897), with the
//              Fortran's linear searches of the 1-degree emissivity map
//   progcld2   namgpu/kernels/phys_rrtm_progcld2.cu:92-444 (radiation_clouds_nmmb.f:787-1323 with
//              rsipath2_tmp :2779-2964 and gethml :2167-2494)
//   clw        namgpu/kernels/phys_rrtm_grrad_clouds.cu:396-416 (grrad_nmmb.f:1556-1571): the condensate of
//              the cloud tracers
//   albedo     namgpu/kernels/phys_rrtm_grrad_clouds.cu:344-393 (grrad_nmmb.f:1722-1794): the IALB = 2 surface
//              albedo from the zenith angle and the atmospheric transmissivity (the TRN / ZA / DZA / ALBD tables)
// Layouts: 2-D fields [n] with n = jm * im columns (row-major, point i of row j at j * im + i), 3-D fields
// [level][n], multi-field outputs [field][level][n].  Never linked into the product.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace orc {
namespace front {

// ------------------------------------------------------------------------------------------ dayparts
// coszmn_nmmb for one point: the daytime mean of max(0, cos zenith) over nrads samples of the SW interval
// (returned) and the whole-interval mean (coszdg).  pid12 is the single-precision literal of dayparts.
inline float dp_cosz(float xlon, float sinlat, float coslat, float solhr, float dtswav, int nrads, float sollag,
                     float sindec, float cosdec, float& coszdg)
{
    const float pid12 = 0.261799388f, f12 = 12.0f, czlimt = 0.0001f;
    const float solang = pid12 * (solhr - f12);
    const float rnstp = dtswav / (float)nrads;
    const float ss = sinlat * sindec, cc = coslat * cosdec;
    float sum = 0.0f;
    int lit = 0;
    for (int it = 1; it <= nrads; ++it) {
        const float cns = solang + (float)(it - 1) * pid12 * rnstp + sollag;
        const float cz = ss + cc * std::cos(cns + xlon);
        sum = sum + std::fmax(0.0f, cz);
        if (cz > czlimt) lit = lit + 1;
    }
    coszdg = sum * rnstp;
    if (lit > 0) sum = sum / (float)lit;
    return sum;
}

// DAYPARTS of every row: a run starts at the row's first point and wherever the day flag (coszen >= 1e-4)
// changes; run k of row j sits in slot j * im + k with its 1-based start point, length and day flag.  Slots
// past the row's run count are left as they are.
inline void dayparts(int im, int jm, const float* xlon, const float* sinlat, const float* coslat, float solhr,
                     float dtswav, int nrads, float sollag, float sindec, float cosdec, float* coszen, float* coszdg,
                     int* dp_start, int* dp_len, int* dp_day, int* ndayparts)
{
    for (int j = 0; j < jm; ++j) {
        const size_t r0 = (size_t)j * im;
        int nrun = 0, prev = -1;
        for (int i = 0; i < im; ++i) {
            const size_t p = r0 + i;
            float dg;
            const float cz = dp_cosz(xlon[p], sinlat[p], coslat[p], solhr, dtswav, nrads, sollag, sindec, cosdec, dg);
            coszen[p] = cz;
            coszdg[p] = dg;
            const int d = cz >= 0.0001f ? 1 : 0;
            if (i == 0 || d != prev) {
                if (nrun > 0) dp_len[r0 + nrun - 1] = (i + 1) - dp_start[r0 + nrun - 1];
                dp_start[r0 + nrun] = i + 1;
                dp_day[r0 + nrun] = d;
                ++nrun;
            }
            prev = d;
        }
        if (nrun > 0) dp_len[r0 + nrun - 1] = (im + 1) - dp_start[r0 + nrun - 1];
        ndayparts[j] = nrun;
    }
}

// ------------------------------------------------------------------------------------------ getgases
// Volume mixing ratios of the 10 radiative gases on lmax levels: the module defaults, CO2 replaced by the
// global mean plus the month's seasonal cycle (ico2flg 1) or, below prsco2 = 788 mb, by the monthly 15-degree
// CO2 map (ico2flg 2).  plvl [lmax + 1][n] mb; co2vmr_sav [12][12][24] ([month][lat][lon]); gasvmr [10][lmax][n].
inline void getgases(int n, int lmax, const float* plvl, const float* xlon, const float* xlat, float co2_glb,
                     const float* gco2cyc, const float* co2vmr_sav, int ico2flg, int kmonsav, int ivflip, float* gasvmr)
{
    const float defv[10] = {350.0e-6f, 0.31e-6f, 1.50e-6f, 0.209f, 1.50e-8f,
                            3.520e-10f, 6.358e-10f, 1.500e-10f, 1.397e-10f, 8.2000e-11f};
    const float con_pi = 3.14159265358979323846f, hfpi = 0.5f * con_pi, raddeg = 180.0f / con_pi;
    const float tmp = raddeg / 15.0f;
    const size_t N = (size_t)n, LN = (size_t)lmax * n;
    for (int c = 0; c < n; ++c) {
        for (int g = 0; g < 10; ++g)
            for (int l = 0; l < lmax; ++l) gasvmr[g * LN + l * N + c] = defv[g];
        if (ico2flg == 1) {
            const float base = co2_glb + gco2cyc[kmonsav - 1];
            for (int l = 0; l < lmax; ++l) gasvmr[l * N + c] = base;
        } else if (ico2flg == 2) {
            float lon = xlon[c];
            if (lon < 0.0f) lon = lon + con_pi;
            const float colat = hfpi - xlat[c];
            int ilon = std::min(24, (int)(lon * tmp + 1.0f));
            int ilat = std::min(12, (int)(colat * tmp + 1.0f));
            ilon = std::max(ilon, 1);
            ilat = std::max(ilat, 1);
            const float map = co2vmr_sav[((size_t)(kmonsav - 1) * 12 + (ilat - 1)) * 24 + (ilon - 1)];
            const float base = co2_glb + gco2cyc[kmonsav - 1];
            for (int l = 0; l < lmax; ++l) {
                const float pl = plvl[(size_t)(ivflip == 0 ? l : l + 1) * N + c];
                gasvmr[l * N + c] = pl >= 788.0f ? map : base;
            }
        }
    }
}

// ------------------------------------------------------------------------------------------ getozn
// Climatological ozone (ntoz 0): the latitude- and time-interpolated profile o3i of the climatology o3r
// [12][loz][jmr], then, per level, linear interpolation in the Exner function between the bracketing
// climatology levels pkstr [loz], the end values outside them.  A level with no bracket keeps its value.
inline void getozn(int n, int nlev, const float* prslk, const float* xlat, const float* o3r, const float* pkstr,
                   int jmr, int loz, int k1oz, int k2oz, float facoz, float blte, float dlte, int ivflip,
                   float* o3mmr)
{
    const float raddeg = 57.29578f;
    const float elte = blte + (float)(jmr - 1) * dlte;
    auto R = [&](int j1, int k, int m1) { return o3r[((size_t)(m1 - 1) * loz + k) * jmr + (j1 - 1)]; };
    std::vector<float> o3i(loz);
    for (int c = 0; c < n; ++c) {
        const float deglat = xlat[c] * raddeg;
        int j1, j2;
        float w;
        if (deglat > blte && deglat < elte) {
            w = (deglat - blte) / dlte + 1.0f;
            j1 = (int)w;
            j2 = j1 + 1;
            w = w - (float)j1;
        } else if (deglat <= blte) {
            j1 = j2 = 1;
            w = 1.0f;
        } else if (deglat >= elte) {
            j1 = j2 = jmr;
            w = 1.0f;
        } else {
            continue;   // NaN latitude: no branch of the Fortran applies
        }
        const float w2 = 1.0f - w;
        for (int k = 0; k < loz; ++k) {
            const float a = w2 * R(j1, k, k1oz) + w * R(j2, k, k1oz);
            const float b = w2 * R(j1, k, k2oz) + w * R(j2, k, k2oz);
            o3i[k] = b * facoz + a * (1.0f - facoz);
        }
        for (int l = 1; l <= nlev; ++l) {
            const int ll = ivflip == 1 ? nlev - l + 1 : l;
            const size_t o = (size_t)(ll - 1) * n + c;
            const float x = prslk[o];
            for (int k = 0; k < loz - 1; ++k) {
                const float rdp = 1.0f / (pkstr[k + 1] - pkstr[k]);
                if (x > pkstr[k] && x <= pkstr[k + 1]) {
                    const float t = (pkstr[k + 1] - x) * rdp;
                    o3mmr[o] = t * o3i[k] + (1.0f - t) * o3i[k + 1];
                }
            }
            if (x > pkstr[loz - 1]) o3mmr[o] = o3i[loz - 1];
            if (x < pkstr[0]) o3mmr[o] = o3i[0];
        }
    }
}

// ------------------------------------------------------------------------------------------ setalb
struct AlbIn {
    const float *slmsk, *snowf, *sncovr, *snoalb, *zorlf, *coszf, *tsknf, *hprif, *alvsf, *alnsf, *alvwf, *alnwf,
        *facsf, *facwf, *fice, *tisfc;
};

// The four surface albedo components [4][n] (near-IR direct, near-IR diffuse, visible direct, visible diffuse)
// for the SW call: Briegleb's climatological scheme (ialbflg 0), MODIS land albedo with the land model's snow
// cover (1), or the externally provided albedos as they are (any other value: the NAM path).
inline void setalb(int n, const AlbIn& a, int ialbflg, float* sfcalb)
{
    const float t0c = 273.15f, ttp = 273.16f, tice = 271.20f;
    for (int c = 0; c < n; ++c) {
        float* A0 = sfcalb + c;
        float* A1 = sfcalb + n + c;
        float* A2 = sfcalb + 2 * (size_t)n + c;
        float* A3 = sfcalb + 3 * (size_t)n + c;
        if (ialbflg != 0 && ialbflg != 1) {
            *A0 = a.alnsf[c];
            *A1 = a.alnwf[c];
            *A2 = a.alvsf[c];
            *A3 = a.alvwf[c];
            continue;
        }
        const int msk = (int)std::round(a.slmsk[c]);
        const float ts = a.tsknf[c], cz = a.coszf[c];
        auto snowfrac = [&]() {
            const float asnow = 0.02f * a.snowf[c];
            const float argh = std::fmin(0.50f, std::fmax(0.025f, 0.01f * a.zorlf[c]));
            const float hrgh = std::fmin(1.0f, std::fmax(0.20f, 1.0577f - 1.1538e-3f * a.hprif[c]));
            return asnow / (argh + asnow) * hrgh;
        };
        float fsno0;
        if (ialbflg == 0) {
            fsno0 = snowfrac();
            if (msk == 0 && ts > tice) fsno0 = 0.0f;
        } else {
            fsno0 = a.sncovr[c];
            if (msk == 0 && ts > tice) fsno0 = 0.0f;
            if (msk == 2) fsno0 = snowfrac();
        }
        const float fsno1 = 1.0f - fsno0;
        const float flnd0 = std::fmin(1.0f, a.facsf[c] + a.facwf[c]);
        const float fsea0 = std::fmax(0.0f, 1.0f - flnd0);
        const float fsno = fsno0, fsea = fsea0 * fsno1, flnd = flnd0 * fsno1;
        // diffuse sea albedo
        float asevd, asend;
        if (ts >= 271.5f) {
            asevd = asend = 0.06f;
        } else if (ts < 271.1f) {
            asevd = 0.70f;
            asend = 0.65f;
        } else {
            const float d2 = (ts - 271.1f) * (ts - 271.1f);
            asevd = 0.7f - 4.0f * d2;
            asend = 0.65f - 3.6875f * d2;
        }
        // diffuse snow albedo (sea ice from the ice fraction)
        float asnvd, asnnd;
        if (msk == 2) {
            const float ffw = 1.0f - a.fice[c];
            float b1 = 0.0f;
            if (ffw < 1.0f) b1 = 0.03f * std::fmax(0.0f, std::fmin(5.0f, ttp - a.tisfc[c]));
            const float b3 = 0.06f * ffw;
            asnvd = (0.70f + b1) * a.fice[c] + b3;
            asnnd = (0.60f + b1) * a.fice[c] + b3;
            asevd = 0.70f * a.fice[c] + b3;
            asend = 0.60f * a.fice[c] + b3;
        } else if (ialbflg == 0) {
            asnvd = 0.90f;
            asnnd = 0.75f;
        } else {
            asnvd = asnnd = a.snoalb[c];
        }
        // direct snow albedo
        float asnvb, asnnb;
        if (ialbflg == 1 && msk != 2) {
            asnvb = asnnb = a.snoalb[c];
        } else if (cz < 0.5f) {
            const float csnow = 0.5f * (3.0f / (1.0f + 4.0f * cz) - 1.0f);
            asnvb = std::fmin(0.98f, asnvd + (1.0f - asnvd) * csnow);
            asnnb = std::fmin(0.98f, asnnd + (1.0f - asnnd) * csnow);
        } else {
            asnvb = asnvd;
            asnnb = asnnd;
        }
        // direct sea albedo (zenith-angle dependence)
        float rfcs, rfcw, asevb, asenb;
        if (cz > 0.0001f) {
            rfcs = ialbflg == 0 ? 2.14f / (1.0f + 1.48f * cz) : 1.775f / (1.0f + 1.55f * cz);
            rfcw = rfcs;
            if (ts >= t0c) {
                asevb = std::fmax(asevd, 0.026f / (std::pow(cz, 1.7f) + 0.065f) +
                                             0.15f * (cz - 0.1f) * (cz - 0.5f) * (cz - 1.0f));
                asenb = asevb;
            } else {
                asevb = asevd;
                asenb = asend;
            }
        } else {
            rfcs = rfcw = 1.0f;
            asevb = asevd;
            asenb = asend;
        }
        if (ialbflg == 0) {
            const float a1 = a.alvsf[c] * a.facsf[c], b1 = a.alvwf[c] * a.facwf[c];
            const float a2 = a.alnsf[c] * a.facsf[c], b2 = a.alnwf[c] * a.facwf[c];
            *A0 = (a2 * rfcs + b2 * rfcw) * flnd + asenb * fsea + asnnb * fsno;
            *A1 = (a2 + b2) * 0.96f * flnd + asend * fsea + asnnd * fsno;
            *A2 = (a1 * rfcs + b1 * rfcw) * flnd + asevb * fsea + asnvb * fsno;
            *A3 = (a1 + b1) * 0.96f * flnd + asevd * fsea + asnvd * fsno;
        } else {
            *A0 = a.alnsf[c] * rfcs * flnd + asenb * fsea + asnnb * fsno;
            *A1 = a.alnwf[c] * flnd + asend * fsea + asnnd * fsno;
            *A2 = a.alvsf[c] * rfcs * flnd + asevb * fsea + asnvb * fsno;
            *A3 = a.alvwf[c] * flnd + asevd * fsea + asnvd * fsno;
        }
    }
}

// ------------------------------------------------------------------------------------------ setemis
struct EmisIn {
    const float *glon, *glat, *sm, *sice, *si, *sncovr, *z0, *stdh, *tskin;
    const int* idxems;   // [180][360] surface type of the 1-degree map, row = latitude from 90N
};

// Surface emissivity [n] for the LW call: 1 everywhere (iemslw 0), else the open-water / sea-ice value or the
// land type's value from the 1-degree map (first map cell within half a degree, Fortran search order), blended
// with the snow emissivity by the snow cover.  The sea-land mask is 2 where SICE > 0.5, else 1 - SM.
inline void setemis(int n, const EmisIn& e, int ialbflg, int iemslw, float* sfcemis)
{
    const float emsref[8] = {0.97f, 0.95f, 0.94f, 0.90f, 0.93f, 0.96f, 0.96f, 0.99f};
    const float rad2dg = 57.29578f;
    const float dltg = 360.0f / 360.0f, hdlt = 0.5f * dltg;
    for (int c = 0; c < n; ++c) {
        if (iemslw == 0) {
            sfcemis[c] = 1.0f;
            continue;
        }
        const int msk = e.sice[c] > 0.5f ? 2 : (int)std::round(1.0f - e.sm[c]);
        float em;
        if (msk == 0) {
            em = emsref[0];
        } else if (msk == 2) {
            em = emsref[6];
        } else {
            float lon = e.glon[c] * rad2dg;
            if (lon < 0.0f) lon = lon + 360.0f;
            int i2 = 1;
            for (int i1 = 1; i1 <= 360; ++i1)
                if (std::fabs(lon - (dltg * (float)(i1 - 1) + hdlt)) <= hdlt) {
                    i2 = i1;
                    break;
                }
            const float lat = e.glat[c] * rad2dg;
            int j2 = 1;
            for (int j1 = 1; j1 <= 180; ++j1)
                if (std::fabs(lat - (90.0f - dltg * (float)(j1 - 1))) <= hdlt) {
                    j2 = j1;
                    break;
                }
            int id = std::max(2, e.idxems[(size_t)(j2 - 1) * 360 + (i2 - 1)]);
            if (id >= 7) id = 2;
            em = emsref[id - 1];
        }
        if (ialbflg == 1 && msk == 1) {
            const float f = e.sncovr[c];
            em = em * (1.0f - f) + emsref[7] * f;
        } else if (e.si[c] > 0.0f) {
            const float asnow = 0.02f * e.si[c];
            const float argh = std::fmin(0.50f, std::fmax(0.025f, 0.01f * (100.0f * e.z0[c])));
            const float hrgh = std::fmin(1.0f, std::fmax(0.20f, 1.0577f - 1.1538e-3f * e.stdh[c]));
            float f = asnow / (argh + asnow) * hrgh;
            if (msk == 0 && e.tskin[c] > 271.2f) f = 0.0f;
            em = em * (1.0f - f) + emsref[7] * f;
        }
        sfcemis[c] = em;
    }
}

// ------------------------------------------------------------------------------------------ progcld2
struct CldIn {
    const float *plyr, *plvl, *tlyr, *tvly, *qlyr, *qstl, *rhly, *clw, *f_ice, *f_rain, *cldfk1, *xlat;
};
struct CldCfg {
    int ivflip, llyr, iovr, lcrick, lcnorm, lnoprec, lsashal, cld_fraction;
};

// Cloud fraction from the power-law (p = 0.49) or fourth-root (2000 / ...) humidity forms.
inline float cld_form(float clw2, float pl, float qstl, float rhly, bool fourth_root)
{
    const float clwm = 0.0f / std::fmax(0.01f, pl * 0.001f);
    const float onemrh = std::fmax(1.0e-10f, 1.0f - rhly);
    float t;
    if (fourth_root) {
        t = std::fmin(std::fmax(std::sqrt(std::sqrt(onemrh * qstl)), 0.0001f), 1.0f);
        t = 2000.0f / t;
    } else {
        t = std::fmin(std::fmax(std::pow(onemrh * qstl, 0.49f), 0.0001f), 1.0f);
        t = 100.0f / t;
    }
    const float v = std::fmax(std::fmin(t * (clw2 - clwm), 50.0f), 0.0f);
    return std::fmax(std::sqrt(std::sqrt(rhly)) * (1.0f - std::exp(-v)), 0.0f);
}

// Ferrier's prognostic cloud properties of n columns on nlay layers: clouds [9][nlay][n] (fraction, liquid
// path, liquid radius, ice path, ice radius, rain path, rain radius, snow path 0, snow radius 0), and gethml's
// high / middle / low / total / boundary-layer cloud fractions clds [5][n] with the top and base layer of the
// high, middle and low decks mtop, mbot [3][n] (1-based layers).
inline void progcld2(int n, int nlay, const CldIn& in, const CldCfg& cfg, float* clouds, float* clds, int* mtop,
                     int* mbot)
{
    const float con_pi = 3.1415926535897931f, con_g = 9.80665f, con_rd = 287.05f, con_rv = 461.5f;
    const float fvirt = con_rv / con_rd - 1.0f, t0c = 273.15f, ttp = 273.16f;
    const float cclimit = 0.001f, cclimit2 = 0.05f, climit = 0.001f, ovcst = 1.0f - 1.0e-8f;
    const float recwat = 5.0f, recice = 10.0f, rerain = 100.0f;
    const float re50 = 1250.0f / 9.917f, re40 = 1250.0f / 9.337f, re30 = 1250.0f / 9.208f, re20 = 1250.0f / 9.387f;
    const float recw1 = 620.35f / std::pow(200.0f, 1.0f / 3.0f);
    const size_t N = (size_t)n, LN = (size_t)nlay * n;
    std::vector<float> ct(nlay);
    for (int c = 0; c < n; ++c) {
        auto at = [&](const float* f, int k) { return f[(size_t)k * N + c]; };
        float ptop1[4];
        {
            const float p1[4] = {1050.0f, 650.0f, 400.0f, 0.0f}, p2[4] = {1050.0f, 750.0f, 500.0f, 0.0f};
            const float w = std::fmax(0.0f, 4.0f * std::fabs(in.xlat[c]) / con_pi - 1.0f);
            for (int d = 0; d < 4; ++d) ptop1[d] = p1[d] + (p2[d] - p1[d]) * w;
        }
        for (int k = 0; k < nlay; ++k) {
            const float pl = at(in.plyr, k), plo = at(in.plvl, k), plp = at(in.plvl, k + 1);
            float clwf;
            if (cfg.lcrick) {
                if (k == 0)
                    clwf = 0.75f * at(in.clw, 0) + 0.25f * at(in.clw, 1);
                else if (k == nlay - 1)
                    clwf = 0.75f * at(in.clw, k) + 0.25f * at(in.clw, nlay - 2);
                else
                    clwf = 0.25f * at(in.clw, k - 1) + 0.5f * at(in.clw, k) + 0.25f * at(in.clw, k + 1);
            } else {
                clwf = at(in.clw, k);
            }
            const float fcice = std::fmax(0.0f, std::fmin(1.0f, at(in.f_ice, k)));
            const float frain = std::fmax(0.0f, std::fmin(1.0f, at(in.f_rain, k)));
            const float tk = at(in.tlyr, k);
            float qcice, qrain, qcwat, clw2;
            if (tk - t0c > -40.0f) {
                qcice = clwf * fcice;
                const float liq = clwf - qcice;
                qrain = liq * frain;
                qcwat = liq - qrain;
                clw2 = qcwat + qcice;
            } else {
                qcice = clwf;
                qrain = qcwat = 0.0f;
                clw2 = clwf;
            }
            float cwp = 0.0f, cip = 0.0f, crp = 0.0f, csp = 0.0f, rew = recwat, rei = recice, rer = rerain;
            if (qcwat + qcice + qrain > 1.0e-12f) {
                const float rho = 100.0f * pl / (con_rd * tk * (1.0f + fvirt * at(in.qlyr, k)));
                const float cpath = std::fabs(plp - plo) * (100000.0f / con_g);
                if (qcwat > 0.0f) {
                    rew = std::fmax(recwat, recw1 * std::pow(rho * qcwat, 1.0f / 3.0f));
                    cwp = cpath * qcwat;
                }
                if (qrain > 0.0f) {
                    rer = 1.5f * std::fmax(50.0f, std::fmin(1000.0f, 2511.54f * std::sqrt(std::sqrt(rho * qrain))));
                    crp = cpath * qrain;
                }
                cip = cpath * qcice;
            }
            const float dens = cfg.ivflip == 0 ? (con_g * pl) / (con_rd * (plp - plo)) : (con_g * pl) / (con_rd * (plo - plp));
            float f = 0.0f;
            if (cfg.cld_fraction == 0) {
                if (cfg.ivflip == 0 && !cfg.lsashal) {
                    if (clw2 > 1.0e-8f * (pl * 0.001f)) f = std::fmin(1.0f, 1.0e5f * clw2 * pl * 0.001f);
                } else if (clw2 > 2.0e-6f * (pl * 0.001f)) {
                    f = cld_form(clw2, pl, at(in.qstl, k), at(in.rhly, k), cfg.ivflip != 0 && !cfg.lsashal);
                }
            } else {
                f = at(in.cldfk1, k);
            }
            if (f < cclimit) {
                f = 0.0f;
                cwp = cip = crp = csp = 0.0f;
            }
            if (cfg.lnoprec) crp = csp = 0.0f;
            if (cfg.lcnorm && f >= cclimit) {
                const float r = 1.0f / std::fmax(cclimit2, f);
                cwp = cwp * r;
                cip = cip * r;
                crp = crp * r;
                csp = csp * r;
            }
            if (cip > 0.0f) {
                const float iwc = dens * cip / at(in.tvly, k);
                const float dt = tk - ttp;
                float re;
                if (dt < -50.0f)
                    re = re50 * std::pow(iwc, 0.109f);
                else if (dt < -40.0f)
                    re = re40 * std::pow(iwc, 0.08f);
                else if (dt < -30.0f)
                    re = re30 * std::pow(iwc, 0.055f);
                else
                    re = re20 * std::pow(iwc, 0.031f);
                rei = std::fmax(recice, re * 0.6495f);
            }
            ct[k] = f;
            const float v[9] = {f, cwp, rew, cip, rei, crp, rer, 0.0f, 0.0f};
            for (int q = 0; q < 9; ++q) clouds[q * LN + (size_t)k * N + c] = v[q];
        }
        // gethml: total and boundary-layer cloud, random (iovr 0) or maximum-random overlap
        auto CT = [&](int k1) { return std::fmin(ovcst, std::fmax(ct[k1 - 1], 0.0f)); };
        auto PL = [&](int k1) { return at(in.plyr, k1 - 1); };
        float cl[5] = {0, 0, 0, 0, 0};
        int mt[3] = {0, 0, 0}, mb[3] = {0, 0, 0};
        {
            float c1 = 1.0f, c2 = 1.0f;
            for (int kk = 0; kk < nlay; ++kk) {
                const int k = cfg.ivflip == 0 ? nlay - kk : kk + 1;
                const float cc = CT(k);
                if (cfg.iovr == 0) {
                    if (cc >= climit) c1 = c1 * (1.0f - cc);
                    if (k == cfg.llyr) cl[4] = 1.0f - c1;
                } else {
                    if (cc >= climit) {
                        c2 = std::fmin(c2, 1.0f - cc);
                    } else {
                        c1 = c1 * c2;
                        c2 = 1.0f;
                    }
                    if (k == cfg.llyr) cl[4] = 1.0f - c1 * c2;
                }
            }
            cl[3] = cfg.iovr == 0 ? 1.0f - c1 : 1.0f - c1 * c2;
        }
        // high / middle / low decks: walk from the surface up, merging contiguous cloudy layers into a deck
        // whose top and base are the cloud-weighted layer indices
        {
            const bool top_first = cfg.ivflip == 0;
            const int step = top_first ? -1 : 1;
            const int k0 = top_first ? nlay : 1, kend = top_first ? 0 : nlay + 1;
            float c1 = 0.0f, c2 = 0.0f;
            int kbt1 = k0, kbt2 = k0, kth1 = 0, kth2 = 0, idom = 1;
            mb[0] = mt[0] = k0;
            for (int k = k0; k != kend; k += step) {
                int id = idom, id1 = id + 1;
                const float pcur = PL(k), ccur = CT(k);
                const bool last = k + step == kend;
                const float pnxt = last ? -1.0f : PL(k + step);
                const float cnxt = last ? 0.0f : CT(k + step);
                if (pcur < ptop1[id1 - 1]) {
                    ++id;
                    ++id1;
                    idom = id;
                }
                if (ccur >= climit) {
                    if (kth2 == 0) kbt2 = k;
                    ++kth2;
                    c2 = cfg.iovr == 0 ? c2 + ccur - c2 * ccur : std::fmax(c2, ccur);
                    if (cnxt < climit || pnxt < ptop1[id1 - 1]) {
                        kbt1 = (int)std::round((c1 * (float)kbt1 + c2 * (float)kbt2) / (c1 + c2));
                        kth1 = (int)std::round((c1 * (float)kth1 + c2 * (float)kth2) / (c1 + c2));
                        c1 = c1 + c2 - c1 * c2;
                        kbt2 = k + step;
                        kth2 = 0;
                        c2 = 0.0f;
                    }
                }
                if (pnxt < ptop1[id1 - 1]) {
                    cl[id - 1] = c1;
                    mt[id - 1] = top_first ? std::min(kbt1, kbt1 - kth1 + 1) : std::max(kbt1, kbt1 + kth1 - 1);
                    mb[id - 1] = kbt1;
                    c1 = 0.0f;
                    kbt1 = k + step;
                    kth1 = 0;
                    if (id1 <= 3) {
                        mb[id1 - 1] = kbt1;
                        mt[id1 - 1] = kbt1;
                    }
                }
            }
        }
        for (int q = 0; q < 5; ++q) clds[q * N + c] = cl[q];
        for (int q = 0; q < 3; ++q) {
            mtop[q * N + c] = mt[q];
            mbot[q * N + c] = mb[q];
        }
    }
}

// ------------------------------------------------------------------------------------------ clw
// Total condensate of each layer: the ncld cloud tracers from index ntcw0 (0-based) summed in tracer order, values
// below epsq set to zero.  tracer [ntrac][lmk][n], clw [lmk][n].
inline void grrad_clw(int n, int lmk, const float* tracer, int ntcw0, int ncld, float epsq, float* clw)
{
    const size_t plane = (size_t)lmk * n;
    for (size_t p = 0; p < plane; ++p) {
        float sum = 0.0f;
        for (int j = 0; j < ncld; ++j) sum += tracer[(size_t)(ntcw0 + j) * plane + p];
        clw[p] = sum < epsq ? 0.0f : sum;
    }
}

// ------------------------------------------------------------------------------------------ IALB = 2 albedo
// The albedo tables: trn [21], za [20] (degrees, decreasing), dza [19], albd [20][21] ([zenith row][trn column]).
struct PayneTab {
    const float *trn, *za, *dza, *albd;
};

// Surface albedo of one point: salbedo unless the sun is up over land-mask value sm > 0.5, where the table value at
// the zenith angle and the fixed transmissivity 0.537 (column 11 of the table and its right neighbour) replaces it.
inline float payne_albedo(float salbedo, float sm, float cz, const PayneTab& t)
{
    const float trans = 0.537f;
    const int iq = (int)(20.0f * trans + 1.0f);                      // transmissivity column (1-based)
    if (!(cz > 0.0f && sm > 0.5f)) return salbedo;
    const float deg = 180.0f / 3.14159265f;
    const float zen = deg * std::acos(std::max(cz, 0.0f));
    // zenith row: 2-degree rows above 74 degrees, 4-degree rows from 50, 10-degree rows below (1-based)
    int jx;
    if (zen >= 74.0f) jx = (int)(0.5f * (90.0f - zen) + 1.0f);
    else if (zen >= 50.0f) jx = (int)(0.25f * (74.0f - zen) + 9.0f);
    else jx = (int)(0.1f * (50.0f - zen) + 15.0f);
    jx = std::max(1, std::min(jx, 19));   // rows 1..19 (a coszen above 1 gives a NaN zenith; the CUDA path clamps)
    const float w = -(zen - t.za[jx - 1]) / t.dza[jx - 1];
    auto A = [&](int row, int col) { return t.albd[(row - 1) * 21 + (col - 1)]; };   // 1-based row, column
    const float a1 = A(jx, iq) + w * (A(jx + 1, iq) - A(jx, iq));
    const float a2 = A(jx, iq + 1) + w * (A(jx + 1, iq + 1) - A(jx, iq + 1));
    return a1 + 20.0f * (a2 - a1) * (trans - t.trn[iq - 1]);
}

}  // namespace front
}  // namespace orc
