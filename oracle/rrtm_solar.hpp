// rrtm_solar.hpp -- CPU oracle: the solar geometry of a radiation call (test infrastructure only).
//
// Restates, in the reference's float arithmetic:
//   sol_update_nmmb + solar  namgpu/kernels/phys_rrtm_sol_update.cu:60-210 (radiation_astronomy_nmmb.f:265-739)
//   coszmn_nmmb              namgpu/kernels/phys_rrtm_coszmn.cu:60-114 (radiation_astronomy_nmmb.f:744-848)
// Never linked into the product.
#pragma once
#include <algorithm>
#include <cmath>

namespace orc {
namespace solar {

inline int iw3jdn(int y, int m, int d)
{
    return d - 32075 + 1461 * (y + 4800 + (m - 14) / 12) / 4 + 367 * (m - 2 - (m - 14) / 12 * 12) / 12 -
           3 * ((y + 4900 + (m - 14) / 12) / 100) / 4;
}

// out: sollag, sindec, cosdec, anginc, solcon, nstp
inline void update(int yr, int mon, int day, int hr, int mn, int sec, float deltsw, float deltim, double solc0d,
                   float* out, int* nstp_out)
{
    const float PI = 3.1415926535897931f, TPI = 2.0f * PI, DEGRAD = 180.0f / PI;
    const int JDOR = 2415020;
    const float solc0 = (float)solc0d;
    int jd1 = iw3jdn(yr, mon, day);
    float fjd1;
    if (hr < 12) {
        jd1 = jd1 - 1;
        fjd1 = 0.5f + (float)hr * (1.0f / 24.0f) + (float)mn * (1.0f / 1440.0f) + (float)sec * (1.0f / 86400.0f);
    } else {
        fjd1 = (float)(hr - 12) * (1.0f / 24.0f) + (float)mn * (1.0f / 1440.0f) + (float)sec * (1.0f / 86400.0f);
    }
    fjd1 = fjd1 + (float)jd1;
    const int jd = (int)fjd1;
    const float fjd = fjd1 - (float)jd;
    // solar
    const float t1 = (float)(jd - JDOR) / 36525.0f;
    float year = 0.25964134f + 0.304e-5f * t1;
    const float tyear = 0.24219879f - 0.614e-5f * t1;
    const float ec = 0.01675104f - (0.418e-4f + 0.126e-6f * t1) * t1;
    const float angin = 23.452294f - (0.0130125f + 0.164e-5f * t1) * t1;
    const float ador = (float)JDOR;
    const int jdoe = (int)(ador + (78.035f * 365.25f) / (year - tyear));
    const float deleqn = (float)(jdoe - jd) * (year - tyear) / 365.25f;
    year = year + 365.0f;
    const float sni = std::sin(angin / DEGRAD);
    const float tini = 1.0f / std::tan(angin / DEGRAD);
    const float er = std::sqrt((1.0f + ec) / (1.0f - ec));
    const float qq = deleqn * TPI / year;
    float e1 = 1.0f, cd = 1.0f, ep;
    int iter = 0;
    while (cd > 1.3e-6f) {
        ep = e1 - (e1 - ec * std::sin(e1) - qq) / (1.0f - ec * std::cos(e1));
        cd = std::fabs(e1 - ep);
        e1 = ep;
        iter = iter + 1;
        if (iter > 10) break;
    }
    const float eq = 2.0f * std::atan(er * std::tan(0.5f * e1));
    const float dat = (float)(jd - JDOR) - 1.55f + fjd;
    const float date = std::fmod(dat, year);
    const float em = TPI * date / year;
    e1 = 1.0f;
    float cr = 1.0f;
    iter = 0;
    while (cr > 1.3e-6f) {
        ep = e1 - (e1 - ec * std::sin(e1) - em) / (1.0f - ec * std::cos(e1));
        cr = std::fabs(e1 - ep);
        e1 = ep;
        iter = iter + 1;
        if (iter > 10) break;
    }
    const float w1 = 2.0f * std::atan(er * std::tan(0.5f * e1));
    const float r1 = 1.0f - ec * std::cos(e1);
    const float sindec = sni * std::sin(w1 - eq);
    const float cosdec = std::sqrt(1.0f - sindec * sindec);
    const float dlt = std::asin(sindec);
    float alp = std::asin(std::tan(dlt) * tini);
    const float tst = std::cos(w1 - eq);
    if (tst < 0.0f) alp = PI - alp;
    if (alp < 0.0f) alp = alp + TPI;
    float sun = TPI * (date - deleqn) / year;
    if (sun < 0.0f) sun = sun + TPI;
    const float sollag = sun - alp - 0.03255f;
    const float solcon = solc0 / (r1 * r1);
    const int nswr = (int)std::lround(deltsw / deltim);
    const float dtswh = deltsw / 3600.0f;
    int nstp;
    if (deltsw >= 3600.0f) {
        int nn = (int)std::lround(3600.0f / deltim);
        nn = std::max(6, std::min(12, nn));
        nstp = (int)std::lround(dtswh) * nn + 1;
    } else {
        nstp = std::max(2, std::min(20, nswr)) + 1;
    }
    const float pid12 = (2.0f * std::asin(1.0f)) / 12.0f;
    out[0] = sollag; out[1] = sindec; out[2] = cosdec; out[3] = pid12 * dtswh / (float)(nstp - 1); out[4] = solcon;
    *nstp_out = nstp;
}

inline void coszmn(float xl, float lat, float sollag, float sindec, float cosdec, float solhr, float dtswav, int nrads,
                   float& coszen, float& coszdg)
{
    const float pid12 = (2.0f * std::asin(1.0f)) / 12.0f;
    const float solang = pid12 * (solhr - 12.0f);
    const float rnstp = dtswav / (float)nrads;
    const float sinlat = std::sin(lat), coslat = std::cos(lat);
    float sum = 0.0f;
    int istsun = 0;
    for (int it = 1; it <= nrads; ++it) {
        const float cns = solang + (float)(it - 1) * pid12 * rnstp + sollag;
        const float ss = sinlat * sindec, cc = coslat * cosdec;
        const float cz = ss + cc * std::cos(cns + xl);
        sum += std::max(0.0f, cz);
        if (cz > 1.0e-4f) istsun += 1;
    }
    coszdg = sum * rnstp;
    coszen = istsun > 0 ? sum / (float)istsun : sum;
}

}  // namespace solar
}  // namespace orc
