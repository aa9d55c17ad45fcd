// rad_solar.cuh -- the radiation call's solar geometry: sol_update (host, once per call) and coszmn (device,
// per column).
//
//   rad_sol_update  the sun's declination (sin / cos), the equation of time and the sun-earth-distance-
//                   adjusted solar constant at the forecast time, and the zenith-angle sampling of the SW
//                   interval (sol_update_nmmb and solar of the NMMB astronomy module,
//                   namgpu/kernels/phys_rrtm_sol_update.cu:60-210) -- a handful of scalars, in float as the
//                   single-precision NAM build computes them, on the host.
//   k_coszmn        the cosine of the solar zenith angle sampled nrads times over the SW interval at each
//                   column: its daytime mean (SW_COSZEN / COSZEN_V, the SW's day predicate and input) and its
//                   mean over the whole interval (COSZDG_V) (coszmn_nmmb,
//                   namgpu/kernels/phys_rrtm_coszmn.cu:60-114).  One thread per column; HBM-bound (2 input,
//                   2 output words per column).
#pragma once

namespace rad {

namespace solh {

inline int julian_day_number(int y, int m, int d)   // Gregorian calendar date -> Julian day number
{
    return d - 32075 + 1461 * (y + 4800 + (m - 14) / 12) / 4 + 367 * (m - 2 - (m - 14) / 12 * 12) / 12 -
           3 * ((y + 4900 + (m - 14) / 12) / 100) / 4;
}

// The sun at Julian day jd + fjd (solar, radiation_astronomy_nmmb.f:575-739): sun-earth distance r1 in
// astronomical units, sin / cos of the declination, the equation of time sollag.
inline void sun(int jd, float fjd, float& r1, float& sindec, float& cosdec, float& sollag)
{
    const float pi = 3.1415926535897931f, tpi = 2.0f * pi, degrad = 180.0f / pi;
    const int jd0 = 2415020;                     // epoch: January 0, 1900, 12 h UT
    const float t1 = (float)(jd - jd0) / 36525.0f;                      // Julian centuries since the epoch
    float year = 0.25964134f + 0.304e-5f * t1;                          // anomalistic year - 365 days
    const float tyear = 0.24219879f - 0.614e-5f * t1;                   // tropical year - 365 days
    const float ec = 0.01675104f - (0.418e-4f + 0.126e-6f * t1) * t1;   // orbit eccentricity
    const float angin = 23.452294f - (0.0130125f + 0.164e-5f * t1) * t1;   // obliquity, degrees
    const int jdoe = (int)((float)jd0 + (78.035f * 365.25f) / (year - tyear));
    const float deleqn = (float)(jdoe - jd) * (year - tyear) / 365.25f;
    year = year + 365.0f;
    const float sni = std::sin(angin / degrad), tini = 1.0f / std::tan(angin / degrad);
    const float er = std::sqrt((1.0f + ec) / (1.0f - ec));
    const float qq = deleqn * tpi / year;
    auto kepler = [&](float m) {                 // eccentric anomaly by Newton's method, at most 11 steps
        float e = 1.0f, d = 1.0f;
        for (int it = 0; d > 1.3e-6f; ) {
            const float ep = e - (e - ec * std::sin(e) - m) / (1.0f - ec * std::cos(e));
            d = std::fabs(e - ep);
            e = ep;
            if (++it > 10) break;
        }
        return e;
    };
    const float eq = 2.0f * std::atan(er * std::tan(0.5f * kepler(qq)));   // true anomaly at the equinox
    const float dat = (float)(jd - jd0) - 1.55f + fjd;                     // days since perihelion ...
    const float date = std::fmod(dat, year);
    const float e1 = kepler(tpi * date / year);
    const float w1 = 2.0f * std::atan(er * std::tan(0.5f * e1));
    r1 = 1.0f - ec * std::cos(e1);
    sindec = sni * std::sin(w1 - eq);
    cosdec = std::sqrt(1.0f - sindec * sindec);
    const float dlt = std::asin(sindec);
    float alp = std::asin(std::tan(dlt) * tini);                           // right ascension
    if (std::cos(w1 - eq) < 0.0f) alp = pi - alp;
    if (alp < 0.0f) alp = alp + tpi;
    float s = tpi * (date - deleqn) / year;
    if (s < 0.0f) s = s + tpi;
    sollag = s - alp - 0.03255f;
}

inline void update(const RadSolarIn& in, RadSolarState& st)
{
    int jd1 = julian_day_number(in.year, in.month, in.day);
    float fjd1;
    if (in.hour < 12) {                          // the Julian day starts at noon
        jd1 = jd1 - 1;
        fjd1 = 0.5f + (float)in.hour * (1.0f / 24.0f) + (float)in.minute * (1.0f / 1440.0f) +
               (float)in.second * (1.0f / 86400.0f);
    } else {
        fjd1 = (float)(in.hour - 12) * (1.0f / 24.0f) + (float)in.minute * (1.0f / 1440.0f) +
               (float)in.second * (1.0f / 86400.0f);
    }
    fjd1 = fjd1 + (float)jd1;
    const int jd = (int)fjd1;
    const float fjd = fjd1 - (float)jd;
    float r1;
    sun(jd, fjd, r1, st.sindec, st.cosdec, st.sollag);
    st.solcon = (float)in.solc0 / (r1 * r1);
    const int nswr = (int)std::lround(in.deltsw / in.deltim);   // model steps per SW call
    const float dtswh = in.deltsw / 3600.0f;
    if (in.deltsw >= 3600.0f) {
        const int nn = std::max(6, std::min(12, (int)std::lround(3600.0f / in.deltim)));   // samples per hour
        st.nstp = (int)std::lround(dtswh) * nn + 1;
    } else {
        st.nstp = std::max(2, std::min(20, nswr)) + 1;
    }
    const float pid12 = (2.0f * std::asin(1.0f)) / 12.0f;
    st.anginc = pid12 * dtswh / (float)(st.nstp - 1);
}

}  // namespace solh

struct CoszArgs {
    const float *glon, *glat;
    float *coszen, *coszdg;
    int64_t n;
    float sollag, sindec, cosdec, solhr, dtswav;
    int nrads;
};

__global__ void __launch_bounds__(256) k_coszmn(const __grid_constant__ CoszArgs a)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const float pid12 = (2.0f * asinf(1.0f)) / 12.0f;
    const float solang = pid12 * (a.solhr - 12.0f);          // hour angle of the present time
    const float rnstp = a.dtswav / (float)a.nrads;
    const float xl = __ldg(a.glon + i), lat = __ldg(a.glat + i);
    const float ss = sinf(lat) * a.sindec, cc = cosf(lat) * a.cosdec;
    float sum = 0.0f;
    int lit = 0;
    for (int it = 1; it <= a.nrads; ++it) {
        const float h = solang + (float)(it - 1) * pid12 * rnstp + a.sollag;
        const float cz = ss + cc * cosf(h + xl);
        sum += fmaxf(0.0f, cz);
        if (cz > 1.0e-4f) ++lit;
    }
    a.coszdg[i] = sum * rnstp;
    a.coszen[i] = lit > 0 ? sum / (float)lit : sum;
}

}  // namespace rad
