// rad_rdtemp.cuh -- RDTEMP on the device: the radiative temperature change applied every model step, with
// the shortwave tendency rescaled by the current solar zenith angle between radiation calls.
//
// Restates rdtemp_apply of namgpu/kernels/drv_rdtemp.cu:140-198 (module_RA_GFDL.F90:116-233 with ZENITH,
// :1662-1805, and CAL_MON_DAY, :7823-7856, inlined): per column on the tile ITS..ITE x JTS..JTE
//   CZEN = max(0, sin(dec) sin(lat) + cos(dec) cos(hrang + lon + 2 pi) cos(lat))
//   FACTR = CZEN / CZMEAN (0 where CZMEAN <= 0)
// and on the interior ITS_B1..ITE_B1 x JTS_B1..JTE_B1, every level: T += (RSWTT FACTR + RLWTT) DT.
// The solar declination and hour angle depend only on the step time and the calendar: one thread of each
// CTA evaluates them (float, the reference's statement order) into shared memory for the CTA's columns.
// Layout: [level][j][i], the column fastest; one thread per column, coalesced level rows.  HBM-bound
// (3 LM + 4 words per column).
#pragma once

namespace rad {

struct RdtempArgs {
    int ntsd;                    // step counter (NTSD)
    float dt;                    // model step, s
    int julday, julyr, ihrst, leap_seen;
    const float *glat, *glon;    // [jm][im], radians
    const float* czmean;         // [jm][im]
    const float *rswtt, *rlwtt;  // [lm][jm][im], K/s
    float* czen;                 // [jm][im], written on the tile
    float* t;                    // [lm][jm][im], updated on the interior
    int im, jm, lm;
    int its, ite, jts, jte;      // tile, 1-based inclusive (the loop-limit table's ITS..JTE)
    int its_b1, ite_b1, jts_b1, jte_b1;   // interior, 1-based inclusive
};

// Days per month; February has 29 in a leap year or once a leap year has been seen (CAL_MON_DAY keeps it).
__device__ __forceinline__ int rd_mdays(int m, int year, int leap_seen)
{
    const int d[12] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
    return (m == 1 && (year % 4 == 0 || leap_seen)) ? 29 : d[m];
}

// The call's solar declination and hour angle (ZENITH, module_RA_GFDL.F90:1700-1770), in float.
__device__ void rd_sun(const RdtempArgs& p, float& dec, float& hrang)
{
    const float pi = 3.1415926f, twopi = 2.0f * pi, d2r = 3.1415926f / 180.0f;
    // day of year -> month and day (CAL_MON_DAY)
    int mon = 12, mday = p.julday, left = p.julday;
    for (int m = 0; m < 12; ++m) {
        const int nd = rd_mdays(m, p.julyr, p.leap_seen);
        if (left > nd) {
            left -= nd;
        } else {
            mday = left;
            mon = m + 1;
            break;
        }
    }
    const float times = (float)p.ntsd * p.dt;
    float day = 0.0f;
    for (int m = 0; m < mon - 1; ++m) day = day + (float)rd_mdays(m, p.julyr, p.leap_seen);
    day = day + (float)(mday - 1) + ((float)p.ihrst + times / 3600.0f) / 24.0f;
    const float dayi = (float)((int)day + 1);
    const float hour = (day - dayi + 1.0f) * 24.0f;
    const float yfctr = 2000.0f - (float)p.julyr;
    const int dy = p.julyr - 2000;
    const float addday = dy < 0 ? (float)(dy / 4) : (float)((dy + 3) / 4);
    const float startyr = 2451545.0f + (float)dy * 365.0f + addday - 0.5f;
    const float difjd = startyr + day - 2451545.0f;
    const float slonm = (280.460f + 0.9856474f * difjd) * d2r + yfctr * twopi;
    const float anom = (357.528f + 0.9856003f * difjd) * d2r;
    float slon = slonm + (1.915f * sinf(anom) + 0.020f * sinf(2.0f * anom)) * d2r;
    if (slon > twopi) slon = slon - twopi;
    dec = asinf(sinf(slon) * sinf(23.440f * d2r));
    float ra = acosf(cosf(slon) / cosf(dec));
    if (slon > pi) ra = twopi - ra;
    const float tu = (startyr + dayi - 1.0f - 2451545.0f) / 36525.0f;
    const float stim0 = 24110.54841f + tu * (8640184.812866f + 9.3104E-2f * tu + -6.2E-6f * tu * tu);
    float sidtim = (stim0 / 3600.0f + yfctr * 24.0f + 1.00273791f * hour) * 15.0f * d2r;
    if (sidtim < 0.0f) sidtim = sidtim + twopi;
    if (sidtim > twopi) sidtim = sidtim - twopi;
    hrang = sidtim - ra;
}

__global__ void __launch_bounds__(256) k_rdtemp(const __grid_constant__ RdtempArgs p)
{
    __shared__ float sun[2];
    if (threadIdx.x == 0) rd_sun(p, sun[0], sun[1]);
    __syncthreads();
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = (int64_t)p.im * p.jm;
    if (c >= n) return;
    const int i = (int)(c % p.im), j = (int)(c / p.im);
    if (i < p.its - 1 || i > p.ite - 1 || j < p.jts - 1 || j > p.jte - 1) return;
    const float dec = sun[0], hrang = sun[1];
    const float lat = p.glat[c];
    float sinalt = sinf(dec) * sinf(lat) + cosf(dec) * cosf(hrang + p.glon[c] + 2.0f * 3.1415926f) * cosf(lat);
    if (sinalt < 0.0f) sinalt = 0.0f;
    p.czen[c] = sinalt;
    const float cm = p.czmean[c];
    const float factr = cm > 0.0f ? sinalt / cm : 0.0f;
    if (i < p.its_b1 - 1 || i > p.ite_b1 - 1 || j < p.jts_b1 - 1 || j > p.jte_b1 - 1) return;
    for (int l = 0; l < p.lm; ++l) {
        const size_t q = (size_t)l * n + c;
        p.t[q] = p.t[q] + (__ldg(p.rswtt + q) * factr + __ldg(p.rlwtt + q)) * p.dt;
    }
}

}  // namespace rad
