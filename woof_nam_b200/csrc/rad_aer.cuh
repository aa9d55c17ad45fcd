// rad_aer.cuh -- climatological aerosol optics of the NAM radiation (iaer = 11) for sm_100a.
//
// Host, once per month (rad_load_aerosols): the band tables from the packed OPAC climatology --
//   set_spectrum      solar flux per wavenumber (151 intervals), black-body IR flux at 273.15 K
//                     (namgpu/kernels/phys_rrtm_aer_init.cu:145-173)
//   set_aercoef       the flux of each of the 61 OPAC bands inside each SW / LW band
//                     (namgpu/kernels/phys_rrtm_clim_aerinit.cu:61-160)
//   optavg            flux-weighted extinction, scattering, asymmetry of each species per band, and the
//                     single-scattering albedo that keeps the weighted two-stream reflectance
//                     (phys_rrtm_clim_aerinit.cu:165-284)
//   trop_update fill  the month's 5-degree cells, component fractions closed to one in double
//                     (namgpu/kernels/phys_rrtm_aer_update.cu:40-63)
// Device, every radiation step (rad_setaer -> k_setaer): per column, setaer's prep (longitude / latitude in
// degrees, layer thickness dz and height hz from the hypsometric equation; phys_rrtm_setaer.cu:80-150,
// ivflip 0) and aer_property (namgpu/kernels/phys_rrtm_aer_property.cu:117-434): the cell bracket and profile
// choice, bilinear densities and mixing ratios, each layer's domain and effective thickness, the humidity
// interpolation, the optics of the five domains in the 30 bands, and the smoothing of optical depth across
// domain boundaries.
//
// k_setaer: a CTA takes 32 columns, one per lane, and 8 warps.  Warp 0 maps the climatology onto its
// columns and walks each column up from the surface for the level heights and layer domains (the parts
// that build up layer by layer); then all warps, layers side by side, form each layer's effective thickness
// and humidity bracket into shared memory ([layer][column]); then warp w runs bands w, w + 8, ... down the
// layers, the smoothing (which couples a band's adjacent layers) carried in a register and each optical
// depth stored once the layer below has settled it.  Every store is a 128-byte row of 32 columns.  The
// reference runs one thread per column through 61 layers x 30 bands; splitting the bands over warps cuts
// each thread's dependent chain eightfold.  The output (22 KB per column of 61 layers) bounds it at HBM.
#pragma once

namespace rad {

constexpr int AER_NAERBND = 61, AER_NRHLEV = 8, AER_NCM1 = 6, AER_NCM2 = 4, AER_NCM = 10, AER_NDM = 5, AER_NAE = 7;
constexpr int AER_IMXAE = 72, AER_JMXAE = 37, AER_NXC = 5, AER_NSW = 14, AER_NLW = 16, AER_NBT = 30;
constexpr int AER_COLS = 32, AER_WARPS = 8, AER_THREADS = AER_COLS * AER_WARPS;   // k_setaer CTA
constexpr int AER_NCELL = AER_IMXAE * AER_JMXAE;

// Device tables (one float blob and one int blob of the handle).
struct AerTab {
    const float *haer, *prsref, *sigref;                      // [NAE][NDM]
    const float *extrhi, *scarhi, *ssarhi, *asyrhi;           // [NBT][NCM1]
    const float *extrhd, *scarhd, *ssarhd, *asyrhd;           // [NBT][NCM2][NRHLEV]
    const float *extstra;                                     // [NBT]
    const float *cmixg, *denng;                               // [JMXAE][IMXAE][NXC], [..][2]
    const int *idxcg, *kprfg;                                 // [JMXAE][IMXAE][NXC], [JMXAE][IMXAE]
};
// float blob offsets
constexpr int AF_HAER = 0, AF_PRSREF = 35, AF_SIGREF = 70, AF_EXTRHI = 105, AF_SCARHI = AF_EXTRHI + 180,
              AF_SSARHI = AF_SCARHI + 180, AF_ASYRHI = AF_SSARHI + 180, AF_EXTRHD = AF_ASYRHI + 180,
              AF_SCARHD = AF_EXTRHD + 960, AF_SSARHD = AF_SCARHD + 960, AF_ASYRHD = AF_SSARHD + 960,
              AF_EXTSTRA = AF_ASYRHD + 960, AF_CMIXG = AF_EXTSTRA + 30, AF_DENNG = AF_CMIXG + AER_NCELL * AER_NXC,
              AF_TOTAL = AF_DENNG + AER_NCELL * 2;
constexpr int AI_IDXCG = 0, AI_KPRFG = AER_NCELL * AER_NXC, AI_TOTAL = AI_KPRFG + AER_NCELL;

__constant__ float c_aer_rhlev[AER_NRHLEV] = {0.0f, 0.5f, 0.7f, 0.8f, 0.9f, 0.95f, 0.98f, 0.99f};

// ------------------------------------------------------------------------------------------------------ host
namespace aerh {

// Band limits in cm-1 (radsw_param_nmmb.f wvnum1 / wvnum2, radlw_param_nmmb.f wvnlw1 / wvnlw2).
static const int WSW[2][AER_NSW] = {{2600, 3251, 4001, 4651, 5151, 6151, 7701, 8051, 12851, 16001, 22651, 29001, 38001, 820},
                                    {3250, 4000, 4650, 5150, 6150, 7700, 8050, 12850, 16000, 22650, 29000, 38000, 50000, 2600}};
static const int WLW[2][AER_NLW] = {{10, 251, 501, 631, 701, 821, 981, 1081, 1181, 1391, 1481, 1801, 2081, 2251, 2381, 2601},
                                    {250, 500, 630, 700, 820, 980, 1080, 1180, 1390, 1480, 1800, 2080, 2250, 2380, 2600, 3000}};

// Flux of every OPAC band inside [iw1, iw2] (f = flux per wavenumber, 1-based wavenumber index); the OPAC
// bands it touches are lo..hi (1-based); returns the band total.
inline float band_weights(const int32_t* iendwv, const std::vector<float>& f, int iw1, int iw2, float* w, int& lo,
                          int& hi)
{
    for (int i = 0; i < AER_NAERBND; ++i) w[i] = 0.0f;
    int b = 1;
    while (b != AER_NAERBND && iw1 > iendwv[b - 1]) ++b;
    lo = b;
    float total = 0.0f, run = 0.0f;
    for (int iw = iw1; iw <= iw2; ++iw) {
        total = total + f[iw - 1];
        run = run + f[iw - 1];
        if (iw == iendwv[b - 1]) {
            w[b - 1] = run;
            if (b < AER_NAERBND) { run = 0.0f; ++b; }
        }
    }
    if (iw2 != iendwv[b - 1]) w[b - 1] = run;
    hi = b;
    return total;
}

// Band average of one species (ext, sca, ssa, asy over the 61 OPAC bands).
inline void band_average(const float* ext, const float* sca, const float* ssa, const float* asy, const float* w,
                         int lo, int hi, float rnorm, float* out4)
{
    float se = 0, ss = 0, swe = 0, sweg = 0, sr = 0;
    for (int i = lo; i <= hi; ++i) {
        const float wt = w[i - 1], a = ssa[i - 1], g = asy[i - 1], e = ext[i - 1];
        const float sp = std::sqrt((1.0f - a) / (1.0f - a * g));       // two-stream reflectance of the species
        sr = sr + ((1.0f - sp) / (1.0f + sp)) * wt;
        se = se + e * wt;
        ss = ss + sca[i - 1] * wt;
        swe = swe + a * wt * e;
        sweg = sweg + a * wt * e * g;
    }
    const float r = sr * rnorm, gb = sweg / (swe + 1.0e-10f);
    out4[0] = se * rnorm;
    out4[1] = ss * rnorm;
    out4[2] = 4.0f * r / ((1.0f + r) * (1.0f + r) - gb * ((1.0f - r) * (1.0f - r)));   // albedo of reflectance r
    out4[3] = gb;
}

// All band tables of one month into the float / int blobs (AF_* / AI_* offsets).
inline void build(const RadAerClim& c, std::vector<float>& fb, std::vector<int>& ib)
{
    fb.assign(AF_TOTAL, 0.0f);
    ib.assign(AI_TOTAL, 0);
    // solar flux per wavenumber: each of the 151 intervals holds its constant; IR: Planck at 273.15 K
    std::vector<float> sol, eir(4000);
    for (int b = 0; b < 151; ++b) sol.insert(sol.end(), (size_t)c.nwvns0[b], c.s0intv[b]);
    const float pi = 3.1415926535897931f, cl = 2.99792458e+8f, h = 6.6260693e-34f, kb = 1.3806505e-23f, t0 = 2.7315e+2f;
    const float c1 = 2.0f * pi * h * (cl * cl), c2 = h * cl / (kb * t0);
    for (int nw = 1; nw <= 4000; ++nw) {
        const float x = 100.0f * (float)nw;
        eir[nw - 1] = (c1 * (x * x * x)) / (std::exp(c2 * x) - 1.0f);
    }
    for (int i = 0; i < 35; ++i) {
        fb[AF_HAER + i] = c.haer[i];
        fb[AF_PRSREF + i] = c.prsref[i];
        fb[AF_SIGREF + i] = 0.001f * c.prsref[i];
    }
    const size_t R1 = (size_t)AER_NCM1 * AER_NAERBND, R2 = (size_t)AER_NCM2 * AER_NRHLEV * AER_NAERBND;
    for (int b = 0; b < AER_NBT; ++b) {
        float w[AER_NAERBND];
        int lo, hi;
        const bool sw = b < AER_NSW;
        const float total = sw ? band_weights(c.iendwv, sol, WSW[0][b], WSW[1][b], w, lo, hi)
                               : band_weights(c.iendwv, eir, WLW[0][b - AER_NSW], WLW[1][b - AER_NSW], w, lo, hi);
        const float rnorm = 1.0f / total;
        for (int s = 0; s < AER_NCM1; ++s) {
            const size_t o = (size_t)s * AER_NAERBND;
            float v[4];
            band_average(c.rhid + o, c.rhid + R1 + o, c.rhid + 2 * R1 + o, c.rhid + 3 * R1 + o, w, lo, hi, rnorm, v);
            const int q = b * AER_NCM1 + s;
            fb[AF_EXTRHI + q] = v[0]; fb[AF_SCARHI + q] = v[1]; fb[AF_SSARHI + q] = v[2]; fb[AF_ASYRHI + q] = v[3];
        }
        for (int s = 0; s < AER_NCM2; ++s)
            for (int r = 0; r < AER_NRHLEV; ++r) {
                const size_t o = ((size_t)s * AER_NRHLEV + r) * AER_NAERBND;
                float v[4];
                band_average(c.rhdp + o, c.rhdp + R2 + o, c.rhdp + 2 * R2 + o, c.rhdp + 3 * R2 + o, w, lo, hi, rnorm, v);
                const int q = (b * AER_NCM2 + s) * AER_NRHLEV + r;
                fb[AF_EXTRHD + q] = v[0]; fb[AF_SCARHD + q] = v[1]; fb[AF_SSARHD + q] = v[2]; fb[AF_ASYRHD + q] = v[3];
            }
        float se = 0;
        for (int i = lo; i <= hi; ++i) se = se + c.straext0[i - 1] * w[i - 1];
        fb[AF_EXTSTRA + b] = se * rnorm;
    }
    for (int cell = 0; cell < AER_NCELL; ++cell) {
        const int kp = c.month_kprf[cell];
        ib[AI_KPRFG + cell] = kp;
        double rest = 1.0;
        for (int m = 0; m < AER_NXC; ++m) ib[AI_IDXCG + cell * AER_NXC + m] = c.month_idx[cell * AER_NXC + m];
        for (int m = 0; m < AER_NXC - 1; ++m) {
            fb[AF_CMIXG + cell * AER_NXC + m] = (float)c.month_cmix[cell * AER_NXC + m];
            rest = rest - c.month_cmix[cell * AER_NXC + m];
        }
        fb[AF_CMIXG + cell * AER_NXC + AER_NXC - 1] = (float)rest;     // the fractions close to one
        fb[AF_DENNG + 2 * cell] = (float)c.month_denn[cell];
        fb[AF_DENNG + 2 * cell + 1] = kp >= 6 ? (float)c.month_cmix[cell * AER_NXC + AER_NXC - 1] : 0.0f;
    }
}

}  // namespace aerh

// ------------------------------------------------------------------------------------------------------ device
struct AerArgs {
    const float *plvl, *plyr, *tlyr, *qlyr, *rhly, *xlon, *xlat, *slmsk;
    float *faersw, *faerlw;
    int64_t n;
    int nlay;
};

__global__ void __launch_bounds__(AER_THREADS, 2) k_setaer(const __grid_constant__ AerArgs a, const __grid_constant__ AerTab t)
{
    __shared__ float s_hz[NLAY_MAX + 1][AER_COLS];        // level heights, level 0 = model top
    __shared__ float s_delz[NLAY_MAX][AER_COLS];          // layer thickness, then effective thickness
    __shared__ float s_fr[NLAY_MAX][AER_COLS];            // sigma of the layer top, then humidity weight
    __shared__ int s_code[NLAY_MAX][AER_COLS];            // domain | low humidity level << 4 | high << 8
    __shared__ float s_cmix[AER_NCM + 1][AER_COLS];       // the column's component mixing ratios
    __shared__ float s_col[4][AER_COLS];                  // denn[1], denn[2], h1, profile structure
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t col = (int64_t)blockIdx.x * AER_COLS + lane;
    const bool live = col < a.n;
    const int nlay = a.nlay;
    const int64_t N = a.n;
    const int64_t c = live ? col : a.n - 1;           // idle lanes of the last CTA mirror a real column
    auto L = [&](const float* p, int k) { return __ldg(p + (size_t)k * N + c); };   // [level][col], 0-based
    auto HA = [&](int d, int kp) { return __ldg(t.haer + (kp - 1) * AER_NDM + (d - 1)); };
    const float pi = 3.1415926535897931f;
    const float rovg = 0.001f * 2.8705e+2f / 9.80665e+0f, fvirt = 4.6150e+2f / 2.8705e+2f - 1.0f;
    // layer thickness (k 0-based, top first): hypsometric, the top layer from its mid-level pressure, doubled
    auto DZ = [&](int k) {
        const float lo = k == 0 ? logf(L(a.plyr, 0)) : logf(L(a.plvl, k));
        const float dz = rovg * (logf(L(a.plvl, k + 1)) - lo) * L(a.tlyr, k) * (1.0f + fvirt * L(a.qlyr, k));
        return k == 0 ? 2.0f * dz : dz;
    };

    // layers side by side: thickness and the sigma of each layer's top interface
    {
        const float rps = __fdiv_rn(1.0f, L(a.plvl, nlay));   // decides domains: IEEE division, not the fast one
        for (int k = warp; k < nlay; k += AER_WARPS) {
            s_delz[k][lane] = DZ(k);
            s_fr[k][lane] = L(a.plvl, k) * rps;
        }
    }
    __syncthreads();
    if (warp == 0) {
        // setaer prep: degrees; the 5-degree cells around the column, profile structure, domain-overlay rules
        const float rdg = 180.0f / pi;
        float alon = __ldg(a.xlon + c) * rdg;
        if (alon < 0.0f) alon = alon + 360.0f;
        float alat = __ldg(a.xlat + c) * rdg;
        if (alat < -90.0f) alat = -90.0f;
        if (alat > 90.0f) alat = 90.0f;
        const float slm = __ldg(a.slmsk + c);
        const float dltg = 360.0f / (float)AER_IMXAE, hdlt = 0.5f * dltg, rdlt = 1.0f / dltg;
        // the reference steps cell by cell to the first i with f(i) <= dltg (f(1) = max(alon, 0),
        // f(i) = alon - dltg (i - 1)); f falls with i, so start next to the answer and step to it
        auto fi = [&](int i) { return i == 1 ? (alon < 0.0f ? 0.0f : alon) : alon - dltg * (float)(i - 1); };
        int i3 = min(AER_IMXAE, max(1, (int)(alon * rdlt)));
        while (i3 > 1 && fi(i3 - 1) <= dltg) --i3;
        while (i3 < AER_IMXAE && fi(i3) > dltg) ++i3;
        const float dtmp = fi(i3);
        const int i1 = i3, i2 = i3 % AER_IMXAE + 1;
        const float wi = dtmp * rdlt;
        const int kpi = dtmp <= hdlt ? i3 : i2;
        auto fj = [&](int j) { return j == 1 ? 90.0f - alat : (90.0f - dltg * (float)(j - 1)) - alat; };
        int j3 = min(AER_JMXAE, max(1, (int)((90.0f - alat) * rdlt)));
        while (j3 > 1 && fj(j3 - 1) <= dltg) --j3;
        while (j3 < AER_JMXAE && fj(j3) > dltg) ++j3;
        const float dtl = fj(j3);
        const int j1 = j3, j2 = j3 + 1 > AER_JMXAE ? AER_JMXAE : j3 + 1;
        const float wj = dtl * rdlt;
        const int kpj = dtl <= hdlt ? j3 : j2;
        auto CELL = [&](int i, int j) { return (j - 1) * AER_IMXAE + (i - 1); };
        int kp = __ldg(t.kprfg + CELL(kpi, kpj));
        const int kpa = max(max(__ldg(t.kprfg + CELL(i1, j1)), __ldg(t.kprfg + CELL(i1, j2))),
                            max(__ldg(t.kprfg + CELL(i2, j1)), __ldg(t.kprfg + CELL(i2, j2))));
        float h1 = HA(1, kp);
        int nden = 1;
        if (kp != kpa) {
            if (kpa == 6 || kpa == 7) {                // mineral transport over the ocean / land profile
                nden = 2;
                const bool land = slm > 0.0f;
                if ((kpa == 6) == land) { kp = kpa == 6 ? 7 : 6; h1 = 0.5f * (HA(1, 6) + HA(1, 7)); }
                else { kp = kpa; h1 = HA(1, kpa); }
            } else {
                h1 = HA(1, kpa);
                kp = kpa;
            }
        }
        const float w11 = (1.0f - wi) * (1.0f - wj), w12 = (1.0f - wi) * wj, w21 = wi * (1.0f - wj), w22 = wi * wj;
        const int c11 = CELL(i1, j1), c12 = CELL(i1, j2), c21 = CELL(i2, j1), c22 = CELL(i2, j2);
        float denn[3] = {0.0f, 0.0f, 0.0f};
        for (int m = 1; m <= nden; ++m)
            denn[m] = w11 * __ldg(t.denng + 2 * c11 + m - 1) + w12 * __ldg(t.denng + 2 * c12 + m - 1) +
                      w21 * __ldg(t.denng + 2 * c21 + m - 1) + w22 * __ldg(t.denng + 2 * c22 + m - 1);
        float cmix[AER_NCM + 1];
#pragma unroll
        for (int q = 0; q <= AER_NCM; ++q) cmix[q] = 0.0f;
        for (int m = 0; m < AER_NXC; ++m) {
            const int cc[4] = {c11, c12, c21, c22};
            const float ww[4] = {w11, w12, w21, w22};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int ic = __ldg(t.idxcg + cc[q] * AER_NXC + m);
                const float v = ww[q] * __ldg(t.cmixg + cc[q] * AER_NXC + m);
#pragma unroll
                for (int s = 1; s <= AER_NCM; ++s)    // register-indexed accumulation (ic = 0: no component)
                    if (ic == s) cmix[s] = cmix[s] + v;
            }
        }
#pragma unroll
        for (int q = 0; q <= AER_NCM; ++q) s_cmix[q][lane] = cmix[q];
        s_col[0][lane] = denn[1];
        s_col[1][lane] = denn[2];
        s_col[2][lane] = h1;
        s_col[3][lane] = __int_as_float(kp);
        // bottom-up: heights (surface 0) and each layer's domain, walking up through the profile's
        // reference sigma levels
        s_hz[nlay][lane] = 0.0f;
        float hz = 0.0f;
        int d = 1;
        for (int k = nlay - 1; k >= 0; --k) {
            hz = hz + s_delz[k][lane];
            s_hz[k][lane] = hz;
            if (d <= AER_NDM && s_fr[k][lane] < __ldg(t.sigref + (kp - 1) * AER_NDM + (d - 1))) {
                d = d + 1;
                if (d == 2 && __ldg(t.prsref + (kp - 1) * AER_NDM + 1) == __ldg(t.prsref + (kp - 1) * AER_NDM + 2)) d = 3;
            }
            s_code[k][lane] = d;
        }
    }
    __syncthreads();
    // per layer, the warps side by side: effective thickness and the humidity bracket
    {
        const int kp = __float_as_int(s_col[3][lane]);
        const float h1 = s_col[2][lane];
        for (int k = warp; k < nlay; k += AER_WARPS) {
            const int dom = s_code[k][lane];
            const float hl = dom > 1 ? (dom <= AER_NDM ? HA(dom, kp) : 0.0f) : h1;
            float delz;
            if (hl > 0.0f) {
                const float r = 1.0f / hl;
                delz = hl * (expf(-s_hz[k + 1][lane] * r) - expf(-s_hz[k][lane] * r));
            } else {                                   // the layer's own thickness
                delz = s_delz[k][lane];
            }
            const float rh = L(a.rhly, k);
            int r2 = 1;
            while (r2 <= AER_NRHLEV && rh > c_aer_rhlev[r2 - 1]) ++r2;
            const int r1 = max(1, r2 - 1);
            r2 = min(AER_NRHLEV, r2);
            s_fr[k][lane] = r1 == r2 ? 0.0f : (rh - c_aer_rhlev[r1 - 1]) / (c_aer_rhlev[r2 - 1] - c_aer_rhlev[r1 - 1]);
            s_delz[k][lane] = delz;
            s_code[k][lane] = dom | (r1 << 4) | (r2 << 8);
        }
    }
    __syncthreads();
    if (!live) return;
    // per band (warp w: bands w, w + AER_WARPS, ...): the layers top to bottom; the smoothing against the
    // layer above settles that layer's optical depth, which is stored one layer late
    const float dn1 = s_col[0][lane], dn2 = s_col[1][lane];
    for (int b = warp; b < AER_NBT; b += AER_WARPS) {
        const bool sw = b < AER_NSW;
        float* const o0 = sw ? a.faersw + ((size_t)(0 * AER_NSW + b) * nlay) * N + col
                             : a.faerlw + ((size_t)(0 * AER_NLW + b - AER_NSW) * nlay) * N + col;
        const size_t fstride = (size_t)(sw ? AER_NSW : AER_NLW) * nlay * N;   // field to field
        auto RI = [&](const float* x, int s) { return __ldg(x + b * AER_NCM1 + (s - 1)); };
        float up = 0.0f;
        for (int k = 0; k < nlay; ++k) {
            const int code = s_code[k][lane];
            const int dom = code & 15, r1 = (code >> 4) & 15, r2 = code >> 8;
            const float fr = s_fr[k][lane], delz = s_delz[k][lane];
            auto RD = [&](const float* x, int s) {
                const float* p = x + (b * AER_NCM2 + (s - 1)) * AER_NRHLEV;
                const float v1 = __ldg(p + r1 - 1);
                return v1 + fr * (__ldg(p + r2 - 1) - v1);
            };
            float tau, ssa, asy;
            if (dom == 4 || dom == 5) {                // stratosphere (4) and the aerosol-free top (5)
                tau = dom == 5 ? 0.0f : __ldg(t.extstra + b) * delz;
                ssa = sw ? 0.99f : 0.5f;
                asy = sw ? 0.696f : 0.3f;
            } else if (dom == 3) {                     // free troposphere: fixed mixture of three species
                const float e1 = RI(t.extrhi, 1), s1 = RI(t.scarhi, 1), a1 = RI(t.ssarhi, 1), g1 = RI(t.asyrhi, 1);
                const float e2 = RI(t.extrhi, 2), s2 = RI(t.scarhi, 2), a2 = RI(t.ssarhi, 2), g2 = RI(t.asyrhi, 2);
                const float e3 = RD(t.extrhd, 1), s3 = RD(t.scarhd, 1), a3 = RD(t.ssarhd, 1), g3 = RD(t.asyrhd, 1);
                const float ext = 0.17e-3f * e1 + 0.4f * e2 + 0.59983f * e3;
                const float sca = 0.17e-3f * s1 + 0.4f * s2 + 0.59983f * s3;
                const float se = 0.17e-3f * a1 * e1 + 0.4f * a2 * e2 + 0.59983f * a3 * e3;
                const float sg = 0.17e-3f * g1 * s1 + 0.4f * g2 * s2 + 0.59983f * g3 * s3;
                tau = ext * 730.0f * delz;
                ssa = ext > 0.0f ? fminf(1.0f, se / ext) : 1.0f;
                asy = sca > 0.0f ? fminf(1.0f, sg / sca) : 0.0f;
            } else if (dom == 1) {                     // mixing layer: the cell's components
                float ext = 0.0f, sca = 0.0f, se = 0.0f, sg = 0.0f;
#pragma unroll
                for (int s = 1; s <= AER_NCM; ++s) {
                    const float cm = s_cmix[s][lane];
                    if (!(cm > 0.0f)) continue;
                    float e, sc, al, g;
                    if (s <= AER_NCM1) { e = RI(t.extrhi, s); sc = RI(t.scarhi, s); al = RI(t.ssarhi, s); g = RI(t.asyrhi, s); }
                    else { e = RD(t.extrhd, s - AER_NCM1); sc = RD(t.scarhd, s - AER_NCM1); al = RD(t.ssarhd, s - AER_NCM1); g = RD(t.asyrhd, s - AER_NCM1); }
                    ext = ext + cm * e;
                    sca = sca + cm * sc;
                    se = se + cm * al * e;
                    sg = sg + cm * g * sc;
                }
                tau = ext * dn1 * delz;
                ssa = ext > 0.0f ? fminf(1.0f, se / ext) : 1.0f;
                asy = sca > 0.0f ? fminf(1.0f, sg / sca) : 0.0f;
            } else if (dom == 2) {                     // mineral transport layers
                tau = RI(t.extrhi, 6) * dn2 * delz;
                ssa = RI(t.ssarhi, 6);
                asy = RI(t.asyrhi, 6);
            } else {                                   // above every domain: no aerosol
                tau = 0.0f;
                ssa = 1.0f;
                asy = 0.0f;
            }
            if (k > 0) {                               // smoothing against the layer above (top to surface)
                const float ratio = tau > 0.0f ? __fdiv_rn(up, tau) : 1.0f;
                const float sum = tau + up, lo = 0.2f * sum, hi = sum - lo;
                if (ratio > 30.0f) { tau = lo; up = hi; }
                if (ratio < 0.03333f) { tau = hi; up = lo; }
                o0[(size_t)(k - 1) * N] = up;
            }
            up = tau;
            o0[fstride + (size_t)k * N] = ssa;
            o0[2 * fstride + (size_t)k * N] = asy;
        }
        o0[(size_t)(nlay - 1) * N] = up;
    }
}

}  // namespace rad
