// rad_front.cu -- grrad's front end ahead of the column solve on sm_100a: the inputs of the solve (cos zenith
// and the sunlit runs, gas and ozone profiles, surface albedo and emissivity, cloud properties) from the model
// state, the surface fields and the climatologies.
//
//   k_dayparts   DAYPARTS (grrad_nmmb.f:606-656 with coszmn_nmmb; the reference's three kernels and a library
//                scan, namgpu/kernels/phys_rrtm_dayparts.cu:76-138): one CTA per row.  Each tile of the row
//                computes its points' zenith cosines, flags the run starts (a day flag that differs from the
//                previous point's, read by a warp shuffle, across warps through shared memory and across tiles
//                from a carried flag), numbers them with a warp ballot and a scan over the CTA's warps, and
//                stages each run's start and flag in shared memory; the run table is then written once,
//                coalesced, with each run's length from its successor.  One pass over the row's points.
//   k_getgases   getgases (radiation_gases_nmmb.f:843-979, phys_rrtm_getgases.cu:67-130): one thread per
//                column writes the 10 gases on every level; only CO2 varies (global mean + seasonal cycle, or
//                the monthly 15-degree map below 788 mb).  Store-bound: 40 lmax bytes per column.
//   k_getozn     getozn (radiation_gases_nmmb.f:984-1094, phys_rrtm_getozn.cu:43-111): the two months of the
//                climatology and its levels are staged in shared memory; each thread interpolates its column's
//                profile in latitude and time into its own shared-memory slice, then interpolates every level
//                in the Exner function.
//   k_setalb     setalb (radiation_surface_nmmb.f:407-725, phys_rrtm_setalb.cu:35-248), ialbflg 0, 1, 2.
//   k_setemis    setemis (radiation_surface_nmmb.f:730-897, phys_rrtm_setemis.cu:40-133).  The Fortran finds
//                the map cell by scanning all 360 longitudes and 180 latitudes for the first cell within half
//                a degree; the cell centres are whole and half degrees, so the first match can only be one of
//                the five cells around floor(longitude) (and 91 - latitude): the kernel tests those, in the
//                Fortran's order and with its float expressions, and gets the same cell in O(1).
//   k_progcld2   progcld2 with rsipath2_tmp and gethml (radiation_clouds_nmmb.f:787-1323, 2167-2494,
//                2779-2964; phys_rrtm_progcld2.cu:92-444): one thread per column; the layer cloud fractions
//                that gethml walks twice are kept in shared memory, [layer][thread].
//   k_grrad_clw  grrad's condensate (grrad_nmmb.f:1556-1571, phys_rrtm_grrad_clouds.cu:396-416): one thread per
//                (layer, column), the cloud tracers summed in tracer order.
//   k_payne_albedo  grrad's IALB = 2 surface albedo (grrad_nmmb.f:1722-1794, phys_rrtm_grrad_clouds.cu:344-393):
//                one thread per point; the tables travel in the kernel parameters (1.9 KB).
//   k_setaer_volc  setaer's volcanic stratospheric term (radiation_aerosols.f 2092-2352, the lavoflg branch;
//                namgpu/kernels/phys_rrtm_setaer.cu:178-330): one thread per column finds the aerosol's top
//                (5 mb) and bottom (150-250 mb by latitude) layers and adds its zone's optical depth, spread
//                by pressure depth, to the extinction of every band.  The per-band spectral factors are powf
//                of constants, formed on the host so that they are the host's bits.
//
// Layouts: [field][level][column] with column = row * im + point, as the solve's inputs.  Every kernel is
// HBM-bound: each input word is read once and each output word written once (the per-column bytes are in
// the launchers' comments).  Built alone with -fmad=false -prec-div=true -prec-sqrt=true -ftz=false.
#include "rad_front.h"

#include <cmath>

namespace rad {
namespace front {

namespace {

constexpr unsigned FULL = 0xffffffffu;

// ------------------------------------------------------------------------------------------ DAYPARTS
// 256 threads per row; per point 12 bytes read (xlon, sinlat, coslat) and 8 written (coszen, coszdg), plus the
// run table (12 bytes per run).
constexpr int DP_THREADS = 256;

__global__ void __launch_bounds__(DP_THREADS) k_dayparts(const DaypartsArgs a)
{
    extern __shared__ int dp_sm[];
    int* rstart = dp_sm;             // [im] 1-based start point of each run of the row
    int* rday = dp_sm + a.im;        // [im] its day flag
    __shared__ int wlast[DP_THREADS / 32], wruns[DP_THREADS / 32], tile_last;
    const int j = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t r0 = (size_t)j * a.im;
    const float pid12 = 0.261799388f, czlimt = 0.0001f;
    const float solang = pid12 * (a.solhr - 12.0f);
    const float rnstp = a.dtswav / (float)a.nrads;
    int runs = 0, prev = 0;          // runs so far in the row, day flag of the previous tile's last point
    for (int base = 0; base < a.im; base += DP_THREADS) {
        const int i = base + threadIdx.x;
        const bool in = i < a.im;
        int d = 0;
        if (in) {
            const size_t p = r0 + i;
            const float ss = __ldg(a.sinlat + p) * a.sindec, cc = __ldg(a.coslat + p) * a.cosdec;
            const float xl = __ldg(a.xlon + p);
            float sum = 0.0f;
            int lit = 0;
            for (int it = 1; it <= a.nrads; ++it) {
                const float cns = solang + (float)(it - 1) * pid12 * rnstp + a.sollag;
                const float cz = ss + cc * cosf(cns + xl);
                sum = sum + fmaxf(0.0f, cz);
                if (cz > czlimt) ++lit;
            }
            a.coszdg[p] = sum * rnstp;
            if (lit > 0) sum = sum / (float)lit;
            a.coszen[p] = sum;
            d = sum >= 0.0001f ? 1 : 0;
        }
        if (lane == 31) wlast[warp] = d;
        if (i == (a.im < base + DP_THREADS ? a.im : base + DP_THREADS) - 1) tile_last = d;
        __syncthreads();
        int dprev = __shfl_up_sync(FULL, d, 1);
        if (lane == 0) dprev = warp == 0 ? prev : wlast[warp - 1];
        const bool start = in && (i == 0 || d != dprev);
        const unsigned ball = __ballot_sync(FULL, start);
        if (lane == 0) wruns[warp] = __popc(ball);
        __syncthreads();
        int k = runs + __popc(ball & ((1u << lane) - 1u)), total = 0;
        for (int w = 0; w < DP_THREADS / 32; ++w) {
            if (w < warp) k += wruns[w];
            total += wruns[w];
        }
        if (start) {
            rstart[k] = i + 1;
            rday[k] = d;
        }
        runs += total;
        prev = tile_last;
        __syncthreads();
    }
    for (int k = threadIdx.x; k < runs; k += DP_THREADS) {
        const int s = rstart[k];
        a.dp_start[r0 + k] = s;
        a.dp_day[r0 + k] = rday[k];
        a.dp_len[r0 + k] = (k + 1 < runs ? rstart[k + 1] : a.im + 1) - s;
    }
    if (threadIdx.x == 0) a.ndayparts[j] = runs;
}

// ------------------------------------------------------------------------------------------ getgases
// Per column 4 (lmax + 1) bytes read (plvl, ico2flg 2 only) and 40 lmax written.
__global__ void __launch_bounds__(256) k_getgases(const GasArgs a)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.n) return;
    const float defv[10] = {350.0e-6f, 0.31e-6f, 1.50e-6f, 0.209f, 1.50e-8f,
                            3.520e-10f, 6.358e-10f, 1.500e-10f, 1.397e-10f, 8.2000e-11f};
    const size_t N = (size_t)a.n;
    float* g = a.gasvmr + c;
#pragma unroll
    for (int q = 1; q < 10; ++q)
        for (int l = 0; l < a.lmax; ++l) __stcs(g + ((size_t)q * a.lmax + l) * N, defv[q]);
    if (a.ico2flg == 2) {
        const float con_pi = 3.14159265358979323846f, hfpi = 0.5f * con_pi, raddeg = 180.0f / con_pi;
        const float tmp = raddeg / 15.0f;
        float lon = __ldg(a.xlon + c);
        if (lon < 0.0f) lon = lon + con_pi;
        const float colat = hfpi - __ldg(a.xlat + c);
        const int ilon = max(1, min(24, (int)(lon * tmp + 1.0f)));
        const int ilat = max(1, min(12, (int)(colat * tmp + 1.0f)));
        const float map = __ldg(a.co2vmr_sav + ((size_t)(a.kmonsav - 1) * 12 + (ilat - 1)) * 24 + (ilon - 1));
        const float base = __ldg(a.co2_glb) + __ldg(a.gco2cyc + a.kmonsav - 1);
        const int off = a.ivflip == 0 ? 0 : 1;
        for (int l = 0; l < a.lmax; ++l)
            __stcs(g + (size_t)l * N, __ldg(a.plvl + (size_t)(l + off) * N + c) >= 788.0f ? map : base);
    } else {
        const float v = a.ico2flg == 1 ? __ldg(a.co2_glb) + __ldg(a.gco2cyc + a.kmonsav - 1) : defv[0];
        for (int l = 0; l < a.lmax; ++l) __stcs(g + (size_t)l * N, v);
    }
}

// ------------------------------------------------------------------------------------------ getozn
// Per column 4 nlev bytes read (prslk) and at most 4 nlev written; the climatology comes from shared memory.
constexpr int OZ_THREADS = 128;

__global__ void __launch_bounds__(OZ_THREADS) k_getozn(const OzoneArgs a)
{
    extern __shared__ float oz_sm[];
    const int loz = a.loz, jmr = a.jmr;
    float* s_lo = oz_sm;                      // [loz][jmr] month k1oz
    float* s_hi = s_lo + loz * jmr;           // [loz][jmr] month k2oz
    float* s_pk = s_hi + loz * jmr;           // [loz]
    float* s_o3i = s_pk + loz;                // [loz][OZ_THREADS] each thread's interpolated profile
    for (int e = threadIdx.x; e < loz * jmr; e += OZ_THREADS) {
        s_lo[e] = __ldg(a.o3r + (size_t)(a.k1oz - 1) * loz * jmr + e);
        s_hi[e] = __ldg(a.o3r + (size_t)(a.k2oz - 1) * loz * jmr + e);
    }
    for (int e = threadIdx.x; e < loz; e += OZ_THREADS) s_pk[e] = __ldg(a.pkstr + e);
    __syncthreads();
    const int64_t c = (int64_t)blockIdx.x * OZ_THREADS + threadIdx.x;
    if (c >= a.n) return;
    const float deglat = __ldg(a.xlat + c) * 57.29578f;
    const float elte = a.blte + (float)(jmr - 1) * a.dlte;
    int j1, j2;
    float w;
    if (deglat > a.blte && deglat < elte) {
        w = (deglat - a.blte) / a.dlte + 1.0f;
        j1 = (int)w;
        j2 = j1 + 1;
        w = w - (float)j1;
    } else if (deglat <= a.blte) {
        j1 = j2 = 1;
        w = 1.0f;
    } else if (deglat >= elte) {
        j1 = j2 = jmr;
        w = 1.0f;
    } else {
        return;                               // NaN latitude: the routine writes nothing
    }
    const float w2 = 1.0f - w;
    float* o3i = s_o3i + threadIdx.x;
    for (int k = 0; k < loz; ++k) {
        const float lo = w2 * s_lo[k * jmr + j1 - 1] + w * s_lo[k * jmr + j2 - 1];
        const float hi = w2 * s_hi[k * jmr + j1 - 1] + w * s_hi[k * jmr + j2 - 1];
        o3i[k * OZ_THREADS] = hi * a.facoz + lo * (1.0f - a.facoz);
    }
    const size_t N = (size_t)a.n;
    for (int l = 1; l <= a.nlev; ++l) {
        const int ll = a.ivflip == 1 ? a.nlev - l + 1 : l;
        const size_t o = (size_t)(ll - 1) * N + c;
        const float x = __ldg(a.prslk + o);
        float v = 0.0f;
        bool set = false;
        for (int k = 0; k < loz - 1; ++k) {
            const float rdp = 1.0f / (s_pk[k + 1] - s_pk[k]);
            if (x > s_pk[k] && x <= s_pk[k + 1]) {
                const float t = (s_pk[k + 1] - x) * rdp;
                v = t * o3i[k * OZ_THREADS] + (1.0f - t) * o3i[(k + 1) * OZ_THREADS];
                set = true;
            }
        }
        if (x > s_pk[loz - 1]) {
            v = o3i[(loz - 1) * OZ_THREADS];
            set = true;
        }
        if (x < s_pk[0]) {
            v = o3i[0];
            set = true;
        }
        if (set) a.o3mmr[o] = v;
    }
}

// ------------------------------------------------------------------------------------------ setalb
// Per column up to 64 bytes read and 16 written (ialbflg 2: 16 and 16).
__global__ void __launch_bounds__(256) k_setalb(const AlbedoArgs a)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.n) return;
    const size_t N = (size_t)a.n;
    float* out = a.sfcalb + c;
    if (a.ialbflg != 0 && a.ialbflg != 1) {
        out[0] = __ldg(a.alnsf + c);
        out[N] = __ldg(a.alnwf + c);
        out[2 * N] = __ldg(a.alvsf + c);
        out[3 * N] = __ldg(a.alvwf + c);
        return;
    }
    const bool modis = a.ialbflg == 1;
    const float t0c = 273.15f, ttp = 273.16f, tice = 271.20f;
    const int msk = (int)roundf(__ldg(a.slmsk + c));
    const float ts = __ldg(a.tsknf + c), cz = __ldg(a.coszf + c);
    float fsno0;
    const bool depth_snow = !modis || msk == 2;
    if (depth_snow) {
        const float asnow = 0.02f * __ldg(a.snowf + c);
        const float argh = fminf(0.50f, fmaxf(0.025f, 0.01f * __ldg(a.zorlf + c)));
        const float hrgh = fminf(1.0f, fmaxf(0.20f, 1.0577f - 1.1538e-3f * __ldg(a.hprif + c)));
        fsno0 = asnow / (argh + asnow) * hrgh;
    } else {
        fsno0 = __ldg(a.sncovr + c);
    }
    if (msk == 0 && ts > tice) fsno0 = 0.0f;
    const float fsno1 = 1.0f - fsno0;
    const float facs = __ldg(a.facsf + c), facw = __ldg(a.facwf + c);
    const float flnd0 = fminf(1.0f, facs + facw);
    const float fsea0 = fmaxf(0.0f, 1.0f - flnd0);
    const float fsno = fsno0, fsea = fsea0 * fsno1, flnd = flnd0 * fsno1;
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
    float asnvd, asnnd;
    if (msk == 2) {
        const float fi = __ldg(a.fice + c), ffw = 1.0f - fi;
        float b1 = 0.0f;
        if (ffw < 1.0f) b1 = 0.03f * fmaxf(0.0f, fminf(5.0f, ttp - __ldg(a.tisfc + c)));
        const float b3 = 0.06f * ffw;
        asnvd = (0.70f + b1) * fi + b3;
        asnnd = (0.60f + b1) * fi + b3;
        asevd = 0.70f * fi + b3;
        asend = 0.60f * fi + b3;
    } else if (!modis) {
        asnvd = 0.90f;
        asnnd = 0.75f;
    } else {
        asnvd = asnnd = __ldg(a.snoalb + c);
    }
    float asnvb, asnnb;
    if (modis && msk != 2) {
        asnvb = asnnb = __ldg(a.snoalb + c);
    } else if (cz < 0.5f) {
        const float csnow = 0.5f * (3.0f / (1.0f + 4.0f * cz) - 1.0f);
        asnvb = fminf(0.98f, asnvd + (1.0f - asnvd) * csnow);
        asnnb = fminf(0.98f, asnnd + (1.0f - asnnd) * csnow);
    } else {
        asnvb = asnvd;
        asnnb = asnnd;
    }
    float rfcs = 1.0f, asevb = asevd, asenb = asend;
    if (cz > 0.0001f) {
        rfcs = modis ? 1.775f / (1.0f + 1.55f * cz) : 2.14f / (1.0f + 1.48f * cz);
        if (ts >= t0c) {
            asevb = fmaxf(asevd, 0.026f / (powf(cz, 1.7f) + 0.065f) + 0.15f * (cz - 0.1f) * (cz - 0.5f) * (cz - 1.0f));
            asenb = asevb;
        }
    }
    const float vs = __ldg(a.alvsf + c), ns = __ldg(a.alnsf + c), vw = __ldg(a.alvwf + c), nw = __ldg(a.alnwf + c);
    if (!modis) {
        const float a1 = vs * facs, b1 = vw * facw, a2 = ns * facs, b2 = nw * facw;
        out[0] = (a2 * rfcs + b2 * rfcs) * flnd + asenb * fsea + asnnb * fsno;
        out[N] = (a2 + b2) * 0.96f * flnd + asend * fsea + asnnd * fsno;
        out[2 * N] = (a1 * rfcs + b1 * rfcs) * flnd + asevb * fsea + asnvb * fsno;
        out[3 * N] = (a1 + b1) * 0.96f * flnd + asevd * fsea + asnvd * fsno;
    } else {
        out[0] = ns * rfcs * flnd + asenb * fsea + asnnb * fsno;
        out[N] = nw * flnd + asend * fsea + asnnd * fsno;
        out[2 * N] = vs * rfcs * flnd + asevb * fsea + asnvb * fsno;
        out[3 * N] = vw * flnd + asevd * fsea + asnvd * fsno;
    }
}

// ------------------------------------------------------------------------------------------ setemis
// The first cell index i1 in 1..cells whose centre first + step (i1 - 1) lies within half of `step` of x, or 1
// (the Fortran default) when none does.  Only the cells around the nearest centre can match (the centres are
// exact in float and their spacing is 1, so |x - centre| <= 0.5 leaves two candidates at most); the window
// [c - 2, c + 2] covers them with the Fortran's rounding of x - centre and is scanned in its order.
__device__ __forceinline__ int emis_cell(float x, float first, float step, int cells)
{
    const float hdlt = 0.5f;
    const float pos = (x - first) / step;     // 0-based fractional cell position (NaN / inf: no match)
    if (!(pos > -4.0f && pos < (float)cells + 4.0f)) return 1;
    const int c0 = (int)floorf(pos) + 1;
    for (int i1 = max(1, c0 - 2); i1 <= min(cells, c0 + 2); ++i1) {
        const float centre = step > 0.0f ? 1.0f * (float)(i1 - 1) + hdlt : 90.0f - 1.0f * (float)(i1 - 1);
        if (fabsf(x - centre) <= hdlt) return i1;
    }
    return 1;
}

// Per column up to 36 bytes read (plus one map word) and 4 written.
__global__ void __launch_bounds__(256) k_setemis(const EmisArgs a)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.n) return;
    if (a.iemslw == 0) {
        a.sfcemis[c] = 1.0f;
        return;
    }
    const float emsref[8] = {0.97f, 0.95f, 0.94f, 0.90f, 0.93f, 0.96f, 0.96f, 0.99f};
    const int msk = __ldg(a.sice + c) > 0.5f ? 2 : (int)roundf(1.0f - __ldg(a.sm + c));
    float em;
    if (msk == 0) {
        em = emsref[0];
    } else if (msk == 2) {
        em = emsref[6];
    } else {
        float lon = __ldg(a.glon + c) * 57.29578f;
        if (lon < 0.0f) lon = lon + 360.0f;
        const int i2 = emis_cell(lon, 0.5f, 1.0f, 360);            // centres 0.5, 1.5, ... (eastward)
        const float lat = __ldg(a.glat + c) * 57.29578f;
        const int j2 = emis_cell(lat, 90.0f, -1.0f, 180);           // centres 90, 89, ... (southward)
        int id = max(2, __ldg(a.idxems + (size_t)(j2 - 1) * 360 + (i2 - 1)));
        if (id >= 7) id = 2;
        em = emsref[id - 1];
    }
    if (a.ialbflg == 1 && msk == 1) {
        const float f = __ldg(a.sncovr + c);
        em = em * (1.0f - f) + emsref[7] * f;
    } else {
        const float si = __ldg(a.si + c);
        if (si > 0.0f) {
            const float asnow = 0.02f * si;
            const float argh = fminf(0.50f, fmaxf(0.025f, 0.01f * (100.0f * __ldg(a.z0 + c))));
            const float hrgh = fminf(1.0f, fmaxf(0.20f, 1.0577f - 1.1538e-3f * __ldg(a.stdh + c)));
            float f = asnow / (argh + asnow) * hrgh;
            if (msk == 0 && __ldg(a.tskin + c) > 271.2f) f = 0.0f;
            em = em * (1.0f - f) + emsref[7] * f;
        }
    }
    a.sfcemis[c] = em;
}

// ------------------------------------------------------------------------------------------ progcld2
// Per column 4 (11 nlay + 1) bytes read (plyr twice through L1) and 36 nlay + 44 written.
constexpr int CLD_THREADS = 128;

__device__ __forceinline__ float cld_form(float clw2, float pl, float qstl, float rhly, bool fourth_root)
{
    const float clwm = 0.0f / fmaxf(0.01f, pl * 0.001f);
    const float onemrh = fmaxf(1.0e-10f, 1.0f - rhly);
    float t;
    if (fourth_root) {
        t = fminf(fmaxf(sqrtf(sqrtf(onemrh * qstl)), 0.0001f), 1.0f);
        t = 2000.0f / t;
    } else {
        t = fminf(fmaxf(powf(onemrh * qstl, 0.49f), 0.0001f), 1.0f);
        t = 100.0f / t;
    }
    const float v = fmaxf(fminf(t * (clw2 - clwm), 50.0f), 0.0f);
    return fmaxf(sqrtf(sqrtf(rhly)) * (1.0f - expf(-v)), 0.0f);
}

__global__ void __launch_bounds__(CLD_THREADS) k_progcld2(const CloudArgs a)
{
    extern __shared__ float cld_sm[];          // [nlay][CLD_THREADS] layer cloud fraction
    const int64_t c = (int64_t)blockIdx.x * CLD_THREADS + threadIdx.x;
    if (c >= a.n) return;
    float* ct = cld_sm + threadIdx.x;
    const size_t N = (size_t)a.n, LN = (size_t)a.nlay * N;
    const int nlay = a.nlay;
    auto at = [&](const float* f, int k) { return __ldg(f + (size_t)k * N + c); };
    const float con_pi = 3.1415926535897931f, con_g = 9.80665f, con_rd = 287.05f, con_rv = 461.5f;
    const float fvirt = con_rv / con_rd - 1.0f, t0c = 273.15f, ttp = 273.16f;
    const float cclimit = 0.001f, cclimit2 = 0.05f, climit = 0.001f, ovcst = 1.0f - 1.0e-8f;
    const float recwat = 5.0f, recice = 10.0f, rerain = 100.0f;
    const float recw1 = 620.35f / powf(200.0f, 1.0f / 3.0f);
    float ptop1[4];
    {
        const float p1[4] = {1050.0f, 650.0f, 400.0f, 0.0f}, p2[4] = {1050.0f, 750.0f, 500.0f, 0.0f};
        const float w = fmaxf(0.0f, 4.0f * fabsf(__ldg(a.xlat + c)) / con_pi - 1.0f);
#pragma unroll
        for (int d = 0; d < 4; ++d) ptop1[d] = p1[d] + (p2[d] - p1[d]) * w;
    }
    float clw_m = 0.0f, clw_0 = at(a.clw, 0), clw_p = nlay > 1 ? at(a.clw, 1) : 0.0f;
    float plo = at(a.plvl, 0);
    for (int k = 0; k < nlay; ++k) {
        const float pl = at(a.plyr, k), plp = at(a.plvl, k + 1), tk = at(a.tlyr, k);
        float clwf;
        if (a.lcrick) {
            if (k == 0)
                clwf = 0.75f * clw_0 + 0.25f * clw_p;
            else if (k == nlay - 1)
                clwf = 0.75f * clw_0 + 0.25f * clw_m;
            else
                clwf = 0.25f * clw_m + 0.5f * clw_0 + 0.25f * clw_p;
        } else {
            clwf = clw_0;
        }
        const float fcice = fmaxf(0.0f, fminf(1.0f, at(a.f_ice, k)));
        const float frain = fmaxf(0.0f, fminf(1.0f, at(a.f_rain, k)));
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
            const float rho = 100.0f * pl / (con_rd * tk * (1.0f + fvirt * at(a.qlyr, k)));
            const float cpath = fabsf(plp - plo) * (100000.0f / con_g);
            if (qcwat > 0.0f) {
                rew = fmaxf(recwat, recw1 * powf(rho * qcwat, 1.0f / 3.0f));
                cwp = cpath * qcwat;
            }
            if (qrain > 0.0f) {
                rer = 1.5f * fmaxf(50.0f, fminf(1000.0f, 2511.54f * sqrtf(sqrtf(rho * qrain))));
                crp = cpath * qrain;
            }
            cip = cpath * qcice;
        }
        float f = 0.0f;
        if (a.cld_fraction == 0) {
            if (a.ivflip == 0 && !a.lsashal) {
                if (clw2 > 1.0e-8f * (pl * 0.001f)) f = fminf(1.0f, 1.0e5f * clw2 * pl * 0.001f);
            } else if (clw2 > 2.0e-6f * (pl * 0.001f)) {
                f = cld_form(clw2, pl, at(a.qstl, k), at(a.rhly, k), a.ivflip != 0 && !a.lsashal);
            }
        } else {
            f = at(a.cldfk1, k);
        }
        if (f < cclimit) {
            f = 0.0f;
            cwp = cip = crp = csp = 0.0f;
        }
        if (a.lnoprec) crp = csp = 0.0f;
        if (a.lcnorm && f >= cclimit) {
            const float r = 1.0f / fmaxf(cclimit2, f);
            cwp = cwp * r;
            cip = cip * r;
            crp = crp * r;
            csp = csp * r;
        }
        if (cip > 0.0f) {
            const float dens = a.ivflip == 0 ? (con_g * pl) / (con_rd * (plp - plo)) : (con_g * pl) / (con_rd * (plo - plp));
            const float iwc = dens * cip / at(a.tvly, k);
            const float dt = tk - ttp;
            float re;
            if (dt < -50.0f)
                re = (1250.0f / 9.917f) * powf(iwc, 0.109f);
            else if (dt < -40.0f)
                re = (1250.0f / 9.337f) * powf(iwc, 0.08f);
            else if (dt < -30.0f)
                re = (1250.0f / 9.208f) * powf(iwc, 0.055f);
            else
                re = (1250.0f / 9.387f) * powf(iwc, 0.031f);
            rei = fmaxf(recice, re * 0.6495f);
        }
        ct[k * CLD_THREADS] = f;
        float* o = a.clouds + (size_t)k * N + c;
        __stcs(o, f);
        __stcs(o + LN, cwp);
        __stcs(o + 2 * LN, rew);
        __stcs(o + 3 * LN, cip);
        __stcs(o + 4 * LN, rei);
        __stcs(o + 5 * LN, crp);
        __stcs(o + 6 * LN, rer);
        __stcs(o + 7 * LN, 0.0f);
        __stcs(o + 8 * LN, 0.0f);
        plo = plp;
        clw_m = clw_0;
        clw_0 = clw_p;
        clw_p = k + 2 < nlay ? at(a.clw, k + 2) : 0.0f;
    }
    // gethml: total and boundary-layer cloud (random overlap for iovr 0, maximum-random otherwise)
    auto CT = [&](int k1) { return fminf(ovcst, fmaxf(ct[(k1 - 1) * CLD_THREADS], 0.0f)); };
    float cl[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    int mt[3] = {0, 0, 0}, mb[3] = {0, 0, 0};
    {
        float c1 = 1.0f, c2 = 1.0f;
        for (int kk = 0; kk < nlay; ++kk) {
            const int k = a.ivflip == 0 ? nlay - kk : kk + 1;
            const float cc = CT(k);
            if (a.iovr == 0) {
                if (cc >= climit) c1 = c1 * (1.0f - cc);
                if (k == a.llyr) cl[4] = 1.0f - c1;
            } else {
                if (cc >= climit) {
                    c2 = fminf(c2, 1.0f - cc);
                } else {
                    c1 = c1 * c2;
                    c2 = 1.0f;
                }
                if (k == a.llyr) cl[4] = 1.0f - c1 * c2;
            }
        }
        cl[3] = a.iovr == 0 ? 1.0f - c1 : 1.0f - c1 * c2;
    }
    // high / middle / low decks, walking up from the surface layer
    // (the deck index id1 stays <= 4 for positive pressures: ptop1[3] is 0; the clamp only keeps the reads
    // inside ptop1 for inputs that are not)
    {
        const bool top_first = a.ivflip == 0;
        const int step = top_first ? -1 : 1, k0 = top_first ? nlay : 1, kend = top_first ? 0 : nlay + 1;
        float c1 = 0.0f, c2 = 0.0f;
        int kbt1 = k0, kbt2 = k0, kth1 = 0, kth2 = 0, idom = 1;
        mb[0] = mt[0] = k0;
        float pcur = at(a.plyr, k0 - 1), ccur = CT(k0);
        for (int k = k0; k != kend; k += step) {
            int id = idom, id1 = id + 1;
            const bool last = k + step == kend;
            const float pnxt = last ? -1.0f : at(a.plyr, k + step - 1);
            const float cnxt = last ? 0.0f : CT(k + step);
            if (pcur < ptop1[min(id1, 4) - 1]) {
                ++id;
                ++id1;
                idom = id;
            }
            if (ccur >= climit) {
                if (kth2 == 0) kbt2 = k;
                ++kth2;
                c2 = a.iovr == 0 ? c2 + ccur - c2 * ccur : fmaxf(c2, ccur);
                if (cnxt < climit || pnxt < ptop1[min(id1, 4) - 1]) {
                    kbt1 = (int)roundf((c1 * (float)kbt1 + c2 * (float)kbt2) / (c1 + c2));
                    kth1 = (int)roundf((c1 * (float)kth1 + c2 * (float)kth2) / (c1 + c2));
                    c1 = c1 + c2 - c1 * c2;
                    kbt2 = k + step;
                    kth2 = 0;
                    c2 = 0.0f;
                }
            }
            if (pnxt < ptop1[min(id1, 4) - 1]) {
                cl[min(id, 3) - 1] = c1;
                mt[min(id, 3) - 1] = top_first ? min(kbt1, kbt1 - kth1 + 1) : max(kbt1, kbt1 + kth1 - 1);
                mb[min(id, 3) - 1] = kbt1;
                c1 = 0.0f;
                kbt1 = k + step;
                kth1 = 0;
                if (id1 <= 3) {
                    mb[id1 - 1] = kbt1;
                    mt[id1 - 1] = kbt1;
                }
            }
            pcur = pnxt;
            ccur = cnxt;
        }
    }
#pragma unroll
    for (int q = 0; q < 5; ++q) a.clds[q * N + c] = cl[q];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        a.mtop[q * N + c] = mt[q];
        a.mbot[q * N + c] = mb[q];
    }
}

// ------------------------------------------------------------------------------------------ clw
// Per (layer, column) ncld words read and one written.
__global__ void __launch_bounds__(256) k_grrad_clw(const ClwArgs a)
{
    const int64_t plane = (int64_t)a.lmk * a.n;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= plane) return;
    float sum = 0.0f;
    for (int j = 0; j < a.ncld; ++j) sum += __ldg(a.tracer + (int64_t)(a.ntcw0 + j) * plane + p);
    a.clw[p] = sum < a.epsq ? 0.0f : sum;
}

// ------------------------------------------------------------------------------------------ IALB = 2 albedo
// Per point 12 bytes read and 36 written.
__global__ void __launch_bounds__(256) k_payne_albedo(const __grid_constant__ PayneArgs a)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n) return;
    const float sm = __ldg(a.sm + p), cz = __ldg(a.coszen + p);
    float alb = __ldg(a.salbedo + p);
    const float trans = 0.537f;
    const int iq = (int)(20.0f * trans + 1.0f);          // transmissivity column (1-based)
    if (cz > 0.0f && sm > 0.5f) {
        const float zen = (180.0f / 3.14159265f) * acosf(fmaxf(cz, 0.0f));
        int jx;                                           // zenith row (1-based)
        if (zen >= 74.0f) jx = (int)(0.5f * (90.0f - zen) + 1.0f);
        else if (zen >= 50.0f) jx = (int)(0.25f * (74.0f - zen) + 9.0f);
        else jx = (int)(0.1f * (50.0f - zen) + 15.0f);
        jx = max(1, min(jx, 19));                         // rows 1..19 (a coszen above 1 gives a NaN zenith)
        const float w = -(zen - a.za[jx - 1]) / a.dza[jx - 1];
        const float* r0 = a.albd + (jx - 1) * 21;
        const float* r1 = r0 + 21;
        const float a1 = r0[iq - 1] + w * (r1[iq - 1] - r0[iq - 1]);
        const float a2 = r0[iq] + w * (r1[iq] - r0[iq]);
        alb = a1 + 20.0f * (a2 - a1) * (trans - a.trn[iq - 1]);
    }
    const float v[9] = {alb, sm, cz, alb, alb, alb, alb, 0.0f, 0.0f};
#pragma unroll
    for (int f = 0; f < 9; ++f) a.out[f][p] = v[f];
}

// ------------------------------------------------------------------------------------------ volcanic term
// Per column (nlay + 1) * 4 bytes of pressure read, and the extinction of the 30 bands over the aerosol's
// layers (about 15 of 61 on NAM's levels) read and written.
__global__ void __launch_bounds__(256) k_setaer_volc(const __grid_constant__ VolcArgs a)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.n) return;
    const size_t N = (size_t)a.n;
    const int nlay = a.nlay;
    auto P = [&](int i) { return __ldg(a.plvl + (size_t)i * N + c); };
    const float pi = 3.1415926535897931f, rdg = 180.0f / pi, psrfh = 5.0f;
    float lat = __ldg(a.xlat + c) * rdg;
    if (lat < -90.0f) lat = -90.0f;
    if (lat > 90.0f) lat = 90.0f;
    float volcae;
    if (lat > 46.0f)       volcae = 1.0e-4f * (float)a.iv[0];
    else if (lat > 44.0f)  volcae = 5.0e-5f * (float)(a.iv[0] + a.iv[1]);
    else if (lat > 1.0f)   volcae = 1.0e-4f * (float)a.iv[1];
    else if (lat > -1.0f)  volcae = 5.0e-5f * (float)(a.iv[1] + a.iv[2]);
    else if (lat > -44.0f) volcae = 1.0e-4f * (float)a.iv[2];
    else if (lat > -46.0f) volcae = 5.0e-5f * (float)(a.iv[2] + a.iv[3]);
    else                   volcae = 1.0e-4f * (float)a.iv[3];
    const float alat = fabsf(lat);
    const float psrfl = alat > 70.0f ? 250.0f : (alat < 20.0f ? 150.0f : 110.0f + 2.0f * alat);
    // top and bottom layer (0-based) and 1 / the pressure depth between them
    int kh, kl;
    float rdelp;
    if (a.ivflip == 0) {
        kh = nlay - 2; kl = 1; rdelp = 1.0f / P(1);
        for (int i = 1; i <= nlay - 3; ++i)
            if (P(i) >= psrfh) { kh = i - 1; break; }
        for (int i = 1; i <= nlay - 3; ++i)
            if (P(i) >= psrfl) { kl = i - 1; rdelp = 1.0f / (P(i) - P(kh)); break; }
    } else {
        kh = 1; kl = nlay - 2; rdelp = 1.0f / P(nlay - 2);
        for (int i = nlay - 2; i >= 1; --i)
            if (P(i) >= psrfh) { kh = i; break; }
        for (int i = nlay - 1; i >= 1; --i)
            if (P(i) >= psrfl) { kl = i; rdelp = 1.0f / (P(i) - P(kh + 1)); break; }
    }
    const bool down = a.ivflip == 0;
    const int j0 = down ? kh : kl, j1 = down ? kl : kh, below = down ? kl + 1 : kl - 1;
    auto add = [&](float* x, float tb) {         // x: one band's [nlay][n] extinction at column c
        for (int j = j0; j <= j1; ++j) {
            const float share = down ? (P(j + 1) - P(j)) * rdelp : (P(j) - P(j + 1)) * rdelp;
            const float tmp2 = tb * share;
            x[(size_t)j * N] = x[(size_t)j * N] + tmp2 * volcae;
        }
    };
    if (a.add_sw) {
        for (int b = 0; b < 14; ++b) {
            float* x = a.faersw + (size_t)b * nlay * N + c;
            add(x, a.tsw[b]);
            const float xl = x[(size_t)kl * N], xb = x[(size_t)below * N];
            if (xl > 10.0f * xb) {                  // a sharp bottom edge is spread 80 / 20 over two layers
                const float s2 = xl + xb;
                x[(size_t)kl * N] = 0.8f * s2;
                x[(size_t)below * N] = 0.2f * s2;
            }
        }
    }
    if (a.add_lw)
        for (int b = 0; b < 16; ++b) add(a.faerlw + (size_t)b * nlay * N + c, a.tlw[b]);
}

inline unsigned blocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t dayparts(const DaypartsArgs& a, cudaStream_t st)
{
    const size_t smem = 2 * sizeof(int) * (size_t)a.im;
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(k_dayparts, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_dayparts<<<(unsigned)a.jm, DP_THREADS, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t getgases(const GasArgs& a, cudaStream_t st)
{
    k_getgases<<<blocks(a.n, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t getozn(const OzoneArgs& a, cudaStream_t st)
{
    const size_t smem = sizeof(float) * ((size_t)2 * a.loz * a.jmr + a.loz + (size_t)a.loz * OZ_THREADS);
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(k_getozn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_getozn<<<blocks(a.n, OZ_THREADS), OZ_THREADS, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t setalb(const AlbedoArgs& a, cudaStream_t st)
{
    k_setalb<<<blocks(a.n, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t setemis(const EmisArgs& a, cudaStream_t st)
{
    k_setemis<<<blocks(a.n, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t progcld2(const CloudArgs& a, cudaStream_t st)
{
    const size_t smem = sizeof(float) * (size_t)a.nlay * CLD_THREADS;
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(k_progcld2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k_progcld2<<<blocks(a.n, CLD_THREADS), CLD_THREADS, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t grrad_clw(const ClwArgs& a, cudaStream_t st)
{
    k_grrad_clw<<<blocks((int64_t)a.lmk * a.n, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t payne_albedo(const PayneArgs& a, cudaStream_t st)
{
    k_payne_albedo<<<blocks(a.n, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t setaer_volc(const VolcArgs& a, cudaStream_t st)
{
    k_setaer_volc<<<blocks(a.n, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace front
}  // namespace rad
