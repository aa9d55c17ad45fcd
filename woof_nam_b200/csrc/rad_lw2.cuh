// rad_lw2.cuh -- the production LW column kernel for sm_100a (mixed precision).
//
// Same column physics as rad_lw.cuh (lwrad prep, cldprop, setcoef, taugb01..16, rtrnmr with maximum-
// random overlap; namgpu/kernels/phys_rrtm_lw_*.cu) and the same set-up phases (lw_setup: shared-memory
// layer data, gas optics per (g, layer) in g-major order so a warp stays inside one band).  The sweeps
// differ: one g-point per lane, 28 lanes per warp (5 warps = 140 g-points), and no per-thread layer
// arrays -- the upward sweep recomputes the layer transmittances and sources from the shared-memory
// optical depths instead of keeping them from the downward sweep, and each level's downward and upward
// radiances are summed over the warp's g-points (float64 shuffles) as the sweeps pass it.  Level sums are
// combined over warps in a fixed order, so results are bit-reproducible.
#pragma once
#include "rad_lw.cuh"

namespace rad {

constexpr int LW2_LANES = 28;   // g-points per warp

// LW cloud-overlap transfer of a sweep: lwrad's dispatch (phys_rrtm_lw_lwrad.py:102-111)
constexpr int LW_OVR_MAXRAN = 0;   // rtrnmr: NAM route, iovrlw > 0
constexpr int LW_OVR_MCICA = 1;    // rtrnmc: McICA route
constexpr int LW_OVR_RANDOM = 2;   // rtrn: NAM route, iovrlw = 0

// Layer k (1-based, surface first) of g-point g: gas and total (cloudy) transmittance and the downward /
// upward layer sources of rtrnmr (phys_rrtm_lw_rtrnmr_body.cuh:130-190).
template <class R>
struct LwTerms {
    R trng, gassrcd, gassrcu, trnt, totsrcd, totsrcu;
    R atrg;        // gas absorptance 1 - trng as computed (directly from the depth for thin layers)
    R atrt;        // cloudy: total absorptance 1 - trnt, likewise
};

template <class R>
__device__ __forceinline__ LwTerms<R> lw2_terms(const LwShared<R>& s, const LwLut<R>& lut, int g, int band, int k,
                                                R sdif, bool cloudy)
{
    const R bpade = (R)1.0f / (R)0.278f, tblint = (R)10000, rec_6 = (R)0.166667f, c06 = (R)0.06f;
    LwTerms<R> t;
    R odepth = fmaxR((R)0, sdif * s.taug[g][k - 1]);
    R atrgas, gasfac;
    if (odepth <= c06) {
        atrgas = odepth - (R)0.5f * odepth * odepth;
        t.trng = (R)1 - atrgas;
        gasfac = rec_6 * odepth;
    } else {
        const R tblind = odepth / (bpade + odepth);
        const int it = (int)(tblint * tblind + (R)0.5f);
        t.trng = ldt(lut.ex + it); atrgas = (R)1 - t.trng; gasfac = ldt(lut.tfn + it); odepth = ldt(lut.tau + it);
    }
    const R plfrac = s.fracs[g][k - 1];
    const R blay = s.pklay[k][band];
    const R dplnku = s.pklev[k][band] - blay;
    const R dplnkd = s.pklev[k - 1][band] - blay;
    t.gassrcd = plfrac * (blay + dplnkd * gasfac) * atrgas;
    t.gassrcu = plfrac * (blay + dplnku * gasfac) * atrgas;
    t.atrg = atrgas;
    t.trnt = 1; t.totsrcd = 0; t.totsrcu = 0; t.atrt = 0;
    if (cloudy) {
        const R odtot = odepth + sdif * s.taucld[band][k - 1];
        R totfac, atrtot;
        if (odtot < c06) {
            totfac = rec_6 * odtot; atrtot = odtot - (R)0.5f * odtot * odtot; t.trnt = (R)1 - atrtot;
        } else {
            const R tblind = odtot / (bpade + odtot);
            const int it = (int)(tblint * tblind + (R)0.5f);
            totfac = ldt(lut.tfn + it); t.trnt = ldt(lut.ex + it); atrtot = (R)1 - t.trnt;
        }
        t.totsrcd = plfrac * (blay + dplnkd * totfac) * atrtot;
        t.totsrcu = plfrac * (blay + dplnku * totfac) * atrtot;
        t.atrt = atrtot;
    }
    return t;
}

// MC = false: the NAM route, rtrnmr (maximum-random overlap of the layer cloud fractions), or rtrn when
// a.rnd (random overlap, phys_rrtm_lw_rtrn.cu:94-330): a layer with cloud fraction clfr >= 1e-6 scales the
// gas transmittance by the effective clear fraction 1 - (1 - exp(-odcld)) clfr and adds clfr x (cloudy
// source - gas source).
// MC = true: the McICA route (rtrnmc, phys_rrtm_lw_rtrnmc.cu:85-310): a layer is cloudy for g-point g
// when its sub-column bit is set, with effective clear fraction 1 - (1 - exp(-odcld)) -- rtrn with clfr = 1.
// A column with a cloudy layer thinner than LW_THIN hPa is solved in float64 (lw3_fp64_kernel): such a layer cools
// at thousands of K/day, so 1e-5 of it is already above 0.01 K/day, and its float optical depths put some
// g-points on the neighbouring entry of the 10,001-entry transmittance table.
constexpr float LW_THIN = 1.0f;

// fp64list (NAM route, float, may be null): [count, columns...] of the launch; a listed column is left to the
// float64 column kernel, which runs after this launch.
template <class R, bool MC>
__global__ void __launch_bounds__(LW_THREADS, 2) lw2_column_kernel(const __grid_constant__ LwBatch bt, LwLut<R> lut, int* err,
                                                                   int* fp64list)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    LwShared<R>& s = *reinterpret_cast<LwShared<R>*>(smem_raw);
    const int rq = bt.find((int64_t)blockIdx.x);
    const LwIn& a = bt.req[rq];
    const int nlay = a.nlay;
    const int64_t col = (int64_t)blockIdx.x - bt.off[rq];
    const int64_t N = a.ncol;
    const int tid = threadIdx.x;
    if (nlay > NLAY_MAX || col >= N) {
        if (tid == 0 && nlay > NLAY_MAX) atomicExch(err, RAD_DEV_NLAY);
        return;
    }
    if (MC)
        for (int i = tid; i < 5 * nlay; i += LW_THREADS)
            s.mcw[i / nlay][i % nlay] = __ldg(a.mask + ((size_t)(i / nlay) * nlay + (i % nlay)) * N + col);
    lw_setup<R, LW_THREADS>(s, a, col, tid);
    if (!MC && sizeof(R) == 4 && fp64list) {
        __shared__ int thin;
        if (tid == 0) {
            int f = 0;
            for (int k0 = 0; k0 < nlay; ++k0) f |= s.delp[k0] < (R)LW_THIN && s.cldfrc[k0 + 1] > (R)1.0e-6f;
            thin = f;
            if (f) fp64list[1 + atomicAdd(fp64list, 1)] = (int)blockIdx.x;
        }
        __syncthreads();
        if (thin) return;
    }
    const R eps = (R)1.0e-6f;
    const int warp = tid >> 5, lane = tid & 31;
    const bool act = lane < LW2_LANES;
    const int g = warp * LW2_LANES + (act ? lane : LW2_LANES - 1);
    int band = 0;
    while (g >= c_lw_ns[band + 1]) ++band;
    const R sdif = s.secdiff[band];
    const bool rnd = !MC && a.rnd != 0;
    // ---- downward sweep (top to surface): per level, the warp's sum of the total-sky radiance
    R radtotd = 0, radclrd = 0, totradd = 0, clrradd = 0, rad = 0;
    for (int k = nlay; k >= 1; --k) {
        if (MC || rnd) {
            const R cf = MC ? (R)1 : s.cldfrc[k];
            const bool cl = MC ? ((s.mcw[g >> 5][k - 1] >> (g & 31)) & 1u) != 0 : cf >= eps;
            const LwTerms<R> t = lw2_terms(s, lut, g, band, k, sdif, cl);
            if (cl) {
                const R efclrfr = (R)1 - ((R)1 - rexp(-(sdif * s.taucld[band][k - 1]))) * cf;
                radtotd = radtotd * t.trng * efclrfr + t.gassrcd + cf * (t.totsrcd - t.gassrcd);
            } else {
                radtotd = radtotd * t.trng + t.gassrcd;
            }
            radclrd = radclrd * t.trng + t.gassrcd;
            const double v = warp_sum(act ? (double)radtotd : 0.0);
            if (lane == 0) s.fnet2[warp][k - 1] = v;
            continue;
        }
        const R clfr = s.cldfrc[k];
        const bool cl = clfr >= eps;
        const LwTerms<R> t = lw2_terms(s, lut, g, band, k, sdif, cl);
        if (s.lstd[k]) { totradd = clfr * radtotd; clrradd = radtotd - totradd; rad = 0; }
        if (cl) {
            totradd = totradd * t.trnt + clfr * t.totsrcd;
            clrradd = clrradd * t.trng + ((R)1 - clfr) * t.gassrcd;
            radtotd = totradd + clrradd;
            radclrd = radclrd * t.trng + t.gassrcd;
            const R radmod = rad * (s.facclr1d[k - 1] * t.trng + s.faccld1d[k - 1] * t.trnt) -
                             s.faccmb1d[k - 1] * t.gassrcd + s.faccmb2d[k - 1] * t.totsrcd;
            rad = -radmod + s.facclr2d[k - 1] * (clrradd + radmod) - s.faccld2d[k - 1] * (totradd - radmod);
            totradd = totradd + rad;
            clrradd = clrradd - rad;
        } else {
            radtotd = radtotd * t.trng + t.gassrcd;
            radclrd = radclrd * t.trng + t.gassrcd;
        }
        const double v = warp_sum(act ? (double)radtotd : 0.0);
        if (lane == 0) s.fnet2[warp][k - 1] = v;
    }
    // ---- surface: emission and reflection
    const R semi = s.semiss[band];
    const R reflct = (R)1 - semi;
    const R rad0 = semi * s.fracs[g][0] * s.pklay[0][band];
    R radtotu = rad0 + reflct * radtotd;
    R radclru = rad0 + reflct * radclrd;
    {
        const double v0 = warp_sum(act ? (double)radtotu : 0.0), v1 = warp_sum(act ? (double)radclru : 0.0);
        const double v2 = warp_sum(act ? (double)radtotd : 0.0), v3 = warp_sum(act ? (double)radclrd : 0.0);
        if (lane == 0) {
            s.scal[warp][2] = v0; s.scal[warp][3] = v1; s.scal[warp][4] = v2; s.scal[warp][5] = v3;
            s.fnet[warp][0] = v0;
        }
    }
    // ---- upward sweep (surface to top), layer terms recomputed from shared memory
    R totradu = 0, clrradu = 0;
    rad = 0;
    for (int k = 1; k <= nlay; ++k) {
        if (MC || rnd) {
            const R cf = MC ? (R)1 : s.cldfrc[k];
            const bool cl = MC ? ((s.mcw[g >> 5][k - 1] >> (g & 31)) & 1u) != 0 : cf >= eps;
            const LwTerms<R> t = lw2_terms(s, lut, g, band, k, sdif, cl);
            if (cl) {
                const R efclrfr = (R)1 - ((R)1 - rexp(-(sdif * s.taucld[band][k - 1]))) * cf;
                radtotu = radtotu * t.trng * efclrfr + t.gassrcu + cf * (t.totsrcu - t.gassrcu);
            } else {
                radtotu = radtotu * t.trng + t.gassrcu;
            }
            radclru = radclru * t.trng + t.gassrcu;
            const double v = warp_sum(act ? (double)radtotu : 0.0);
            if (lane == 0) s.fnet[warp][k] = v;
            continue;
        }
        const R clfr = s.cldfrc[k];
        const bool cl = clfr >= eps;
        const LwTerms<R> t = lw2_terms(s, lut, g, band, k, sdif, cl);
        if (s.lstu[k]) { totradu = clfr * radtotu; clrradu = radtotu - totradu; rad = 0; }
        if (cl) {
            totradu = totradu * t.trnt + clfr * t.totsrcu;
            clrradu = clrradu * t.trng + ((R)1 - clfr) * t.gassrcu;
            radtotu = totradu + clrradu;
            radclru = radclru * t.trng + t.gassrcu;
            const R radmod = rad * (s.facclr1u[k + 1] * t.trng + s.faccld1u[k + 1] * t.trnt) -
                             s.faccmb1u[k + 1] * t.gassrcu + s.faccmb2u[k + 1] * t.totsrcu;
            rad = -radmod + s.facclr2u[k + 1] * (clrradu + radmod) - s.faccld2u[k + 1] * (totradu - radmod);
            totradu = totradu + rad;
            clrradu = clrradu - rad;
        } else {
            radtotu = radtotu * t.trng + t.gassrcu;
            radclru = radclru * t.trng + t.gassrcu;
        }
        const double v = warp_sum(act ? (double)radtotu : 0.0);
        if (lane == 0) s.fnet[warp][k] = v;
    }
    {
        const double v0 = warp_sum(act ? (double)radtotu : 0.0), v1 = warp_sum(act ? (double)radclru : 0.0);
        if (lane == 0) { s.scal[warp][0] = v0; s.scal[warp][1] = v1; }
    }
    __syncthreads();
    // ---- outputs: fluxes x flxfac, heating rates from float64 net-flux differences (rtrnmr post)
    const double pi = 3.14159265358979323846;
    const double flxfac = 0.5 * pi * 2.0e4;
    const double heatfac = 9.80665 * 1.0e-2 / 1.0046e3;
    for (int k = tid; k < nlay; k += LW_THREADS) {
        double uk = 0, uk1 = 0, dk = 0, dk1 = 0;
        for (int w = 0; w < LW_WARPS; ++w) {
            uk += s.fnet[w][k]; uk1 += s.fnet[w][k + 1];
            dk += s.fnet2[w][k]; dk1 += k + 1 < nlay ? s.fnet2[w][k + 1] : 0.0;
        }
        const int kin = nlay - 1 - k;
        const double dl = (double)__ldg(a.plvl + (size_t)(kin + 1) * N + col) - (double)__ldg(a.plvl + (size_t)kin * N + col);
        const double h = ((uk - dk) - (uk1 - dk1)) * flxfac * (heatfac / dl);
        a.htlw[(size_t)kin * N + col] = (float)h;
    }
    if (tid == 0) {
        double sc[6] = {0, 0, 0, 0, 0, 0};
        for (int w = 0; w < LW_WARPS; ++w)
            for (int i = 0; i < 6; ++i) sc[i] += s.scal[w][i];
        a.topflw[col] = (float)(sc[0] * flxfac);
        a.topflw[N + col] = (float)(sc[1] * flxfac);
        a.sfcflw[col] = (float)(sc[2] * flxfac);
        a.sfcflw[N + col] = (float)(sc[3] * flxfac);
        a.sfcflw[2 * N + col] = (float)(sc[4] * flxfac);
        a.sfcflw[3 * N + col] = (float)(sc[5] * flxfac);
    }
}

}  // namespace rad
