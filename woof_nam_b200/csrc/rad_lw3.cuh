// rad_lw3.cuh -- the LW column solve as two kernels over chunks of columns (mixed precision, sm_100a).
//
// The single-kernel LW (rad_lw2.cuh) holds a column's gas optics (taug, fracs: 140 g x 61 layers x 2 floats,
// 68 KB) in shared memory, so two CTAs fit an SM and the latency-bound table gathers and sweep recurrences
// run with ten warps per SM.  Here the gas optics go through HBM instead:
//
//   lw3_optics_kernel  one CTA (160 threads) per column: phases A and B of lw_setup_core (absorber amounts,
//                      cldprop, setcoef, Planck functions, taugb01..16, the max-random overlap factors of
//                      rtrnmr), with taug / fracs written straight to the chunk's scratch and the sweep inputs
//                      copied after them.  Shared memory is the set-up data only (~32 KB).
//   lw3_sweep_kernel   one warp per column: lane l carries g-points l, l + 32, ..., l + 128 (five
//                      independent recurrences interleaved per lane), reading each layer's optical depths as
//                      coalesced 128-byte rows; per level the lane sums its g-points in float64 and one warp
//                      reduction gives the column's radiance sum.
//
// Scratch block of one column (floats, 128-byte aligned): taug [nlay][160], fracs [nlay][160] (g-points
// 140..159 unused), then one 80-word record per layer k = 1..nlay holding everything the sweeps read at that
// layer (so a layer step touches one contiguous record), and a head record (k = 0) for the surface.  The
// arithmetic of every term and recurrence is that of rad_lw2.cuh (rtrnmr, phys_rrtm_lw_rtrnmr_body.cuh:
// 130-330; rtrnmc, phys_rrtm_lw_rtrnmc.cu:85-310); only the order of the float64 level sums differs.
#pragma once
#include "rad_lw2.cuh"

namespace rad {

constexpr int LW3_GSTRIDE = 160;                         // floats per layer row of taug / fracs
constexpr int LW3_SLOTS = 5;                             // g-points per lane in the sweeps
constexpr int LW3_SWEEP_WARPS = 4;                       // columns per sweep CTA
constexpr int LW3_REC = 80;                              // words per layer record
// layer record k (1..nlay)
constexpr int R_PKLAY = 0;      // [16] pklay[k]
constexpr int R_PKLEVU = 16;    // [16] pklev[k]
constexpr int R_PKLEVD = 32;    // [16] pklev[k - 1]
constexpr int R_TAUCLD = 48;    // [16] cloud optical depth of layer k
constexpr int R_CLDFRC = 64;    // cldfrc[k]
constexpr int R_LSTU = 65;      // int lstu[k]
constexpr int R_LSTD = 66;      // int lstd[k]
constexpr int R_FACD = 67;      // [6] downward factors at k - 1: clr1 cld1 cmb1 cmb2 clr2 cld2
constexpr int R_FACU = 73;      // [6] upward factors at k + 1, same order
// head record (k = 0)
constexpr int H_PKLAY0 = 0;     // [16] pklay[0] (surface)
constexpr int H_SECDIFF = 16;   // [16]
constexpr int H_SEMISS = 32;    // [16]

__host__ __device__ constexpr int64_t lw3_block_floats(int nlay)
{
    return (int64_t)2 * nlay * LW3_GSTRIDE + ((((int64_t)nlay + 1) * LW3_REC + 31) / 32) * 32;
}

__global__ void __launch_bounds__(LW_THREADS, 3) lw3_optics_kernel(const __grid_constant__ LwBatch bt, int64_t c0,
                                                                   float* __restrict__ scr, int* err)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    LwSetup<float>& s = *reinterpret_cast<LwSetup<float>*>(smem_raw);
    const int64_t gc = c0 + blockIdx.x;
    const int rq = bt.find(gc);
    const LwIn& a = bt.req[rq];
    const int nlay = a.nlay;
    const int64_t col = gc - bt.off[rq];
    const int tid = threadIdx.x;
    if (nlay > NLAY_MAX || col >= a.ncol) {
        if (tid == 0 && nlay > NLAY_MAX) atomicExch(err, RAD_DEV_NLAY);
        return;
    }
    float* blk = scr + (int64_t)blockIdx.x * lw3_block_floats(nlay);
    float* tgo = blk;
    float* fro = blk + (size_t)nlay * LW3_GSTRIDE;
    lw_setup_core<float, LW_THREADS>(s, a, col, tid, [&](int g, int k0, float tg, float fr) {
        tgo[k0 * LW3_GSTRIDE + g] = tg;
        fro[k0 * LW3_GSTRIDE + g] = fr;
    });
    float* aux = blk + (size_t)2 * nlay * LW3_GSTRIDE;
    for (int i = tid; i < nlay * 64; i += LW_THREADS) {
        const int k = 1 + (i >> 6), w = i & 63, b = w & 15;
        float* r = aux + (size_t)k * LW3_REC;
        r[w] = w < 16 ? s.pklay[k][b] : w < 32 ? s.pklev[k][b] : w < 48 ? s.pklev[k - 1][b] : s.taucld[b][k - 1];
    }
    for (int k = 1 + tid; k <= nlay; k += LW_THREADS) {
        float* r = aux + (size_t)k * LW3_REC;
        r[R_CLDFRC] = s.cldfrc[k];
        r[R_LSTU] = __int_as_float(s.lstu[k]);
        r[R_LSTD] = __int_as_float(s.lstd[k]);
        const float fd[6] = {s.facclr1d[k - 1], s.faccld1d[k - 1], s.faccmb1d[k - 1], s.faccmb2d[k - 1],
                             s.facclr2d[k - 1], s.faccld2d[k - 1]};
        const float fu[6] = {s.facclr1u[k + 1], s.faccld1u[k + 1], s.faccmb1u[k + 1], s.faccmb2u[k + 1],
                             s.facclr2u[k + 1], s.faccld2u[k + 1]};
        for (int f = 0; f < 6; ++f) { r[R_FACD + f] = fd[f]; r[R_FACU + f] = fu[f]; }
        r[LW3_REC - 1] = 0.0f;
    }
    if (tid < 16) {
        aux[H_PKLAY0 + tid] = s.pklay[0][tid];
        aux[H_SECDIFF + tid] = s.secdiff[tid];
        aux[H_SEMISS + tid] = s.semiss[tid];
    }
}

// Layer k (1-based, surface first) terms of one g-point from the chunk scratch (lw2_terms arithmetic).
__device__ __forceinline__ LwTerms<float> lw3_terms(const LwLut<float>& lut, float taug, float plfrac, float blay,
                                                    float plev_u, float plev_d, float taucld, float sdif, bool cloudy)
{
    const float bpade = 1.0f / 0.278f, tblint = 10000.0f, rec_6 = 0.166667f, c06 = 0.06f;
    LwTerms<float> t;
    float odepth = fmaxf(0.0f, sdif * taug);
    float atrgas, gasfac;
    if (odepth <= c06) {
        atrgas = odepth - 0.5f * odepth * odepth;
        t.trng = 1.0f - atrgas;
        gasfac = rec_6 * odepth;
    } else {
        const float tblind = odepth / (bpade + odepth);
        const int it = (int)(tblint * tblind + 0.5f);
        t.trng = ldt(lut.ex + it); atrgas = 1.0f - t.trng; gasfac = ldt(lut.tfn + it); odepth = ldt(lut.tau + it);
    }
    const float dplnku = plev_u - blay;
    const float dplnkd = plev_d - blay;
    t.gassrcd = plfrac * (blay + dplnkd * gasfac) * atrgas;
    t.gassrcu = plfrac * (blay + dplnku * gasfac) * atrgas;
    t.trnt = 1; t.totsrcd = 0; t.totsrcu = 0;
    if (cloudy) {
        const float odtot = odepth + sdif * taucld;
        float totfac, atrtot;
        if (odtot < c06) {
            totfac = rec_6 * odtot; atrtot = odtot - 0.5f * odtot * odtot; t.trnt = 1.0f - atrtot;
        } else {
            const float tblind = odtot / (bpade + odtot);
            const int it = (int)(tblint * tblind + 0.5f);
            totfac = ldt(lut.tfn + it); t.trnt = ldt(lut.ex + it); atrtot = 1.0f - t.trnt;
        }
        t.totsrcd = plfrac * (blay + dplnkd * totfac) * atrtot;
        t.totsrcu = plfrac * (blay + dplnku * totfac) * atrtot;
    }
    return t;
}

// L1 prefetch of one 128-byte line (PTX prefetch.global.L1): the sweeps fetch the next layer's rows and
// record while the current layer computes, so the scratch's DRAM latency is not paid once per layer.
__device__ __forceinline__ void lw3_prefetch(const void* p)
{
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// Lanes 0..9 prefetch the five 128-byte lines of layer k's taug row and of its fracs row, lanes 10..12 the
// (up to three) lines of its record.
__device__ __forceinline__ void lw3_prefetch_layer(const float* tg, const float* fr, const float* aux, int k, int lane)
{
    if (lane < 5) lw3_prefetch(tg + (size_t)(k - 1) * LW3_GSTRIDE + 32 * lane);
    else if (lane < 10) lw3_prefetch(fr + (size_t)(k - 1) * LW3_GSTRIDE + 32 * (lane - 5));
    else if (lane < 13) lw3_prefetch(aux + (size_t)k * LW3_REC + 32 * (lane - 10));
}

template <bool MC>
__global__ void __launch_bounds__(LW3_SWEEP_WARPS * 32) lw3_sweep_kernel(const __grid_constant__ LwBatch bt, int64_t c0,
                                                                         int64_t nc, const float* __restrict__ scr,
                                                                         LwLut<float> lut)
{
    __shared__ double fup[LW3_SWEEP_WARPS][NLAY_MAX + 1], fdn[LW3_SWEEP_WARPS][NLAY_MAX + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t lc = (int64_t)blockIdx.x * LW3_SWEEP_WARPS + warp;
    if (lc >= nc) return;
    const int64_t gc = c0 + lc;
    const int rq = bt.find(gc);
    const LwIn& a = bt.req[rq];
    const int nlay = a.nlay;
    const int64_t col = gc - bt.off[rq];
    const int64_t N = a.ncol;
    if (nlay > NLAY_MAX || col >= N) return;    // the optics kernel has flagged a bad nlay
    const float* blk = scr + lc * lw3_block_floats(nlay);
    const float* tg = blk;
    const float* fr = blk + (size_t)nlay * LW3_GSTRIDE;
    const float* aux = blk + (size_t)2 * nlay * LW3_GSTRIDE;
    lw3_prefetch_layer(tg, fr, aux, nlay, lane);
    const float eps = 1.0e-6f;
    int gi[LW3_SLOTS], band[LW3_SLOTS];
    float sdif[LW3_SLOTS];
    bool val[LW3_SLOTS];
#pragma unroll
    for (int j = 0; j < LW3_SLOTS; ++j) {
        const int g = lane + 32 * j;
        val[j] = g < LW_NGPT;
        gi[j] = val[j] ? g : LW_NGPT - 1;
        int b = 0;
        while (gi[j] >= c_lw_ns[b + 1]) ++b;
        band[j] = b;
        sdif[j] = __ldg(aux + H_SECDIFF + b);
    }
    auto mask_bit = [&](int j, int k) {   // McICA: word j holds g-points 32 j .. 32 j + 31
        return ((__ldg(a.mask + ((size_t)j * nlay + (k - 1)) * N + col) >> lane) & 1u) != 0;
    };
    // ---- downward sweep
    float radtotd[LW3_SLOTS], radclrd[LW3_SLOTS], totradd[LW3_SLOTS], clrradd[LW3_SLOTS], rad[LW3_SLOTS];
#pragma unroll
    for (int j = 0; j < LW3_SLOTS; ++j) { radtotd[j] = 0; radclrd[j] = 0; totradd[j] = 0; clrradd[j] = 0; rad[j] = 0; }
    for (int k = nlay; k >= 1; --k) {
        if (k > 1) lw3_prefetch_layer(tg, fr, aux, k - 1, lane);
        const float* tgr = tg + (size_t)(k - 1) * LW3_GSTRIDE;
        const float* frr = fr + (size_t)(k - 1) * LW3_GSTRIDE;
        const float* r = aux + (size_t)k * LW3_REC;
        const float clfr = __ldg(r + R_CLDFRC);
        const bool lst = __float_as_int(__ldg(r + R_LSTD)) != 0;
        const float c1 = __ldg(r + R_FACD), d1 = __ldg(r + R_FACD + 1), m1 = __ldg(r + R_FACD + 2),
                    m2 = __ldg(r + R_FACD + 3), c2 = __ldg(r + R_FACD + 4), d2 = __ldg(r + R_FACD + 5);
        double sum = 0.0;
#pragma unroll
        for (int j = 0; j < LW3_SLOTS; ++j) {
            const int g = gi[j], b = band[j];
            const bool cl = MC ? mask_bit(j, k) : clfr >= eps;
            const float tcb = __ldg(r + R_TAUCLD + b);
            const LwTerms<float> t = lw3_terms(lut, __ldg(tgr + g), __ldg(frr + g), __ldg(r + R_PKLAY + b),
                                               __ldg(r + R_PKLEVU + b), __ldg(r + R_PKLEVD + b), tcb, sdif[j], cl);
            if (MC) {
                if (cl) {
                    const float efclrfr = 1.0f - (1.0f - rexp(-(sdif[j] * tcb)));
                    radtotd[j] = radtotd[j] * t.trng * efclrfr + t.gassrcd + (t.totsrcd - t.gassrcd);
                } else {
                    radtotd[j] = radtotd[j] * t.trng + t.gassrcd;
                }
                radclrd[j] = radclrd[j] * t.trng + t.gassrcd;
            } else {
                if (lst) { totradd[j] = clfr * radtotd[j]; clrradd[j] = radtotd[j] - totradd[j]; rad[j] = 0; }
                if (cl) {
                    totradd[j] = totradd[j] * t.trnt + clfr * t.totsrcd;
                    clrradd[j] = clrradd[j] * t.trng + (1.0f - clfr) * t.gassrcd;
                    radtotd[j] = totradd[j] + clrradd[j];
                    radclrd[j] = radclrd[j] * t.trng + t.gassrcd;
                    const float radmod = rad[j] * (c1 * t.trng + d1 * t.trnt) - m1 * t.gassrcd + m2 * t.totsrcd;
                    rad[j] = -radmod + c2 * (clrradd[j] + radmod) - d2 * (totradd[j] - radmod);
                    totradd[j] = totradd[j] + rad[j];
                    clrradd[j] = clrradd[j] - rad[j];
                } else {
                    radtotd[j] = radtotd[j] * t.trng + t.gassrcd;
                    radclrd[j] = radclrd[j] * t.trng + t.gassrcd;
                }
            }
            if (val[j]) sum += (double)radtotd[j];
        }
        sum = warp_sum(sum);
        if (lane == 0) fdn[warp][k - 1] = sum;
    }
    // ---- surface: emission and reflection
    lw3_prefetch_layer(tg, fr, aux, 1, lane);
    float radtotu[LW3_SLOTS], radclru[LW3_SLOTS];
    double s_tu = 0, s_cu = 0, s_td = 0, s_cd = 0;
#pragma unroll
    for (int j = 0; j < LW3_SLOTS; ++j) {
        const int b = band[j];
        const float semi = __ldg(aux + H_SEMISS + b);
        const float reflct = 1.0f - semi;
        const float rad0 = semi * __ldg(fr + gi[j]) * __ldg(aux + H_PKLAY0 + b);
        radtotu[j] = rad0 + reflct * radtotd[j];
        radclru[j] = rad0 + reflct * radclrd[j];
        if (val[j]) {
            s_tu += (double)radtotu[j]; s_cu += (double)radclru[j];
            s_td += (double)radtotd[j]; s_cd += (double)radclrd[j];
        }
    }
    s_tu = warp_sum(s_tu); s_cu = warp_sum(s_cu); s_td = warp_sum(s_td); s_cd = warp_sum(s_cd);
    if (lane == 0) fup[warp][0] = s_tu;
    // ---- upward sweep
    float totradu[LW3_SLOTS], clrradu[LW3_SLOTS];
#pragma unroll
    for (int j = 0; j < LW3_SLOTS; ++j) { totradu[j] = 0; clrradu[j] = 0; rad[j] = 0; }
    for (int k = 1; k <= nlay; ++k) {
        if (k < nlay) lw3_prefetch_layer(tg, fr, aux, k + 1, lane);
        const float* tgr = tg + (size_t)(k - 1) * LW3_GSTRIDE;
        const float* frr = fr + (size_t)(k - 1) * LW3_GSTRIDE;
        const float* r = aux + (size_t)k * LW3_REC;
        const float clfr = __ldg(r + R_CLDFRC);
        const bool lst = __float_as_int(__ldg(r + R_LSTU)) != 0;
        const float c1 = __ldg(r + R_FACU), d1 = __ldg(r + R_FACU + 1), m1 = __ldg(r + R_FACU + 2),
                    m2 = __ldg(r + R_FACU + 3), c2 = __ldg(r + R_FACU + 4), d2 = __ldg(r + R_FACU + 5);
        double sum = 0.0;
#pragma unroll
        for (int j = 0; j < LW3_SLOTS; ++j) {
            const int g = gi[j], b = band[j];
            const bool cl = MC ? mask_bit(j, k) : clfr >= eps;
            const float tcb = __ldg(r + R_TAUCLD + b);
            const LwTerms<float> t = lw3_terms(lut, __ldg(tgr + g), __ldg(frr + g), __ldg(r + R_PKLAY + b),
                                               __ldg(r + R_PKLEVU + b), __ldg(r + R_PKLEVD + b), tcb, sdif[j], cl);
            if (MC) {
                if (cl) {
                    const float efclrfr = 1.0f - (1.0f - rexp(-(sdif[j] * tcb)));
                    radtotu[j] = radtotu[j] * t.trng * efclrfr + t.gassrcu + (t.totsrcu - t.gassrcu);
                } else {
                    radtotu[j] = radtotu[j] * t.trng + t.gassrcu;
                }
                radclru[j] = radclru[j] * t.trng + t.gassrcu;
            } else {
                if (lst) { totradu[j] = clfr * radtotu[j]; clrradu[j] = radtotu[j] - totradu[j]; rad[j] = 0; }
                if (cl) {
                    totradu[j] = totradu[j] * t.trnt + clfr * t.totsrcu;
                    clrradu[j] = clrradu[j] * t.trng + (1.0f - clfr) * t.gassrcu;
                    radtotu[j] = totradu[j] + clrradu[j];
                    radclru[j] = radclru[j] * t.trng + t.gassrcu;
                    const float radmod = rad[j] * (c1 * t.trng + d1 * t.trnt) - m1 * t.gassrcu + m2 * t.totsrcu;
                    rad[j] = -radmod + c2 * (clrradu[j] + radmod) - d2 * (totradu[j] - radmod);
                    totradu[j] = totradu[j] + rad[j];
                    clrradu[j] = clrradu[j] - rad[j];
                } else {
                    radtotu[j] = radtotu[j] * t.trng + t.gassrcu;
                    radclru[j] = radclru[j] * t.trng + t.gassrcu;
                }
            }
            if (val[j]) sum += (double)radtotu[j];
        }
        sum = warp_sum(sum);
        if (lane == 0) fup[warp][k] = sum;
    }
    double t_tu = 0, t_cu = 0;
#pragma unroll
    for (int j = 0; j < LW3_SLOTS; ++j)
        if (val[j]) { t_tu += (double)radtotu[j]; t_cu += (double)radclru[j]; }
    t_tu = warp_sum(t_tu);
    t_cu = warp_sum(t_cu);
    __syncwarp();
    // ---- outputs: fluxes x flxfac, heating rates from float64 net-flux differences (rtrnmr post)
    const double pi = 3.14159265358979323846;
    const double flxfac = 0.5 * pi * 2.0e4;
    const double heatfac = 9.80665 * 1.0e-2 / 1.0046e3;
    for (int k = lane; k < nlay; k += 32) {
        const double uk = fup[warp][k], uk1 = fup[warp][k + 1];
        const double dk = fdn[warp][k], dk1 = k + 1 < nlay ? fdn[warp][k + 1] : 0.0;
        const int kin = nlay - 1 - k;
        const double dl = (double)__ldg(a.plvl + (size_t)(kin + 1) * N + col) - (double)__ldg(a.plvl + (size_t)kin * N + col);
        a.htlw[(size_t)kin * N + col] = (float)(((uk - dk) - (uk1 - dk1)) * flxfac * (heatfac / dl));
    }
    if (lane == 0) {
        a.topflw[col] = (float)(t_tu * flxfac);
        a.topflw[N + col] = (float)(t_cu * flxfac);
        a.sfcflw[col] = (float)(s_tu * flxfac);
        a.sfcflw[N + col] = (float)(s_cu * flxfac);
        a.sfcflw[2 * N + col] = (float)(s_td * flxfac);
        a.sfcflw[3 * N + col] = (float)(s_cd * flxfac);
    }
}

}  // namespace rad
