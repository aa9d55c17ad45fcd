// rad_lw3.cuh -- the LW column solve as kernels over chunks of columns (mixed precision, sm_100a).
//
// The single-kernel LW (rad_lw2.cuh) holds a column's gas optics (taug, fracs: 140 g x 61 layers x 2 floats,
// 68 KB) in shared memory, so two CTAs fit an SM and the latency-bound table gathers and sweep recurrences
// run with ten warps per SM.  Here the gas optics go through HBM instead:
//
//   lw3_optics_kernel  one CTA (288 threads) per column: phases A and B of lw_setup_core (absorber amounts,
//                      cldprop, setcoef, Planck functions, taugb01..16, the max-random overlap factors of
//                      rtrnmr), with taug / fracs written straight to the chunk's scratch and the sweep inputs
//                      copied after them.  Shared memory is the set-up data and the species keys of bands 3,
//                      4, 5, 7 and 9 (LwSetupK, ~50 KB).
//   lw3_sweep_kernel   one warp per column: lane l carries g-points l, l + 32, ..., l + 128 (five independent
//                      recurrences interleaved per lane), reading each layer's optical depths as coalesced
//                      128-byte rows staged through shared memory by asynchronous copies.  Per layer each
//                      g-point's radiance CHANGE across the layer is formed directly (source minus radiance x
//                      absorptance) and summed over g-points in float64; the
//                      heating rates come from those changes, not from differences of ~300 W/m^2 level
//                      fluxes.
//   lw3_fp64_kernel    the plain float64 LW column (lw_column_body<double>) for the columns the optics kernel
//                      flags: a cloudy layer thinner than LW3_THIN hPa.  Such a layer (a cloud in the 0.1 hPa
//                      top layer of the precision-stress request) cools at thousands of K/day, and 1e-5 of
//                      that is already above 0.01 K/day: float optical depths put some g-points on the
//                      neighbouring entry of the 10,001-entry transmittance table, and float radiances
//                      carry ~1e-6 through the column.  Other columns exit at once.
//
// Scratch block of one column (floats, 128-byte aligned): taug [nlay][160], fracs [nlay][160] (g-points
// 140..159 unused), then one 80-word record per layer k = 1..nlay holding everything the sweeps read at that
// layer (so a layer step touches one contiguous record) and a head record (k = 0) for the surface.  The
// arithmetic of every term and recurrence is that of rad_lw2.cuh (rtrnmr,
// phys_rrtm_lw_rtrnmr_body.cuh:130-330; rtrnmc, phys_rrtm_lw_rtrnmc.cu:85-310; rtrn,
// phys_rrtm_lw_rtrn.cu:94-330).
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
constexpr int H_FP64 = 48;      // int: 1 when the column is to be solved in float64 (lw3_fp64_kernel)

constexpr float LW3_THIN = LW_THIN;   // hPa: a cloudy layer thinner than this sends the column to float64

__host__ __device__ constexpr int64_t lw3_rec_floats(int nlay) { return ((((int64_t)nlay + 1) * LW3_REC + 31) / 32) * 32; }
__host__ __device__ constexpr int64_t lw3_block_floats(int nlay)
{
    return (int64_t)2 * nlay * LW3_GSTRIDE + lw3_rec_floats(nlay);
}

// Optics CTA: 9 warps, 3 CTAs per SM (27 warps, at most 72 registers a thread, no spills).  The CTAs per SM set
// how many columns share an SM's L1 for the table gathers, and more than 3 cost more than they gain; more warps
// per CTA share a column's (g-point, layer) tasks and hide the gathers' latency.  Measured over the LW of 262,144
// columns: 160 threads 66.1 ms, 192 63.3, 224 61.4, 256 60.5, 288 60.0, 320 63.8 (spills); 4 CTAs of 224 / 256
// threads 64.0 / 70.1, 2 of 320 / 384 threads 64.0 / 62.6.  Same bits for every shape.
constexpr int LW3_OPT_THREADS = 288;
constexpr int LW3_OPT_MINB = 3;        // CTAs per SM the optics kernel is compiled for

__global__ void __launch_bounds__(LW3_OPT_THREADS, LW3_OPT_MINB) lw3_optics_kernel(const __grid_constant__ LwBatch bt, int64_t c0,
                                                                   float* __restrict__ scr, int* fp64list, int* err)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    LwSetupK<float>& s = *reinterpret_cast<LwSetupK<float>*>(smem_raw);
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
    lw_setup_core<float, LW3_OPT_THREADS>(s, a, col, tid, [&](int g, int k0, float tg, float fr) {
        tgo[k0 * LW3_GSTRIDE + g] = tg;
        fro[k0 * LW3_GSTRIDE + g] = fr;
    });
    float* aux = blk + (size_t)2 * nlay * LW3_GSTRIDE;
    for (int i = tid; i < nlay * 64; i += LW3_OPT_THREADS) {
        const int k = 1 + (i >> 6), w = i & 63, b = w & 15;
        float* r = aux + (size_t)k * LW3_REC;
        r[w] = w < 16 ? s.pklay[k][b] : w < 32 ? s.pklev[k][b] : w < 48 ? s.pklev[k - 1][b] : s.taucld[b][k - 1];
    }
    for (int k = 1 + tid; k <= nlay; k += LW3_OPT_THREADS) {
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
    if (tid == 0) {
        int fp64 = 0;
        for (int k0 = 0; k0 < nlay; ++k0)
            fp64 |= s.delp[k0] < LW3_THIN && s.cldfrc[k0 + 1] > 1.0e-6f;
        aux[H_FP64] = __int_as_float(fp64);
        if (fp64) fp64list[1 + atomicAdd(fp64list, 1)] = blockIdx.x;    // the chunk's list for lw3_fp64_kernel
    }
}

// The flagged columns of a chunk in float64: list = [count, chunk-local columns...] appended by the optics
// kernel; a grid of one CTA per SM walks it (the float64 layout's shared memory allows one CTA per SM).
__global__ void __launch_bounds__(LW_THREADS) lw3_fp64_kernel(const __grid_constant__ LwBatch bt, int64_t c0,
                                                              const int* __restrict__ list, LwLut<double> lutd,
                                                              int* err)
{
    const int n = list[0];
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        lw_column_body<double>(bt, lutd, err, c0 + list[1 + i]);
        __syncthreads();                          // shared memory is reused by the next column
    }
}

// Layer k (1-based, surface first) terms of one g-point (lw2_terms arithmetic), in float or float64.
template <class R>
__device__ __forceinline__ LwTerms<R> lw3_terms(const LwLut<R>& lut, R taug, R plfrac, R blay, R plev_u, R plev_d,
                                                R taucld, R sdif, bool cloudy)
{
    const R bpade = (R)1.0f / (R)0.278f, tblint = (R)10000, rec_6 = (R)0.166667f, c06 = (R)0.06f;
    LwTerms<R> t;
    R odepth = fmaxR((R)0, sdif * taug);
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
    const R dplnku = plev_u - blay;
    const R dplnkd = plev_d - blay;
    t.gassrcd = plfrac * (blay + dplnkd * gasfac) * atrgas;
    t.gassrcu = plfrac * (blay + dplnku * gasfac) * atrgas;
    t.atrg = atrgas;
    t.trnt = 1; t.totsrcd = 0; t.totsrcu = 0; t.atrt = 0;
    if (cloudy) {
        const R odtot = odepth + sdif * taucld;
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

// One layer of one g-point's sweep in arithmetic R on the float state (radtot, radclr and, with the
// max-random overlap, totrad / clrrad / rad): the recurrences of rtrnmr, rtrnmc and rtrn (OVR, the
// LW_OVR_* transfer).  Returns the total-sky radiance change across the layer formed directly -- source -
// radiance x absorptance, per overlap part -- so it keeps its relative precision however small it is beside
// the radiance.  f = the layer's six max-random overlap factors (clr1 cld1 cmb1 cmb2 clr2 cld2), x = sdif x
// cloud optical depth.  rtrnmc is rtrn with a cloud fraction of 1 in its cloudy sub-columns.
template <class R, int OVR>
__device__ __forceinline__ R lw3_step(float& rtot, float& rclr, float& trad, float& crad, float& radv,
                                      const LwTerms<R>& t, bool down, bool cl, bool lst, R clfr, const float* f, R x)
{
    const R src = down ? t.gassrcd : t.gassrcu, tsrc = down ? t.totsrcd : t.totsrcu;
    const R prev = (R)rtot;
    R inc;
    if (OVR != LW_OVR_MAXRAN) {
        if (cl) {
            const R cf = OVR == LW_OVR_MCICA ? (R)1 : clfr;
            const R efclrfr = (R)1 - ((R)1 - rexp(-x)) * cf;
            const R S = src + cf * (tsrc - src);
            rtot = (float)(prev * t.trng * efclrfr + S);
            const R cabs = -expm1(-x) * cf;        // 1 - efclrfr without the cancellation
            inc = S - prev * (t.atrg + cabs - t.atrg * cabs);
        } else {
            rtot = (float)(prev * t.trng + src);
            inc = src - prev * t.atrg;
        }
        rclr = (float)((R)rclr * t.trng + src);
        return inc;
    }
    R tt = trad, cc = crad, r = radv;
    if (lst) { tt = clfr * prev; cc = prev - tt; r = 0; }
    if (cl) {
        const R tp = tt, cp = cc;
        tt = tt * t.trnt + clfr * tsrc;
        cc = cc * t.trng + ((R)1 - clfr) * src;
        rtot = (float)(tt + cc);
        rclr = (float)((R)rclr * t.trng + src);
        const R radmod = r * ((R)f[0] * t.trng + (R)f[1] * t.trnt) - (R)f[2] * src + (R)f[3] * tsrc;
        r = -radmod + (R)f[4] * (cc + radmod) - (R)f[5] * (tt - radmod);
        tt = tt + r;
        cc = cc - r;
        inc = (clfr * tsrc + ((R)1 - clfr) * src) - (tp * t.atrt + cp * t.atrg);
    } else {
        rtot = (float)(prev * t.trng + src);
        rclr = (float)((R)rclr * t.trng + src);
        inc = src - prev * t.atrg;
    }
    trad = (float)tt;
    crad = (float)cc;
    radv = (float)r;
    return inc;
}

// The sweeps stream each layer's taug row, fracs row and record (400 floats) through a LW3_NSTAGE-stage ring in
// shared memory with asynchronous 16-byte copies (cp.async.cg: L2 to shared, no L1 allocation), LW3_NSTAGE - 1
// layers ahead of the one being computed, so the scratch's DRAM latency overlaps the arithmetic.
constexpr int LW3_STAGE = 2 * LW3_GSTRIDE + LW3_REC;   // floats per stage
constexpr int LW3_NSTAGE = 3;
// LW3_TMA fills the ring by bulk copies instead (cp.async.bulk: the layer's taug row, fracs row and record, three
// contiguous runs) that lane 0 issues and an mbarrier per slot completes.  Same bits; measured 2.5 % slower over
// the LW on the B200 (lane 0 alone issues and waits, where the 16-byte copies spread over the warp), so off.
constexpr bool LW3_TMA = false;
constexpr int LW3_WAIT_LIMIT = 1 << 16;   // mbarrier tests before a wait gives up (flags RAD_DEV_TIMEOUT)

__device__ __forceinline__ void lw3_cp16(float* dst, const float* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

// Layer k's rows and record into stage st: 100 16-byte pieces over the warp's lanes, one commit group.
// Sources are 16-byte aligned: rows start at multiples of 640 bytes and records at multiples of 320 bytes
// of a 128-byte aligned block.
__device__ __forceinline__ void lw3_stage_layer(float* st, const float* tg, const float* fr, const float* aux, int k,
                                                int lane)
{
    for (int c = lane; c < LW3_STAGE / 4; c += 32) {
        const float* src = c < 40   ? tg + (size_t)(k - 1) * LW3_GSTRIDE + 4 * c
                           : c < 80 ? fr + (size_t)(k - 1) * LW3_GSTRIDE + 4 * (c - 40)
                                    : aux + (size_t)k * LW3_REC + 4 * (c - 80);
        lw3_cp16(st + 4 * c, src);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Per-g-point profiles of one column for lwrad's optional outputs (DIAG sweeps): [nlay + 1][LW3_PGQ][LW_NGPT]
// floats: at level L (surface first) the upward and downward radiance, total sky then clear sky (q 0..3); at
// layer L (1..nlay) the radiance changes across it formed directly, upward pass U(L) - U(L-1) and downward
// pass D(L-1) - D(L), total sky then clear sky (q 4..7).
constexpr int LW3_PGQ = 8;
__host__ __device__ constexpr int64_t lw3_pg_floats(int nlay) { return (int64_t)(nlay + 1) * LW3_PGQ * LW_NGPT; }

template <int OVR, bool DIAG = false>
__global__ void __launch_bounds__(LW3_SWEEP_WARPS * 32) lw3_sweep_kernel(const __grid_constant__ LwBatch bt, int64_t c0,
                                                                         int64_t nc, const float* __restrict__ scr,
                                                                         LwLut<float> lut, int* err,
                                                                         float* __restrict__ pg = nullptr)
{
    __shared__ double fup[LW3_SWEEP_WARPS][NLAY_MAX + 1], fdn[LW3_SWEEP_WARPS][NLAY_MAX + 1];
    __shared__ __align__(16) float ring[LW3_SWEEP_WARPS][LW3_NSTAGE][LW3_STAGE];
    __shared__ __align__(8) uint64_t rbar[LW3_SWEEP_WARPS][LW3_NSTAGE];
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
    if (DIAG) pg += lc * lw3_pg_floats(nlay);
    // sweep steps: s = 0 .. nlay-1 downward (layer nlay - s), s = nlay .. 2 nlay - 1 upward (layer s - nlay + 1)
    const int nstep = 2 * nlay;
    auto layer_of = [&](int st) { return st < nlay ? nlay - st : st - nlay + 1; };
    if (LW3_TMA) {
        if (lane == 0) {
            for (int q = 0; q < LW3_NSTAGE; ++q) mbar_init(&rbar[warp][q], 1);
            mbar_init_fence();
        }
        __syncwarp();
    }
    // layer k's rows and record into ring slot q: lane 0 issues three bulk copies completed on the slot's barrier,
    // after the warp's reads of the slot's previous layer (ordered by the __syncwarp and the proxy fence)
    auto stage = [&](int q, int k) {
        if (LW3_TMA) {
            __syncwarp();
            if (lane == 0) {
                async_proxy_fence();
                uint64_t* b = &rbar[warp][q];
                float* dst = ring[warp][q];
                mbar_expect_tx(b, (unsigned)(LW3_STAGE * sizeof(float)));
                bulk_copy_g2s(dst, tg + (size_t)(k - 1) * LW3_GSTRIDE, LW3_GSTRIDE * sizeof(float), b);
                bulk_copy_g2s(dst + LW3_GSTRIDE, fr + (size_t)(k - 1) * LW3_GSTRIDE, LW3_GSTRIDE * sizeof(float), b);
                bulk_copy_g2s(dst + 2 * LW3_GSTRIDE, aux + (size_t)k * LW3_REC, LW3_REC * sizeof(float), b);
            }
        } else {
            lw3_stage_layer(ring[warp][q], tg, fr, aux, k, lane);
        }
    };
#pragma unroll
    for (int q = 0; q < LW3_NSTAGE - 1; ++q) stage(q, layer_of(q));
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
    float radtot[LW3_SLOTS], radclr[LW3_SLOTS], trad[LW3_SLOTS], crad[LW3_SLOTS], rad[LW3_SLOTS];
    // One layer of the sweep for the warp's g-points; returns the warp's float64 sum of the radiance changes.
    auto layer = [&](const float* stg, int k, bool down) -> double {
        const float* tgr = stg;
        const float* frr = stg + LW3_GSTRIDE;
        const float* r = stg + 2 * LW3_GSTRIDE;
        const float clfr = r[R_CLDFRC];
        const bool lst = __float_as_int(r[down ? R_LSTD : R_LSTU]) != 0;
        float f[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) f[i] = r[(down ? R_FACD : R_FACU) + i];
        double sum = 0.0;
#pragma unroll
        for (int j = 0; j < LW3_SLOTS; ++j) {
            const int g = gi[j], b = band[j];
            const bool cl = OVR == LW_OVR_MCICA ? mask_bit(j, k) : clfr >= eps;
            const float tcb = r[R_TAUCLD + b];
            const LwTerms<float> t = lw3_terms<float>(lut, tgr[g], frr[g], r[R_PKLAY + b], r[R_PKLEVU + b],
                                                      r[R_PKLEVD + b], tcb, sdif[j], cl);
            const float pclr = radclr[j];
            const float inc = lw3_step<float, OVR>(radtot[j], radclr[j], trad[j], crad[j], rad[j], t, down, cl, lst,
                                                  clfr, f, sdif[j] * tcb);
            if (val[j]) sum += (double)inc;
            if (DIAG && val[j]) {
                // the clear-sky change across the layer, formed directly like inc; the radiances at the level
                // the step ends on (k - 1 going down, k going up)
                const float incc = (down ? t.gassrcd : t.gassrcu) - pclr * t.atrg;
                float* p = pg + (size_t)k * LW3_PGQ * LW_NGPT + g;
                p[(down ? 5 : 4) * LW_NGPT] = inc;
                p[(down ? 7 : 6) * LW_NGPT] = incc;
                float* q = pg + (size_t)(down ? k - 1 : k) * LW3_PGQ * LW_NGPT + g;
                q[(down ? 1 : 0) * LW_NGPT] = radtot[j];
                q[(down ? 3 : 2) * LW_NGPT] = radclr[j];
            }
        }
        return warp_sum(sum);
    };
    // ---- the sweeps: downward, the surface, upward; layer s + LW3_NSTAGE - 1 is copied in while layer s computes
#pragma unroll
    for (int j = 0; j < LW3_SLOTS; ++j) { radtot[j] = 0; radclr[j] = 0; trad[j] = 0; crad[j] = 0; rad[j] = 0; }
    double s_tu = 0, s_cu = 0, s_td = 0, s_cd = 0;
    for (int st = 0; st < nstep; ++st) {
        if (st + LW3_NSTAGE - 1 < nstep)
            stage((st + LW3_NSTAGE - 1) % LW3_NSTAGE, layer_of(st + LW3_NSTAGE - 1));
        else if (!LW3_TMA)
            asm volatile("cp.async.commit_group;" ::: "memory");
        if (LW3_TMA) {
            // slot st % LW3_NSTAGE completes its (st / LW3_NSTAGE)-th phase when the step's copies have landed
            // lane 0 waits for the phase; the __syncwarp then orders the landed data for the other lanes
            bool ok = true;
            if (lane == 0)
                ok = mbar_wait_bounded(&rbar[warp][st % LW3_NSTAGE], (unsigned)((st / LW3_NSTAGE) & 1), LW3_WAIT_LIMIT);
            __syncwarp();
            if (!__shfl_sync(0xffffffffu, ok, 0)) {
                // a copy did not land: flag it, wait (bounded) for the copies still in flight, stop this column
                if (lane == 0) atomicExch(err, RAD_DEV_TIMEOUT);
                if (lane == 0)
                    for (int s2 = st + 1; s2 < min(nstep, st + LW3_NSTAGE); ++s2)
                        mbar_wait_bounded(&rbar[warp][s2 % LW3_NSTAGE], (unsigned)((s2 / LW3_NSTAGE) & 1),
                                          LW3_WAIT_LIMIT);
                return;
            }
        } else {
            // this lane's copies of step st have landed (the LW3_NSTAGE - 1 later groups may still be in flight)
            asm volatile("cp.async.wait_group %0;" ::"n"(LW3_NSTAGE - 1) : "memory");
            __syncwarp();                                        // ... and every lane's
        }
        if (st == nlay) {
            // surface: emission and reflection
#pragma unroll
            for (int j = 0; j < LW3_SLOTS; ++j) {
                const int b = band[j];
                const float semi = __ldg(aux + H_SEMISS + b);
                const float reflct = 1.0f - semi;
                const float rad0 = semi * __ldg(fr + gi[j]) * __ldg(aux + H_PKLAY0 + b);
                const float rtd = radtot[j], rcd = radclr[j];
                radtot[j] = rad0 + reflct * rtd;
                radclr[j] = rad0 + reflct * rcd;
                if (DIAG && val[j]) {   // the upward radiances leaving the surface; nothing comes down at the top
                    pg[(size_t)0 * LW_NGPT + gi[j]] = radtot[j];
                    pg[(size_t)2 * LW_NGPT + gi[j]] = radclr[j];
                    pg[((size_t)nlay * LW3_PGQ + 1) * LW_NGPT + gi[j]] = 0.0f;
                    pg[((size_t)nlay * LW3_PGQ + 3) * LW_NGPT + gi[j]] = 0.0f;
                }
                if (val[j]) {
                    s_tu += (double)radtot[j]; s_cu += (double)radclr[j];
                    s_td += (double)rtd; s_cd += (double)rcd;
                }
                trad[j] = 0; crad[j] = 0; rad[j] = 0;
            }
            s_tu = warp_sum(s_tu); s_cu = warp_sum(s_cu); s_td = warp_sum(s_td); s_cd = warp_sum(s_cd);
        }
        const bool down = st < nlay;
        const int k = layer_of(st);
        const double v = layer(ring[warp][st % LW3_NSTAGE], k, down);
        if (lane == 0) {
            if (down) fdn[warp][k - 1] = v;           // D(k-1) - D(k), summed over g
            else fup[warp][k] = v;                    // U(k) - U(k-1), summed over g
        }
        __syncwarp();                                 // the stage is free for the copy two steps on
    }
    double t_tu = 0, t_cu = 0;
#pragma unroll
    for (int j = 0; j < LW3_SLOTS; ++j)
        if (val[j]) { t_tu += (double)radtot[j]; t_cu += (double)radclr[j]; }
    t_tu = warp_sum(t_tu);
    t_cu = warp_sum(t_cu);
    __syncwarp();
    // ---- outputs: fluxes x flxfac; heating rates from the per-layer net-flux changes (rtrnmr post)
    const double pi = 3.14159265358979323846;
    const double flxfac = 0.5 * pi * 2.0e4;
    const double heatfac = 9.80665 * 1.0e-2 / 1.0046e3;
    for (int k = lane; k < nlay; k += 32) {
        // layer k + 1 (surface first): (U(k) - D(k)) - (U(k+1) - D(k+1)) = -(dU + dD)
        const double du = fup[warp][k + 1], dd = fdn[warp][k];
        const int kin = nlay - 1 - k;
        const double dl = (double)__ldg(a.plvl + (size_t)(kin + 1) * N + col) - (double)__ldg(a.plvl + (size_t)kin * N + col);
        a.htlw[(size_t)kin * N + col] = (float)(-(du + dd) * flxfac * (heatfac / dl));
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

// lwrad's optional outputs of a chunk from the DIAG sweeps' profiles: one warp per column, lane q < 16 band q
// (hlwb: htrb of rtrnmr's lhlwb block, from the band's per-layer changes), lane 16 the totals (lwflxprf, the
// level fluxes; hlw0 from the clear-sky per-layer changes).  Sums over g-points in float64 in g order, times
// flxfac; heating as the sweeps form htlw: -(dU + dD) flxfac heatfac / delp.
// Optional-output pointers of a launch's requests: hlw0, hlwb, lwflxprf, hsw0, htswb, swflxprf (null = not wanted).
struct DiagOuts {
    float* p[RAD_MAXREQ][6];
};
__global__ void __launch_bounds__(128) k_lw_diag(const __grid_constant__ LwBatch bt, int64_t c0, int64_t nc,
                                                 const float* __restrict__ pg, const __grid_constant__ DiagOuts outs)
{
    const int64_t lc = (int64_t)blockIdx.x * 4 + (threadIdx.x >> 5);
    const int q = threadIdx.x & 31;
    if (lc >= nc || q > 16) return;
    const int64_t gc = c0 + lc;
    const int rq = bt.find(gc);
    const LwIn& a = bt.req[rq];
    const int nlay = a.nlay;
    const int64_t col = gc - bt.off[rq], N = a.ncol;
    if (nlay > NLAY_MAX || col >= N) return;
    float* hlw0 = outs.p[rq][0];
    float* hlwb = outs.p[rq][1];
    float* flx = outs.p[rq][2];
    const float* p = pg + lc * lw3_pg_floats(nlay);
    const double flxfac = 0.5 * 3.14159265358979323846 * 2.0e4;
    const double heatfac = 9.80665 * 1.0e-2 / 1.0046e3;
    const int g0 = q < 16 ? c_lw_ns[q] : 0, g1 = q < 16 ? c_lw_ns[q + 1] : LW_NGPT;
    auto S = [&](int L, int f) {
        double v = 0.0;
        for (int g = g0; g < g1; ++g) v += (double)p[((size_t)L * LW3_PGQ + f) * LW_NGPT + g];
        return v;
    };
    for (int k = 1; k <= nlay; ++k) {
        const int kin = nlay - k;   // top-first index of layer k
        const double dl = (double)__ldg(a.plvl + (size_t)(kin + 1) * N + col) - (double)__ldg(a.plvl + (size_t)kin * N + col);
        const double rf = flxfac * (heatfac / dl);
        if (q < 16) {
            if (hlwb) hlwb[((size_t)q * nlay + kin) * N + col] = (float)(-(S(k, 4) + S(k, 5)) * rf);
        } else if (hlw0) {
            hlw0[(size_t)kin * N + col] = (float)(-(S(k, 6) + S(k, 7)) * rf);
        }
    }
    if (q == 16 && flx)
        for (int L = 0; L <= nlay; ++L)
            for (int f = 0; f < 4; ++f) flx[((size_t)f * (nlay + 1) + (nlay - L)) * N + col] = (float)(S(L, f) * flxfac);
}

}  // namespace rad
