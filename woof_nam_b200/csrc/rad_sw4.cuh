// rad_sw4.cuh -- the chunked SW of rad_solve (mixed precision): set-up and gas optics, the layer reflectances
// and transmittances, and the adding sweeps in three kernels per chunk of sunlit columns.
//
// Same statements as sw2_column (rad_sw2.cuh), split where the work changes shape, and each kernel small enough
// that the CTAs resident on an SM run out of the instruction cache (one kernel with all three phases spent most
// of its stalls waiting for instructions):
//  * sw4_gas_kernel, one CTA (128 threads) per sunlit column, six per SM: set-up and cloud optics
//    (sw2_setup), gas and Rayleigh optical depths per (g-point, layer); writes the column image (the part of the
//    shared-memory layout the later phases read, taug included).
//  * sw4_rt_kernel, one CTA per column: loads the image, then the layer R/T of the clear pass and, in the
//    layers with cloud, of the cloudy pass (spcvrtc.cu:112-173, 330-460), lanes on 32 consecutive
//    (layer, g-point) tasks so that a warp shares the cloudy branch, two tasks per thread side by side, in
//    float without branches.  A task whose R/T needs a float64 step (the resonance, or an exp-table argument
//    near an entry bound whose neighbouring entry matters) is queued and formed afterwards by sw2_layer, the
//    sweep kernels' own function, one per thread.  Output per column: a header (solar source per g-point,
//    albedos, overlap fractions, heating factors, the cloudy-pass slot of each layer) and the R/T as
//    [layer][field][g-point] (a warp of the sweep kernel reads 32 consecutive g-points of one field and
//    layer: one 128-byte line).
//  * sw4_sweep_kernel, one CTA per column: the adding method alone (swflux, spcvrtc.cu:178-215) -- the upward
//    sweep with segment checkpoints, the downward sweep re-reading each segment's R/T, float64 level sums and
//    the swrad epilogue.
// The outputs agree with sw2_column's to float rounding (tests/test_gpu_sw_split.py).
#pragma once
#include <type_traits>
#include "rad_sw2.cuh"

namespace rad {

constexpr int SW4_FIELDS = 6;                       // rb, rd, tb, td, e3 (delta-scaled beam), e4 (unscaled beam)
constexpr int SW4_LAYER = SW4_FIELDS * SW_NGPT;     // floats per layer and pass, [field][g]
// CTA shapes of the three kernels, swept on the B200 (same bits): the gas-optics kernel at 128 threads x 6 CTAs
// per SM against 160 x 5, 192 x 4, 256 x 3, 320 x 2, 384 x 2 (SW +0.2 to +9.8 %); the R/T kernel at 128 x 4
// against 160 x 3, 192 x 3, 224 x 2, 256 x 2 (+1.8 to +8.3 %).
constexpr int SW4_RT_THREADS = 128;                 // threads of an R/T CTA
constexpr int SW4_OPT_MINB = 4;                     // CTAs per SM the R/T kernel is compiled for
constexpr bool SW4_RT_PAIR = false;                 // two R/T tasks per thread side by side (else one)
constexpr int SW4_SWEEP_MINB = 6;                   // ... and the sweep kernel
constexpr int SW4_GAS_THREADS = 128;               // threads of a gas-optics CTA
constexpr int SW4_GAS_MINB = 6;                     // ... and the gas-optics kernel
constexpr bool SW4_L2PF = true;                     // the sweeps prefetch the R/T rows two segments ahead into L2

struct Sw4Hdr {
    double rdelp[NLAY_MAX];          // heatfac / delp, float64
    float zsolar[SW_NGPT];           // ssolar * sfluxzen of each g-point
    float albbm[2], albdf[2], zcf0, zcf1, pad0[2];
    int cloudy;                      // the cloudy pass runs
    int ncl;                         // layers with a cloudy-pass R/T
    int pad1[2];
    signed char slot[NLAY_MAX];      // cloudy-pass slot of each layer; -1: the clear R/T serve both passes
};
static_assert(sizeof(Sw4Hdr) % 16 == 0, "the header is copied in 16-byte pieces");
__host__ __device__ constexpr size_t sw4_hdr_bytes() { return (sizeof(Sw4Hdr) + 15) / 16 * 16; }
// One column's block of the chunk scratch: header, clear R/T [nlay][SW4_LAYER], cloudy R/T [nlay][SW4_LAYER]
// (the first ncl slots used).
__host__ __device__ constexpr size_t sw4_block_bytes(int nlay)
{
    return sw4_hdr_bytes() + (size_t)2 * nlay * SW4_LAYER * sizeof(float);
}
static_assert(sw4_hdr_bytes() % 16 == 0 && (SW4_LAYER * sizeof(float)) % 16 == 0, "16-byte aligned parts");

// ---- branch-free float R/T (the phase-R fast path).  Two tasks per thread run side by side, so the
// compiler can interleave their long dependency chains; the float64 decisions become flags.
__device__ __forceinline__ bool sw4_near(float zb)            // sw2_near without branches
{
    const float ft = zb / ((float)1.0f / (float)0.278f + zb);
    const float pos = ft * (float)10000 + (float)0.5f;
    const float fr = pos - floorf(pos);
    const float m = 10000.0f * ft * (SW2_ZB_EPS * (1.0f - ft) + 3.0e-7f);
    const bool tbl = fr < m || fr > 1.0f - m;
    const bool ser = zb > 0.06f * (1.0f - SW2_ZB_EPS);
    return zb <= 0.06f * (1.0f + SW2_ZB_EPS) ? ser : tbl;
}
__device__ __forceinline__ float sw4_tblexp(float zb, float& em)   // sw2_tblexp without branches
{
    const float ftind = zb / ((float)1.0f / (float)0.278f + zb);
    const int it = min(10000, (int)(ftind * (float)10000 + (float)0.5f));
    const float et = it >= 10000 ? 1.0e-20f : __expf(-(3.59712230f * (float)it) / (float)(10000 - it));
    const bool ser = zb <= 0.06f;
    em = ser ? zb - 0.5f * zb * zb : 1.0f - et;
    return ser ? 1.0f - zb + 0.5f * zb * zb : et;
}
// sw2_rt_float (prologue of two-stream mode MODE, R/T, direct transmissions) without branches; ok = false where
// sw2_rt_mixed would take a float64 step or test a neighbouring table entry (the outputs are then not used).
template <int MODE>
__device__ __forceinline__ void sw4_rt(float t0, float tabs, float s0, float y0, float cz, float snt, float wk, float wf,
                                       SwLayerRT& r, bool& ok)
{
    const float ftiny = 1.0e-12f;
    const float cwmin = (float)(1.0 - ((double)1.0f - (double)1.0e-6f));
    const float cw = fmaxf(cwmin, tabs / t0);
    const float zssaw = 1.0f - cw;
    const float zasyw = y0 / fmaxf(ftiny, s0);
    const float za2s = zssaw * (zasyw * zasyw);
    const float om = 1.0f - za2s;
    SwPro<float> p;
    p.ztau1 = om * t0;
    p.zssa1 = (zssaw - za2s) / om;
    const float cw1 = cw / om;
    const float zasy1 = zasyw / (1.0f + zasyw), zasy3 = 0.75f * zasy1;
    float gm, gp;
    if constexpr (MODE == 2) {
        p.g1 = 2.0f - p.zssa1 * (1.25f + zasy3);
        p.g2 = 0.75f * p.zssa1 * (1.0f - zasy1);
        p.g3 = 0.5f - zasy3 * cz;
        gm = 2.0f * cw1;
        gp = 2.0f - p.zssa1 * (0.5f + 1.5f * zasy1);
    } else if constexpr (MODE == 1) {
        p.g1 = 1.75f - p.zssa1 * (1.0f + zasy3);
        p.g2 = -0.25f - p.zssa1 * (1.0f - zasy3);
        p.g3 = 0.5f - zasy3 * cz;
        gm = p.g1 - p.g2;
        gp = p.g1 + p.g2;
    } else {
        const float zsr3 = 1.7320508f;
        p.g1 = zsr3 * (2.0f - p.zssa1 * (1.0f + zasy1)) * 0.5f;
        p.g2 = zsr3 * p.zssa1 * (1.0f - zasy1) * 0.5f;
        p.g3 = (1.0f - zsr3 * zasy1 * cz) * 0.5f;
        gm = zsr3 * cw1;
        gp = zsr3 * (1.0f - p.zssa1 * zasy1);
    }
    p.g4 = 1.0f - p.g3;
    p.zrk = sqrtf(gm * gp);
    p.zrp = p.zrk * cz;
    p.zrpp = (1.0f - p.zrp) * (1.0f + p.zrp);
    const float zb1 = fminf(p.zrk * p.ztau1, 500.0f), zb2 = fminf(p.ztau1 * snt, 500.0f), zb4 = t0 * snt;
    ok = !(fabsf(p.zrpp) < SW2_RESONANCE) && !(wk > 0.0f && (sw4_near(zb1) || sw4_near(zb2))) &&
         !(wf * 4.0e-4f > 1.0f && sw4_near(zb4));
    float em1, em2, em;
    const float e1 = sw4_tblexp(zb1, em1), e2 = sw4_tblexp(zb2, em2);
    // sw2_rt_core with the clamp and the degenerate-denominator case as selects
    const float eps1 = 1.0e-8f;
    const float zrpp = fabsf(p.zrpp) < eps1 ? (p.zrpp < 0 ? -eps1 : eps1) : p.zrpp;
    const float g1 = p.g1, g2 = p.g2, g3 = p.g3, g4 = p.g4, zrk = p.zrk, zrp = p.zrp;
    const float za1 = g1 * g4 + g2 * g3, za2 = g1 * g3 + g2 * g4;
    const float e11 = e1 * e1, em11 = em1 * (2.0f - em1);
    const float B = zrk * (1.0f + e11) + g1 * em11;
    const float D = zrpp * B;
    const bool degen = D >= -eps1 * e1 && D <= eps1 * e1;
    const float q = p.zssa1 / D;
    const float nr = em11 * (za2 - zrk * g3 * zrp) + zrk * (g3 - za2 * cz) * (em1 * em1 + 2.0f * e1 * em2);
    const float nt = zrk * (g4 + za1 * cz) * (2.0f * e1 * em2 - e2 * em1 * em1) - e2 * em11 * (za1 + zrk * g4 * zrp);
    r.rb = degen ? eps1 : fmaxf(0.0f, fminf(1.0f, nr * q));
    r.tb = degen ? e2 : fmaxf(0.0f, fminf(1.0f, e2 + nt * q));
    r.rd = fmaxf(0.0f, fminf(1.0f, g2 * em11 / B));
    r.td = fmaxf(0.0f, fminf(1.0f, 2.0f * zrk * e1 / B));
    r.e3 = sw4_tblexp(p.ztau1 * snt, em);
    r.e4 = sw4_tblexp(zb4, em);
}

// The column image handed from the gas-optics kernel to the R/T kernel: SwSh2 from colmol to its end (taug last)
// and, with aerosol, the aerosol block after it, rounded up to 16-byte units.
__host__ __device__ constexpr size_t sw4_image_begin() { return offsetof(SwSh2, colmol); }
__host__ __device__ constexpr size_t sw4_image_bytes(bool aer)
{
    return ((sizeof(SwSh2) - sw4_image_begin() + (aer ? sizeof(SwAer) : 0)) + 15) / 16 * 16;
}
static_assert(offsetof(SwSh2, colmol) % 16 == 0, "the image starts on a 16-byte boundary");
static_assert(offsetof(SwSh2, taug) + sizeof(SwSh2::taug) == sizeof(SwSh2) && sizeof(SwAer) % 16 == 0,
              "taug closes SwSh2 and the aerosol block is whole 16-byte units");
// Shared memory of the gas-optics kernel: SwSh2 up to taug (taug goes to the image directly), the aerosol block
// where taug would be.
__host__ __device__ constexpr size_t sw4_gas_smem(bool aer) { return offsetof(SwSh2, taug) + (aer ? sizeof(SwAer) : 0); }

// The image's taug part holds the gas optical depths as [layer][g-point]: the R/T kernel reads them straight from
// the image, 32 consecutive (layer, g-point) tasks per warp on one 128-byte line, instead of staging them.
static_assert((size_t)NLAY_MAX * SW_NGPT * sizeof(float) <= sizeof(SwSh2::taug), "[layer][g] fits the taug part");
__host__ __device__ inline const float* sw4_image_taug(const int4* im)
{
    return reinterpret_cast<const float*>(reinterpret_cast<const unsigned char*>(im) + (offsetof(SwSh2, taug) - sw4_image_begin()));
}

// Set-up, cloud optics and gas optics of one sunlit column (one CTA, six per SM) into its image.
__global__ void __launch_bounds__(SW4_GAS_THREADS, SW4_GAS_MINB)
sw4_gas_kernel(const __grid_constant__ SwBatch bt, int any_aer, int* err, int d0, int4* img)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SwSh2& s = *reinterpret_cast<SwSh2*>(smem_raw);
    const int d = d0 + (int)blockIdx.x;
    if (d >= *bt.req[0].nday) return;
    const int64_t gcol = bt.req[0].daycol[d];
    const int rq = bt.find(gcol);
    const SwIn& a = bt.req[rq];
    const int nlay = a.nlay;
    if (nlay > NLAY_MAX) {
        if (threadIdx.x == 0) atomicExch(err, RAD_DEV_NLAY);
        return;
    }
    SwAer* aer = a.faersw ? reinterpret_cast<SwAer*>(smem_raw + offsetof(SwSh2, taug)) : nullptr;
    const int64_t col = gcol - bt.off[rq];
    const int tid = threadIdx.x;
    int4* im = img + (size_t)blockIdx.x * (sw4_image_bytes(any_aer) / 16);
    float* img_taug = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(im) + (offsetof(SwSh2, taug) - sw4_image_begin()));
    sw2_setup<SW4_GAS_THREADS>(s, aer, a, col, d, tid);
    for_each_band_flat(c_sw_ns, 14, nlay, &s.task_next, tid & 31, [&](int g, int k0, int b) {
        float tg, tr;
        sw_gas<float>(s, g, k0, tg, tr, b);
        img_taug[k0 * SW_NGPT + g] = tg;
        if (g >= 66 && g < 74 && k0 < s.laytrop) s.taur24[g - 66][k0] = tr;
    });
    __syncthreads();
    const int4* sm = reinterpret_cast<const int4*>(smem_raw + sw4_image_begin());
    const int n1 = (int)((offsetof(SwSh2, taug) - sw4_image_begin()) / 16);
    const int n2 = any_aer ? (int)(sizeof(SwAer) / 16) : 0;
    const int skip = (int)(sizeof(SwSh2::taug) / 16);
    for (int i = tid; i < n1 + n2; i += SW4_GAS_THREADS) im[i < n1 ? i : i + skip] = sm[i];
}

__global__ void __launch_bounds__(SW4_RT_THREADS, SW4_OPT_MINB)
sw4_rt_kernel(const __grid_constant__ SwBatch bt, int any_aer, const float* ex, const double* exd, int d0,
              const int4* img, unsigned char* scr, size_t blk_bytes)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SwSh2& s = *reinterpret_cast<SwSh2*>(smem_raw);
    __shared__ signed char slot[NLAY_MAX];
    const int d = d0 + (int)blockIdx.x;
    if (d >= *bt.req[0].nday) return;
    const int64_t gcol = bt.req[0].daycol[d];
    const int rq = bt.find(gcol);
    const SwIn& a = bt.req[rq];
    const int nlay = a.nlay;
    if (nlay > NLAY_MAX) return;                                   // flagged by the gas-optics kernel
    SwAer* aer = a.faersw ? reinterpret_cast<SwAer*>(smem_raw + offsetof(SwSh2, taug)) : nullptr;
    const int64_t col = gcol - bt.off[rq];
    const int tid = threadIdx.x;
    const int4* im = img + (size_t)blockIdx.x * (sw4_image_bytes(any_aer) / 16);
    const float* tgi = sw4_image_taug(im);   // [layer][g], read from the image as the tasks need it
    if (SW4_L2PF && tid == 0) l2_prefetch(tgi, (uint32_t)(nlay * SW_NGPT * sizeof(float)));
    {   // the rest of the image into shared memory (the aerosol block where taug would be), every 16-byte piece
        // in flight at once (cp.async.cg: L2 to shared)
        const uint32_t sb = (uint32_t)__cvta_generic_to_shared(smem_raw + sw4_image_begin());
        const int n1 = (int)((offsetof(SwSh2, taug) - sw4_image_begin()) / 16);
        const int n2 = any_aer ? (int)(sizeof(SwAer) / 16) : 0;
        const int skip = (int)(sizeof(SwSh2::taug) / 16);
        for (int i = tid; i < n1 + n2; i += SW4_RT_THREADS)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sb + 16u * (uint32_t)i),
                         "l"(im + (i < n1 ? i : i + skip))
                         : "memory");
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();
    }
    unsigned char* blk = scr + (size_t)blockIdx.x * blk_bytes;
    Sw4Hdr& H = *reinterpret_cast<Sw4Hdr*>(blk);
    float* rtc = reinterpret_cast<float*>(blk + sw4_hdr_bytes());
    float* rto = rtc + (size_t)nlay * SW4_LAYER;
    const bool mc = a.mask != nullptr;
    const bool cloudy = mc ? s.zcf1 > 0.0f : s.zcf1 > 1.0e-6f;
    // the queue of (layer, g-point) tasks whose float64 work is left for the pass after the R/T (the level-sum
    // scratch fn is not used by this kernel): count, then entries k0 * SW_NGPT + g
    int* qn = reinterpret_cast<int*>(&s.fn[0][0]);
    int* qe = qn + 1;
    constexpr int QCAP = (int)(sizeof(SwSh2::fn) / sizeof(int)) - 1;
    if (tid == 0) {
        int n = 0;
        for (int k0 = 0; k0 < nlay; ++k0) {
            const bool cl = cloudy && s.cldfrc[k0] > 1.0e-12f;
            slot[k0] = cl ? (signed char)n : (signed char)-1;
            H.slot[k0] = slot[k0];
            n += cl ? 1 : 0;
        }
        H.ncl = n;
        H.cloudy = cloudy ? 1 : 0;
        H.albbm[0] = s.albbm[0]; H.albbm[1] = s.albbm[1];
        H.albdf[0] = s.albdf[0]; H.albdf[1] = s.albdf[1];
        H.zcf0 = s.zcf0; H.zcf1 = s.zcf1;
        *qn = 0;
    }
    for (int k0 = tid; k0 < nlay; k0 += SW4_RT_THREADS) H.rdelp[k0] = s.rdelp[k0];
    for (int g = tid; g < SW_NGPT; g += SW4_RT_THREADS) H.zsolar[g] = s.ssolar * s.sfluxzen[g];
    __syncthreads();
    const float cz = s.cosz, snt = s.sntz;
    const double czd = (double)__ldg(a.coszen + col);
    __shared__ unsigned char gband[SW_NGPT];
    for (int g = tid; g < SW_NGPT; g += SW4_RT_THREADS) {
        int ib = 0;
        while (g >= c_sw_ns[ib + 1]) ++ib;
        gband[g] = (unsigned char)ib;
    }
    __syncthreads();
    auto store = [&](int k0, int g, const SwLayerRT2& L) {
        float* pc = rtc + (size_t)k0 * SW4_LAYER + g;
        pc[0] = L.c.rb; pc[SW_NGPT] = L.c.rd; pc[2 * SW_NGPT] = L.c.tb; pc[3 * SW_NGPT] = L.c.td;
        pc[4 * SW_NGPT] = L.c.e3; pc[5 * SW_NGPT] = L.c.e4;
        const int sl = slot[k0];
        if (sl >= 0) {
            float* po = rto + (size_t)sl * SW4_LAYER + g;
            po[0] = L.o.rb; po[SW_NGPT] = L.o.rd; po[2 * SW_NGPT] = L.o.tb; po[3 * SW_NGPT] = L.o.td;
            po[4 * SW_NGPT] = L.o.e3; po[5 * SW_NGPT] = L.o.e4;
        }
    };
    // the complete layer function (sw2_layer, float64 steps included) for task i = k0 * SW_NGPT + g
    auto full = [&](int i) {
        const int k0 = i / SW_NGPT, g = i - k0 * SW_NGPT, ib = gband[g];
        const float zsolar = s.ssolar * s.sfluxzen[g];
        const SwExactCtx x{&a, col, s.laytrop, s.kmin8, s.kminw, a.iswmode, czd, 1.0 / czd, exd,
                           zsolar * (1.5f * 86400.0f / SW2_HEAT_T), zsolar * (1.0f / SW2_FLUX_T)};
        store(k0, g, sw2_layer(s, aer, x, k0, g, ib, cloudy, mc, cz, snt, ex, __ldg(tgi + i)));
    };
    // ---- layer R/T in two passes over the column, each with lanes on 32 consecutive (layer, g-point) tasks and
    // two tasks per thread side by side; a task whose R/T needs a float64 step or a table-entry test is queued
    // (qbit marks it) and formed afterwards by sw2_layer, one per thread
    __shared__ unsigned qbit[NLAY_MAX][4];
    __shared__ signed char slotk[NLAY_MAX];
    for (int j = tid; j < NLAY_MAX * 4; j += SW4_RT_THREADS) qbit[j >> 2][j & 3] = 0u;
    if (tid < nlay && slot[tid] >= 0) slotk[slot[tid]] = (signed char)tid;
    __syncthreads();
    const int ncl = H.ncl;
    auto enqueue = [&](int i) {
        const int k0 = i / SW_NGPT, g = i - k0 * SW_NGPT;
        if (atomicOr(&qbit[k0][g >> 5], 1u << (g & 31)) & (1u << (g & 31))) return;   // queued already
        const int j = atomicAdd(qn, 1);
        if (j < QCAP) qe[j] = i;
        else full(i);
    };
    // clear-pass inputs of task i
    auto inputs = [&](int i, float& t0, float& ab, float& s0, float& y0, int& ib) {
        const int k0 = i / SW_NGPT, g = i - k0 * SW_NGPT;
        ib = gband[g];
        const float tr = sw2_taur(s, g, k0), tg = __ldg(tgi + i);
        float ta = 0, tasa = 0, tay = 0, taab = 0;
        if (aer) { ta = aer->tau[ib][k0]; tasa = aer->tasa[ib][k0]; tay = aer->tay[ib][k0]; taab = aer->tabs[ib][k0]; }
        t0 = fmaxf(1.0e-12f, tr + tg + ta); s0 = tr + tasa; y0 = tay; ab = tg + taab;
    };
    auto weights = [&](int i, float& wk, float& wf) {
        const int k0 = i / SW_NGPT, g = i - k0 * SW_NGPT;
        const float zsolar = s.ssolar * s.sfluxzen[g];
        wf = zsolar * (1.0f / SW2_FLUX_T);
        wk = zsolar * (1.5f * 86400.0f / SW2_HEAT_T) * (float)s.rdelp[k0];
    };
    auto put = [&](float* base, int i, const SwLayerRT& r) {
        float* p = base + i;   // i = k0 * SW_NGPT + g indexes [layer][g]; fields are SW_NGPT apart
        const int k0 = i / SW_NGPT;
        p += (size_t)k0 * (SW4_LAYER - SW_NGPT);
        p[0] = r.rb; p[SW_NGPT] = r.rd; p[2 * SW_NGPT] = r.tb; p[3 * SW_NGPT] = r.td; p[4 * SW_NGPT] = r.e3;
        p[5 * SW_NGPT] = r.e4;
    };
    auto run = [&](auto mode_tag) {
        constexpr int MODE = decltype(mode_tag)::value;
        const int nt = nlay * SW_NGPT;
        // clear pass
        if constexpr (!SW4_RT_PAIR) {
            for (int i0 = tid; i0 < nt; i0 += SW4_RT_THREADS) {
                float t0a, aba, s0a, y0a, wka, wfa;
                int iba;
                inputs(i0, t0a, aba, s0a, y0a, iba);
                weights(i0, wka, wfa);
                SwLayerRT ra;
                bool oka;
                sw4_rt<MODE>(t0a, aba, s0a, y0a, cz, snt, wka, wfa, ra, oka);
                put(rtc, i0, ra);
                if (!oka) enqueue(i0);
            }
        }
        for (int i0 = tid; SW4_RT_PAIR && i0 < nt; i0 += 2 * SW4_RT_THREADS) {
            const int i1 = min(i0 + SW4_RT_THREADS, nt - 1);
            float t0a, aba, s0a, y0a, t0b, abb, s0b, y0b, wka, wfa, wkb, wfb;
            int iba, ibb;
            inputs(i0, t0a, aba, s0a, y0a, iba);
            inputs(i1, t0b, abb, s0b, y0b, ibb);
            weights(i0, wka, wfa);
            weights(i1, wkb, wfb);
            SwLayerRT ra, rb;
            bool oka, okb;
            sw4_rt<MODE>(t0a, aba, s0a, y0a, cz, snt, wka, wfa, ra, oka);
            sw4_rt<MODE>(t0b, abb, s0b, y0b, cz, snt, wkb, wfb, rb, okb);
            put(rtc, i0, ra);
            if (!oka) enqueue(i0);
            if (i0 + SW4_RT_THREADS < nt) {
                put(rtc, i1, rb);
                if (!okb) enqueue(i1);
            }
        }
        __syncthreads();
        // cloudy pass: the layers with a slot, mixture R/T blended with the clear R/T (or, McICA, taken
        // unblended where the g-point's sub-column bit is set)
        const int nc2 = ncl * SW_NGPT;
        auto mix = [&](int j, SwLayerRT& o, bool& ok, int& i) {
            const int sl = j / SW_NGPT, g = j - sl * SW_NGPT, k0 = slotk[sl];
            i = k0 * SW_NGPT + g;
            float t0, ab, s0, y0, wk, wf;
            int ib;
            inputs(i, t0, ab, s0, y0, ib);
            weights(i, wk, wf);
            const float* pc = rtc + (size_t)k0 * SW4_LAYER + g;
            SwLayerRT c;
            c.rb = pc[0]; c.rd = pc[SW_NGPT]; c.tb = pc[2 * SW_NGPT]; c.td = pc[3 * SW_NGPT]; c.e3 = pc[4 * SW_NGPT];
            c.e4 = pc[5 * SW_NGPT];
            const bool bit = !mc || ((s.mcw[g >> 5][k0] >> (g & 31)) & 1u);
            SwLayerRT m;
            sw4_rt<MODE>(t0 + s.taucw[ib][k0], ab + s.tabsc[ib][k0], s0 + s.ssacw[ib][k0], y0 + s.asycw[ib][k0], cz,
                         snt, wk, wf, m, ok);
            ok = ok || !bit;
            if (!bit) {
                o = c;
            } else if (mc) {
                o = m;
            } else {
                const float zc1 = s.cldfrc[k0], zc0 = 1.0f - zc1;
                o.rb = zc0 * c.rb + zc1 * m.rb;
                o.rd = zc0 * c.rd + zc1 * m.rd;
                o.tb = zc0 * c.tb + zc1 * m.tb;
                o.td = zc0 * c.td + zc1 * m.td;
                o.e3 = zc0 * c.e3 + zc1 * m.e3;
                o.e4 = zc0 * c.e4 + zc1 * m.e4;
            }
        };
        if constexpr (!SW4_RT_PAIR) {
            for (int j0 = tid; j0 < nc2; j0 += SW4_RT_THREADS) {
                SwLayerRT oa;
                bool oka;
                int ia;
                mix(j0, oa, oka, ia);
                const int k0 = ia / SW_NGPT, g = ia - k0 * SW_NGPT;
                if (!(qbit[k0][g >> 5] & (1u << (g & 31)))) {
                    put(rto, (int)(slot[k0]) * SW_NGPT + g, oa);
                    if (!oka) enqueue(ia);
                }
            }
        }
        for (int j0 = tid; SW4_RT_PAIR && j0 < nc2; j0 += 2 * SW4_RT_THREADS) {
            const int j1 = min(j0 + SW4_RT_THREADS, nc2 - 1);
            SwLayerRT oa, ob;
            bool oka, okb;
            int ia, ib_;
            mix(j0, oa, oka, ia);
            mix(j1, ob, okb, ib_);
            {
                const int k0 = ia / SW_NGPT, g = ia - k0 * SW_NGPT;
                if (!(qbit[k0][g >> 5] & (1u << (g & 31)))) {
                    put(rto, (int)(slot[k0]) * SW_NGPT + g, oa);
                    if (!oka) enqueue(ia);
                }
            }
            if (j0 + SW4_RT_THREADS < nc2) {
                const int k0 = ib_ / SW_NGPT, g = ib_ - k0 * SW_NGPT;
                if (!(qbit[k0][g >> 5] & (1u << (g & 31)))) {
                    put(rto, (int)(slot[k0]) * SW_NGPT + g, ob);
                    if (!okb) enqueue(ib_);
                }
            }
        }
    };
    if (a.iswmode == 1) run(std::integral_constant<int, 1>{});
    else if (a.iswmode == 2) run(std::integral_constant<int, 2>{});
    else run(std::integral_constant<int, 3>{});
    __syncthreads();
    // ---- the queued tasks with their float64 steps, one per thread
    const int nq = min(*qn, QCAP);
    for (int j = tid; j < nq; j += SW4_RT_THREADS) full(qe[j]);
}

// Per-g-point level fluxes of one sunlit column for swrad's optional outputs (DIAG sweeps):
// [nlay + 1][SW4_PGQ][SW_NGPT] floats at level L (surface first), each x zsolar: up total, down total, up clear,
// down clear, net (down - up) total, net clear.
constexpr int SW4_PGQ = 6;
__host__ __device__ constexpr int64_t sw4_pg_floats(int nlay) { return (int64_t)(nlay + 1) * SW4_PGQ * SW_NGPT; }

// One level of the DIAG profile of g-point g (see sw4_pg_floats): clear fluxes fu / fd, cloudy-pass fuo / fdo,
// pass weights w0 / w1 and the sweep's net total.
__device__ __forceinline__ void sw4_pg_level(float* pg, int L, int g, float zsolar, bool cloudy, double w0, double w1,
                                             float fu, float fd, float fuo, float fdo, double net)
{
    const double zs = (double)zsolar;
    float* p = pg + (size_t)L * SW4_PGQ * SW_NGPT + g;
    p[0] = (float)(zs * (cloudy ? w0 * fu + w1 * fuo : (double)fu));
    p[SW_NGPT] = (float)(zs * (cloudy ? w0 * fd + w1 * fdo : (double)fd));
    p[2 * SW_NGPT] = (float)(zs * fu);
    p[3 * SW_NGPT] = (float)(zs * fd);
    p[4 * SW_NGPT] = (float)(zs * net);
    p[5 * SW_NGPT] = (float)(zs * ((double)fd - (double)fu));
}

// The adding method of one sunlit column from its block (sw2_column phase C with the R/T read instead of
// formed; the same operations in the same order).
template <bool DIAG = false>
__global__ void __launch_bounds__(SW2_THREADS, SW4_SWEEP_MINB)
sw4_sweep_kernel(const __grid_constant__ SwBatch bt, int* err, int d0, int nc, const unsigned char* scr,
                 size_t blk_bytes, float* __restrict__ pg = nullptr)
{
    extern __shared__ __align__(16) float ckpt[];                  // [(nseg - 1) x 4][SW2_THREADS]
    __shared__ __align__(16) Sw4Hdr H;
    __shared__ double fn[SW2_WARPS][NLAY_MAX + 2];
    __shared__ double scs[SW2_WARPS][18];
    const int i = (int)blockIdx.x;
    const int d = d0 + i;
    if (i >= nc || d >= *bt.req[0].nday) return;
    const int64_t gcol = bt.req[0].daycol[d];
    const int rq = bt.find(gcol);
    const SwIn& a = bt.req[rq];
    const int nlay = a.nlay, nlp1 = nlay + 1;
    if (nlay > NLAY_MAX) return;                                   // flagged by the optics kernel
    const int64_t N = a.ncol;
    const int64_t col = gcol - bt.off[rq];
    const int tid = threadIdx.x;
    const unsigned char* blk = scr + (size_t)i * blk_bytes;
    {
        const int4* src = reinterpret_cast<const int4*>(blk);
        int4* dst = reinterpret_cast<int4*>(&H);
        for (int j = tid; j < (int)(sizeof(Sw4Hdr) / 16); j += SW2_THREADS) dst[j] = __ldg(src + j);
    }
    __syncthreads();
    const float* rtc = reinterpret_cast<const float*>(blk + sw4_hdr_bytes());
    const float* rto = rtc + (size_t)nlay * SW4_LAYER;
    if (DIAG) pg += (int64_t)i * sw4_pg_floats(nlay);
    const int warp = tid >> 5, lane = tid & 31;
    bool act;
    const int g = sw2_lane_g(tid, act);
    int ib0 = 0;
    while (g >= c_sw_ns[ib0 + 1]) ++ib0;
    const int ibd = ib0 == 8 ? 0 : ((ib0 >= 9 && ib0 <= 12) ? 2 : 1);   // idxsfc
    const bool mc = a.mask != nullptr;
    const bool cloudy = H.cloudy != 0;
    const float zsolar = act ? H.zsolar[g] : 0.0f;
    const float ab = ibd ? H.albbm[ibd - 1] : 0.5f * (H.albbm[0] + H.albbm[1]);
    const float ad = ibd ? H.albdf[ibd - 1] : 0.5f * (H.albdf[0] + H.albdf[1]);
    const int nseg = (nlay + SW2_SEG - 1) / SW2_SEG;
    float* ck = ckpt + tid;
    auto CK = [&](int sg, int q) -> float& { return ck[((sg - 1) * 4 + q) * SW2_THREADS]; };
    // R/T of layer k0, both passes (transparent padding above the model top)
    auto load = [&](int k0, SwLayerRT& c, SwLayerRT& o) {
        if (k0 >= nlay) {
            c.rb = 0; c.rd = 0; c.tb = 1; c.td = 1; c.e3 = 1; c.e4 = 1;
            o = c;
            return;
        }
        const float* p = rtc + (size_t)k0 * SW4_LAYER + g;
        c.rb = __ldg(p); c.rd = __ldg(p + SW_NGPT); c.tb = __ldg(p + 2 * SW_NGPT); c.td = __ldg(p + 3 * SW_NGPT);
        c.e3 = __ldg(p + 4 * SW_NGPT); c.e4 = __ldg(p + 5 * SW_NGPT);
        const int sl = H.slot[k0];
        if (cloudy && sl >= 0) {
            const float* q = rto + (size_t)sl * SW4_LAYER + g;
            o.rb = __ldg(q); o.rd = __ldg(q + SW_NGPT); o.tb = __ldg(q + 2 * SW_NGPT); o.td = __ldg(q + 3 * SW_NGPT);
            o.e3 = __ldg(q + 4 * SW_NGPT); o.e4 = __ldg(q + 5 * SW_NGPT);
        } else {
            o = c;
        }
    };
    // The R/T rows of segment sg into L2 ahead of its loads (thread 0, one bulk prefetch per pass): the clear rows
    // of its layers and the cloudy rows of their slots, each a contiguous run inside the column's block.
    auto prefetch = [&](int sg) {
        if (!SW4_L2PF || tid != 0 || sg < 0 || sg >= nseg) return;
        const int k0 = sg * SW2_SEG, k1 = min(nlay, k0 + SW2_SEG);
        if (k0 >= k1) return;
        l2_prefetch(rtc + (size_t)k0 * SW4_LAYER, (uint32_t)((k1 - k0) * SW4_LAYER * sizeof(float)));
        if (!cloudy) return;
        int s0 = -1, s1 = -1;
        for (int k = k0; k < k1; ++k)
            if (H.slot[k] >= 0) { if (s0 < 0) s0 = H.slot[k]; s1 = H.slot[k]; }
        if (s0 >= 0) l2_prefetch(rto + (size_t)s0 * SW4_LAYER, (uint32_t)((s1 - s0 + 1) * SW4_LAYER * sizeof(float)));
    };
    // ---- upward sweep: reflectances of the atmosphere below each level, clear (c) and cloudy (o) passes
    float ubc = ab, udc = ad, ubo = ab, udo = ad;
    prefetch(0);
    prefetch(1);
    for (int sg = 0; sg < nseg; ++sg) {
        prefetch(sg + 2);
        if (sg > 0) { CK(sg, 0) = ubc; CK(sg, 1) = udc; CK(sg, 2) = ubo; CK(sg, 3) = udo; }
        SwLayerRT Lc[SW2_SEG], Lo[SW2_SEG];
#pragma unroll
        for (int j = 0; j < SW2_SEG; ++j) load(sg * SW2_SEG + j, Lc[j], Lo[j]);
#pragma unroll
        for (int j = 0; j < SW2_SEG; ++j) {
            sw2_up(Lc[j], ubc, udc);
            if (cloudy) sw2_up(Lo[j], ubo, udo);
        }
    }
    // ---- downward sweep, segment by segment from the top: the segment's R/T again, its upward states from
    // the checkpoint, then the walk down through it
    const double w0 = cloudy ? (mc ? 0.0 : (double)H.zcf0) : 1.0, w1 = cloudy ? (mc ? 1.0 : (double)H.zcf1) : 0.0;
    float tdnc = 1, rdnc = 0, tdbc = 1, tdbc0 = 1, tdno = 1, rdno = 0, tdbo = 1, tdbo0 = 1;
    float toa_c = 0, toa_o = 0;
    prefetch(nseg - 2);
    for (int sg = nseg - 1; sg >= 0; --sg) {
        prefetch(sg - 2);
        SwLayerRT Lc[SW2_SEG], Lo[SW2_SEG];
        float zubc[SW2_SEG + 1], zudc[SW2_SEG + 1], zubo[SW2_SEG + 1], zudo[SW2_SEG + 1];
        zubc[0] = sg ? CK(sg, 0) : ab;
        zudc[0] = sg ? CK(sg, 1) : ad;
        zubo[0] = sg ? CK(sg, 2) : ab;
        zudo[0] = sg ? CK(sg, 3) : ad;
#pragma unroll
        for (int j = 0; j < SW2_SEG; ++j) load(sg * SW2_SEG + j, Lc[j], Lo[j]);
        float e4c = 1, e4o = 1;
#pragma unroll
        for (int j = 0; j < SW2_SEG; ++j) {
            e4c = e4c * Lc[j].e4;
            if (cloudy) e4o = e4o * Lo[j].e4;
            zubc[j + 1] = zubc[j]; zudc[j + 1] = zudc[j];
            sw2_up(Lc[j], zubc[j + 1], zudc[j + 1]);
            if (cloudy) {
                zubo[j + 1] = zubo[j]; zudo[j + 1] = zudo[j];
                sw2_up(Lo[j], zubo[j + 1], zudo[j + 1]);
            }
        }
#pragma unroll
        for (int j = SW2_SEG - 1; j >= 0; --j) {
            const int lev = sg * SW2_SEG + j + 2;        // level above layer j (1 = surface)
            if (lev <= nlp1) {
                float fu, fd, fuo = 0, fdo = 0;
                sw2_flux(zubc[j + 1], zudc[j + 1], tdnc, rdnc, tdbc, fu, fd);
                double net = w0 * ((double)fd - (double)fu);
                if (lev == nlp1) toa_c = fu;
                if (cloudy) {
                    sw2_flux(zubo[j + 1], zudo[j + 1], tdno, rdno, tdbo, fuo, fdo);
                    net += w1 * ((double)fdo - (double)fuo);
                    if (lev == nlp1) toa_o = fuo;
                }
                const double v = warp_sum(act ? (double)zsolar * net : 0.0);
                if (lane == 0) fn[warp][lev - 1] = v;
                if (DIAG && act) sw4_pg_level(pg, lev - 1, g, zsolar, cloudy, w0, w1, fu, fd, fuo, fdo, net);
            }
            sw2_down(Lc[j], tdnc, rdnc, tdbc);
            if (cloudy) sw2_down(Lo[j], tdno, rdno, tdbo);
        }
        tdbc0 = tdbc0 * e4c;
        tdbo0 = tdbo0 * e4o;
    }
    // ---- surface level, the per-lane scalars (zero for idle lanes), column end and swrad_post
    double scv[18];
#pragma unroll
    for (int q = 0; q < 18; ++q) scv[q] = 0;
    {
        float fu, fd, fuo = 0, fdo = 0;
        sw2_flux(ab, ad, tdnc, rdnc, tdbc, fu, fd);
        double net = w0 * ((double)fd - (double)fu);
        if (cloudy) {
            sw2_flux(ab, ad, tdno, rdno, tdbo, fuo, fdo);
            net += w1 * ((double)fdo - (double)fuo);
        }
        const double v = warp_sum(act ? (double)zsolar * net : 0.0);
        if (lane == 0) fn[warp][0] = v;
        if (DIAG && act) sw4_pg_level(pg, 0, g, zsolar, cloudy, w0, w1, fu, fd, fuo, fdo, net);
        if (act) {
            const double zs = (double)zsolar;
            // slots: 0 toa up, 1 sfc up, 2 sfc dn, 3 uv-b, 4 nir beam, 5 nir diffuse, 6 vis beam, 7 vis diffuse, 8 toa down
            auto fill = [&](double* o, float tu, float su, float sd, float sdir) {
                o[0] = zs * (double)tu;
                o[1] = zs * (double)su;
                o[2] = zs * (double)sd;
                o[3] = ib0 == 11 ? zs * (double)sd : 0.0;
                const double zb1 = (double)(zsolar * sdir), zb2 = (double)(zsolar * (sd - sdir));
                if (ibd == 1) { o[4] = zb1; o[5] = zb2; }
                else if (ibd == 2) { o[6] = zb1; o[7] = zb2; }
                else { o[4] = 0.5 * zb1; o[5] = 0.5 * zb2; o[6] = 0.5 * zb1; o[7] = 0.5 * zb2; }
                o[8] = zs;
            };
            fill(scv, toa_c, fu, fd, tdbc0);
            if (cloudy) fill(scv + 9, toa_o, fuo, fdo, tdbo0);
        }
    }
#pragma unroll
    for (int q = 0; q < 18; ++q) {
        const double v = warp_sum(scv[q]);
        if (lane == 0) scs[warp][q] = v;
    }
    __syncthreads();
    auto tot = [&](double clr, double cld) { return cloudy ? w1 * cld + w0 * clr : clr; };
    for (int k = tid; k < nlay; k += SW2_THREADS) {
        double f0 = 0, f1 = 0;
        for (int w = 0; w < SW2_WARPS; ++w) { f0 += fn[w][k]; f1 += fn[w][k + 1]; }
        a.htsw[(size_t)(nlay - 1 - k) * N + col] = (float)((f1 - f0) * H.rdelp[k]);
    }
    if (tid == 0) {
        double c[9], t[9];
        for (int q = 0; q < 9; ++q) {
            c[q] = 0; t[q] = 0;
            for (int w = 0; w < SW2_WARPS; ++w) { c[q] += scs[w][q]; t[q] += scs[w][9 + q]; }
        }
        a.topfsw[col] = (float)tot(c[0], t[0]);
        a.topfsw[N + col] = (float)c[8];
        a.topfsw[2 * N + col] = (float)c[0];
        a.sfcfsw[col] = (float)tot(c[1], t[1]);
        a.sfcfsw[N + col] = (float)tot(c[2], t[2]);
        a.sfcfsw[2 * N + col] = (float)c[1];
        a.sfcfsw[3 * N + col] = (float)c[2];
        if (a.fdncmp) {
            a.fdncmp[col] = (float)c[3];
            a.fdncmp[N + col] = (float)tot(c[3], t[3]);
            a.fdncmp[2 * N + col] = (float)tot(c[4], t[4]);
            a.fdncmp[3 * N + col] = (float)tot(c[5], t[5]);
            a.fdncmp[4 * N + col] = (float)tot(c[6], t[6]);
            a.fdncmp[5 * N + col] = (float)tot(c[7], t[7]);
        }
    }
    (void)err;
}

// swrad's optional outputs of a chunk from the DIAG sweeps' profiles (swrad_post's lhsw0 / lhswb / lflxprf
// blocks): one warp per sunlit column, lane q < 14 band q (htswb from the band's net fluxes), lane 14 the totals
// (swflxprf, hsw0 from the clear net fluxes).  Sums over g-points in float64 in g order; heating
// (F(k + 1) - F(k)) heatfac / delp as the sweeps form htsw.
__global__ void __launch_bounds__(128) k_sw_diag(const __grid_constant__ SwBatch bt, int d0, int nc,
                                                 const unsigned char* scr, size_t blk_bytes,
                                                 const float* __restrict__ pg, const __grid_constant__ DiagOuts outs)
{
    const int i = (int)blockIdx.x * 4 + (threadIdx.x >> 5);
    const int q = threadIdx.x & 31;
    const int d = d0 + i;
    if (i >= nc || q > 14 || d >= *bt.req[0].nday) return;
    const int64_t gcol = bt.req[0].daycol[d];
    const int rq = bt.find(gcol);
    const SwIn& a = bt.req[rq];
    const int nlay = a.nlay, nlp1 = nlay + 1;
    if (nlay > NLAY_MAX) return;
    const int64_t col = gcol - bt.off[rq], N = a.ncol;
    const Sw4Hdr& H = *reinterpret_cast<const Sw4Hdr*>(scr + (size_t)i * blk_bytes);
    const float* p = pg + (int64_t)i * sw4_pg_floats(nlay);
    float* hsw0 = outs.p[rq][3];
    float* htswb = outs.p[rq][4];
    float* flx = outs.p[rq][5];
    const int g0 = q < 14 ? c_sw_ns[q] : 0, g1 = q < 14 ? c_sw_ns[q + 1] : SW_NGPT;
    auto S = [&](int L, int f) {
        double v = 0.0;
        for (int g = g0; g < g1; ++g) v += (double)p[((size_t)L * SW4_PGQ + f) * SW_NGPT + g];
        return v;
    };
    if (q < 14) {
        if (htswb) {
            double f0 = S(0, 4);
            for (int k0 = 0; k0 < nlay; ++k0) {
                const double f1 = S(k0 + 1, 4);
                htswb[((size_t)q * nlay + (nlay - 1 - k0)) * N + col] = (float)((f1 - f0) * H.rdelp[k0]);
                f0 = f1;
            }
        }
        return;
    }
    if (hsw0) {
        double f0 = S(0, 5);
        for (int k0 = 0; k0 < nlay; ++k0) {
            const double f1 = S(k0 + 1, 5);
            hsw0[(size_t)(nlay - 1 - k0) * N + col] = (float)((f1 - f0) * H.rdelp[k0]);
            f0 = f1;
        }
    }
    if (flx)
        for (int L = 0; L < nlp1; ++L)
            for (int f = 0; f < 4; ++f) flx[((size_t)f * nlp1 + (nlp1 - 1 - L)) * N + col] = (float)S(L, f);
}

}  // namespace rad
