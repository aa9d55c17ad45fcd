// rad_common.cuh -- device-side pieces shared by the LW and SW column kernels.
//
// Tables: every packed RRTM table lives in one float32 and one float64 device buffer; the offset of each
// table (by RadTableId) is published in constant memory, so a kernel instantiated for float reads the
// float32 copy and one instantiated for double reads the float64 copy, with the same index arithmetic.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "rad_tabids.h"

namespace rad {

constexpr int NLAY_MAX = 64;        // per-thread sweep arrays are sized for this many layers
constexpr int LW_NGPT = 140, SW_NGPT = 112;

__constant__ int64_t c_toff[T_COUNT];
__constant__ const float* c_tf;
__constant__ const double* c_td;

// Scalars the reference's wrappers compute on the host (band 4, 5 and 15 reference ratios), float32.
struct LwHostConsts {
    float b4_rpa, b4_rpb, b5_rpa, b5_rpb, b5_rma, b15_r;
};
__constant__ LwHostConsts c_lwk;

template <class R> __device__ __forceinline__ const R* tab(int id);
template <> __device__ __forceinline__ const float* tab<float>(int id) { return c_tf + c_toff[id]; }
template <> __device__ __forceinline__ const double* tab<double>(int id) { return c_td + c_toff[id]; }

template <class R> __device__ __forceinline__ R ldt(const R* p) { return __ldg(p); }

// IEEE minNum/maxNum as CUDA's fminf/fmaxf: a NaN operand yields the other one.
__device__ __forceinline__ float fminR(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ float fmaxR(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double fminR(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ double fmaxR(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float rlog(float x) { return logf(x); }
__device__ __forceinline__ double rlog(double x) { return log(x); }
__device__ __forceinline__ float rexp(float x) { return expf(x); }
__device__ __forceinline__ double rexp(double x) { return exp(x); }
__device__ __forceinline__ float rpow(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double rpow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float sqrtR(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrtR(double x) { return sqrt(x); }
// MOD(x, 1.0): by fmod's definition x - n with n = trunc(x / 1) = trunc(x).  The subtraction is exact for every
// finite x (x and trunc(x) share x's exponent range and the difference is its fraction bits), and inf / NaN give
// NaN as fmod does, so this is fmod(x, 1) bit for bit -- at two instructions instead of the library's general
// remainder loop, in the per-(g-point, layer) species keys of the gas optics.
__device__ __forceinline__ float rfmod1(float x) { return x - truncf(x); }
__device__ __forceinline__ double rfmod1(double x) { return x - trunc(x); }

// ---- bulk copies into shared memory completed on an mbarrier (cp.async.bulk, no multicast) ----
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// Make the barriers' initialisation visible to the bulk-copy (async) proxy.
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Order this thread's earlier generic accesses to shared memory before the async proxy writes it.
__device__ __forceinline__ void async_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// One arrival that also expects `bytes` of bulk copies to complete the barrier's current phase.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// [dst, dst + bytes) <- [src, src + bytes): both 16-byte aligned, bytes a multiple of 16; completes on bar.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(__cvta_generic_to_global(src)), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// One bounded test of the barrier's phase `parity` (the hardware suspends the thread for a while inside).
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}
// Wait for the phase with at most `limit` tests; false when it did not complete (the caller flags and stops).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, int limit)
{
    for (int i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Bulk prefetch of [p, p + bytes) from global memory into L2 (cp.async.bulk.prefetch.L2, no shared memory, no
// multicast): one instruction brings a contiguous run of a column's scratch in ahead of the loads that read it.
// p must be 16-byte aligned and bytes a multiple of 16; the range must lie inside one allocation.
__device__ __forceinline__ void l2_prefetch(const void* p, uint32_t bytes)
{
    if (bytes == 0) return;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(__cvta_generic_to_global(p)), "r"(bytes)
                 : "memory");
}

// t(ig, ind) + frac * (t(ig, ind+1) - t(ig, ind)) for a [ind][g] table, 1-based ind.
template <class R>
__device__ __forceinline__ R interp(const R* t, int ng, int ind, int ig, R frac)
{
    const R a = ldt(t + ((ind - 1) * ng + ig)), b = ldt(t + (ind * ng + ig));   // tables < 2^31 entries
    return a + frac * (b - a);
}

// Warp sum of a double, lanes 0..31 (result valid in lane 0); a fixed tree, so bit-reproducible.
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Visit every (g-point, layer) pair of a column with the CTA's warps such that each warp works on one band
// at a time: lane l of a task of band b takes g-point ns[b] + l % ng and layer k0 + l / ng (ng = the band's
// g-point count, 32 / ng layers per task).  Neighbouring lanes then read neighbouring g entries of the
// band's [..][g] k-tables (coalesced) and take the same band branch.  Tasks are handed out in order from
// the shared counter *next (zero before the first call of the CTA), so a warp that arrives late (after
// other work) takes fewer tasks.  f(g, k0, b) runs once per pair.
template <class F>
__device__ __forceinline__ void for_each_band_pair(const int* ns, int nbands, int nlay, int* next, int lane, F f)
{
    int b = 0, t0 = 0;   // band of the current task and the index of its first task
    // the band's shape and this lane's (layer, g-point) offset in its tasks, formed when the band changes
    int ng, kpw, nt, kk, jg;
    auto shape = [&](int bb) {
        ng = ns[bb + 1] - ns[bb];
        kpw = 32 / ng;
        nt = (nlay + kpw - 1) / kpw;
        kk = lane / ng;
        jg = lane - kk * ng;
    };
    shape(0);
    // the next task is claimed while the current one runs, so the atomic's latency is hidden behind it (a warp
    // claims one id past the end before it stops; ids only grow, so no task is skipped or repeated)
    int tn = 0;
    if (lane == 0) tn = atomicAdd(next, 1);
    for (;;) {
        const int t = __shfl_sync(0xffffffffu, tn, 0);
        if (lane == 0) tn = atomicAdd(next, 1);
        while (b < nbands && t >= t0 + nt) {
            t0 += nt;
            ++b;
            if (b < nbands) shape(b);
        }
        if (b >= nbands) break;
        const int k0 = (t - t0) * kpw + kk;
        if (kk < kpw && k0 < nlay) f(ns[b] + jg, k0, b);
    }
}

// As for_each_band_pair, but a band's tasks tile its nlay * ng (layer, g-point) pairs, in [layer][g] order,
// 32 at a time: lane l of task j of band b takes pair i = 32 j + l, g-point ns[b] + i % ng, layer i / ng.  Only
// a band's last task has idle lanes, where the fixed layers-per-task mapping leaves 32 mod ng lanes idle in every
// task (a quarter of them in the 12-g-point bands): 274 tasks instead of 304 for the LW's 140 g-points on 61
// layers, 222 instead of 245 for the SW's 112 (LW -5 %, SW -2 % on the B200, same bits).  i / ng is
// (i * ceil(2^16 / ng)) >> 16, exact for ng <= 16 and i < 2^12 (checked exhaustively).
template <class F>
__device__ __forceinline__ void for_each_band_flat(const int* ns, int nbands, int nlay, int* next, int lane, F f)
{
    int b = 0, t0 = 0;   // band of the current task and the index of its first task
    int g0, ng, np, nt, mg;
    auto shape = [&](int bb) {
        g0 = ns[bb];
        ng = ns[bb + 1] - g0;
        np = ng * nlay;
        nt = (np + 31) >> 5;
        mg = (65536 + ng - 1) / ng;
    };
    shape(0);
    int tn = 0;
    if (lane == 0) tn = atomicAdd(next, 1);
    for (;;) {
        const int t = __shfl_sync(0xffffffffu, tn, 0);
        if (lane == 0) tn = atomicAdd(next, 1);
        while (b < nbands && t >= t0 + nt) {
            t0 += nt;
            ++b;
            if (b < nbands) shape(b);
        }
        if (b >= nbands) break;
        const int i = ((t - t0) << 5) + lane;
        if (i < np) {
            const int k0 = (i * mg) >> 16;
            f(g0 + (i - k0 * ng), k0, b);
        }
    }
}

// The requests of one launch (passed by value as a kernel parameter): request r covers columns
// [off[r], off[r+1]) of the launch's concatenated column space.  A CTA finds its request by bisection.
constexpr int RAD_MAXREQ = 32;
template <class In>
struct ReqBatch {
    int nreq;
    int64_t off[RAD_MAXREQ + 1];
    In req[RAD_MAXREQ];
    __device__ __forceinline__ int find(int64_t g) const
    {
        int lo = 0, hi = nreq - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (off[mid] <= g) lo = mid;
            else hi = mid - 1;
        }
        return lo;
    }
};

// Error word written by kernels on bad input (host reads it after a synchronising call).
enum : int { RAD_DEV_OK = 0, RAD_DEV_NLAY = 1, RAD_DEV_INDEX = 2, RAD_DEV_TIMEOUT = 3 };

}  // namespace rad
