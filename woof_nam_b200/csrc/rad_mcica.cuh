// rad_mcica.cuh -- McICA sub-column cloud generator for sm_100a: one warp per column.
//
// The reference runs the generator one thread per column with the 624-word MT19937 state in local memory
// (namgpu/kernels/phys_rrtm_lw_mcica_subcol.cu:48-191, phys_rrtm_sw_mcica_subcol.cu:63-203).  Here a warp
// owns a column and keeps the state in shared memory: the seeding mt[i] = seed * 69069^i (mod 2^32, the
// powers precomputed), the twist in three read-before-write phases of 32 words (MT19937's dependencies
// allow it: words 0..226 read only old words, 227..622 read words already renewed 227 places earlier,
// 623 reads the renewed words 0 and 396), the tempering and float conversion of a whole generation at once.
// Lane l owns g-points l, l+32, ...; it walks its draws generation by generation in the reference's
// consumption order (g outer, layer inner; one draw per g for maximum overlap), carrying the max-random
// recursion, and keeps its layer bits in a 64-bit word per g-point.  The packed words are assembled with
// ballots.  Output: bit g & 31 of word [g >> 5][layer][column], layers surface first -- the reference's.
#pragma once
#include "rad_common.cuh"

namespace rad {

constexpr int MC_WARPS = 4;
__constant__ uint32_t c_mt_pow[624];   // 69069^i mod 2^32

__device__ __forceinline__ float mc_real(uint32_t y)
{
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    const int ys = (int)y;
    const float two32 = 4294967296.0f;
    return ys < 0 ? ((float)ys + two32) / two32 : (float)ys / two32;
}

// One MT19937 twist of mt[0..623] by the 32 lanes of a warp.
__device__ __forceinline__ void mc_twist(uint32_t* mt, int lane)
{
    const uint32_t up = 0x80000000u, lo = 0x7fffffffu, a = 0x9908b0dfu;
    for (int base = 0; base < 227; base += 32) {
        const int k = base + lane;
        uint32_t v = 0;
        if (k < 227) {
            const uint32_t y = (mt[k] & up) | (mt[k + 1] & lo);
            v = mt[k + 397] ^ (y >> 1) ^ ((y & 1u) ? a : 0u);
        }
        __syncwarp();
        if (k < 227) mt[k] = v;
        __syncwarp();
    }
    for (int base = 227; base < 623; base += 32) {
        const int k = base + lane;
        uint32_t v = 0;
        if (k < 623) {
            const uint32_t y = (mt[k] & up) | (mt[k + 1] & lo);
            v = mt[k - 227] ^ (y >> 1) ^ ((y & 1u) ? a : 0u);
        }
        __syncwarp();
        if (k < 623) mt[k] = v;
        __syncwarp();
    }
    if (lane == 0) {
        const uint32_t y = (mt[623] & up) | (mt[0] & lo);
        mt[623] = mt[396] ^ (y >> 1) ^ ((y & 1u) ? a : 0u);
    }
    __syncwarp();
}

// Masks of NGPT g-points for every column of the request.  lw: the cloud fraction is the input's, zero
// for a column with no layer above 1e-6 (the LW cldprop gate); otherwise (SW) values below 1e-12 are zero.
// seed: icseed[seedrow][col] when icseed is given, else seed0 + col + 1.
template <int NGPT>
__global__ void __launch_bounds__(MC_WARPS * 32) k_mcica(const float* clouds, int64_t ncol, int nlay, const int* icseed,
                                                         int seedrow, int seed0, int iovr, int lw, uint32_t* out)
{
    constexpr int NW = (NGPT + 31) / 32;
    __shared__ uint32_t mt_s[MC_WARPS][624];
    __shared__ float buf_s[MC_WARPS][624];
    __shared__ float cf_s[MC_WARPS][NLAY_MAX];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t col = (int64_t)blockIdx.x * MC_WARPS + warp;
    if (col >= ncol || nlay > NLAY_MAX) return;   // whole warps only; the warp-level steps below stay inside
    uint32_t* mt = mt_s[warp];
    float* buf = buf_s[warp];
    float* cf = cf_s[warp];
    bool any = false;
    for (int k0 = lane; k0 < nlay; k0 += 32) {
        const float x = __ldg(clouds + (size_t)(nlay - 1 - k0) * ncol + col);
        cf[k0] = lw ? x : (x < 1.0e-12f ? 0.0f : x);
        any = any || x > 1.0e-6f;
    }
    if (lw && !__any_sync(0xffffffffu, any))
        for (int k0 = lane; k0 < nlay; k0 += 32) cf[k0] = 0.0f;
    const int seed = icseed ? __ldg(icseed + (size_t)seedrow * ncol + col) : seed0 + (int)(col + 1);
    const uint32_t s0 = seed == 0 ? 4357u : (uint32_t)seed;
    for (int i = lane; i < 624; i += 32) mt[i] = s0 * c_mt_pow[i];
    __syncwarp();
    uint64_t bits[NW];
    float prev[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) { bits[w] = 0; prev[w] = 0; }
    const int ndraw = iovr == 2 ? NGPT : NGPT * nlay;
    for (int lo0 = 0; lo0 < ndraw; lo0 += 624) {
        mc_twist(mt, lane);
        for (int i = lane; i < 624; i += 32) buf[i] = mc_real(mt[i]);
        __syncwarp();
        const int hi0 = min(ndraw, lo0 + 624);
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            const int g = w * 32 + lane;
            if (g >= NGPT) continue;
            if (iovr == 2) {
                if (g >= lo0 && g < hi0) {
                    const float r = buf[g - lo0];
                    for (int k0 = 0; k0 < nlay; ++k0)
                        if (r >= 1.0f - cf[k0]) bits[w] |= 1ull << k0;
                }
                continue;
            }
            const int d0 = g * nlay;
            const int ka = max(0, lo0 - d0), kb = min(nlay, hi0 - d0);
            for (int k0 = ka; k0 < kb; ++k0) {
                const float r = buf[d0 + k0 - lo0];
                float cd = r;
                if (iovr == 1) {
                    if (k0 > 0) {
                        const float tem1 = 1.0f - cf[k0 - 1];
                        cd = prev[w] > tem1 ? prev[w] : r * tem1;
                    }
                    prev[w] = cd;
                }
                if (cd >= 1.0f - cf[k0]) bits[w] |= 1ull << k0;
            }
        }
        __syncwarp();
    }
#pragma unroll
    for (int w = 0; w < NW; ++w)
        for (int k0 = 0; k0 < nlay; ++k0) {
            const uint32_t word = __ballot_sync(0xffffffffu, (bits[w] >> k0) & 1ull);
            if (lane == (k0 & 31)) out[((size_t)w * nlay + k0) * ncol + col] = word;
        }
}

}  // namespace rad
