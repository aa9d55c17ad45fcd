// rad_capi.cu -- the C ABI of libradb200.so (include/radb200.h): handle, tables, the SW day list and
// MINVAL(laytrop) groups on the device, and the LW / SW column kernel launches.
//
// The reference drives its radiation per row window from the host with one device-to-host read of the
// day counts per call and ~52k launches (namgpu/physics/rrtm/rrtm_call.py:44-48, :206-235).  Here one
// rad_solve is a fixed, host-sync-free sequence of launches on the caller's stream: day flags, an
// exclusive scan (CUB), the day list, per-day-column laytrop and group minima, the LW kernel over all
// columns and the SW kernel over the day columns (its grid is the column count; CTAs past the device day
// count exit at once).
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <chrono>
#include <thread>
#include <string>
#include <vector>

#define RAD_WANT_TABLE_NAMES
#include "../../include/radb200.h"
#include "rad_tabids.h"
#include "rad_front.h"

namespace rad {
__constant__ int c_lw_ns[17] = {0, 10, 22, 38, 52, 68, 76, 88, 96, 108, 114, 122, 130, 134, 136, 138, 140};
__constant__ int c_sw_ns[15] = {0, 6, 18, 26, 34, 44, 54, 56, 66, 74, 80, 86, 94, 100, 112};
}  // namespace rad

#include "rad_lw.cuh"
#include "rad_sw.cuh"
#include "rad_sw2.cuh"
#include "rad_lw2.cuh"
#include "rad_lw3.cuh"
#include "rad_sw4.cuh"
#include "rad_mcica.cuh"
#include "rad_post.cuh"
#include "rad_rdtemp.cuh"
#include "rad_aer.cuh"
#include "rad_solar.cuh"
#include "rad_grrad.cuh"

using namespace rad;

struct RadHandle {
    RadConfig cfg{};
    int device = 0;
    bool tables_ok = false;
    float *d_lwf = nullptr, *d_swf = nullptr;      // LW LUT (3 x 10001) and SW exp table, float32
    double *d_lwd = nullptr, *d_swd = nullptr;     // the same in float64
    int* d_err = nullptr;
    // day-list scratch
    int64_t cap = 0;
    int *d_flag = nullptr, *d_pos = nullptr, *d_daycol = nullptr, *d_lt = nullptr, *d_k8 = nullptr, *d_kw = nullptr;
    int *d_cmin = nullptr, *d_nday = nullptr;
    int64_t cmin_cap = 0;
    uint32_t *d_lwm = nullptr, *d_swm = nullptr;   // McICA sub-column words when the caller passes no mask
    int64_t mask_cap = 0;                          // columns x layers the mask scratch holds
    void* d_cub = nullptr;
    size_t cub_bytes = 0;
    float* d_lw3 = nullptr;                        // two-kernel LW: gas optics and sweep inputs of one chunk
    int64_t lw3_cap = 0;                           // columns d_lw3 holds
    int* d_lw3list = nullptr;                      // [1 + lw3_cap]: count, then the chunk's float64 columns
    float* d_swrt = nullptr;                       // SW layer R/T stores, sw2_rt_floats() per CTA of the SW grid
    float* d_lwpg = nullptr;                       // optional LW outputs: g-point profiles of one chunk (DIAG sweeps)
    float* d_swpg = nullptr;                       // optional SW outputs: g-point level fluxes of one chunk
    int64_t lwpg_cap = 0, swpg_cap = 0;            // columns they hold
    int4* d_sw4img = nullptr;                      // chunked SW: set-up and gas-optics images of one chunk's columns
    unsigned char* d_sw4 = nullptr;                // chunked SW: header and layer R/T of one chunk's columns
    int64_t sw4_cap = 0;                           // columns d_sw4 and d_sw4img hold
    float* d_aerf = nullptr;                       // aerosol band tables of the loaded month (AF_* offsets)
    int* d_aeri = nullptr;                         // their integer part (AI_* offsets)
    int nsm = 148;                                 // SMs of the device (grid of the float64 column kernel)
    std::string err;
    // kernel accounting
    int64_t launches = 0;
    bool profiling = false;
    std::vector<cudaEvent_t> ev;      // 4 events per profiled solve: before LW, after LW, after prep, after SW
    size_t ev_used = 0;
    int64_t prof_solves = 0, prof_columns = 0;
};

namespace {
thread_local std::string g_err;

// Per-device k-table store shared by every handle of the process (see rad_load_tables).
struct DeviceTables {
    float* tf = nullptr;
    double* td = nullptr;
    std::vector<int64_t> off;
    std::vector<float> hf;
    LwHostConsts k{};
};
std::mutex g_tab_mu;
std::map<int, DeviceTables> g_tabs;

int fail(RadHandle* h, int code, const std::string& msg)
{
    if (h) h->err = msg;
    g_err = msg;
    return code;
}
#define RAD_CUDA(h, call)                                                                                  \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return fail((h), RAD_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// ---------------------------------------------------------------------------------- device helpers
// The SW day list of a launch's requests (their columns concatenated; phys_rrtm_grrad_sw.cu:69,80 per
// request) and, per day column, laytrop and the MINVAL(laytrop) minima of its 8-column group and of its
// chunk (sw_seam.py:23-37, rrtm_sw_kmin_windows.cu).  Windows and chunks restart with every request.
struct DayReq {
    const float* coszen;
    const float* plyr;
    int64_t ncol;
    int wc, maxc;          // window columns, chunks per window
    int64_t cmin_off;      // first chunk-minimum slot of the request
};
using DayBatch = ReqBatch<DayReq>;

__global__ void k_dayflags(const __grid_constant__ DayBatch b, int64_t n, int* flag)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n) {
        const int r = b.find(c);
        flag[c] = b.req[r].coszen[c - b.off[r]] >= 1.0e-4f ? 1 : 0;
    }
    if (c == n) flag[c] = 0;
}
__global__ void k_scatter(const int* flag, const int* pos, int64_t n, int* daycol, int* nday)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c < n && flag[c]) daycol[pos[c]] = (int)c;
    if (c == n) *nday = pos[n];
}
// SW setcoef laytrop of each day column (setcoef.cu:28-73): the last layer (surface first) with
// ln(p) > 4.56, nlay when there is none.
__global__ void k_laytrop(const __grid_constant__ DayBatch b, int nlay, const int* daycol, const int* nday, int* lt,
                          int* cmin, int chunk, const int* pos)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= *nday) return;
    const int64_t g = daycol[d];
    const int r = b.find(g);
    const DayReq& q = b.req[r];
    const int64_t c = g - b.off[r];
    int l = nlay;
    for (int k0 = 0; k0 < nlay; ++k0)
        if (log((double)q.plyr[(size_t)(nlay - 1 - k0) * q.ncol + c]) > (double)4.56f) l = k0 + 1;
    lt[d] = l;
    const int w = (int)(c / q.wc);
    const int dw0 = pos[b.off[r] + (int64_t)w * q.wc];
    const int ci = (d - dw0) / chunk;
    atomicMin(cmin + q.cmin_off + (int64_t)w * q.maxc + ci, l);
}
__global__ void k_groups(const __grid_constant__ DayBatch b, const int* daycol, const int* nday, const int* lt,
                         const int* cmin, int chunk, const int* pos, int* k8, int* kw)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= *nday) return;
    const int64_t g = daycol[d];
    const int r = b.find(g);
    const DayReq& q = b.req[r];
    const int64_t c = g - b.off[r];
    const int w = (int)(c / q.wc);
    const int dw0 = pos[b.off[r] + (int64_t)w * q.wc];
    const int64_t wend = ((int64_t)w + 1) * q.wc < q.ncol ? ((int64_t)w + 1) * q.wc : q.ncol;
    const int dw1 = pos[b.off[r] + wend];
    const int ci = (d - dw0) / chunk;
    const int dc0 = dw0 + ci * chunk;
    const int dc1 = dc0 + chunk < dw1 ? dc0 + chunk : dw1;
    const int g0 = dc0 + ((d - dc0) / 8) * 8;
    const int g1 = g0 + 8 < dc1 ? g0 + 8 : dc1;
    int m = lt[d];
    for (int i = g0; i < g1; ++i) m = min(m, lt[i]);
    k8[d] = m;
    kw[d] = cmin[q.cmin_off + (int64_t)w * q.maxc + ci];
}
__global__ void k_fill_int(int* p, int64_t n, int v)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// ---------------------------------------------------------------------------------- host tables
template <class R>
void lw_lut(std::vector<R>& v)   // [ex | tfn | tau], 3 x 10001 (phys_rrtm_lw_rtrnmr.py:108-131 recipe)
{
    const int n = 10000;
    v.assign(3 * (n + 1), 0);
    R* ex = v.data();
    R* tfn = ex + n + 1;
    R* tau = tfn + n + 1;
    const R bpade = (R)1.0f / (R)0.278f, expeps = (R)1.0e-20f;
    const R explimit = (R)std::trunc(-std::log((double)std::numeric_limits<R>::min()));
    ex[0] = 1; tau[0] = 0; tfn[0] = 0;
    for (int i = 1; i < n; ++i) {
        const R tf = (R)i / (R)(n - i);
        const R ta = bpade * tf;
        const R e = ta >= explimit ? expeps : (R)std::exp(-(double)ta);
        tau[i] = ta; ex[i] = e;
        tfn[i] = ta < (R)0.06f ? ta / (R)6 : (R)1 - (R)2 * (((R)1 / ta) - (e / ((R)1 - e)));
    }
    ex[n] = expeps; tau[n] = (R)1.0e10f; tfn[n] = 1;
}
template <class R>
void sw_lut(std::vector<R>& v)   // exp_tbl(0:10000) (phys_rrtm_sw_spcvrtc.py:60-73)
{
    const int n = 10000;
    v.assign(n + 1, 0);
    v[0] = 1;
    const double bpade = 1.0 / 0.278;
    for (int i = 1; i < n; ++i) v[i] = (R)std::exp(-bpade * ((double)i / ((double)n - i)));
    v[n] = (R)1.0e-20f;
}

// The plain FP64 precision runs the first-design kernels (lw_column_kernel / sw_column_kernel<double>);
// the mixed precision runs the production kernels (lw2_column_kernel<float> / sw2_column_kernel).
template <class R>
void* kernel_ptr_lw(bool mc) { return sizeof(R) == 4 ? (mc ? (void*)lw2_column_kernel<float, true> : (void*)lw2_column_kernel<float, false>) : (void*)lw_column_kernel<double>; }
template <class R>
void* kernel_ptr_sw() { return (void*)sw_column_kernel<R>; }

template <class T>
int upload(RadHandle* h, T** dptr, const std::vector<T>& host)
{
    if (*dptr) cudaFree(*dptr);
    *dptr = nullptr;
    RAD_CUDA(h, cudaMalloc((void**)dptr, host.size() * sizeof(T)));
    RAD_CUDA(h, cudaMemcpy(*dptr, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice));
    return RAD_OK;
}

int ensure_scratch(RadHandle* h, int64_t n)
{
    if (n + 1 > h->cap) {
        const int64_t cap = n + 1 + (n >> 3);
        for (int** p : {&h->d_flag, &h->d_pos, &h->d_daycol, &h->d_lt, &h->d_k8, &h->d_kw})
            if (*p) cudaFree(*p);
        for (int** p : {&h->d_flag, &h->d_pos, &h->d_daycol, &h->d_lt, &h->d_k8, &h->d_kw})
            RAD_CUDA(h, cudaMalloc((void**)p, (size_t)cap * sizeof(int)));
        size_t need = 0;
        RAD_CUDA(h, cub::DeviceScan::ExclusiveSum(nullptr, need, h->d_flag, h->d_pos, (int)cap));
        if (need > h->cub_bytes) {
            if (h->d_cub) cudaFree(h->d_cub);
            RAD_CUDA(h, cudaMalloc(&h->d_cub, need));
            h->cub_bytes = need;
        }
        h->cap = cap;
    }
    return RAD_OK;
}

// Columns per LW chunk when the optional LW outputs are wanted (their g-point profiles: 278 KB per column).
constexpr int64_t LW_DIAG_CHUNK = 8192;
int64_t sw4_chunk(const RadConfig& cfg);
int64_t lw3_chunk(const RadConfig& cfg);

// The g-point profile buffers of the optional outputs (allocated on the first solve that asks for them).
int ensure_diag_scratch(RadHandle* h, int64_t ntot, bool lw, bool sw)
{
    const int nlay = h->cfg.nlay;
    if (lw) {
        const int64_t need = std::min(std::min(lw3_chunk(h->cfg), LW_DIAG_CHUNK), ntot);
        if (need > h->lwpg_cap) {
            if (h->d_lwpg) cudaFree(h->d_lwpg);
            h->d_lwpg = nullptr;
            h->lwpg_cap = 0;
            RAD_CUDA(h, cudaMalloc((void**)&h->d_lwpg, (size_t)need * lw3_pg_floats(nlay) * sizeof(float)));
            h->lwpg_cap = need;
        }
    }
    if (sw) {
        const int64_t need = std::min(sw4_chunk(h->cfg), ntot);
        if (need > h->swpg_cap) {
            if (h->d_swpg) cudaFree(h->d_swpg);
            h->d_swpg = nullptr;
            h->swpg_cap = 0;
            RAD_CUDA(h, cudaMalloc((void**)&h->d_swpg, (size_t)need * sw4_pg_floats(nlay) * sizeof(float)));
            h->swpg_cap = need;
        }
    }
    return RAD_OK;
}

// McICA: LW and SW sub-column words of every column of request r, into the caller's mask outputs when
// given, else into the handle's scratch at the request's column offset (scratch holds the launch's columns).
// Seeds: icseed [2][ncol] (LW row, SW row) or seed0 + column + 1.
int mcica_masks(RadHandle* h, const RadColumns* in, const RadOutputs* out, int64_t n, int64_t scratch_off,
                cudaStream_t st, const uint32_t** lwm, const uint32_t** swm)
{
    const RadConfig& cfg = h->cfg;
    const int nlay = cfg.nlay;
    uint32_t* lw = out->lw_mask;
    uint32_t* sw = out->sw_mask;
    // scratch layout per request: [5][nlay][n] LW words then [4][nlay][n] SW words, at 9 nlay offset
    if (!lw) lw = h->d_lwm + (size_t)9 * nlay * scratch_off;
    if (!sw) sw = (out->lw_mask ? h->d_lwm + (size_t)9 * nlay * scratch_off : lw + (size_t)5 * nlay * n);
    const unsigned grid = (unsigned)((n + MC_WARPS - 1) / MC_WARPS);
    k_mcica<140><<<grid, MC_WARPS * 32, 0, st>>>(in->clouds, n, nlay, in->icseed, 0, cfg.lw_seed0, cfg.iovrlw, 1, lw);
    k_mcica<112><<<grid, MC_WARPS * 32, 0, st>>>(in->clouds, n, nlay, in->icseed, 1, cfg.sw_seed0, cfg.iovrsw, 0, sw);
    h->launches += 2;
    RAD_CUDA(h, cudaGetLastError());
    *lwm = lw;
    *swm = sw;
    return RAD_OK;
}

// Record the next profiling event on st (no-op while profiling is off).
int mark(RadHandle* h, cudaStream_t st, size_t base, int i)
{
    if (!h->profiling) return RAD_OK;
    RAD_CUDA(h, cudaEventRecord(h->ev[base + i], st));
    return RAD_OK;
}

// Columns per chunk of the two-kernel LW (mixed precision), 0 when the single-kernel LW runs.
int64_t lw3_chunk(const RadConfig& cfg)
{
    if (cfg.precision != RAD_PREC_MIXED || cfg.lw_chunk < 0) return 0;
    return cfg.lw_chunk > 0 ? cfg.lw_chunk : 32768;
}

// Day columns per chunk of the two-kernel SW (mixed precision), 0 when the single-kernel SW runs.
int64_t sw4_chunk(const RadConfig& cfg)
{
    if (cfg.precision != RAD_PREC_MIXED || cfg.sw_sweep_chunk < 0) return 0;
    return cfg.sw_sweep_chunk > 0 ? cfg.sw_sweep_chunk : 16384;
}

// Scratch for a launch of ntot columns: day list arrays, CUB temp, chunk minima, McICA words.
int ensure_launch_scratch(RadHandle* h, int64_t ntot, int64_t ncmin)
{
    int rc = ensure_scratch(h, ntot);
    if (rc) return rc;
    if (ncmin > h->cmin_cap) {
        if (h->d_cmin) cudaFree(h->d_cmin);
        h->d_cmin = nullptr;
        h->cmin_cap = 0;
        RAD_CUDA(h, cudaMalloc((void**)&h->d_cmin, (size_t)ncmin * sizeof(int)));
        h->cmin_cap = ncmin;
    }
    const int64_t lwc = lw3_chunk(h->cfg);
    if (lwc > 0 && (h->cfg.parts & RAD_PART_LW)) {
        const int64_t need = std::min(lwc, ntot);
        if (need > h->lw3_cap) {
            if (h->d_lw3) cudaFree(h->d_lw3);
            if (h->d_lw3list) cudaFree(h->d_lw3list);
            h->d_lw3 = nullptr;
            h->d_lw3list = nullptr;
            h->lw3_cap = 0;
            RAD_CUDA(h, cudaMalloc((void**)&h->d_lw3, (size_t)need * lw3_block_floats(h->cfg.nlay) * sizeof(float)));
            RAD_CUDA(h, cudaMalloc((void**)&h->d_lw3list, (size_t)(need + 1) * sizeof(int)));
            h->lw3_cap = need;
        }
    }
    const int64_t swc = sw4_chunk(h->cfg);
    if (h->cfg.precision == RAD_PREC_MIXED && (h->cfg.parts & RAD_PART_SW) && swc <= 0 && !h->d_swrt)
        RAD_CUDA(h, cudaMalloc((void**)&h->d_swrt, (size_t)sw2_rt_bytes(h->nsm)));
    if (swc > 0 && (h->cfg.parts & RAD_PART_SW) && std::min(swc, ntot) > h->sw4_cap) {
        if (h->d_sw4) cudaFree(h->d_sw4);
        if (h->d_sw4img) cudaFree(h->d_sw4img);
        h->d_sw4 = nullptr;
        h->d_sw4img = nullptr;
        h->sw4_cap = 0;
        const int64_t need = std::min(swc, ntot);
        RAD_CUDA(h, cudaMalloc((void**)&h->d_sw4, (size_t)need * sw4_block_bytes(h->cfg.nlay)));
        RAD_CUDA(h, cudaMalloc((void**)&h->d_sw4img, (size_t)need * sw4_image_bytes(true)));
        h->sw4_cap = need;
    }
    if (h->cfg.route == RAD_ROUTE_MCICA && ntot * h->cfg.nlay > h->mask_cap) {
        if (h->d_lwm) cudaFree(h->d_lwm);
        h->d_lwm = nullptr;
        h->mask_cap = 0;
        RAD_CUDA(h, cudaMalloc((void**)&h->d_lwm, (size_t)9 * h->cfg.nlay * ntot * sizeof(uint32_t)));
        h->mask_cap = ntot * h->cfg.nlay;
    }
    return RAD_OK;
}

// One launch set for up to RAD_MAXREQ requests: the McICA generators (McICA route), one LW launch over all
// the requests' columns, the day list and group minima of all of them, one SW launch over all their sunlit
// columns.  No host synchronisation.
// Day-list scratch of one launch: the handle's growing buffers, or a fixed region (rad_solve_noalloc).
struct LaunchScratch {
    int *flag, *pos, *daycol, *lt, *k8, *kw, *cmin, *nday;
    void* cub;
    size_t cub_bytes;
    int64_t max_cols, max_cmin;   // capacity of a fixed region (unused for the handle's buffers)
};

template <class R>
int launch_batch(RadHandle* h, int nreq, const RadColumns* ins, const RadOutputs* outs, const int64_t* ncols,
                 cudaStream_t st, const LaunchScratch* fixed = nullptr)
{
    const RadConfig& cfg = h->cfg;
    const int nlay = cfg.nlay;
    const int chunk = cfg.sw_chunk > 0 ? cfg.sw_chunk : 32768;
    int64_t ntot = 0, ncmin = 0;
    bool any_aer = false;
    DayBatch db{};
    db.nreq = nreq;
    for (int r = 0; r < nreq; ++r) {
        const int64_t n = ncols[r];
        DayReq& q = db.req[r];
        q.coszen = ins[r].coszen;
        q.plyr = ins[r].plyr;
        q.ncol = n;
        q.wc = cfg.window_cols > 0 ? (int)std::min<int64_t>(cfg.window_cols, std::max<int64_t>(n, 1)) : (int)std::max<int64_t>(n, 1);
        q.maxc = (q.wc + chunk - 1) / chunk;
        q.cmin_off = ncmin;
        ncmin += ((n + q.wc - 1) / q.wc) * q.maxc;
        db.off[r] = ntot;
        ntot += n;
        any_aer = any_aer || ins[r].faersw != nullptr;
    }
    db.off[nreq] = ntot;
    if (ntot == 0) return RAD_OK;
    if (ntot > (int64_t)std::numeric_limits<int>::max() - 1)
        return fail(h, RAD_E_INVALID, "rad_solve: more than 2^31 - 2 columns in one launch");
    int rc = RAD_OK;
    LaunchScratch sc;
    if (fixed) {
        if (ntot > fixed->max_cols || ncmin > fixed->max_cmin)
            return fail(h, RAD_E_INVALID, "rad_solve_noalloc: request larger than the fixed scratch region");
        sc = *fixed;
    } else {
        if ((rc = ensure_launch_scratch(h, ntot, std::max<int64_t>(ncmin, 1)))) return rc;
        sc = LaunchScratch{h->d_flag, h->d_pos, h->d_daycol, h->d_lt, h->d_k8, h->d_kw, h->d_cmin, h->d_nday,
                           h->d_cub, h->cub_bytes, 0, 0};
    }
    size_t eb = 0;
    if (h->profiling && !fixed) {
        eb = h->ev_used;
        while (h->ev.size() < eb + 4) {
            cudaEvent_t e;
            RAD_CUDA(h, cudaEventCreate(&e));
            h->ev.push_back(e);
        }
        h->ev_used += 4;
        h->prof_solves += 1;
        h->prof_columns += ntot;
    }
    const bool prof = h->profiling && !fixed;
    auto mark_if = [&](int i) { return prof ? mark(h, st, eb, i) : RAD_OK; };
    int mrc = mark_if(0);
    if (mrc) return mrc;
    // ---- McICA route: sub-column cloud words of every column (LW and SW generators)
    const uint32_t* lwm[RAD_MAXREQ] = {};
    const uint32_t* swm[RAD_MAXREQ] = {};
    if (cfg.route == RAD_ROUTE_MCICA)
        for (int r = 0; r < nreq; ++r)
            if (ncols[r] > 0 && (rc = mcica_masks(h, ins + r, outs + r, ncols[r], db.off[r], st, &lwm[r], &swm[r])))
                return rc;
    const bool do_lw = cfg.parts & RAD_PART_LW, do_sw = cfg.parts & RAD_PART_SW;
    // lwrad's / swrad's optional outputs: profiles of every g-point from the chunked sweeps, then per chunk a
    // reduction into the requested fields
    DiagOuts dout{};
    bool diag_lw = false, diag_sw = false;
    for (int r = 0; r < nreq; ++r) {
        const RadOutputs* o = outs + r;
        dout.p[r][0] = o->hlw0; dout.p[r][1] = o->hlwb; dout.p[r][2] = o->lwflxprf;
        dout.p[r][3] = o->hsw0; dout.p[r][4] = o->htswb; dout.p[r][5] = o->swflxprf;
        diag_lw = diag_lw || (do_lw && (o->hlw0 || o->hlwb || o->lwflxprf));
        diag_sw = diag_sw || (do_sw && (o->hsw0 || o->htswb || o->swflxprf));
    }
    if ((diag_lw && (fixed || sizeof(R) != 4 || lw3_chunk(cfg) <= 0)) ||
        (diag_sw && (fixed || sizeof(R) != 4 || sw4_chunk(cfg) <= 0)))
        return fail(h, RAD_E_INVALID, "optional outputs (hlw0, hlwb, lwflxprf, hsw0, htswb, swflxprf) are produced by "
                                      "rad_solve's mixed precision with the chunked LW and SW (lw_chunk >= 0, "
                                      "sw_sweep_chunk >= 0)");
    if (diag_lw || diag_sw) {
        if ((rc = ensure_diag_scratch(h, ntot, diag_lw, diag_sw))) return rc;
    }
    // ---- LW over every column
    if (do_lw) {
        LwBatch bt{};
        bt.nreq = nreq;
        for (int r = 0; r <= nreq; ++r) bt.off[r] = db.off[r];
        for (int r = 0; r < nreq; ++r) {
            const RadColumns* in = ins + r;
            const RadOutputs* out = outs + r;
            bt.req[r] = LwIn{in->plyr, in->plvl, in->tlyr, in->tlvl, in->qlyr, in->olyr, in->gasvmr, in->clouds,
                             in->faerlw, in->sfcemis, in->tsfg, out->htlw, out->topflw, out->sfcflw, ncols[r], nlay,
                             cfg.diagnostic, cfg.cpathfac, lwm[r], cfg.route == RAD_ROUTE_NAM && cfg.iovrlw == 0};
        }
        LwLut<R> lut;
        const R* base = sizeof(R) == 4 ? (const R*)h->d_lwf : (const R*)h->d_lwd;
        lut.ex = base; lut.tfn = base + 10001; lut.tau = base + 2 * 10001;
        const bool mc = cfg.route == RAD_ROUTE_MCICA;
        const int64_t lwc = fixed ? 0 : lw3_chunk(cfg);
        if (sizeof(R) == 4 && lwc > 0) {
            // per chunk: gas optics into the scratch, one warp per column sweeps, then (NAM route) the flagged
            // columns -- a cloudy layer under 1 hPa -- again by the float64 column kernel
            LwLut<float> fl;
            fl.ex = h->d_lwf; fl.tfn = h->d_lwf + 10001; fl.tau = h->d_lwf + 2 * 10001;
            LwLut<double> dl;
            dl.ex = h->d_lwd; dl.tfn = h->d_lwd + 10001; dl.tau = h->d_lwd + 2 * 10001;
            const size_t smem1 = sizeof(LwSetupK<float>), smemd = sizeof(LwShared<double>);
            RAD_CUDA(h, cudaFuncSetAttribute((void*)lw3_optics_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1));
            RAD_CUDA(h, cudaFuncSetAttribute((void*)lw3_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemd));
            const int64_t lstep = diag_lw ? std::min(lwc, (int64_t)LW_DIAG_CHUNK) : lwc;
            for (int64_t c0 = 0; c0 < ntot; c0 += lstep) {
                const int64_t nc = std::min(lstep, ntot - c0);
                RAD_CUDA(h, cudaMemsetAsync(h->d_lw3list, 0, sizeof(int), st));
                lw3_optics_kernel<<<(unsigned)nc, LW3_OPT_THREADS, smem1, st>>>(bt, c0, h->d_lw3, h->d_lw3list, h->d_err);
                const unsigned g2 = (unsigned)((nc + LW3_SWEEP_WARPS - 1) / LW3_SWEEP_WARPS);
                float* pg = h->d_lwpg;
                if (mc) {
                    if (diag_lw) lw3_sweep_kernel<LW_OVR_MCICA, true><<<g2, LW3_SWEEP_WARPS * 32, 0, st>>>(bt, c0, nc, h->d_lw3, fl, h->d_err, pg);
                    else lw3_sweep_kernel<LW_OVR_MCICA><<<g2, LW3_SWEEP_WARPS * 32, 0, st>>>(bt, c0, nc, h->d_lw3, fl, h->d_err);
                    h->launches += 2;
                } else {
                    if (cfg.iovrlw == 0) {
                        if (diag_lw) lw3_sweep_kernel<LW_OVR_RANDOM, true><<<g2, LW3_SWEEP_WARPS * 32, 0, st>>>(bt, c0, nc, h->d_lw3, fl, h->d_err, pg);
                        else lw3_sweep_kernel<LW_OVR_RANDOM><<<g2, LW3_SWEEP_WARPS * 32, 0, st>>>(bt, c0, nc, h->d_lw3, fl, h->d_err);
                    } else {
                        if (diag_lw) lw3_sweep_kernel<LW_OVR_MAXRAN, true><<<g2, LW3_SWEEP_WARPS * 32, 0, st>>>(bt, c0, nc, h->d_lw3, fl, h->d_err, pg);
                        else lw3_sweep_kernel<LW_OVR_MAXRAN><<<g2, LW3_SWEEP_WARPS * 32, 0, st>>>(bt, c0, nc, h->d_lw3, fl, h->d_err);
                    }
                    lw3_fp64_kernel<<<(unsigned)h->nsm, LW_THREADS, smemd, st>>>(bt, c0, h->d_lw3list, dl, h->d_err);
                    h->launches += 3;
                }
                if (diag_lw) {
                    k_lw_diag<<<(unsigned)((nc + 3) / 4), 128, 0, st>>>(bt, c0, nc, pg, dout);
                    h->launches += 1;
                }
            }
            RAD_CUDA(h, cudaGetLastError());
        } else {
        const size_t smem = sizeof(LwShared<R>);
        RAD_CUDA(h, cudaFuncSetAttribute(kernel_ptr_lw<R>(mc), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        if (sizeof(R) == 4 && mc) {
            lw2_column_kernel<R, true><<<(unsigned)ntot, LW_THREADS, smem, st>>>(bt, lut, h->d_err, nullptr);
            h->launches += 1;
        } else if (sizeof(R) == 4) {
            // NAM route: columns with a cloudy layer under 1 hPa go to the float64 column kernel through a list
            // in the day-list scratch's pos array (ntot + 1 words; the SW part rewrites it afterwards)
            LwLut<double> dl;
            dl.ex = h->d_lwd; dl.tfn = h->d_lwd + 10001; dl.tau = h->d_lwd + 2 * 10001;
            const size_t smemd = sizeof(LwShared<double>);
            RAD_CUDA(h, cudaFuncSetAttribute((void*)lw3_fp64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemd));
            RAD_CUDA(h, cudaMemsetAsync(sc.pos, 0, sizeof(int), st));
            lw2_column_kernel<R, false><<<(unsigned)ntot, LW_THREADS, smem, st>>>(bt, lut, h->d_err, sc.pos);
            lw3_fp64_kernel<<<(unsigned)h->nsm, LW_THREADS, smemd, st>>>(bt, 0, sc.pos, dl, h->d_err);
            h->launches += 2;
        } else {
            lw_column_kernel<R><<<(unsigned)ntot, LW_THREADS, smem, st>>>(bt, lut, h->d_err);
            h->launches += 1;
        }
        RAD_CUDA(h, cudaGetLastError());
        }
    }
    if ((mrc = mark_if(1))) return mrc;
    if (!do_sw) {
        if ((mrc = mark_if(2))) return mrc;
        return mark_if(3);
    }
    // ---- SW day list, laytrop, groups
    const int T = 256;
    const unsigned gb = (unsigned)((ntot + 1 + T - 1) / T);
    k_dayflags<<<gb, T, 0, st>>>(db, ntot, sc.flag);
    size_t tb = sc.cub_bytes;
    RAD_CUDA(h, cub::DeviceScan::ExclusiveSum(sc.cub, tb, sc.flag, sc.pos, (int)(ntot + 1), st));
    k_scatter<<<gb, T, 0, st>>>(sc.flag, sc.pos, ntot, sc.daycol, sc.nday);
    k_fill_int<<<(unsigned)((ncmin + T - 1) / T), T, 0, st>>>(sc.cmin, ncmin, std::numeric_limits<int>::max());
    k_laytrop<<<gb, T, 0, st>>>(db, nlay, sc.daycol, sc.nday, sc.lt, sc.cmin, chunk, sc.pos);
    k_groups<<<gb, T, 0, st>>>(db, sc.daycol, sc.nday, sc.lt, sc.cmin, chunk, sc.pos, sc.k8, sc.kw);
    h->launches += 7;   // day flags, scan (2 kernels), scatter, fill, laytrop, groups
    RAD_CUDA(h, cudaGetLastError());
    // ---- SW over the day columns; zeros first (night columns keep them, as swrad does)
    for (int r = 0; r < nreq; ++r) {
        const int64_t n = ncols[r];
        if (!n) continue;
        const RadOutputs* out = outs + r;
        RAD_CUDA(h, cudaMemsetAsync(out->htsw, 0, (size_t)nlay * n * sizeof(float), st));
        RAD_CUDA(h, cudaMemsetAsync(out->topfsw, 0, (size_t)3 * n * sizeof(float), st));
        RAD_CUDA(h, cudaMemsetAsync(out->sfcfsw, 0, (size_t)4 * n * sizeof(float), st));
        if (out->fdncmp) RAD_CUDA(h, cudaMemsetAsync(out->fdncmp, 0, (size_t)6 * n * sizeof(float), st));
        if (out->hsw0) RAD_CUDA(h, cudaMemsetAsync(out->hsw0, 0, (size_t)nlay * n * sizeof(float), st));
        if (out->htswb) RAD_CUDA(h, cudaMemsetAsync(out->htswb, 0, (size_t)14 * nlay * n * sizeof(float), st));
        if (out->swflxprf) RAD_CUDA(h, cudaMemsetAsync(out->swflxprf, 0, (size_t)4 * (nlay + 1) * n * sizeof(float), st));
    }
    {
        SwBatch bt{};
        bt.nreq = nreq;
        for (int r = 0; r <= nreq; ++r) bt.off[r] = db.off[r];
        for (int r = 0; r < nreq; ++r) {
            const RadColumns* in = ins + r;
            const RadOutputs* out = outs + r;
            bt.req[r] = SwIn{in->plyr, in->plvl, in->tlyr, in->qlyr, in->olyr, in->gasvmr, in->clouds, in->faersw,
                             in->sfcalb, in->coszen, sc.daycol, sc.nday, sc.k8, sc.kw, out->htsw, out->topfsw,
                             out->sfcfsw, out->fdncmp, ncols[r], nlay, cfg.diagnostic, cfg.iswmode, in->solcon, swm[r],
                             cfg.iovrsw};
        }
        if ((mrc = mark_if(2))) return mrc;
        int64_t nlaunch = 1;
        if (sizeof(R) == 4) {
            const size_t smem = sw2_smem_bytes(any_aer);
            if (fixed) {   // no scratch: one CTA per sunlit column, R/T recomputed on the way down
                RAD_CUDA(h, cudaFuncSetAttribute((void*)sw2_column_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                sw2_column_kernel<false><<<(unsigned)ntot, SW2_THREADS, smem, st>>>(bt, any_aer ? 1 : 0, h->d_swf, h->d_swd,
                                                                                     h->d_err, nullptr);
            } else if (sw4_chunk(cfg) > 0) {
                // per chunk of day indices (the day count stays on the device: chunks past it exit at once):
                // set-up and gas optics one CTA per column into the images, the layer R/T one CTA per column
                // into the chunk scratch, then the adding sweeps one CTA per column
                const int64_t swc = sw4_chunk(cfg);
                const size_t smem0 = sw4_gas_smem(any_aer);
                const size_t smem1 = sw4_gas_smem(any_aer);   // the image without taug (read from the image)
                const size_t smem2 = (size_t)(SW2_NSEG - 1) * 4 * SW2_THREADS * sizeof(float);
                const size_t bb = sw4_block_bytes(nlay);
                RAD_CUDA(h, cudaFuncSetAttribute((void*)sw4_gas_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem0));
                RAD_CUDA(h, cudaFuncSetAttribute((void*)sw4_rt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1));
                RAD_CUDA(h, cudaFuncSetAttribute((void*)sw4_sweep_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
                RAD_CUDA(h, cudaFuncSetAttribute((void*)sw4_sweep_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
                for (int64_t d0 = 0; d0 < ntot; d0 += swc) {
                    const int64_t nc = std::min(swc, ntot - d0);
                    sw4_gas_kernel<<<(unsigned)nc, SW4_GAS_THREADS, smem0, st>>>(bt, any_aer ? 1 : 0, h->d_err, (int)d0, h->d_sw4img);
                    sw4_rt_kernel<<<(unsigned)nc, SW4_RT_THREADS, smem1, st>>>(bt, any_aer ? 1 : 0, h->d_swf, h->d_swd, (int)d0,
                                                                         h->d_sw4img, h->d_sw4, bb);
                    if (diag_sw) {
                        sw4_sweep_kernel<true><<<(unsigned)nc, SW2_THREADS, smem2, st>>>(bt, h->d_err, (int)d0, (int)nc,
                                                                                        h->d_sw4, bb, h->d_swpg);
                        k_sw_diag<<<(unsigned)((nc + 3) / 4), 128, 0, st>>>(bt, (int)d0, (int)nc, h->d_sw4, bb, h->d_swpg, dout);
                    } else {
                        sw4_sweep_kernel<false><<<(unsigned)nc, SW2_THREADS, smem2, st>>>(bt, h->d_err, (int)d0, (int)nc,
                                                                                         h->d_sw4, bb);
                    }
                }
                nlaunch = (diag_sw ? 4 : 3) * ((ntot + swc - 1) / swc);
            } else {       // SW2_CTAS_PER_SM CTAs per SM walk the day list, each with its R/T store
                RAD_CUDA(h, cudaFuncSetAttribute((void*)sw2_column_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                sw2_column_kernel<true><<<(unsigned)(SW2_CTAS_PER_SM * h->nsm), SW2_THREADS, smem, st>>>(
                    bt, any_aer ? 1 : 0, h->d_swf, h->d_swd, h->d_err, h->d_swrt);
            }
        } else {
            SwLut<R> lut;
            lut.ex = (const R*)h->d_swd;
            const size_t smem = sizeof(SwShared<R>);
            RAD_CUDA(h, cudaFuncSetAttribute(kernel_ptr_sw<R>(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            sw_column_kernel<R><<<(unsigned)ntot, SW_THREADS, smem, st>>>(bt, lut, h->d_swd, h->d_err);
        }
        h->launches += nlaunch;
        RAD_CUDA(h, cudaGetLastError());
    }
    return mark_if(3);
}
}  // namespace

// ============================================================================================== C ABI
extern "C" {

int rad_version(void) { return RAD_ABI_VERSION; }

void rad_config_default(RadConfig* cfg, int32_t nlay)
{
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->nlay = nlay;
    cfg->precision = RAD_PREC_MIXED;
    cfg->route = RAD_ROUTE_NAM;
    cfg->iswmode = 2;
    cfg->diagnostic = 0;
    cfg->window_cols = 0;
    cfg->sw_chunk = 32768;
    cfg->iovrlw = 1;
    cfg->iovrsw = 1;
    cfg->lw_seed0 = 140;
    cfg->sw_seed0 = 1;
    cfg->cpathfac = 1.5f;
    cfg->parts = RAD_PART_LW | RAD_PART_SW;
    cfg->lw_chunk = 0;
    cfg->sw_sweep_chunk = 0;
}

int rad_create(const RadConfig* cfg, RadHandle** out)
{
    if (!cfg || !out) return fail(nullptr, RAD_E_INVALID, "rad_create: null argument");
    if (cfg->nlay < 2 || cfg->nlay > NLAY_MAX)
        return fail(nullptr, RAD_E_INVALID, "rad_create: nlay must be in [2, " + std::to_string(NLAY_MAX) + "]");
    if (cfg->iswmode < 1 || cfg->iswmode > 3) return fail(nullptr, RAD_E_INVALID, "rad_create: iswmode must be 1, 2 or 3");
    if (cfg->parts < 1 || cfg->parts > 3) return fail(nullptr, RAD_E_INVALID, "rad_create: parts must be RAD_PART_LW, RAD_PART_SW or both");
    if (cfg->precision != RAD_PREC_FP64 && cfg->precision != RAD_PREC_MIXED)
        return fail(nullptr, RAD_E_INVALID, "rad_create: precision must be RAD_PREC_FP64 or RAD_PREC_MIXED");
    if (cfg->route != RAD_ROUTE_NAM && cfg->route != RAD_ROUTE_MCICA)
        return fail(nullptr, RAD_E_INVALID, "rad_create: unknown route");
    if (cfg->route == RAD_ROUTE_MCICA && cfg->precision != RAD_PREC_MIXED)
        return fail(nullptr, RAD_E_INVALID, "rad_create: the McICA route runs in the mixed precision");
    if (cfg->iovrlw < 0 || cfg->iovrlw > 2 || cfg->iovrsw < 0 || cfg->iovrsw > 2)
        return fail(nullptr, RAD_E_INVALID, "rad_create: iovrlw and iovrsw must be 0, 1 or 2");
    int device = 0, nsm = 0;
    if (cudaGetDevice(&device) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return fail(nullptr, RAD_E_CUDA, "rad_create: no usable CUDA device");
    RadHandle* h = new RadHandle();
    h->cfg = *cfg;
    h->device = device;
    h->nsm = nsm;
    if (cudaMalloc((void**)&h->d_err, sizeof(int)) != cudaSuccess ||
        cudaMalloc((void**)&h->d_nday, sizeof(int)) != cudaSuccess) {
        delete h;
        return fail(nullptr, RAD_E_NOMEM, "rad_create: device allocation failed");
    }
    cudaMemset(h->d_err, 0, sizeof(int));
    *out = h;
    return RAD_OK;
}

// Blob: "RADTBL01", uint32 count, then per table: uint16 name length, name, uint8 dtype (0 f32, 1 f64,
// 2 i32), uint64 element count, data.
int rad_load_tables(RadHandle* h, const void* blob, size_t nbytes)
{
    if (!h || !blob) return fail(h, RAD_E_INVALID, "rad_load_tables: null argument");
    const unsigned char* p = (const unsigned char*)blob;
    const unsigned char* end = p + nbytes;
    if (nbytes < 12 || std::memcmp(p, "RADTBL01", 8) != 0) return fail(h, RAD_E_TABLES, "rad_load_tables: bad magic");
    uint32_t count;
    std::memcpy(&count, p + 8, 4);
    p += 12;
    std::vector<std::vector<double>> vals(T_COUNT);
    std::vector<bool> seen(T_COUNT, false);
    std::vector<double> chi64;
    for (uint32_t e = 0; e < count; ++e) {
        if (p + 2 > end) return fail(h, RAD_E_TABLES, "rad_load_tables: truncated blob");
        uint16_t ln;
        std::memcpy(&ln, p, 2);
        p += 2;
        if (p + ln + 9 > end) return fail(h, RAD_E_TABLES, "rad_load_tables: truncated blob");
        std::string name((const char*)p, ln);
        p += ln;
        const uint8_t dt = *p++;
        uint64_t cnt;
        std::memcpy(&cnt, p, 8);
        p += 8;
        const size_t es = dt == 1 ? 8 : 4;
        if (p + cnt * es > end) return fail(h, RAD_E_TABLES, "rad_load_tables: truncated data of " + name);
        std::vector<double> v(cnt);
        for (uint64_t i = 0; i < cnt; ++i) {
            if (dt == 0) { float f; std::memcpy(&f, p + 4 * i, 4); v[i] = f; }
            else if (dt == 1) { double x; std::memcpy(&x, p + 8 * i, 8); v[i] = x; }
            else { int32_t x; std::memcpy(&x, p + 4 * i, 4); v[i] = x; }
        }
        p += cnt * es;
        if (name == "lw05_chi_mls_f64") { chi64 = v; continue; }
        for (int t = 0; t < T_COUNT; ++t)
            if (name == RAD_TABLE_NAMES[t]) { vals[t] = std::move(v); seen[t] = true; break; }
    }
    for (int t = 0; t < T_COUNT; ++t)
        if (!seen[t]) return fail(h, RAD_E_TABLES, std::string("rad_load_tables: missing table ") + RAD_TABLE_NAMES[t]);
    if (chi64.size() != 59 * 7) return fail(h, RAD_E_TABLES, "rad_load_tables: missing lw05_chi_mls_f64");
    std::vector<int64_t> off(T_COUNT);
    int64_t tot = 0;
    for (int t = 0; t < T_COUNT; ++t) { off[t] = tot; tot += (int64_t)vals[t].size(); }
    std::vector<float> hf(tot);
    std::vector<double> hd(tot);
    for (int t = 0; t < T_COUNT; ++t)
        for (size_t i = 0; i < vals[t].size(); ++i) {
            hf[off[t] + i] = (float)vals[t][i];
            hd[off[t] + i] = (double)(float)vals[t][i];   // the float32 table values, exactly
        }
    // host-side reference ratios (phys_rrtm_lw_taugb04.py:87-99, taugb05.py:81-85, taugb15.py:135-136)
    const std::vector<double>& chi = vals[T_LW_CHI_MLS];   // [59][7]
    LwHostConsts k;
    k.b4_rpa = (float)chi[10 * 7 + 0] / (float)chi[10 * 7 + 1];
    k.b4_rpb = (float)chi[12 * 7 + 2] / (float)chi[12 * 7 + 1];
    k.b5_rpa = (float)(chi64[4 * 7 + 0] / chi64[4 * 7 + 1]);
    k.b5_rpb = (float)(chi64[42 * 7 + 2] / chi64[42 * 7 + 1]);
    k.b5_rma = (float)(chi64[6 * 7 + 0] / chi64[6 * 7 + 1]);
    k.b15_r = (float)chi[0 * 7 + 3] / (float)chi[0 * 7 + 1];
    std::vector<float> lwf, swf;
    std::vector<double> lwd, swd;
    lw_lut(lwf); lw_lut(lwd); sw_lut(swf); sw_lut(swd);
    int rc;
    if ((rc = upload(h, &h->d_lwf, lwf)) || (rc = upload(h, &h->d_lwd, lwd)) || (rc = upload(h, &h->d_swf, swf)) ||
        (rc = upload(h, &h->d_swd, swd)))
        return rc;
    // The k-tables are read through __constant__ pointers, which are per device, not per handle: the
    // first load on a device uploads them and sets the constants; they stay until the process exits and
    // every later handle on that device shares them.  A later blob with different content is refused, so a
    // handle can never leave another handle's kernels reading freed or different tables.
    std::lock_guard<std::mutex> lock(g_tab_mu);
    DeviceTables& dt = g_tabs[h->device];
    if (dt.tf) {
        if (dt.off != off || dt.hf != hf || std::memcmp(&dt.k, &k, sizeof(k)) != 0)
            return fail(h, RAD_E_TABLES, "rad_load_tables: tables with different content are already loaded on this "
                                         "device (one table set per device and process)");
    } else {
        float* tf = nullptr;
        double* td = nullptr;
        if ((rc = upload(h, &tf, hf)) || (rc = upload(h, &td, hd))) {
            if (tf) cudaFree(tf);
            return rc;
        }
        RAD_CUDA(h, cudaMemcpyToSymbol(c_toff, off.data(), T_COUNT * sizeof(int64_t)));
        RAD_CUDA(h, cudaMemcpyToSymbol(c_tf, &tf, sizeof(float*)));
        RAD_CUDA(h, cudaMemcpyToSymbol(c_td, &td, sizeof(double*)));
        RAD_CUDA(h, cudaMemcpyToSymbol(c_lwk, &k, sizeof(k)));
        uint32_t pw[624];
        pw[0] = 1u;
        for (int i = 1; i < 624; ++i) pw[i] = 69069u * pw[i - 1];
        RAD_CUDA(h, cudaMemcpyToSymbol(c_mt_pow, pw, sizeof(pw)));
        RAD_CUDA(h, cudaDeviceSynchronize());
        dt.tf = tf;
        dt.td = td;
        dt.off = off;
        dt.hf = std::move(hf);
        dt.k = k;
    }
    h->tables_ok = true;
    return RAD_OK;
}

int64_t rad_workspace_bytes(const RadHandle* h, int64_t ncol)
{
    int64_t b = (ncol + 1) * 6 * (int64_t)sizeof(int) + (1 << 20);
    if (h) {
        const int64_t lwc = lw3_chunk(h->cfg);
        if (lwc > 0 && (h->cfg.parts & RAD_PART_LW))
            b += std::min(lwc, ncol) * lw3_block_floats(h->cfg.nlay) * (int64_t)sizeof(float);
        if (h->cfg.route == RAD_ROUTE_MCICA) b += 9 * (int64_t)h->cfg.nlay * ncol * (int64_t)sizeof(uint32_t);
        const int64_t swc = sw4_chunk(h->cfg);
        if (h->cfg.precision == RAD_PREC_MIXED && (h->cfg.parts & RAD_PART_SW) && swc <= 0) b += sw2_rt_bytes(h->nsm);
        if (swc > 0 && (h->cfg.parts & RAD_PART_SW))
            b += std::min(swc, ncol) * (int64_t)(sw4_block_bytes(h->cfg.nlay) + sw4_image_bytes(true));
    }
    return b;
}

// Argument checks of one request.
static int check_request(RadHandle* h, const RadColumns* in, const RadOutputs* out, int64_t ncol, const char* what)
{
    if (!in || !out) return fail(h, RAD_E_INVALID, std::string(what) + ": null argument");
    if (ncol < 0 || ncol > (int64_t)std::numeric_limits<int>::max() - 1)
        return fail(h, RAD_E_INVALID, std::string(what) + ": ncol out of range");
    if (ncol == 0) return RAD_OK;
    const bool lw = h->cfg.parts & RAD_PART_LW, sw = h->cfg.parts & RAD_PART_SW;
    if (!in->plyr || !in->plvl || !in->tlyr || !in->qlyr || !in->olyr || !in->gasvmr || !in->clouds ||
        (lw && (!in->tlvl || !in->sfcemis || !in->tsfg)) || (sw && (!in->sfcalb || !in->coszen)))
        return fail(h, RAD_E_INVALID, std::string(what) + ": a required input pointer is null");
    if ((lw && (!out->htlw || !out->topflw || !out->sfcflw)) || (sw && (!out->htsw || !out->topfsw || !out->sfcfsw)))
        return fail(h, RAD_E_INVALID, std::string(what) + ": a required output pointer is null");
    return RAD_OK;
}

int rad_solve_batch(RadHandle* h, int32_t nreq, const RadColumns* ins, const RadOutputs* outs, const int64_t* ncols,
                    void* stream)
{
    if (!h) return fail(h, RAD_E_INVALID, "rad_solve_batch: null handle");
    if (nreq < 0 || (nreq > 0 && (!ins || !outs || !ncols))) return fail(h, RAD_E_INVALID, "rad_solve_batch: bad arguments");
    if (!h->tables_ok) return fail(h, RAD_E_TABLES, "rad_solve: tables not loaded (rad_load_tables)");
    for (int32_t r = 0; r < nreq; ++r) {
        const int rc = check_request(h, ins + r, outs + r, ncols[r], "rad_solve");
        if (rc) return rc;
    }
    int dev = 0;
    RAD_CUDA(h, cudaGetDevice(&dev));
    if (dev != h->device) return fail(h, RAD_E_INVALID, "rad_solve: handle belongs to another device");
    cudaStream_t st = (cudaStream_t)stream;
    int32_t r0 = 0;
    while (r0 < nreq) {
        // one launch set per group of at most RAD_MAXREQ requests and 2^31 - 2 columns
        int32_t r1 = r0;
        int64_t cols = 0;
        while (r1 < nreq && r1 - r0 < RAD_MAXREQ && (r1 == r0 || cols + ncols[r1] <= (int64_t)std::numeric_limits<int>::max() - 1))
            cols += ncols[r1++];
        const int rc = h->cfg.precision == RAD_PREC_FP64
                           ? launch_batch<double>(h, r1 - r0, ins + r0, outs + r0, ncols + r0, st)
                           : launch_batch<float>(h, r1 - r0, ins + r0, outs + r0, ncols + r0, st);
        if (rc) return rc;
        r0 = r1;
    }
    return RAD_OK;
}

struct RadGraph {
    RadHandle* h = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t launches = 0;    // kernels one replay runs
};

int rad_graph_create(RadHandle* h, int32_t nreq, const RadColumns* ins, const RadOutputs* outs, const int64_t* ncols,
                     RadGraph** out)
{
    if (!h || !out) return fail(h, RAD_E_INVALID, "rad_graph_create: null argument");
    *out = nullptr;
    // a first, uncaptured pass validates the arguments and grows the scratch to this batch
    cudaStream_t st;
    RAD_CUDA(h, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const bool prof = h->profiling;
    h->profiling = false;
    const int64_t l0 = h->launches;
    int rc = rad_solve_batch(h, nreq, ins, outs, ncols, st);
    const int64_t per = h->launches - l0;
    if (rc == RAD_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = fail(h, RAD_E_CUDA, "rad_graph_create: warm-up solve failed");
    RadGraph* g = nullptr;
    if (rc == RAD_OK) {
        g = new RadGraph();
        g->h = h;
        g->launches = per;
        cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            rc = rad_solve_batch(h, nreq, ins, outs, ncols, st);
            const cudaError_t e2 = cudaStreamEndCapture(st, &g->graph);
            if (rc == RAD_OK && e2 != cudaSuccess) rc = fail(h, RAD_E_CUDA, std::string("rad_graph_create: capture: ") + cudaGetErrorString(e2));
        } else {
            rc = fail(h, RAD_E_CUDA, std::string("rad_graph_create: begin capture: ") + cudaGetErrorString(e));
        }
        if (rc == RAD_OK && cudaGraphInstantiate(&g->exec, g->graph, 0) != cudaSuccess)
            rc = fail(h, RAD_E_CUDA, "rad_graph_create: instantiate failed");
        h->launches = l0 + per;
    }
    h->profiling = prof;
    cudaStreamDestroy(st);
    if (rc != RAD_OK) {
        if (g) {
            if (g->exec) cudaGraphExecDestroy(g->exec);
            if (g->graph) cudaGraphDestroy(g->graph);
            delete g;
        }
        return rc;
    }
    *out = g;
    return RAD_OK;
}

int rad_graph_launch(RadGraph* g, void* stream)
{
    if (!g) return fail(nullptr, RAD_E_INVALID, "rad_graph_launch: null graph");
    RAD_CUDA(g->h, cudaGraphLaunch(g->exec, (cudaStream_t)stream));
    g->h->launches += g->launches;
    return RAD_OK;
}

void rad_graph_destroy(RadGraph* g)
{
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
}

int rad_solve(RadHandle* h, const RadColumns* in, const RadOutputs* out, int64_t ncol, void* stream)
{
    if (!h || !in || !out) return fail(h, RAD_E_INVALID, "rad_solve: null argument");
    return rad_solve_batch(h, 1, in, out, &ncol, stream);
}

// ---------------------------------------------------------------------------- fixed-scratch solve
// rad_solve_noalloc: the day-list scratch of a solve lives in this file-scope device array instead of the
// handle's growing buffers, so the call reaches no allocator.  Layout in 32-bit words, each part 256-byte
// aligned: flag, pos, daycol, lt, k8, kw ([NA_W] each), cmin ([2 NA_W]), nday ([64]), CUB scan temp.  The LW
// part uses pos first, as the [count, columns...] list of the columns it leaves to the float64 column kernel.
// Nothing else in it has to start at zero (the list count is cleared by the solve): every word a solve reads is
// written earlier in the same solve.
namespace {
constexpr int64_t NA_W = ((RAD_NOALLOC_MAX_COLS + 1 + 63) / 64) * 64;
constexpr int64_t NA_CUB_WORDS = 16384;   // 64 KiB for the device-wide scan
constexpr int64_t NA_WORDS = 8 * NA_W + 64 + NA_CUB_WORDS;
__device__ __align__(256) uint32_t g_noalloc_scratch[NA_WORDS];

// The array's address on the current device and the layout over it.  cudaGetSymbolAddress is a runtime
// query that allocates nothing; resolving it on every call keeps the address right after a device reset
// (which gives the array a new address).
int noalloc_scratch(RadHandle* h, LaunchScratch* out)
{
    uint32_t* base = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&base, g_noalloc_scratch);
    if (e != cudaSuccess)
        return fail(h, RAD_E_CUDA, std::string("rad_solve_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    size_t need = 0;
    RAD_CUDA(h, cub::DeviceScan::ExclusiveSum(nullptr, need, (int*)nullptr, (int*)nullptr, (int)(RAD_NOALLOC_MAX_COLS + 1)));
    if (need > (size_t)NA_CUB_WORDS * 4)
        return fail(h, RAD_E_INVALID, "rad_solve_noalloc: the scan needs more temp space than the fixed region holds");
    int* w = (int*)base;
    LaunchScratch& c = *out;
    c.flag = w;
    c.pos = w + NA_W;
    c.daycol = w + 2 * NA_W;
    c.lt = w + 3 * NA_W;
    c.k8 = w + 4 * NA_W;
    c.kw = w + 5 * NA_W;
    c.cmin = w + 6 * NA_W;
    c.nday = w + 8 * NA_W;
    c.cub = (void*)(w + 8 * NA_W + 64);
    c.cub_bytes = (size_t)NA_CUB_WORDS * 4;
    c.max_cols = RAD_NOALLOC_MAX_COLS;
    c.max_cmin = 2 * NA_W;
    return RAD_OK;
}
}  // namespace

int rad_solve_noalloc(RadHandle* h, const RadColumns* in, const RadOutputs* out, int64_t ncol, void* stream)
{
    if (!h || !in || !out) return fail(h, RAD_E_INVALID, "rad_solve_noalloc: null argument");
    if (!h->tables_ok) return fail(h, RAD_E_TABLES, "rad_solve_noalloc: tables not loaded (rad_load_tables)");
    int rc = check_request(h, in, out, ncol, "rad_solve_noalloc");
    if (rc) return rc;
    if (ncol > RAD_NOALLOC_MAX_COLS)
        return fail(h, RAD_E_INVALID, "rad_solve_noalloc: ncol above RAD_NOALLOC_MAX_COLS (65536); use rad_solve");
    if (h->cfg.route == RAD_ROUTE_MCICA && (!out->lw_mask || !out->sw_mask))
        return fail(h, RAD_E_INVALID, "rad_solve_noalloc: the McICA route needs the caller's lw_mask and sw_mask buffers");
    int dev = 0;
    const cudaError_t de = cudaGetDevice(&dev);
    if (de != cudaSuccess) return fail(h, RAD_E_CUDA, std::string("rad_solve_noalloc: cudaGetDevice: ") + cudaGetErrorString(de));
    if (dev != h->device) return fail(h, RAD_E_INVALID, "rad_solve_noalloc: handle belongs to another device");
    if (ncol == 0) return RAD_OK;
    LaunchScratch sc;
    if ((rc = noalloc_scratch(h, &sc))) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    return h->cfg.precision == RAD_PREC_FP64 ? launch_batch<double>(h, 1, in, out, &ncol, st, &sc)
                                             : launch_batch<float>(h, 1, in, out, &ncol, st, &sc);
}

int rad_post_outputs(RadHandle* h, const RadPostIn* in, const RadPostOut* out, int64_t ncol, int32_t lm,
                     int32_t kd, int32_t cloud_block, int32_t lw_step, void* stream)
{
    if (!h || !in || !out) return fail(h, RAD_E_INVALID, "rad_post_outputs: null argument");
    if (ncol < 0 || lm < 1 || kd < 0 || kd > 1) return fail(h, RAD_E_INVALID, "rad_post_outputs: ncol, lm or kd out of range");
    if (ncol == 0) return RAD_OK;
    if (!in->hlw || !in->swh || !in->coszdg_v || !in->coszen_v || !in->sfcflw_dnfxc || !in->topflw_upfxc ||
        !in->sfcfsw_upfxc || !in->sfcfsw_dnfxc || !in->sfcfsw_dnfx0 || !in->topfsw_upfxc || !out->rlwtt ||
        !out->rswtt || !out->rlwin || !out->rswin || !out->rswinc || !out->rswout || !out->rlwtoa || !out->rswtoa ||
        !out->czmean || !out->coszdg)
        return fail(h, RAD_E_INVALID, "rad_post_outputs: a required pointer is null");
    if (cloud_block && (!in->cldcov || !in->cldsa || !in->cw || !in->cu_cloud || !out->cldfra || !out->csmid ||
                        !out->cfracl || !out->cfracm || !out->cfrach || !out->acfrst || !out->acfrcv ||
                        !out->ncfrst || !out->ncfrcv))
        return fail(h, RAD_E_INVALID, "rad_post_outputs: a cloud-diagnostic pointer is null");
    if (lw_step && (!in->t || !out->sigt4)) return fail(h, RAD_E_INVALID, "rad_post_outputs: T / SIGT4 null on an LW step");
    PostArgs a{in->hlw, in->swh, in->coszdg_v, in->coszen_v, in->sfcflw_dnfxc, in->topflw_upfxc, in->sfcfsw_upfxc,
               in->sfcfsw_dnfxc, in->sfcfsw_dnfx0, in->topfsw_upfxc, in->cldcov, in->cldsa, in->cw, in->t,
               in->cu_cloud, out->rlwtt, out->rswtt, out->cldfra, out->csmid, out->rlwin, out->rswin, out->rswinc,
               out->rswout, out->rlwtoa, out->rswtoa, out->czmean, out->sigt4, out->coszdg, out->cfracl, out->cfracm,
               out->cfrach, out->acfrst, out->acfrcv, out->ncfrst, out->ncfrcv, ncol, lm, kd, cloud_block ? 1 : 0,
               lw_step ? 1 : 0};
    const unsigned grid = (unsigned)((ncol + 255) / 256);
    k_post_outputs<<<grid, 256, 0, (cudaStream_t)stream>>>(a);
    h->launches += 1;
    RAD_CUDA(h, cudaGetLastError());
    return RAD_OK;
}

int rad_load_aerosols(RadHandle* h, const RadAerClim* c)
{
    if (!h || !c) return fail(h, RAD_E_INVALID, "rad_load_aerosols: null argument");
    if (!c->iendwv || !c->haer || !c->prsref || !c->rhid || !c->rhdp || !c->straext0 || !c->nwvns0 || !c->s0intv ||
        !c->month_idx || !c->month_cmix || !c->month_kprf || !c->month_denn)
        return fail(h, RAD_E_INVALID, "rad_load_aerosols: a climatology pointer is null");
    int64_t nw = 0;
    for (int b = 0; b < 151; ++b) nw += c->nwvns0[b];
    if (nw != 57600) return fail(h, RAD_E_INVALID, "rad_load_aerosols: the solar spectrum must cover 57,600 wavenumbers");
    for (int i = 0; i < AER_NCELL; ++i)
        if (c->month_kprf[i] < 1 || c->month_kprf[i] > AER_NAE)
            return fail(h, RAD_E_INVALID, "rad_load_aerosols: a profile structure is outside 1..7");
    for (int i = 0; i < AER_NCELL * AER_NXC; ++i)
        if (c->month_idx[i] < 0 || c->month_idx[i] > AER_NCM)
            return fail(h, RAD_E_INVALID, "rad_load_aerosols: a component index is outside 0..10");
    std::vector<float> fb;
    std::vector<int> ib;
    aerh::build(*c, fb, ib);
    RAD_CUDA(h, cudaSetDevice(h->device));
    if (!h->d_aerf) RAD_CUDA(h, cudaMalloc((void**)&h->d_aerf, (size_t)AF_TOTAL * sizeof(float)));
    if (!h->d_aeri) RAD_CUDA(h, cudaMalloc((void**)&h->d_aeri, (size_t)AI_TOTAL * sizeof(int)));
    RAD_CUDA(h, cudaMemcpy(h->d_aerf, fb.data(), fb.size() * sizeof(float), cudaMemcpyHostToDevice));
    RAD_CUDA(h, cudaMemcpy(h->d_aeri, ib.data(), ib.size() * sizeof(int), cudaMemcpyHostToDevice));
    return RAD_OK;
}

int rad_setaer(RadHandle* h, const RadAerColumns* in, int64_t ncol, float* faersw, float* faerlw, void* stream)
{
    if (!h || !in) return fail(h, RAD_E_INVALID, "rad_setaer: null argument");
    if (!h->d_aerf) return fail(h, RAD_E_INVALID, "rad_setaer: no climatology loaded (rad_load_aerosols)");
    if (ncol < 0 || ncol > (int64_t)std::numeric_limits<int>::max() - 1)
        return fail(h, RAD_E_INVALID, "rad_setaer: ncol out of range");
    if (ncol == 0) return RAD_OK;
    if (!in->plvl || !in->plyr || !in->tlyr || !in->qlyr || !in->rhly || !in->xlon || !in->xlat || !in->slmsk ||
        !faersw || !faerlw)
        return fail(h, RAD_E_INVALID, "rad_setaer: a required pointer is null");
    if (h->cfg.nlay > NLAY_MAX) return fail(h, RAD_E_INVALID, "rad_setaer: nlay above NLAY_MAX");
    const float* f = h->d_aerf;
    const int* i = h->d_aeri;
    AerTab t{f + AF_HAER, f + AF_PRSREF, f + AF_SIGREF, f + AF_EXTRHI, f + AF_SCARHI, f + AF_SSARHI, f + AF_ASYRHI,
             f + AF_EXTRHD, f + AF_SCARHD, f + AF_SSARHD, f + AF_ASYRHD, f + AF_EXTSTRA, f + AF_CMIXG, f + AF_DENNG,
             i + AI_IDXCG, i + AI_KPRFG};
    AerArgs a{in->plvl, in->plyr, in->tlyr, in->qlyr, in->rhly, in->xlon, in->xlat, in->slmsk, faersw, faerlw, ncol,
              h->cfg.nlay};
    k_setaer<<<(unsigned)((ncol + AER_COLS - 1) / AER_COLS), AER_THREADS, 0, (cudaStream_t)stream>>>(a, t);
    h->launches += 1;
    RAD_CUDA(h, cudaGetLastError());
    return RAD_OK;
}

int rad_grrad_clw(RadHandle* h, const float* tracer, int32_t ntrac, int32_t lmk, int64_t ncol, int32_t ntcw,
                  int32_t ncld, float epsq, float* clw, void* stream)
{
    if (!h) return fail(h, RAD_E_INVALID, "rad_grrad_clw: null argument");
    if (ncol < 0 || lmk < 1 || ncld < 1 || ntcw < 1 || ntcw - 1 + ncld > ntrac)
        return fail(h, RAD_E_INVALID, "rad_grrad_clw: sizes or tracer range out of range");
    if ((int64_t)lmk * ncol > (int64_t)std::numeric_limits<int>::max() * 256)
        return fail(h, RAD_E_INVALID, "rad_grrad_clw: too many points for one launch");
    if (ncol == 0) return RAD_OK;
    if (!tracer || !clw) return fail(h, RAD_E_INVALID, "rad_grrad_clw: a required pointer is null");
    const front::ClwArgs a{tracer, clw, ncol, lmk, ntcw - 1, ncld, epsq};
    h->launches += 1;
    RAD_CUDA(h, front::grrad_clw(a, (cudaStream_t)stream));
    return RAD_OK;
}

int rad_payne_albedo(RadHandle* h, const float* salbedo, const float* sm, const float* coszen, int64_t ncol,
                     const RadPayneTables* t, float* const* out, void* stream)
{
    if (!h || !t || !out) return fail(h, RAD_E_INVALID, "rad_payne_albedo: null argument");
    if (ncol < 0 || ncol > (int64_t)std::numeric_limits<int>::max() * 256)
        return fail(h, RAD_E_INVALID, "rad_payne_albedo: ncol out of range");
    if (ncol == 0) return RAD_OK;
    if (!salbedo || !sm || !coszen || !t->trn || !t->za || !t->dza || !t->albd)
        return fail(h, RAD_E_INVALID, "rad_payne_albedo: a required pointer is null");
    front::PayneArgs a{};
    a.salbedo = salbedo; a.sm = sm; a.coszen = coszen; a.n = ncol;
    for (int f = 0; f < 9; ++f) {
        if (!out[f]) return fail(h, RAD_E_INVALID, "rad_payne_albedo: an output pointer is null");
        a.out[f] = out[f];
    }
    std::copy(t->trn, t->trn + 21, a.trn);
    std::copy(t->za, t->za + 20, a.za);
    std::copy(t->dza, t->dza + 19, a.dza);
    std::copy(t->albd, t->albd + 20 * 21, a.albd);
    h->launches += 1;
    RAD_CUDA(h, front::payne_albedo(a, (cudaStream_t)stream));
    return RAD_OK;
}

int rad_setaer_volc(RadHandle* h, const float* plvl, const float* xlat, int64_t ncol, int32_t ivflip,
                    const int32_t* ivolae, int32_t kyrsav, int32_t kmonsav, int32_t add_sw, int32_t add_lw,
                    int32_t lw1bd, float* faersw, float* faerlw, void* stream)
{
    if (!h) return fail(h, RAD_E_INVALID, "rad_setaer_volc: null argument");
    if (ncol < 0 || ncol > (int64_t)std::numeric_limits<int>::max() - 1)
        return fail(h, RAD_E_INVALID, "rad_setaer_volc: ncol out of range");
    if (h->cfg.nlay < 4 || h->cfg.nlay > NLAY_MAX) return fail(h, RAD_E_INVALID, "rad_setaer_volc: nlay out of range");
    if (ivflip != 0 && ivflip != 1) return fail(h, RAD_E_INVALID, "rad_setaer_volc: ivflip must be 0 or 1");
    if (kmonsav < 1 || kmonsav > 12) return fail(h, RAD_E_INVALID, "rad_setaer_volc: kmonsav outside 1..12");
    if (!ivolae) return fail(h, RAD_E_INVALID, "rad_setaer_volc: ivolae is null");
    if (ncol == 0 || (!add_sw && !add_lw)) return RAD_OK;
    if (!plvl || !xlat || (add_sw && !faersw) || (add_lw && !faerlw))
        return fail(h, RAD_E_INVALID, "rad_setaer_volc: a required pointer is null");
    front::VolcArgs a{};
    a.plvl = plvl; a.xlat = xlat; a.faersw = faersw; a.faerlw = faerlw; a.n = ncol;
    a.nlay = h->cfg.nlay; a.ivflip = ivflip; a.add_sw = add_sw != 0; a.add_lw = add_lw != 0;
    const int y = ((kyrsav % 10) + 10) % 10;                // Python's kyrsav % 10, as the reference's wrapper
    for (int z = 0; z < 4; ++z) a.iv[z] = ivolae[(y * 4 + z) * 12 + (kmonsav - 1)];
    for (int b = 0; b < AER_NSW; ++b) {
        const float w1 = (float)aerh::WSW[0][b], w2 = (float)aerh::WSW[1][b];
        const float e = w1 > 20000.0f ? 0.74f : (w2 < 20000.0f ? 1.14f : 0.94f);
        a.tsw[b] = powf(0.275e-4f * (w2 + w1), e);
    }
    for (int b = 0; b < AER_NLW; ++b)
        a.tlw[b] = lw1bd ? powf(0.55f / 11.0f, 1.2f)
                         : powf(0.275e-4f * ((float)aerh::WLW[1][b] + (float)aerh::WLW[0][b]), 1.2f);
    h->launches += 1;
    RAD_CUDA(h, front::setaer_volc(a, (cudaStream_t)stream));
    return RAD_OK;
}

int rad_grrad_setup(RadHandle* h, const RadModelColumns* in, int64_t ncol, int32_t lm, const RadLayerFields* out,
                    void* stream)
{
    if (!h || !in || !out) return fail(h, RAD_E_INVALID, "rad_grrad_setup: null argument");
    if (ncol < 0 || lm < 1 || lm + 1 > NLAY_MAX) return fail(h, RAD_E_INVALID, "rad_grrad_setup: ncol or lm out of range");
    if (ncol == 0) return RAD_OK;
    if (!in->pint || !in->pmid || !in->prslk || !in->t || !in->q || !in->tsfc || !out->plvl || !out->plyr ||
        !out->tlyr || !out->tlvl || !out->qlyr || !out->rhly || !out->qstl || !out->prslk1 || !out->tvly || !out->tsfg)
        return fail(h, RAD_E_INVALID, "rad_grrad_setup: a required pointer is null");
    GrradArgs a{in->pint, in->pmid, in->prslk, in->t, in->q, in->tsfc, out->plvl, out->plyr, out->tlyr, out->tlvl,
                out->qlyr, out->rhly, out->qstl, out->prslk1, out->tvly, out->tsfg, ncol, lm};
    k_grrad_setup<<<(unsigned)((ncol + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a);
    h->launches += 1;
    RAD_CUDA(h, cudaGetLastError());
    return RAD_OK;
}

int rad_sol_update(const RadSolarIn* in, RadSolarState* out)
{
    if (!in || !out) return fail(nullptr, RAD_E_INVALID, "rad_sol_update: null argument");
    if (in->month < 1 || in->month > 12 || in->day < 1 || in->day > 31 || in->hour < 0 || in->hour > 23 ||
        in->minute < 0 || in->minute > 59 || in->second < 0 || in->second > 60)
        return fail(nullptr, RAD_E_INVALID, "rad_sol_update: date or time out of range");
    if (!(in->deltim > 0.0f) || !(in->deltsw > 0.0f) || !(in->solc0 > 0.0))
        return fail(nullptr, RAD_E_INVALID, "rad_sol_update: deltsw, deltim and solc0 must be positive");
    solh::update(*in, *out);
    return RAD_OK;
}

int rad_coszmn(RadHandle* h, const RadSolarState* s, const float* glon, const float* glat, int64_t n, float solhr,
               float dtswav, int32_t nrads, float* coszen, float* coszdg, void* stream)
{
    if (!h || !s) return fail(h, RAD_E_INVALID, "rad_coszmn: null argument");
    if (n < 0 || nrads < 1 || !(dtswav > 0.0f)) return fail(h, RAD_E_INVALID, "rad_coszmn: n, nrads or dtswav out of range");
    if (n == 0) return RAD_OK;
    if (!glon || !glat || !coszen || !coszdg) return fail(h, RAD_E_INVALID, "rad_coszmn: a required pointer is null");
    CoszArgs a{glon, glat, coszen, coszdg, n, s->sollag, s->sindec, s->cosdec, solhr, dtswav, nrads};
    k_coszmn<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a);
    h->launches += 1;
    RAD_CUDA(h, cudaGetLastError());
    return RAD_OK;
}

// ---- grrad's front end (kernels in rad_front.cu) ----

int rad_dayparts(RadHandle* h, const RadSolarState* s, const float* xlon, const float* sinlat, const float* coslat,
                 int32_t im, int32_t jm, float solhr, float dtswav, int32_t nrads, const RadDayparts* out, void* stream)
{
    if (!h || !s || !out) return fail(h, RAD_E_INVALID, "rad_dayparts: null argument");
    if (im < 0 || jm < 0 || nrads < 1 || !(dtswav > 0.0f))
        return fail(h, RAD_E_INVALID, "rad_dayparts: im, jm, nrads or dtswav out of range");
    if (im > front::DAYPARTS_MAX_IM) return fail(h, RAD_E_INVALID, "rad_dayparts: a row is longer than 24576 points");
    if ((int64_t)im * jm == 0) return RAD_OK;
    if (!xlon || !sinlat || !coslat || !out->coszen || !out->coszdg || !out->dp_start || !out->dp_len ||
        !out->dp_day || !out->ndayparts)
        return fail(h, RAD_E_INVALID, "rad_dayparts: a required pointer is null");
    const front::DaypartsArgs a{xlon, sinlat, coslat, out->coszen, out->coszdg, out->dp_start, out->dp_len,
                                out->dp_day, out->ndayparts, im, jm, nrads, solhr, dtswav, s->sollag, s->sindec,
                                s->cosdec};
    h->launches += 1;
    RAD_CUDA(h, front::dayparts(a, (cudaStream_t)stream));
    return RAD_OK;
}

int rad_getgases(RadHandle* h, const float* plvl, const float* xlon, const float* xlat, int64_t ncol, int32_t lmax,
                 const RadGasSetup* g, float* gasvmr, void* stream)
{
    if (!h || !g) return fail(h, RAD_E_INVALID, "rad_getgases: null argument");
    if (ncol < 0 || lmax < 1) return fail(h, RAD_E_INVALID, "rad_getgases: ncol or lmax out of range");
    if (g->ico2flg < 0 || g->ico2flg > 2) return fail(h, RAD_E_INVALID, "rad_getgases: ico2flg is not 0, 1 or 2");
    if (g->ico2flg != 0 && (g->kmonsav < 1 || g->kmonsav > 12))
        return fail(h, RAD_E_INVALID, "rad_getgases: kmonsav must be 1..12 when ico2flg is 1 or 2");
    if (g->ivflip != 0 && g->ivflip != 1) return fail(h, RAD_E_INVALID, "rad_getgases: ivflip must be 0 or 1");
    if (ncol == 0) return RAD_OK;
    if (!gasvmr || (g->ico2flg != 0 && (!g->co2_glb || !g->gco2cyc)) ||
        (g->ico2flg == 2 && (!plvl || !xlon || !xlat || !g->co2vmr_sav)))
        return fail(h, RAD_E_INVALID, "rad_getgases: a required pointer is null");
    const front::GasArgs a{plvl, xlon, xlat, g->co2_glb, g->gco2cyc, g->co2vmr_sav, gasvmr, ncol, lmax, g->ico2flg,
                           g->kmonsav, g->ivflip};
    h->launches += 1;
    RAD_CUDA(h, front::getgases(a, (cudaStream_t)stream));
    return RAD_OK;
}

int rad_getozn(RadHandle* h, const float* prslk, const float* xlat, int64_t ncol, int32_t nlev, const RadOzoneClim* oz,
               float* o3mmr, void* stream)
{
    if (!h || !oz) return fail(h, RAD_E_INVALID, "rad_getozn: null argument");
    if (ncol < 0 || nlev < 1) return fail(h, RAD_E_INVALID, "rad_getozn: ncol or nlev out of range");
    if (oz->loz < 2 || oz->loz > front::OZONE_MAX_LOZ || oz->jmr < 1 || oz->jmr > front::OZONE_MAX_JMR)
        return fail(h, RAD_E_INVALID, "rad_getozn: loz must be 2..64 and jmr 1..360");
    if (oz->k1oz < 1 || oz->k1oz > 12 || oz->k2oz < 1 || oz->k2oz > 12)
        return fail(h, RAD_E_INVALID, "rad_getozn: the ozone months are not set (k1oz, k2oz must be 1..12)");
    if (oz->ivflip != 0 && oz->ivflip != 1) return fail(h, RAD_E_INVALID, "rad_getozn: ivflip must be 0 or 1");
    if (!(oz->dlte > 0.0f)) return fail(h, RAD_E_INVALID, "rad_getozn: dlte must be positive");
    if (ncol == 0) return RAD_OK;
    if (!prslk || !xlat || !oz->o3r || !oz->pkstr || !o3mmr)
        return fail(h, RAD_E_INVALID, "rad_getozn: a required pointer is null");
    const front::OzoneArgs a{prslk, xlat, oz->o3r, oz->pkstr, o3mmr, ncol, nlev, oz->jmr, oz->loz, oz->k1oz, oz->k2oz,
                             oz->ivflip, oz->facoz, oz->blte, oz->dlte};
    h->launches += 1;
    RAD_CUDA(h, front::getozn(a, (cudaStream_t)stream));
    return RAD_OK;
}

int rad_setalb(RadHandle* h, const RadAlbedoIn* in, int64_t ncol, int32_t ialbflg, float* sfcalb, void* stream)
{
    if (!h || !in) return fail(h, RAD_E_INVALID, "rad_setalb: null argument");
    if (ncol < 0) return fail(h, RAD_E_INVALID, "rad_setalb: ncol out of range");
    if (ncol == 0) return RAD_OK;
    const bool all = ialbflg == 0 || ialbflg == 1;
    if (!sfcalb || !in->alvsf || !in->alnsf || !in->alvwf || !in->alnwf ||
        (all && (!in->slmsk || !in->snowf || !in->zorlf || !in->coszf || !in->tsknf || !in->hprif || !in->facsf ||
                 !in->facwf || !in->fice || !in->tisfc)) ||
        (ialbflg == 1 && (!in->sncovr || !in->snoalb)))
        return fail(h, RAD_E_INVALID, "rad_setalb: a required pointer is null");
    const front::AlbedoArgs a{in->slmsk, in->snowf, in->sncovr, in->snoalb, in->zorlf, in->coszf, in->tsknf, in->hprif,
                              in->alvsf, in->alnsf, in->alvwf, in->alnwf, in->facsf, in->facwf, in->fice, in->tisfc,
                              sfcalb, ncol, ialbflg};
    h->launches += 1;
    RAD_CUDA(h, front::setalb(a, (cudaStream_t)stream));
    return RAD_OK;
}

int rad_setemis(RadHandle* h, const RadEmisIn* in, int64_t ncol, int32_t ialbflg, int32_t iemslw, float* sfcemis,
                void* stream)
{
    if (!h || !in) return fail(h, RAD_E_INVALID, "rad_setemis: null argument");
    if (ncol < 0) return fail(h, RAD_E_INVALID, "rad_setemis: ncol out of range");
    if (ncol == 0) return RAD_OK;
    if (!sfcemis || (iemslw != 0 && (!in->glon || !in->glat || !in->sm || !in->sice || !in->si || !in->z0 ||
                                     !in->stdh || !in->tskin || !in->idxems || (ialbflg == 1 && !in->sncovr))))
        return fail(h, RAD_E_INVALID, "rad_setemis: a required pointer is null");
    const front::EmisArgs a{in->glon, in->glat, in->sm, in->sice, in->si, in->sncovr, in->z0, in->stdh, in->tskin,
                            in->idxems, sfcemis, ncol, ialbflg, iemslw};
    h->launches += 1;
    RAD_CUDA(h, front::setemis(a, (cudaStream_t)stream));
    return RAD_OK;
}

int rad_progcld2(RadHandle* h, const RadCloudIn* in, int64_t ncol, int32_t nlay, const RadCloudCfg* cfg,
                 const RadCloudOut* out, void* stream)
{
    if (!h || !in || !cfg || !out) return fail(h, RAD_E_INVALID, "rad_progcld2: null argument");
    if (ncol < 0 || nlay < 2 || nlay > front::CLOUD_MAX_LAY)
        return fail(h, RAD_E_INVALID, "rad_progcld2: ncol or nlay out of range (2 <= nlay <= 128)");
    if (cfg->ivflip != 0 && cfg->ivflip != 1) return fail(h, RAD_E_INVALID, "rad_progcld2: ivflip must be 0 or 1");
    if (cfg->llyr < 1 || cfg->llyr > nlay) return fail(h, RAD_E_INVALID, "rad_progcld2: llyr outside 1..nlay");
    if (ncol == 0) return RAD_OK;
    if (!in->plyr || !in->plvl || !in->tlyr || !in->tvly || !in->qlyr || !in->qstl || !in->rhly || !in->clw ||
        !in->f_ice || !in->f_rain || !in->xlat || (cfg->cld_fraction != 0 && !in->cldfk1) || !out->clouds ||
        !out->clds || !out->mtop || !out->mbot)
        return fail(h, RAD_E_INVALID, "rad_progcld2: a required pointer is null");
    const front::CloudArgs a{in->plyr, in->plvl, in->tlyr, in->tvly, in->qlyr, in->qstl, in->rhly, in->clw, in->f_ice,
                             in->f_rain, in->cldfk1, in->xlat, out->clouds, out->clds, out->mtop, out->mbot, ncol,
                             nlay, cfg->ivflip, cfg->llyr, cfg->iovr, cfg->lcrick, cfg->lcnorm, cfg->lnoprec,
                             cfg->lsashal, cfg->cld_fraction};
    h->launches += 1;
    RAD_CUDA(h, front::progcld2(a, (cudaStream_t)stream));
    return RAD_OK;
}

int rad_rdtemp(RadHandle* h, const RadRdtemp* p, void* stream)
{
    if (!h || !p) return fail(h, RAD_E_INVALID, "rad_rdtemp: null argument");
    if (p->im < 1 || p->jm < 1 || p->lm < 1) return fail(h, RAD_E_INVALID, "rad_rdtemp: empty grid");
    if (!p->glat || !p->glon || !p->czmean || !p->rswtt || !p->rlwtt || !p->czen || !p->t)
        return fail(h, RAD_E_INVALID, "rad_rdtemp: a required pointer is null");
    if (p->julday < 1 || p->julday > 366) return fail(h, RAD_E_INVALID, "rad_rdtemp: julday out of range");
    RdtempArgs a{p->ntsd, p->dt, p->julday, p->julyr, p->ihrst, p->leap_seen, p->glat, p->glon, p->czmean,
                 p->rswtt, p->rlwtt, p->czen, p->t, p->im, p->jm, p->lm, p->its, p->ite, p->jts, p->jte,
                 p->its_b1, p->ite_b1, p->jts_b1, p->jte_b1};
    const int64_t n = (int64_t)p->im * p->jm;
    k_rdtemp<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a);
    h->launches += 1;
    RAD_CUDA(h, cudaGetLastError());
    return RAD_OK;
}

// ------------------------------------------------------------------------------------------------- queue
struct RadQueue {
    struct Slot {
        RadHandle* h = nullptr;
        cudaStream_t st = nullptr;
        cudaEvent_t ev = nullptr;
        int64_t ticket = 0;          // 0: free
        int64_t bytes = 0;           // scratch charged against the budget while the ticket runs
    };
    std::vector<Slot> slots;
    int64_t budget = 0, in_use = 0, next = 1;
    std::mutex mu;
};

int rad_queue_create(RadHandle* const* slots, int32_t nslots, int64_t hbm_budget_bytes, RadQueue** out)
{
    if (!slots || !out || nslots < 1 || hbm_budget_bytes < 0)
        return fail(nullptr, RAD_E_INVALID, "rad_queue_create: null argument, no slot or a negative budget");
    *out = nullptr;
    RadQueue* q = new RadQueue();
    q->budget = hbm_budget_bytes;
    for (int i = 0; i < nslots; ++i) {
        RadQueue::Slot sl;
        sl.h = slots[i];
        if (!sl.h || !sl.h->tables_ok ||
            cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) != cudaSuccess) {
            if (sl.st) cudaStreamDestroy(sl.st);
            q->slots.push_back(sl);
            rad_queue_destroy(q);
            return fail(nullptr, RAD_E_INVALID, "rad_queue_create: a slot handle is null or has no tables, or a "
                                                 "stream / event could not be created");
        }
        q->slots.push_back(sl);
    }
    *out = q;
    return RAD_OK;
}

int rad_submit(RadQueue* q, const RadColumns* in, const RadOutputs* out, int64_t ncol, int64_t* ticket)
{
    if (!q || !in || !out || !ticket) return fail(nullptr, RAD_E_INVALID, "rad_submit: null argument");
    std::lock_guard<std::mutex> lock(q->mu);
    *ticket = 0;
    RadQueue::Slot* free_slot = nullptr;
    for (auto& sl : q->slots)
        if (!sl.ticket) { free_slot = &sl; break; }
    if (!free_slot) return fail(nullptr, RAD_E_BUSY, "rad_submit: every slot is in use");
    const int64_t need = rad_workspace_bytes(free_slot->h, ncol);
    if (q->budget > 0 && need > q->budget)
        return fail(free_slot->h, RAD_E_INVALID, "rad_submit: the request's scratch exceeds the whole HBM budget");
    if (q->budget > 0 && q->in_use + need > q->budget)
        return fail(free_slot->h, RAD_E_BUDGET, "rad_submit: the request's scratch does not fit beside those in flight");
    int rc = rad_solve(free_slot->h, in, out, ncol, free_slot->st);
    if (rc) return rc;
    RAD_CUDA(free_slot->h, cudaEventRecord(free_slot->ev, free_slot->st));
    free_slot->ticket = q->next++;
    free_slot->bytes = need;
    q->in_use += need;
    *ticket = free_slot->ticket;
    return RAD_OK;
}

int rad_poll(RadQueue* q, int64_t ticket, int32_t* done)
{
    if (!q || !done) return fail(nullptr, RAD_E_INVALID, "rad_poll: null argument");
    std::lock_guard<std::mutex> lock(q->mu);
    *done = 0;
    if (ticket < 1 || ticket >= q->next) return fail(nullptr, RAD_E_INVALID, "rad_poll: unknown ticket");
    for (auto& sl : q->slots) {
        if (sl.ticket != ticket) continue;
        const cudaError_t e = cudaEventQuery(sl.ev);
        if (e == cudaErrorNotReady) return RAD_OK;
        sl.ticket = 0;
        q->in_use -= sl.bytes;
        sl.bytes = 0;
        if (e != cudaSuccess) return fail(sl.h, RAD_E_CUDA, std::string("rad_poll: ") + cudaGetErrorString(e));
        *done = 1;
        return RAD_OK;
    }
    *done = 1;   // completed and reaped by an earlier poll
    return RAD_OK;
}

int rad_wait(RadQueue* q, int64_t ticket, int32_t timeout_ms)
{
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        int32_t done = 0;
        const int rc = rad_poll(q, ticket, &done);
        if (rc || done) return rc;
        if (std::chrono::steady_clock::now() - t0 >= std::chrono::milliseconds(std::max(timeout_ms, 0)))
            return fail(nullptr, RAD_E_TIMEOUT, "rad_wait: the ticket is still running");
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

void rad_queue_destroy(RadQueue* q)
{
    if (!q) return;
    for (auto& sl : q->slots) {
        if (sl.st) {
            cudaStreamSynchronize(sl.st);
            cudaStreamDestroy(sl.st);
        }
        if (sl.ev) cudaEventDestroy(sl.ev);
    }
    delete q;
}

int rad_device_error(RadHandle* h, int32_t* code)
{
    if (!h || !code) return fail(h, RAD_E_INVALID, "rad_device_error: null argument");
    int v = 0;
    RAD_CUDA(h, cudaMemcpy(&v, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    RAD_CUDA(h, cudaMemset(h->d_err, 0, sizeof(int)));
    *code = v;
    return RAD_OK;
}

int rad_profile_enable(RadHandle* h, int on)
{
    if (!h) return fail(h, RAD_E_INVALID, "rad_profile_enable: null handle");
    h->profiling = on != 0;
    h->ev_used = 0;
    h->prof_solves = h->prof_columns = 0;
    return RAD_OK;
}

int rad_profile_read(RadHandle* h, RadProfile* p)
{
    if (!h || !p) return fail(h, RAD_E_INVALID, "rad_profile_read: null argument");
    *p = RadProfile{};
    p->launches = h->launches;
    p->solves = h->prof_solves;
    p->columns = h->prof_columns;
    if (h->ev_used) RAD_CUDA(h, cudaEventSynchronize(h->ev[h->ev_used - 1]));
    for (size_t b = 0; b + 4 <= h->ev_used; b += 4) {
        float t[3];
        for (int i = 0; i < 3; ++i) RAD_CUDA(h, cudaEventElapsedTime(&t[i], h->ev[b + i], h->ev[b + i + 1]));
        p->lw_ms += t[0];
        p->prep_ms += t[1];
        p->sw_ms += t[2];
    }
    return RAD_OK;
}

const char* rad_last_error(const RadHandle* h) { return h ? h->err.c_str() : g_err.c_str(); }

void rad_destroy(RadHandle* h)
{
    if (!h) return;
    for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
    for (void* p : {(void*)h->d_lwf, (void*)h->d_swf, (void*)h->d_lwd, (void*)h->d_swd,
                    (void*)h->d_err, (void*)h->d_flag, (void*)h->d_pos, (void*)h->d_daycol, (void*)h->d_lt,
                    (void*)h->d_k8, (void*)h->d_kw, (void*)h->d_cmin, (void*)h->d_nday, h->d_cub, (void*)h->d_lwm,
                    (void*)h->d_swm, (void*)h->d_lw3, (void*)h->d_lw3list, (void*)h->d_swrt, (void*)h->d_sw4, (void*)h->d_sw4img, (void*)h->d_lwpg, (void*)h->d_swpg, (void*)h->d_aerf,
                    (void*)h->d_aeri})
        if (p) cudaFree(p);
    delete h;
}

}  // extern "C"
