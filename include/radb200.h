/* radb200.h -- C ABI of the B200 RRTM longwave + shortwave column-radiation library (libradb200.so).
 *
 * The library replaces the column solve that WOOF-NAM's radiation driver hook runs between the grrad
 * input set-up and driver_post: the reference binds it as the callable `rrtm_call(ctx, args)` handed to
 * `phys_rad_driver.run(ctx, *, radupdate=None, rrtm_call=None, mype=0)`
 * (namgpu/physics/driver/phys_rad_driver.py:25-30, :171, :255-262), whose column work is
 * `lwrad.run(ctx)` (namgpu/physics/rrtm/phys_rrtm_lw_lwrad.py:247) and `swrad.run(ctx, has_htrswb, nc)`
 * (namgpu/physics/rrtm/phys_rrtm_sw_swrad.py:282).  Inputs and outputs keep the reference's arrays,
 * names, units and layout: float32, [field][level][column] with the column index fastest and level 0 the
 * model top (the reference's [field, level, JM, IM] with JM*IM columns flattened).
 *
 * Conventions: every entry returns 0 or a negative RAD_E_* code; rad_last_error() gives the message.
 * Device pointers only in rad_solve (the caller owns inputs and outputs, the library owns its scratch
 * and tables); rad_solve is asynchronous on the given stream and performs no host synchronisation.
 * One handle per host thread or stream; calls on distinct handles are thread-safe.
 */
#ifndef RADB200_H
#define RADB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RAD_ABI_VERSION 2

enum {
    RAD_OK = 0,
    RAD_E_INVALID = -1,      /* bad argument, shape or configuration */
    RAD_E_TABLES = -2,       /* tables missing or malformed */
    RAD_E_CUDA = -3,         /* a CUDA call failed */
    RAD_E_NOMEM = -4,        /* device allocation failed */
    RAD_E_BUDGET = -5,       /* request refused by the HBM budget (serving queue) */
    RAD_E_TIMEOUT = -6,      /* a bounded wait gave up (serving queue) */
    RAD_E_BUSY = -7          /* queue full or slot in use */
};

enum { RAD_PREC_FP64 = 0, RAD_PREC_MIXED = 1 };
enum { RAD_ROUTE_NAM = 0, RAD_ROUTE_MCICA = 1 };
enum { RAD_PART_LW = 1, RAD_PART_SW = 2 };   /* RadConfig.parts bits */

typedef struct RadHandle RadHandle;

/* Solve configuration.  Defaults (rad_config_default) are NAM's runtime switches: iswmode 2 (PIFM),
 * iovrlw = iovrsw = 1 (maximum-random), prognostic clouds, cloud-path factor 1.5 for LW
 * (module_RA_RRTM.F90:212 as cited at namgpu/physics/rrtm/phys_rrtm_grrad_lw.py:75). */
typedef struct {
    int32_t nlay;            /* radiation layers, including the extra top layer (61 for 60 model layers) */
    int32_t precision;       /* RAD_PREC_FP64 or RAD_PREC_MIXED */
    int32_t route;           /* RAD_ROUTE_NAM (rtrnmr or rtrn + spcvrtc) or RAD_ROUTE_MCICA */
    int32_t iswmode;         /* SW two-stream: 1 delta-Eddington, 2 PIFM, 3 discrete ordinates */
    int32_t diagnostic;      /* 1: clouds hold optical depth / SSA / asymmetry (ilwcliq = iswcliq = 0) */
    int32_t window_cols;     /* columns per SW MINVAL(laytrop) window, 0 = the whole request */
    int32_t sw_chunk;        /* SW day columns per chunk (reference 32768) */
    int32_t iovrlw, iovrsw;  /* cloud overlap, 0 random, 1 max-random, 2 maximum.  McICA route: the sub-column
                                generators' overlap.  NAM route: iovrlw 0 runs rtrn (random overlap,
                                phys_rrtm_lw_rtrn.cu), 1 or 2 rtrnmr (lwrad's dispatch,
                                phys_rrtm_lw_lwrad.py:102-111); iovrsw sets swrad's clear-sky view fraction
                                zcf0 (phys_rrtm_sw_swrad.cu:251-279) */
    int32_t lw_seed0, sw_seed0;   /* McICA permutation seed offsets (ipsdlw0 = 140, ipsdsw0 = 1) */
    float cpathfac;          /* LW cloud-path factor (1.5) */
    int32_t parts;           /* RAD_PART_LW | RAD_PART_SW (default both): which solves rad_solve runs, for
                                steps where only one of lslwr / lsswr holds (module_RA_RRTM.F90:842-846 as
                                cited at namgpu/physics/rrtm/rrtm_call.py:37); the other part's inputs and
                                outputs may then be NULL */
    int32_t lw_chunk;        /* mixed precision: columns per LW chunk of the two-kernel LW (gas optics through
                                ~95 KB per column of scratch, then the sweeps); 0 = 32768; negative = the
                                single-kernel LW (gas optics in shared memory, no scratch) */
    int32_t sw_sweep_chunk;  /* mixed precision: day columns per chunk of the two-kernel SW (set-up, optics and
                                the layer reflectances / transmittances through ~330 KB per column of scratch, then
                                the adding sweeps); 0 = 16384; negative = the single-kernel SW (no scratch besides
                                the R/T stores) */
} RadConfig;

/* Column inputs (device pointers, float32).  ncol columns, nlay layers, nlp1 = nlay + 1 levels. */
typedef struct {
    const float* plyr;       /* [nlay][ncol]    layer pressure, mb        (RAD_PLYR) */
    const float* plvl;       /* [nlp1][ncol]    interface pressure, mb    (RAD_PLVL) */
    const float* tlyr;       /* [nlay][ncol]    layer temperature, K      (RAD_TLYR) */
    const float* tlvl;       /* [nlp1][ncol]    level temperature, K      (TLVL) */
    const float* qlyr;       /* [nlay][ncol]    specific humidity, kg/kg  (QLYR) */
    const float* olyr;       /* [nlay][ncol]    ozone mass mixing ratio   (RAD_OLYR) */
    const float* gasvmr;     /* [10][nlay][ncol] co2 n2o ch4 o2 co cfc11 cfc12 cfc22 ccl4 cfc113 (GASVMR) */
    const float* clouds;     /* [9][nlay][ncol]  cfrac clwp relw ciwp reiw rain rrain snow rsnow (RAD_CLOUDS) */
    const float* faerlw;     /* [3][16][nlay][ncol] tau, ssa, asy per LW band, or NULL (no aerosol) */
    const float* faersw;     /* [3][14][nlay][ncol] tau, ssa, asy per SW band, or NULL */
    const float* sfcemis;    /* [ncol] surface emissivity */
    const float* tsfg;       /* [ncol] ground temperature, K (RAD_TSFG) */
    const float* sfcalb;     /* [4][ncol] nir-beam, nir-diffuse, uv-vis beam, uv-vis diffuse (SFCALB) */
    const float* coszen;     /* [ncol] cosine of the solar zenith angle (SW_COSZEN) */
    const int32_t* icseed;   /* [2][ncol] McICA seeds, LW row then SW row (icsdlw, icsdsw), or NULL for
                                seed0 + column + 1 (isubcl 1, radlw/radsw_main_nmmb.f) */
    float solcon;            /* solar constant of this call, W/m2 */
} RadColumns;

/* Outputs (device pointers, float32); any optional pointer may be NULL. */
typedef struct {
    float* htlw;             /* [nlay][ncol] LW total-sky heating rate, K/s   (htlwc) */
    float* htsw;             /* [nlay][ncol] SW total-sky heating rate, K/s   (HTSWC) */
    float* topflw;           /* [2][ncol] TOA upward LW: total, clear         (topflw upfxc, upfx0) */
    float* sfcflw;           /* [4][ncol] sfc LW: up total, up clear, down total, down clear */
    float* topfsw;           /* [3][ncol] TOA SW: up total, down, up clear    (TOPFLX) */
    float* sfcfsw;           /* [4][ncol] sfc SW: up total, down total, up clear, down clear (SFCFLX) */
    float* fdncmp;           /* [6][ncol] uvbf0 uvbfc nirbm nirdf visbm visdf (FDNCMP), optional */
    uint32_t* lw_mask;       /* [5][nlay][ncol] McICA LW sub-column cloud words, optional (McICA route):
                                bit g & 31 of word g >> 5 for g-point g, layers surface first (lcloudy) */
    uint32_t* sw_mask;       /* [4][nlay][ncol] McICA SW sub-column cloud words, optional, same packing */
    /* Optional outputs of lwrad / swrad (NULL = not wanted), levels top first, as the reference's units write
     * them when their switches are on (phys_rrtm_sw_swrad.py:49-51, phys_rrtm_lw_lwrad.py:47-50; kernels
     * phys_rrtm_sw_swrad.cu:393-418, phys_rrtm_lw_rtrnmr_body.cuh:328-362, phys_rrtm_lw_lwrad.cu:343-363).
     * They run on rad_solve's mixed-precision path with the chunked LW and SW (lw_chunk >= 0,
     * sw_sweep_chunk >= 0); another configuration, or rad_solve_noalloc, refuses them with RAD_E_INVALID. */
    float* hsw0;             /* [nlay][ncol] SW clear-sky heating rate, K/s (HSW0, lhsw0) */
    float* htswb;            /* [14][nlay][ncol] SW heating rate per band, K/s (HTSWB, lhswb) */
    float* swflxprf;         /* [4][nlay + 1][ncol] SW level fluxes: up total, down total, up clear, down clear
                                (FLXPRF, lflxprf) */
    float* hlw0;             /* [nlay][ncol] LW clear-sky heating rate, K/s (htlw0, lhlw0) */
    float* hlwb;             /* [16][nlay][ncol] LW heating rate per band, K/s (htlwb, lhlwb) */
    float* lwflxprf;         /* [4][nlay + 1][ncol] LW level fluxes, same order (flwprf, lflxprf) */
} RadOutputs;

/* Library version (RAD_ABI_VERSION).  Replaces: nothing in the reference (a versioned ABI). */
int rad_version(void);

/* Fill *cfg with the NAM defaults for nlay layers. */
void rad_config_default(RadConfig* cfg, int32_t nlay);

/* Create a handle on the current CUDA device.  Replaces the reference's per-unit table and scratch set-up
 * (namgpu/physics/rrtm/lw_core.py:217-286 seam, phys_rrtm_sw_swrad.py:168-212 chunk_scratch). */
int rad_create(const RadConfig* cfg, RadHandle** out);

/* Load the packed k-distribution / cloud-optics / Planck tables (blob made by woof_nam_b200.tables).
 * Replaces the reference's npz loads (namgpu/physics/rrtm/phys_rrtm_lw_setcoef.py:160-169 and the band
 * units' load_tables). */
int rad_load_tables(RadHandle* h, const void* blob, size_t nbytes);

/* Solve ncol columns: LW on every column, SW on the sunlit ones (coszen >= 1e-4).  Replaces
 * lwrad.run (phys_rrtm_lw_lwrad.py:247) + swrad.run (phys_rrtm_sw_swrad.py:282) as rrtm_call drives them
 * (namgpu/physics/rrtm/rrtm_call.py:246).  stream is a cudaStream_t (NULL = legacy default stream). */
int rad_solve(RadHandle* h, const RadColumns* in, const RadOutputs* out, int64_t ncol, void* stream);

/* Scratch bytes rad_solve needs for ncol columns (the HBM admission budget uses it). */
int64_t rad_workspace_bytes(const RadHandle* h, int64_t ncol);

/* Batched solve of several independent requests in one launch set (uneven domains).  Each request keeps
 * its own SW MINVAL(laytrop) groups, so every result equals the result of solving it alone. */
int rad_solve_batch(RadHandle* h, int32_t nreq, const RadColumns* ins, const RadOutputs* outs,
                    const int64_t* ncols, void* stream);

/* A batched solve captured once into a CUDA graph and replayed (no counterpart in the reference, which
 * launches ~52k kernels per radiation call).  The graph binds the requests' buffers and solcon at capture
 * time: refill the input buffers in place between launches; re-capture when a pointer, a column count or
 * solcon changes.  rad_graph_create allocates the handle's scratch for the batch before capturing, so the
 * replay allocates nothing.  A graph belongs to its handle and must be destroyed before it. */
typedef struct RadGraph RadGraph;
int rad_graph_create(RadHandle* h, int32_t nreq, const RadColumns* ins, const RadOutputs* outs,
                     const int64_t* ncols, RadGraph** out);
int rad_graph_launch(RadGraph* g, void* stream);
void rad_graph_destroy(RadGraph* g);

/* ---- serving queue: continuous batching of whole-request solves (the rad_submit / rad_poll pair of the
 * boundary; the reference has no serving path -- its rrtm_call is synchronous per model step,
 * namgpu/physics/rrtm/rrtm_call.py:246) ----
 * A queue owns one CUDA stream per slot handle.  rad_submit starts a request's solve at once on a free slot,
 * so requests submitted while others run overlap on the device; the caller keeps its own arrival queue and
 * retries on RAD_E_BUSY / RAD_E_BUDGET.  Results are the same bits as rad_solve on that slot's handle. */
typedef struct RadQueue RadQueue;

/* slots: handles with tables loaded, one per solve that may run at a time (the queue does not own them;
 * destroy the queue first).  hbm_budget_bytes: the library scratch (rad_workspace_bytes) that the requests
 * in flight may hold together, 0 = no limit. */
int rad_queue_create(RadHandle* const* slots, int32_t nslots, int64_t hbm_budget_bytes, RadQueue** out);

/* Start the solve of ncol columns (device pointers, as rad_solve) and return its ticket (>= 1).
 * RAD_E_BUSY: every slot is in use; RAD_E_BUDGET: its scratch does not fit beside the requests in flight
 * (a request larger than the whole budget is refused with RAD_E_INVALID).  Inputs must stay valid and outputs
 * untouched until the ticket is done. */
int rad_submit(RadQueue* q, const RadColumns* in, const RadOutputs* out, int64_t ncol, int64_t* ticket);

/* *done = 1 once the ticket's solve has completed (its outputs are then valid for any reader), which frees
 * its slot; 0 while it runs.  A ticket never issued is RAD_E_INVALID. */
int rad_poll(RadQueue* q, int64_t ticket, int32_t* done);

/* Poll until the ticket is done or timeout_ms elapse: RAD_OK or RAD_E_TIMEOUT (the solve keeps running). */
int rad_wait(RadQueue* q, int64_t ticket, int32_t timeout_ms);

/* Waits for the solves in flight, then releases the streams and events. */
void rad_queue_destroy(RadQueue* q);

/* Solve without reaching any allocator (no counterpart in the reference).  rad_solve grows the handle's
 * day-list scratch with cudaMalloc / cudaFree when a request is larger than any before it; cudaFree waits
 * for the whole device, and a host model that has handed its memory to its own pool, or keeps a fixed HBM
 * budget, may not want the library to allocate in the middle of a time step at all.  This entry runs the
 * same kernels with that scratch in a fixed device array of the library (about 2 MB), so it takes at most
 * RAD_NOALLOC_MAX_COLS columns (larger requests fail with RAD_E_INVALID) and, on the McICA route, needs the
 * caller's lw_mask and sw_mask buffers.  Every call looks the array's address up on the current device (a
 * runtime query, no allocation); the library's first use on a device may load its kernels and the array
 * there, so make the first call of the library on a device before any stream capture.  Every call on every
 * handle of the process shares the one array: calls whose work may overlap on the device (other streams,
 * other host threads) race on it, so issue them on one stream or one after another.  Profiling events are
 * not recorded by this entry.  The LW runs in its single-kernel form (no scratch; columns with a cloudy layer
 * thinner than 1 hPa are solved again in float64 from a list kept in the array) and the SW in its single-kernel
 * form, so results equal rad_solve's on a handle configured with lw_chunk < 0 and sw_sweep_chunk < 0. */
#define RAD_NOALLOC_MAX_COLS 65536
int rad_solve_noalloc(RadHandle* h, const RadColumns* in, const RadOutputs* out, int64_t ncol, void* stream);

/* The radiation call's post step (rrtm_post_outputs, namgpu/kernels/phys_rrtm_driver_post.cu:71-145, the
 * ICWP /= -1 path of module_RA_RRTM.F90:1142-1240): heating rates and fluxes into the model's radiation
 * state, the radiation-step cloud diagnostics, SIGT4 on LW steps.  All arrays [level or component][ncol],
 * float32 unless noted, device pointers.  hlw / swh hold lm + kd levels: kd = 1 reads the solve's
 * [nlay = lm + 1] htlw / htsw directly (the extra top layer skipped, as grrad's htrlw / htrsw copies do),
 * kd = 0 reads [lm] arrays (htrlw / HTRSW, the reference kernel's interface).  cloud_block = 0 skips the
 * cloud diagnostics (then cldcov ... ncfrcv may be NULL). */
typedef struct {
    const float* hlw;            /* [lm + kd][ncol] LW heating, K/s (htrlw, or the solve's htlw with kd 1) */
    const float* swh;            /* [lm + kd][ncol] SW heating, K/s (HTRSW, or the solve's htsw with kd 1) */
    const float* coszdg_v;       /* [ncol] GRRAD_COSZDG_V */
    const float* coszen_v;       /* [ncol] GRRAD_COSZEN_V */
    const float* sfcflw_dnfxc;   /* [ncol] sfc LW down, total sky (row 2 of the solve's sfcflw) */
    const float* topflw_upfxc;   /* [ncol] TOA LW up, total sky (row 0 of topflw) */
    const float* sfcfsw_upfxc;   /* [ncol] SFCFSW row 0 */
    const float* sfcfsw_dnfxc;   /* [ncol] SFCFSW row 1 */
    const float* sfcfsw_dnfx0;   /* [ncol] SFCFSW row 3 */
    const float* topfsw_upfxc;   /* [ncol] TOPFSW row 0 */
    float* cldcov;               /* [lm][ncol] cldcov, zeroed in place on columns with max CW < 1e-8 */
    float* cldsa;                /* [5][ncol] cldsa, zeroed in place on the same columns */
    const float* cw;             /* [lm][ncol] total condensate CW */
    const float* t;              /* [lm][ncol] temperature T (level lm - 1 used) */
    const int32_t* cu_cloud;     /* [ncol] CU_cloud flag */
} RadPostIn;

typedef struct {
    float *rlwtt, *rswtt, *cldfra, *csmid;                       /* [lm][ncol] */
    float *rlwin, *rswin, *rswinc, *rswout, *rlwtoa, *rswtoa;    /* [ncol] */
    float *czmean, *sigt4, *coszdg;                              /* [ncol] */
    float *cfracl, *cfracm, *cfrach, *acfrst, *acfrcv;           /* [ncol]; acfrst / acfrcv accumulate */
    int32_t *ncfrst, *ncfrcv;                                    /* [ncol]; counters, incremented */
} RadPostOut;

int rad_post_outputs(RadHandle* h, const RadPostIn* in, const RadPostOut* out, int64_t ncol, int32_t lm,
                     int32_t kd, int32_t cloud_block, int32_t lw_step, void* stream);

/* RDTEMP, the radiative temperature change of every model step (rdtemp_apply, namgpu/kernels/
 * drv_rdtemp.cu:140-198; module_RA_GFDL.F90:116-233): the solar zenith cosine CZEN of this step on the
 * tile, and T += (RSWTT x CZEN / CZMEAN + RLWTT) x DT on the interior, every level.  Arrays [level][jm][im]
 * or [jm][im], float32, device pointers; limits 1-based inclusive as in the loop-limit table. */
typedef struct {
    int32_t ntsd;                /* step counter */
    float dt;                    /* model step, s */
    int32_t julday, julyr, ihrst, leap_seen;   /* start day of year, year, hour; sticky leap flag */
    const float* glat;           /* [jm][im] latitude, radians */
    const float* glon;           /* [jm][im] longitude, radians */
    const float* czmean;         /* [jm][im] mean cos(zenith) of the last SW call (CZMEAN) */
    const float* rswtt;          /* [lm][jm][im] SW heating, K/s (RSWTT) */
    const float* rlwtt;          /* [lm][jm][im] LW heating, K/s (RLWTT) */
    float* czen;                 /* [jm][im] out: cos(zenith) of this step, on the tile */
    float* t;                    /* [lm][jm][im] in/out: temperature, on the interior */
    int32_t im, jm, lm;
    int32_t its, ite, jts, jte;              /* tile */
    int32_t its_b1, ite_b1, jts_b1, jte_b1;  /* interior (T update) */
} RadRdtemp;

int rad_rdtemp(RadHandle* h, const RadRdtemp* p, void* stream);

/* ---- climatological aerosol optics (NAM iaer = 11: SW and LW aerosol), and the volcanic term ----
 * The monthly 5-degree OPAC climatology as packed (woof_nam_b200/data/aer_tables.npz from the NAM data file
 * nam_climaeropac_global.txt), host pointers. */
typedef struct {
    const int32_t* iendwv;      /* [61] ending wavenumber of each OPAC band, cm-1 */
    const float* haer;          /* [7][5] scale height, km, per profile structure and domain */
    const float* prsref;        /* [7][5] reference pressure of each domain's top, mb */
    const float* rhid;          /* [4][6][61] extinction, scattering, single-scattering albedo, asymmetry of the
                                   six humidity-independent species per OPAC band */
    const float* rhdp;          /* [4][4][8][61] the same of the four humidity-dependent species at 8 humidities */
    const float* straext0;      /* [61] stratospheric background extinction */
    const int32_t* nwvns0;      /* [151] wavenumbers of each interval of the solar spectrum */
    const float* s0intv;        /* [151] solar flux per wavenumber of each interval */
    const int32_t* month_idx;   /* [37][72][5] component (1..10, 0 = none) of each 5-degree cell of the month */
    const double* month_cmix;   /* [37][72][5] its mixing ratio */
    const int32_t* month_kprf;  /* [37][72] profile structure (1..7) */
    const double* month_denn;   /* [37][72] number density of the mixing layer */
} RadAerClim;

/* The band tables of one month (aer_init's set_spectrum, clim_aerinit's set_aercoef and optavg, aer_update's
 * month fill: namgpu/physics/rrtm/phys_rrtm_aer_init.py, phys_rrtm_clim_aerinit.py:196-235,
 * phys_rrtm_aer_update.py:139-165), built on the host and copied to the handle's device (synchronous; call it
 * at start-up and at each month change, outside stream capture). */
int rad_load_aerosols(RadHandle* h, const RadAerClim* c);

/* Column inputs of rad_setaer (device pointers, float32, levels top first). */
typedef struct {
    const float* plvl;          /* [nlay + 1][ncol] interface pressure, mb (RAD_PLVL) */
    const float* plyr;          /* [nlay][ncol] layer pressure, mb (RAD_PLYR) */
    const float* tlyr;          /* [nlay][ncol] layer temperature, K */
    const float* qlyr;          /* [nlay][ncol] specific humidity, kg/kg */
    const float* rhly;          /* [nlay][ncol] layer relative humidity, 0..1 (RAD_RHLY) */
    const float* xlon;          /* [ncol] longitude, radians (XLON) */
    const float* xlat;          /* [ncol] latitude, radians (XLAT) */
    const float* slmsk;         /* [ncol] sea-land mask: 0 sea, 1 land, 2 sea ice (SLMSK) */
} RadAerColumns;

/* The aerosol optics of ncol columns (setaer with aer_property, ivflip 0: replaces the setaer call of grrad,
 * namgpu/physics/rrtm/phys_rrtm_grrad_aerosols.py:85-121, phys_rrtm_setaer.py, phys_rrtm_aer_property.py:176):
 * faersw [3][14][nlay][ncol] and faerlw [3][16][nlay][ncol] (optical depth, single-scattering albedo,
 * asymmetry per band; the layouts RadColumns.faersw / faerlw take), nlay = the handle's.  Asynchronous on
 * stream; needs rad_load_aerosols first. */
int rad_setaer(RadHandle* h, const RadAerColumns* in, int64_t ncol, float* faersw, float* faerlw, void* stream);

/* grrad's condensate clw [lmk][ncol] = the sum of the ncld cloud tracers ntcw .. ntcw + ncld - 1 (1-based) of
 * tracer [ntrac][lmk][ncol], values below epsq set to zero (replaces grrad_clouds_clw,
 * namgpu/kernels/phys_rrtm_grrad_clouds.cu:396-416, as phys_rrtm_grrad_clouds.py:183-193 launches it; NAM: ncld 1,
 * epsq 1e-12).  Device pointers; asynchronous on stream. */
int rad_grrad_clw(RadHandle* h, const float* tracer, int32_t ntrac, int32_t lmk, int64_t ncol, int32_t ntcw,
                  int32_t ncld, float epsq, float* clw, void* stream);

/* The IALB = 2 albedo tables (grrad_nmmb.f DATA TRN, ZA, DZA, ALBD; woof_nam_b200/data/payne_albedo.npz): host
 * pointers, copied into each launch. */
typedef struct {
    const float* trn;        /* [21] */
    const float* za;         /* [20] zenith angles, degrees */
    const float* dza;        /* [19] */
    const float* albd;       /* [20][21] albedo by zenith row and transmissivity column */
} RadPayneTables;

/* grrad's IALB = 2 surface albedo of ncol points (replaces grrad_clouds_albedo,
 * namgpu/kernels/phys_rrtm_grrad_clouds.cu:344-393, phys_rrtm_grrad_clouds.py:230-245): from salbedo, sm and
 * coszen [ncol] (device) the nine fields out[0..8] [ncol] (device): sfcalbedo, smx, czmean, alvsf, alnsf, alvwf,
 * alnwf, facsf, facwf, the last six being what rad_setalb (ialbflg 2) reads.  Asynchronous on stream. */
int rad_payne_albedo(RadHandle* h, const float* salbedo, const float* sm, const float* coszen, int64_t ncol,
                     const RadPayneTables* t, float* const* out, void* stream);

/* setaer's stratospheric volcanic aerosol term (the lavoflg branch, iaer >= 100; off on NAM): replaces
 * phys_rrtm_setaer_volc (namgpu/kernels/phys_rrtm_setaer.cu:178-330) as phys_rrtm_setaer.py:177-192 calls it
 * after the climatological optics.  Adds, in place, each column's zone optical depth, spread over the layers
 * between 5 mb and 150-250 mb by pressure depth, to the extinction (component 0) of faersw [3][14][nlay][ncol]
 * (add_sw) and faerlw [3][16][nlay][ncol] (add_lw; lw1bd: the one-broad-band LW factor in all 16 bands), nlay =
 * the handle's.  plvl [nlay + 1][ncol] interface pressure, mb, and xlat [ncol], radians: device pointers;
 * levels top first (ivflip 0) or surface first (ivflip 1).  ivolae: HOST int32 [10][4][12] (year, zone,
 * month) as the reference's table; the call reads year (kyrsav mod 10, non-negative) and month kmonsav
 * (1..12).  Needs no climatology loaded.  Asynchronous on stream; nlay >= 4. */
int rad_setaer_volc(RadHandle* h, const float* plvl, const float* xlat, int64_t ncol, int32_t ivflip,
                    const int32_t* ivolae, int32_t kyrsav, int32_t kmonsav, int32_t add_sw, int32_t add_lw,
                    int32_t lw1bd, float* faersw, float* faerlw, void* stream);

/* ---- grrad's radiation layers from the model state ---- */
typedef struct {              /* model state of ncol columns: device pointers, float32, levels top first */
    const float* pint;        /* [lm + 1][ncol] interface pressure, Pa (PINT) */
    const float* pmid;        /* [lm][ncol] layer pressure, Pa (P_PHY) */
    const float* prslk;       /* [lm][ncol] Exner function of the layer pressure (PRSLK) */
    const float* t;           /* [lm][ncol] temperature, K (T) */
    const float* q;           /* [lm][ncol] specific humidity, kg/kg (Q) */
    const float* tsfc;        /* [ncol] surface (skin) temperature, K (TSFC) */
} RadModelColumns;
typedef struct {              /* radiation layers: device pointers, float32, lmk = lm + 1 layers, top first */
    float* plvl;              /* [lmk + 1][ncol] level pressure, mb (RAD_PLVL; RadColumns.plvl) */
    float* plyr;              /* [lmk][ncol] layer pressure, mb (RAD_PLYR) */
    float* tlyr;              /* [lmk][ncol] layer temperature, K (RAD_TLYR) */
    float* tlvl;              /* [lmk + 1][ncol] level temperature, K (TLVL) */
    float* qlyr;              /* [lmk][ncol] specific humidity with the moisture floor (QLYR) */
    float* rhly;              /* [lmk][ncol] relative humidity (RAD_RHLY; RadAerColumns.rhly) */
    float* qstl;              /* [lmk][ncol] saturation specific humidity (RAD_QSTL) */
    float* prslk1;            /* [lmk][ncol] Exner function (RAD_PRSLK1) */
    float* tvly;              /* [lmk][ncol] virtual temperature, K (RAD_TVLY) */
    float* tsfg;              /* [ncol] ground temperature, K (RAD_TSFG) */
} RadLayerFields;

/* grrad_nmmb's set-up of the radiation layers (phys-rrtm-grrad-setup and the layer part of
 * phys-rrtm-grrad-gases: namgpu/physics/rrtm/phys_rrtm_grrad_setup.py, phys_rrtm_grrad_gases.cu:55-110),
 * for the NAM orientation (model top first) with the extra top layer: lm model layers -> lm + 1 radiation
 * layers.  Asynchronous on stream. */
int rad_grrad_setup(RadHandle* h, const RadModelColumns* in, int64_t ncol, int32_t lm, const RadLayerFields* out,
                    void* stream);

/* ---- solar geometry of a radiation call ---- */
typedef struct {
    int32_t year, month, day, hour, minute, second;   /* forecast time (JDAT 1, 2, 3, 5, 6, 7) */
    float deltsw;            /* SW calling interval, s */
    float deltim;            /* model time step, s */
    double solc0;            /* solar constant at 1 AU, W/m^2 (the year's table value, or 1366) */
} RadSolarIn;
typedef struct {
    float sollag;            /* equation of time, radians */
    float sindec, cosdec;    /* sin / cos of the solar declination */
    float anginc;            /* solar angle increment per zenith-angle sample */
    float solcon;            /* solar constant at today's sun-earth distance, W/m^2 */
    int32_t nstp;            /* zenith-angle samples per SW call */
} RadSolarState;

/* The sun at the forecast time (sol_update_nmmb with solar, namgpu/physics/rrtm/phys_rrtm_sol_update.py,
 * namgpu/kernels/phys_rrtm_sol_update.cu:60-210), on the host: no handle, no device. */
int rad_sol_update(const RadSolarIn* in, RadSolarState* out);

/* Mean cosine of the solar zenith angle of n columns over the SW interval (coszmn_nmmb,
 * namgpu/physics/rrtm/phys_rrtm_coszmn.py:51-67, namgpu/kernels/phys_rrtm_coszmn.cu:60-114): glon, glat [n]
 * radians (device); solhr = hours after 00 UTC; dtswav = SW interval in hours, sampled nrads times.  Writes
 * coszen [n] (daytime mean: SW_COSZEN / COSZEN_V) and coszdg [n] (whole-interval mean: COSZDG_V).
 * Asynchronous on stream. */
int rad_coszmn(RadHandle* h, const RadSolarState* s, const float* glon, const float* glat, int64_t n, float solhr,
               float dtswav, int32_t nrads, float* coszen, float* coszdg, void* stream);

/* ---- grrad's front end: the solve's inputs from the model state, the surface and the climatologies ----
 * Each entry is one kernel, asynchronous on stream, over device pointers in the solve's layout ([field][level]
 * [column], column = row * im + point, levels top first for ivflip 0).  Column counts of 0 do nothing. */

/* DAYPARTS (grrad_nmmb.f:606-656 with coszmn_nmmb; replaces phys_rrtm_dayparts.dayparts,
 * namgpu/physics/rrtm/phys_rrtm_dayparts.py:67, and its three kernels phys_rrtm_dayparts_cosz / _scatter / _len,
 * namgpu/kernels/phys_rrtm_dayparts.cu:76,108,125, and the library scan between them): for jm rows of im points
 * (im <= 24576), xlon, sinlat, coslat [jm * im], the sun of s (sollag, sindec, cosdec), solhr = hours after
 * 00 UTC and the SW interval dtswav (hours) sampled nrads times.  Writes coszen, coszdg [jm * im] (as
 * rad_coszmn), the run table of each row -- run k of row j in slot j * im + k for k < ndayparts[j]: dp_start
 * (1-based point in the row), dp_len (points), dp_day (0 / 1: coszen >= 1e-4) -- and ndayparts [jm].  Slots
 * past a row's runs are not written. */
typedef struct {
    float* coszen;           /* [jm * im] */
    float* coszdg;           /* [jm * im] */
    int32_t* dp_start;       /* [jm * im] */
    int32_t* dp_len;         /* [jm * im] */
    int32_t* dp_day;         /* [jm * im] */
    int32_t* ndayparts;      /* [jm] */
} RadDayparts;
int rad_dayparts(RadHandle* h, const RadSolarState* s, const float* xlon, const float* sinlat, const float* coslat,
                 int32_t im, int32_t jm, float solhr, float dtswav, int32_t nrads, const RadDayparts* out,
                 void* stream);

/* The CO2 set-up getgases reads (module variables of gas_init / gas_update, device pointers). */
typedef struct {
    const float* co2_glb;    /* [1] global mean CO2 volume mixing ratio */
    const float* gco2cyc;    /* [12] its seasonal cycle */
    const float* co2vmr_sav; /* [12][12][24] monthly 15-degree CO2 map ([month][latitude from 90N][longitude]) */
    int32_t ico2flg;         /* 0: prescribed default, 1: global mean + cycle, 2: the map below 788 mb */
    int32_t kmonsav;         /* month 1..12 (ico2flg 1, 2) */
    int32_t ivflip;          /* 0: level 0 is the model top (NAM); 1: the surface */
} RadGasSetup;

/* getgases (radiation_gases_nmmb.f:843-979; replaces phys_rrtm_getgases.getgases,
 * namgpu/physics/rrtm/phys_rrtm_getgases.py:65, kernel phys_rrtm_getgases.cu:67): the 10 gases' volume mixing
 * ratios gasvmr [10][lmax][ncol] (RadColumns.gasvmr) from plvl [lmax + 1][ncol] (mb) and xlon, xlat [ncol]
 * (radians).  RAD_E_INVALID for ico2flg outside 0..2, kmonsav outside 1..12 where used, ivflip outside 0..1. */
int rad_getgases(RadHandle* h, const float* plvl, const float* xlon, const float* xlat, int64_t ncol, int32_t lmax,
                 const RadGasSetup* g, float* gasvmr, void* stream);

/* The ozone climatology getozn reads (gas_init / gas_update module variables; o3r and pkstr on the device). */
typedef struct {
    const float* o3r;        /* [12][loz][jmr] mass mixing ratio ([month][level][latitude]) */
    const float* pkstr;      /* [loz] Exner function of its levels (increasing) */
    int32_t jmr, loz;        /* latitudes (<= 360), levels (<= 64) */
    int32_t k1oz, k2oz;      /* the two months interpolated, 1..12 */
    float facoz;             /* weight of k2oz */
    float blte, dlte;        /* first latitude and spacing, degrees */
    int32_t ivflip;
} RadOzoneClim;

/* getozn (radiation_gases_nmmb.f:984-1094; replaces the phys_rrtm_getozn kernel launch,
 * namgpu/physics/rrtm/phys_rrtm_getozn.py:117, kernel phys_rrtm_getozn.cu:43): ozone mass mixing ratio o3mmr
 * [nlev][ncol] from the Exner function prslk [nlev][ncol] (grrad's prslk1) and xlat [ncol].  A level whose
 * Exner function equals the climatology's first level, or a column with a NaN latitude, is not written (the
 * routine leaves it as it was). */
int rad_getozn(RadHandle* h, const float* prslk, const float* xlat, int64_t ncol, int32_t nlev, const RadOzoneClim* oz,
               float* o3mmr, void* stream);

/* setalb's inputs (device pointers, [ncol] each; grrad's names and units: snowf mm of water, zorlf cm). */
typedef struct {
    const float *slmsk, *snowf, *sncovr, *snoalb, *zorlf, *coszf, *tsknf, *hprif;
    const float *alvsf, *alnsf, *alvwf, *alnwf, *facsf, *facwf, *fice, *tisfc;
} RadAlbedoIn;

/* setalb (radiation_surface_nmmb.f:407-725; replaces phys_rrtm_setalb.run, namgpu/physics/rrtm/
 * phys_rrtm_setalb.py:78, kernel phys_rrtm_setalb.cu:35): sfcalb [4][ncol] (RadColumns.sfcalb: near-IR direct,
 * near-IR diffuse, visible direct, visible diffuse) by Briegleb's scheme (ialbflg 0), MODIS land albedo with the
 * land model's snow cover (1) or the provided albedos as they are (2, the NAM path; only alvsf..alnwf read). */
int rad_setalb(RadHandle* h, const RadAlbedoIn* in, int64_t ncol, int32_t ialbflg, float* sfcalb, void* stream);

/* setemis's inputs (device pointers, [ncol] each; SM 1 sea / 0 land, SICE > 0.5 sea ice, SI snow mm, Z0 m). */
typedef struct {
    const float *glon, *glat, *sm, *sice, *si, *sncovr, *z0, *stdh, *tskin;
    const int32_t* idxems;   /* [180][360] surface type of the 1-degree map (read when iemslw is 1) */
} RadEmisIn;

/* setemis (radiation_surface_nmmb.f:730-897; replaces phys_rrtm_setemis.run, namgpu/physics/rrtm/
 * phys_rrtm_setemis.py:54, kernel phys_rrtm_setemis.cu:40, whose sfc_flags [ialbflg, iemsflg, iemslw] come as
 * ialbflg and iemslw): sfcemis [ncol] (RadColumns.sfcemis). */
int rad_setemis(RadHandle* h, const RadEmisIn* in, int64_t ncol, int32_t ialbflg, int32_t iemslw, float* sfcemis,
                void* stream);

/* progcld2's inputs: the radiation layers ([nlay][ncol], plvl [nlay + 1][ncol], mb / K / kg/kg) and xlat. */
typedef struct {
    const float *plyr, *plvl, *tlyr, *tvly, *qlyr, *qstl, *rhly;
    const float *clw;        /* total condensate (grrad clw) */
    const float *f_ice, *f_rain, *r_rime;   /* Ferrier fractions (r_rime is not read) */
    const float *cldfk1;     /* Thompson cloud fraction (read when cld_fraction != 0) */
    const float *xlat;       /* [ncol] radians */
} RadCloudIn;
typedef struct {
    int32_t ivflip, llyr;    /* llyr: 1-based boundary-layer top layer (1..nlay) */
    int32_t iovr;            /* 0 random, else maximum-random overlap in gethml */
    int32_t lcrick, lcnorm, lnoprec, lsashal, cld_fraction;
} RadCloudCfg;
typedef struct {
    float* clouds;           /* [9][nlay][ncol] RadColumns.clouds */
    float* clds;             /* [5][ncol] high, middle, low, total, boundary-layer cloud */
    int32_t* mtop;           /* [3][ncol] 1-based top layer of the high, middle, low deck */
    int32_t* mbot;           /* [3][ncol] 1-based base layer */
} RadCloudOut;

/* progcld2 with gethml (radiation_clouds_nmmb.f:787-1323, 2167-2494; replaces phys_rrtm_progcld2.run,
 * namgpu/physics/rrtm/phys_rrtm_progcld2.py:75, kernel phys_rrtm_progcld2.cu:92).  2 <= nlay <= 128. */
int rad_progcld2(RadHandle* h, const RadCloudIn* in, int64_t ncol, int32_t nlay, const RadCloudCfg* cfg,
                 const RadCloudOut* out, void* stream);

/* Reads and clears the handle's device error word: *code = 0, or the code a kernel flagged since the last read
 * (1: a request with more layers than the kernels hold; 2: an index out of range; 3: a bounded wait inside a
 * kernel gave up -- an asynchronous copy did not land -- and the kernel stopped that column).  Waits for the
 * handle's device to finish its work first. */
int rad_device_error(RadHandle* h, int32_t* code);

/* Device-time accounting of the library's own kernels (instrumentation; no counterpart in the reference,
 * which has none).  While enabled, rad_solve records CUDA events on its stream around the LW kernel, the
 * SW day-list kernels and the SW kernel; rad_profile_read waits for the last recorded event and returns
 * the sums since the last enable.  `launches` counts every kernel the handle launched since rad_create. */
typedef struct {
    int64_t launches;        /* kernels launched by this handle since rad_create (profiling on or off) */
    int64_t solves;          /* rad_solve calls profiled */
    int64_t columns;         /* columns of the profiled solves */
    double lw_ms;            /* device time of the LW column kernel */
    double prep_ms;          /* device time of the SW day list and group kernels */
    double sw_ms;            /* device time of the SW column kernel */
} RadProfile;

int rad_profile_enable(RadHandle* h, int on);
int rad_profile_read(RadHandle* h, RadProfile* p);

/* Thread-local message of the last failing call on this handle (or a global message when h is NULL). */
const char* rad_last_error(const RadHandle* h);

void rad_destroy(RadHandle* h);

#ifdef __cplusplus
}
#endif
#endif /* RADB200_H */
