// rad_front.h -- launchers of grrad's front-end kernels (rad_front.cu), called by the C-ABI in rad_capi.cu.
//
// rad_front.cu is its own translation unit, compiled with IEEE division and square root, denormals kept and
// no multiply-add contraction, so that every statement rounds as the single-precision routines it restates
// (only the library's cosf / expf / powf differ from the host's in the last bits).  Arguments are checked by
// the C-ABI before a launcher runs; each launcher issues exactly one kernel on the stream and returns the
// launch status.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace rad {
namespace front {

// DAYPARTS of jm rows of im points (one CTA per row).
struct DaypartsArgs {
    const float *xlon, *sinlat, *coslat;                // [jm * im]
    float *coszen, *coszdg;                             // [jm * im]
    int32_t *dp_start, *dp_len, *dp_day, *ndayparts;    // [jm * im] run table (slot row * im + k), [jm]
    int32_t im, jm, nrads;
    float solhr, dtswav, sollag, sindec, cosdec;
};
constexpr int DAYPARTS_MAX_IM = 24576;                 // run table of a row staged in shared memory
cudaError_t dayparts(const DaypartsArgs& a, cudaStream_t st);

// getgases on lmax levels of n columns.
struct GasArgs {
    const float *plvl, *xlon, *xlat;                    // [lmax + 1][n] mb, [n], [n] radians
    const float *co2_glb, *gco2cyc, *co2vmr_sav;        // [1], [12], [12][12][24]
    float* gasvmr;                                      // [10][lmax][n]
    int64_t n;
    int32_t lmax, ico2flg, kmonsav, ivflip;
};
cudaError_t getgases(const GasArgs& a, cudaStream_t st);

// getozn on nlev levels of n columns.
struct OzoneArgs {
    const float *prslk, *xlat, *o3r, *pkstr;            // [nlev][n], [n], [12][loz][jmr], [loz]
    float* o3mmr;                                       // [nlev][n]
    int64_t n;
    int32_t nlev, jmr, loz, k1oz, k2oz, ivflip;
    float facoz, blte, dlte;
};
constexpr int OZONE_MAX_LOZ = 64;
constexpr int OZONE_MAX_JMR = 360;
cudaError_t getozn(const OzoneArgs& a, cudaStream_t st);

// setalb of n columns.
struct AlbedoArgs {
    const float *slmsk, *snowf, *sncovr, *snoalb, *zorlf, *coszf, *tsknf, *hprif, *alvsf, *alnsf, *alvwf, *alnwf,
        *facsf, *facwf, *fice, *tisfc;                  // [n]
    float* sfcalb;                                      // [4][n]
    int64_t n;
    int32_t ialbflg;
};
cudaError_t setalb(const AlbedoArgs& a, cudaStream_t st);

// setemis of n columns.
struct EmisArgs {
    const float *glon, *glat, *sm, *sice, *si, *sncovr, *z0, *stdh, *tskin;   // [n]
    const int32_t* idxems;                              // [180][360]
    float* sfcemis;                                     // [n]
    int64_t n;
    int32_t ialbflg, iemslw;
};
cudaError_t setemis(const EmisArgs& a, cudaStream_t st);

// progcld2 with gethml on nlay layers of n columns.
struct CloudArgs {
    const float *plyr, *plvl, *tlyr, *tvly, *qlyr, *qstl, *rhly, *clw, *f_ice, *f_rain, *cldfk1, *xlat;
    float *clouds, *clds;                               // [9][nlay][n], [5][n]
    int32_t *mtop, *mbot;                               // [3][n]
    int64_t n;
    int32_t nlay, ivflip, llyr, iovr, lcrick, lcnorm, lnoprec, lsashal, cld_fraction;
};
constexpr int CLOUD_MAX_LAY = 128;
cudaError_t progcld2(const CloudArgs& a, cudaStream_t st);

// grrad's condensate: clw [lmk][n] = the ncld tracers from ntcw0 (0-based) of tracer [ntrac][lmk][n], summed,
// below epsq set to zero.
struct ClwArgs {
    const float* tracer;
    float* clw;
    int64_t n;
    int32_t lmk, ntcw0, ncld;
    float epsq;
};
cudaError_t grrad_clw(const ClwArgs& a, cudaStream_t st);

// grrad's IALB = 2 surface albedo of n points, the tables by value.
struct PayneArgs {
    const float *salbedo, *sm, *coszen;                 // [n]
    float* out[9];                                      // sfcalbedo, smx, czmean, alvsf, alnsf, alvwf, alnwf, facsf, facwf
    int64_t n;
    float trn[21], za[20], dza[19], albd[20 * 21];      // albd [zenith row][transmissivity column]
};
cudaError_t payne_albedo(const PayneArgs& a, cudaStream_t st);

// setaer's volcanic stratospheric term on nlay layers of n columns, added in place to component 0 (extinction).
struct VolcArgs {
    const float *plvl, *xlat;                           // [nlay + 1][n] mb in the order of ivflip, [n] radians
    float *faersw, *faerlw;                             // [3][14][nlay][n], [3][16][nlay][n]
    int64_t n;
    int32_t nlay, ivflip, add_sw, add_lw;
    int32_t iv[4];                                      // the table's values of the 4 latitude zones, year and month
    float tsw[14], tlw[16];                             // per band (0.275e-4 (w1 + w2))^e, by the host's powf
};
cudaError_t setaer_volc(const VolcArgs& a, cudaStream_t st);

}  // namespace front
}  // namespace rad
