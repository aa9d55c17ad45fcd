// rad_post.cuh -- the radiation call's post step on the device: the solve's heating rates and fluxes into
// the model's radiation state, the radiation-step cloud diagnostics and SIGT4.
//
// Restates rrtm_post_outputs of namgpu/kernels/phys_rrtm_driver_post.cu:71-145 (module_RA_RRTM.F90:1142-1240,
// the ICWP /= -1 path NAM runs): per column
//   COSZDG = COSZDG_V, CZMEAN = COSZEN_V, RLWIN = sfc LW down (total sky), RSWIN / RSWOUT / RSWINC = sfc SW
//   down / up / clear-sky down, RLWTOA / RSWTOA = TOA LW / SW up                        (1142-1143, 1164-1170)
//   RLWTT(l) = HLW(l + kd), RSWTT(l) = SWH(l + kd), l = 0..LM-1                          (1145-1148)
//   if max_l CW(l) < EPSQ2 (1e-8): cloud cover and the five cloud-amount fields zeroed in place (1180-1194)
//   CLDFRA = CSMID = cloud cover; CFRACL/M/H = cloud amounts 1..3; ACFRST += amount 4, NCFRST += 1;
//   ACFRCV += amount 4 where CU_cloud, NCFRCV += 1                                     (1197-1214)
//   SIGT4 = STBOLT * T * T * T * T at the lowest model layer on LW steps                (1232-1240)
// kd lets the heating rates come straight from the solve's [nlay = LM + 1] arrays (kd = 1: the extra top
// layer is level 0, grrad_nmmb.f:1177-1178 as cited at phys_rrtm_grrad_sw.cu:31-34), which fuses grrad's
// htrlw / htrsw copies into this pass; kd = 0 with [LM] arrays is the reference kernel's own interface.
//
// Layout: every array is [level][column] (or [component][column]) with the column fastest, so one thread
// per column and a loop over levels gives coalesced rows; the pass is HBM-bound (about 8 LM + 20 words per
// column) and has no reuse to stage.
#pragma once

namespace rad {

struct PostArgs {
    const float *hlw, *swh;              // [LM + kd][n]
    const float *coszdg_v, *coszen_v;    // [n]
    const float *sfcflw_dnfxc, *topflw_upfxc;           // [n] (rows of the solve's sfcflw / topflw)
    const float *sfcfsw_upfxc, *sfcfsw_dnfxc, *sfcfsw_dnfx0, *topfsw_upfxc;   // [n]
    float *cldcov, *cldsa;               // [LM][n], [5][n]; zeroed in place on dry columns
    const float *cw, *t;                 // [LM][n]
    const int32_t* cu_cloud;             // [n]
    float *rlwtt, *rswtt, *cldfra, *csmid;               // [LM][n]
    float *rlwin, *rswin, *rswinc, *rswout, *rlwtoa, *rswtoa, *czmean, *sigt4, *coszdg;   // [n]
    float *cfracl, *cfracm, *cfrach, *acfrst, *acfrcv;   // [n]
    int32_t *ncfrst, *ncfrcv;            // [n]
    int64_t n;
    int lm, kd, cloud_block, lw_step;
};

constexpr float POST_EPSQ2 = 1.0e-8f;        // module_RA_RRTM.F90:286
constexpr float POST_STBOLT = 5.67051e-8f;   // nmmb_common STBOLT

__global__ void __launch_bounds__(256) k_post_outputs(const __grid_constant__ PostArgs a)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.n) return;
    const int64_t N = a.n;
    a.coszdg[c] = a.coszdg_v[c];
    a.czmean[c] = a.coszen_v[c];
    a.rlwin[c] = a.sfcflw_dnfxc[c];
    a.rswin[c] = a.sfcfsw_dnfxc[c];
    a.rswout[c] = a.sfcfsw_upfxc[c];
    a.rswinc[c] = a.sfcfsw_dnfx0[c];
    a.rlwtoa[c] = a.topflw_upfxc[c];
    a.rswtoa[c] = a.topfsw_upfxc[c];
    for (int l = 0; l < a.lm; ++l) {
        a.rlwtt[(size_t)l * N + c] = __ldg(a.hlw + (size_t)(l + a.kd) * N + c);
        a.rswtt[(size_t)l * N + c] = __ldg(a.swh + (size_t)(l + a.kd) * N + c);
    }
    if (a.cloud_block) {
        float mx = -3.402823466e38f;
        for (int l = 0; l < a.lm; ++l) {
            const float v = __ldg(a.cw + (size_t)l * N + c);
            if (v > mx) mx = v;
        }
        const bool dry = mx < POST_EPSQ2;
        for (int l = 0; l < a.lm; ++l) {
            const size_t p = (size_t)l * N + c;
            float v = a.cldcov[p];
            if (dry) {
                v = 0.0f;
                a.cldcov[p] = 0.0f;
            }
            a.cldfra[p] = v;
            a.csmid[p] = v;
        }
        float s[5];
        for (int k = 0; k < 5; ++k) {
            s[k] = dry ? 0.0f : a.cldsa[(size_t)k * N + c];
            if (dry) a.cldsa[(size_t)k * N + c] = 0.0f;
        }
        a.cfracl[c] = s[0];
        a.cfracm[c] = s[1];
        a.cfrach[c] = s[2];
        a.acfrst[c] = a.acfrst[c] + s[3];
        a.ncfrst[c] = a.ncfrst[c] + 1;
        if (a.cu_cloud[c] != 0) a.acfrcv[c] = a.acfrcv[c] + s[3];
        a.ncfrcv[c] = a.ncfrcv[c] + 1;
    }
    if (a.lw_step) {
        const float td = a.t[(size_t)(a.lm - 1) * N + c];
        a.sigt4[c] = POST_STBOLT * td * td * td * td;
    }
}

}  // namespace rad
