// rad_grrad.cuh -- grrad's radiation-layer set-up of the model state (one thread per column, sm_100a).
//
// Restates, for the NAM orientation (ivflip 0: the model top first) and its extra top layer (LTP = 1):
//   grrad_nmmb set-up  namgpu/kernels/phys_rrtm_grrad_setup.cu:112-225 (grrad_nmmb.f:1166-1396): Pa -> mb
//                      pressures, layer temperatures and Exner function, saturation specific humidity from
//                      funcphys' table fpvs (its nodes are the closed form fpvsx), relative humidity, the
//                      extra top layer (interface at 1e-6 mb, mid-pressure half the model top), ground = skin
//                      temperature
//   grrad_nmmb gases   namgpu/kernels/phys_rrtm_grrad_gases.cu:55-110 (grrad_nmmb.f:1427-1488): the moisture
//                      floor carried down from the top (qlyr), virtual temperature, and level temperatures by
//                      log-pressure interpolation between layers (model top = top layer, surface = skin)
// into the arrays the radiation takes (plvl, plyr, tlyr, tlvl, qlyr, tsfg of RadColumns) and the ones the
// aerosol and cloud set-up read (rhly, qstl, prslk1, tvly).  Every layer is read once and every output
// written once: the pass is HBM-bound (about 5 lm input and 10 lm output words per column).
#pragma once

namespace rad {

struct GrradArgs {
    const float *pint, *pmid, *prslk, *t, *q, *tsfc;        // model state [lm (+1)][n], [n]
    float *plvl, *plyr, *tlyr, *tlvl, *qlyr, *rhly, *qstl, *prslk1, *tvly, *tsfg;   // [lmk (+1)][n], [n]
    int64_t n;
    int lm;
};

// Saturation vapour pressure (Pa) in closed form: over liquid at or above the triple point, over ice 20 K
// below it, a linear blend between (funcphys.f fpvsx; physcons.f constants).
__device__ __forceinline__ float gr_fpvsx(float t)
{
    const float ttp = 2.7316e+2f, psat = 6.1078e+2f, rv = 4.6150e+2f;
    const float cvap = 1.8460e+3f, cliq = 4.1855e+3f, csol = 2.1060e+3f, hvap = 2.5000e+6f, hfus = 3.3358e+5f;
    const float dldtl = cvap - cliq, dldti = cvap - csol;
    const float xal = -dldtl / rv, xbl = -dldtl / rv + hvap / (rv * ttp);
    const float xai = -dldti / rv, xbi = -dldti / rv + (hvap + hfus) / (rv * ttp);
    const float tr = ttp / t;
    const float pl = psat * powf(tr, xal) * expf(xbl * (1.0f - tr));
    const float pi = psat * powf(tr, xai) * expf(xbi * (1.0f - tr));
    const float tice = ttp - 20.0f;
    if (t >= ttp) return pl;
    if (t < tice) return pi;
    const float w = (t - tice) / (ttp - tice);
    return w * pl + (1.0f - w) * pi;
}
// funcphys.f fpvs: linear interpolation between the 7,501 nodes 180 + 0.02 j K of fpvsx (Pa).
__device__ __forceinline__ float gr_fpvs(float t)
{
    const float c2 = 1.0f / 0.02f, c1 = 1.0f - 180.0f * c2;
    const float xj = fminf(fmaxf(c1 + c2 * t, 1.0f), 7501.0f);
    const int jx = (int)fminf(xj, 7500.0f);
    const float f0 = gr_fpvsx(180.0f + (float)(jx - 1) * 0.02f), f1 = gr_fpvsx(180.0f + (float)jx * 0.02f);
    return f0 + (xj - (float)jx) * (f1 - f0);
}

__global__ void __launch_bounds__(256) k_grrad_setup(const __grid_constant__ GrradArgs a)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.n) return;
    const int lm = a.lm, lmk = lm + 1;
    const int64_t N = a.n;
    auto I = [&](const float* p, int k) { return __ldg(p + (size_t)k * N + c); };
    auto O = [&](float* p, int k) -> float& { return p[(size_t)k * N + c]; };
    const float rd = 2.8705e+2f, rv = 4.6150e+2f, cp = 1.0046e+3f;
    const float eps = rd / rv, epsm1 = rd / rv - 1.0f, fvirt = rv / rd - 1.0f, qmin = 1.0e-10f, qme = 1.0e-7f;
    // model layers (local layer l = k + 1 below the extra top layer)
    float qfloor = qme;                            // the moisture floor carried down from the top
    float tl_prev = 0.0f, la_prev = 0.0f;          // the layer above: temperature, log(layer pressure)
    float t1 = 0.0f, rh1 = 0.0f, qs1 = 0.0f, q1 = 0.0f, tv1 = 0.0f;   // model layer 1, copied to the extra layer
    const float ptop = 10.0f * (I(a.pint, 0) * 1.0e-3f);
    const float plvl0 = 1.0e-6f, plvl1 = ptop <= 1.0e-6f ? 2.0e-6f : ptop;
    const float pl0 = 0.5f * plvl1;                // the extra top layer's pressure, mb
    O(a.plvl, 0) = plvl0;
    O(a.plvl, 1) = plvl1;
    O(a.plyr, 0) = pl0;
    O(a.prslk1, 0) = powf((pl0 * 100.0f) / 1.0e5f, rd / cp);
    for (int k = 0; k < lm; ++k) {
        const int l = k + 1;
        const float pl_cb = I(a.pmid, k) * 1.0e-3f;
        const float tg = I(a.t, k), qg = I(a.q, k);
        if (k > 0) O(a.plvl, l) = 10.0f * (I(a.pint, k) * 1.0e-3f);
        const float plyr = 10.0f * pl_cb;
        O(a.plyr, l) = plyr;
        O(a.tlyr, l) = tg;
        O(a.prslk1, l) = I(a.prslk, k);
        const float es = fminf(pl_cb, 0.001f * gr_fpvs(tg));
        const float qs = fmaxf(qmin, eps * es / (pl_cb + epsm1 * es));
        const float rh = fmaxf(0.0f, fminf(1.0f, fmaxf(qmin, qg) / qs));
        O(a.rhly, l) = rh;
        O(a.qstl, l) = qs;
        const float ql = fmaxf(qfloor, qg);
        qfloor = fminf(qme, ql);
        const float tv = tg * (1.0f + fvirt * ql);
        O(a.qlyr, l) = ql;
        O(a.tvly, l) = tv;
        // level above this layer: between the layer above and this one in log pressure
        const float la = logf(plyr);
        if (k == 0) {
            t1 = tg; rh1 = rh; qs1 = qs; q1 = ql; tv1 = tv;
            // the extra top layer has this layer's temperature; its level 1 sits between the two
            const float la0 = logf(pl0), lb = logf(plvl1);
            O(a.tlvl, 1) = tg + (tg - tg) * (lb - la) / (la0 - la);
        } else {
            const float lb = logf(O(a.plvl, l));
            O(a.tlvl, l) = tg + (tl_prev - tg) * (lb - la) / (la_prev - la);
        }
        tl_prev = tg;
        la_prev = la;
    }
    O(a.plvl, lmk) = 10.0f * (I(a.pint, lm) * 1.0e-3f);
    O(a.tlyr, 0) = t1;
    O(a.rhly, 0) = rh1;
    O(a.qstl, 0) = qs1;
    O(a.qlyr, 0) = q1;
    O(a.tvly, 0) = tv1;
    O(a.tlvl, 0) = t1;                             // the model top: the top layer's temperature
    const float ts = __ldg(a.tsfc + c);
    O(a.tlvl, lmk) = ts;                           // the surface: the skin temperature
    a.tsfg[c] = ts;
}

}  // namespace rad
