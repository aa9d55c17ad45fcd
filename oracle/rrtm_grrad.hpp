// rrtm_grrad.hpp -- CPU oracle: grrad's radiation-layer set-up of the model state (test infrastructure only).
//
// Restates, in the reference's float arithmetic, for ivflip 0 and the extra top layer:
//   namgpu/kernels/phys_rrtm_grrad_setup.cu:112-225 (rrtm_grrad_setup; fpvs / fpvsx / fpkapx of funcphys)
//   namgpu/kernels/phys_rrtm_grrad_gases.cu:55-110 (phys_rrtm_grrad_gases, the ivflip 0 branch)
// Never linked into the product.
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

namespace orc {
namespace grrad {

inline float fpvsx(float t)
{
    const float ttp = 2.7316e+2f, psat = 6.1078e+2f, rv = 4.6150e+2f, cvap = 1.8460e+3f, cliq = 4.1855e+3f,
                csol = 2.1060e+3f, hvap = 2.5000e+6f, hfus = 3.3358e+5f;
    const float tliq = ttp, tice = ttp - 20.0f;
    const float dldtl = cvap - cliq, xponal = -dldtl / rv, xponbl = -dldtl / rv + hvap / (rv * ttp);
    const float dldti = cvap - csol, heati = hvap + hfus, xponai = -dldti / rv, xponbi = -dldti / rv + heati / (rv * ttp);
    const float tr = ttp / t;
    if (t >= tliq) return psat * std::pow(tr, xponal) * std::exp(xponbl * (1.0f - tr));
    if (t < tice) return psat * std::pow(tr, xponai) * std::exp(xponbi * (1.0f - tr));
    const float w = (t - tice) / (tliq - tice);
    const float pvl = psat * std::pow(tr, xponal) * std::exp(xponbl * (1.0f - tr));
    const float pvi = psat * std::pow(tr, xponai) * std::exp(xponbi * (1.0f - tr));
    return w * pvl + (1.0f - w) * pvi;
}

inline float fpvs(float t)
{
    const float c2 = 1.0f / 0.02f, c1 = 1.0f - 180.0f * c2;
    const float xj = std::min(std::max(c1 + c2 * t, 1.0f), 7501.0f);
    const int jx = (int)std::min(xj, 7500.0f);
    const float f0 = fpvsx(180.0f + (float)(jx - 1) * 0.02f), f1 = fpvsx(180.0f + (float)jx * 0.02f);
    return f0 + (xj - (float)jx) * (f1 - f0);
}

// One column: pint [lm + 1], pmid, prslk, t, q [lm] (Pa, K), tsfc -> the radiation layers (lmk = lm + 1).
inline void column(int lm, const float* pint, const float* pmid, const float* prslk, const float* t, const float* q,
                   float tsfc, float* plvl, float* plyr, float* tlyr, float* tlvl, float* qlyr, float* rhly,
                   float* qstl, float* prslk1, float* tvly, float& tsfg)
{
    const float rd = 2.8705e+2f, rv = 4.6150e+2f, cp = 1.0046e+3f;
    const float eps = rd / rv, epsm1 = rd / rv - 1.0f, fvirt = rv / rd - 1.0f, qmin = 1.0e-10f;
    const int lmk = lm + 1, lmp = lmk + 1;
    for (int k0 = 0; k0 < lm; ++k0) {
        const int l = k0 + 1;
        const float pi_cb = pint[k0] * 1.0e-3f, pl_cb = pmid[k0] * 1.0e-3f, tg = t[k0], qg = q[k0];
        plvl[l] = 10.0f * pi_cb;
        plyr[l] = 10.0f * pl_cb;
        tlyr[l] = tg;
        prslk1[l] = prslk[k0];
        const float es = std::min(pl_cb, 0.001f * fpvs(tg));
        const float qs = std::max(qmin, eps * es / (pl_cb + epsm1 * es));
        rhly[l] = std::max(0.0f, std::min(1.0f, std::max(qmin, qg) / qs));
        qstl[l] = qs;
    }
    plvl[lm + 1] = 10.0f * (pint[lm] * 1.0e-3f);
    float tem1d = 1.0e-7f;
    for (int k0 = 0; k0 < lm; ++k0) {
        const int l = k0 + 1;
        const float ql = std::max(tem1d, q[k0]);
        tem1d = std::min(1.0e-7f, ql);
        qlyr[l] = ql;
        tvly[l] = t[k0] * (1.0f + fvirt * ql);
    }
    plvl[0] = 1.0e-6f;
    if (plvl[1] <= 1.0e-6f) plvl[1] = 2.0f * 1.0e-6f;
    plyr[0] = 0.5f * plvl[1];
    tlyr[0] = tlyr[1];
    rhly[0] = rhly[1];
    qstl[0] = qstl[1];
    prslk1[0] = std::pow((plyr[0] * 100.0f) / 1.0e5f, rd / cp);
    qlyr[0] = qlyr[1];
    tvly[0] = tvly[1];
    tsfg = tsfc;
    // grrad gases, ivflip 0: level temperatures by log-pressure interpolation
    std::vector<float> lda(lmk), ldb(lmp);
    for (int k = 2; k <= lmk; ++k) { lda[k - 1] = std::log(plyr[k - 1]); ldb[k - 1] = std::log(plvl[k - 1]); }
    lda[0] = std::log(plyr[0]);
    ldb[0] = plvl[0] == 0.0f ? -14.0f : std::log(plvl[0]);
    tlvl[0] = tlyr[0];
    tlvl[lmp - 1] = tsfc;
    for (int k = 2; k <= lmk; ++k)
        tlvl[k - 1] = tlyr[k - 1] + (tlyr[k - 2] - tlyr[k - 1]) * (ldb[k - 1] - lda[k - 1]) / (lda[k - 2] - lda[k - 1]);
}

}  // namespace grrad
}  // namespace orc
