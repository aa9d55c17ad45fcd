// rad_sw2.cuh -- the production SW column kernel for sm_100a (mixed precision).
//
// Same column physics as rad_sw.cuh (swrad prep, cldprop, setcoef, taumol16..29, spcvrtc + swflux,
// namgpu/kernels/phys_rrtm_sw_*.cu), organised for throughput:
//
//  * 128 threads per sunlit column.  Phase A: threads = layers / (band, layer) pairs / bands build the
//    layer coefficients, cloud optics and solar source in shared memory.  Phase B: threads = (g, layer)
//    pairs in g-major order compute the gas and Rayleigh optical depths once (a warp stays inside one
//    band, so the band switch does not diverge).  Phase C: one g-point per lane (28/28/30/26 lanes per
//    warp, the Rayleigh-dominated bands 23-26 grouped in one warp), each lane carrying the clear and the
//    cloudy pass of spcvrtc.
//  * No per-thread layer arrays.  The adding method needs the upward reflectances of every level while
//    it walks down; the upward sweep keeps only one checkpoint per segment of SEG layers (shared memory),
//    and the downward sweep rebuilds each segment's upward states from it.  The layer R/T of the upward
//    sweep go to a per-CTA store in global memory (~340 KB, L2-resident across the grid's CTAs) and the
//    downward sweep reads them back; without a store (rad_solve_noalloc) it recomputes them.
//  * Level fluxes are summed over the g-points of a warp in float64 (shuffles) and over warps in a fixed
//    order: results are bit-reproducible and do not depend on what else runs on the GPU.
//
// Precision (mixed):
//  * The layer R/T (sw2_rt) is an algebraically equal rearrangement of the reference's statements that
//    float evaluates accurately: co-albedo carried from the optics (no 1 - ssa cancellation), the
//    complements 1 - exp(-x) carried next to exp(-x), and exp(-k tau) multiplied through instead of
//    divided (the reference's float form overflows and returns NaN once k tau > ~88).  Near-conservative
//    and thin layers need no float64.
//  * Within 1 % of the two-stream resonance k mu0 = 1 the reference's formula divides two small
//    quantities, clamps 1 - (k mu0)^2 at 1e-8 and compares exp-table entries of two nearly equal depths;
//    there the R/T is evaluated in float64 from the float optical properties, and where a table entry it
//    takes could differ from the one the float64 optical properties select, the layer's optical properties
//    are recomputed from the column inputs in float64 (prep, setcoef, gas, aerosol and cloud optics) and
//    the reference's statements are evaluated in float64 (sw2_exact), so the result follows the
//    reference's own arithmetic.  Both run inline in the lane that needs them.
//  * The layer coefficients and the key-species ratios are formed in float64 and rounded once, so a float
//    exponent argument is within ~2e-6 of the float64 one.  Where an argument lies that close to a bound of
//    the reference's exp table and taking the neighbouring entry would move the layer's heating or the
//    surface beam by more than the guard allows (sw2_near, sw2_flip_matters), the layer is recomputed in
//    float64 (sw2_exact): one entry step can move a thin layer's heating by ~0.05 K/day.
//  * Flux sums over g-points and bands and the heating-rate flux differences are float64.
#pragma once
#include "rad_sw.cuh"

namespace rad {

constexpr int SW2_WARPS = 4, SW2_THREADS = 128;
#ifndef RAD_SW2_SEG
#define RAD_SW2_SEG 4
#endif
constexpr int SW2_SEG = RAD_SW2_SEG;                              // layers per checkpoint segment
constexpr int SW2_NSEG = (NLAY_MAX + SW2_SEG - 1) / SW2_SEG;
constexpr float SW2_RESONANCE = 1.0e-2f;                          // float64 R/T where |1-(k mu0)^2| < this
constexpr double SW2_TBL_MARGIN = 0.01;                           // table-index rounding margin (see sw2_tbl_sure)
// Table-entry guard of the float R/T (sw2_near, sw2_flip_matters): relative error bound of a float exponent
// argument against the float64 one, and the largest output change one entry of the 10,001-entry exp table may
// make unchecked (the heating weight carries a safety factor of 1.5 on top).
constexpr float SW2_ZB_EPS = 2.0e-6f;
constexpr float SW2_HEAT_T = 2.0e-3f;                             // K/day
constexpr float SW2_FLUX_T = 5.0e-3f;                             // W/m^2

// Rain and snow optical coefficients per SW band (phys_rrtm_sw_cldprop.cu): b0r, c0r, b0s, b1s, c0s.
__constant__ float c_sw_rain_snow[5][14] = {
    {0.466f, 0.437f, 0.416f, 0.391f, 0.374f, 0.352f, 0.183f, 0.048f, 0.012f, 0.000f, 0.000f, 0.000f, 0.000f, 0.496f},
    {0.975f, 0.965f, 0.960f, 0.955f, 0.952f, 0.950f, 0.944f, 0.894f, 0.884f, 0.883f, 0.883f, 0.883f, 0.883f, 0.980f},
    {0.460f, 0.460f, 0.460f, 0.460f, 0.460f, 0.460f, 0.460f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.460f},
    {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.62e-5f, 1.62e-5f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f},
    {0.970f, 0.970f, 0.970f, 0.970f, 0.970f, 0.970f, 0.970f, 0.970f, 0.970f, 0.700f, 0.700f, 0.700f, 0.700f, 0.970f}};

template <class T>
struct One {   // a scalar read through the array syntax of the shared-memory layer arrays
    T v;
    __device__ __forceinline__ T operator[](int) const { return v; }
};

// One layer after swrad_prep + setcoef (swrad.cu:166-240, setcoef.cu:17-97).
template <class R>
struct SwCoef {
    R fac00, fac01, fac10, fac11, selffac, selffrac, forfac, forfrac, colmol;
    R colamt[6];
    int jp, jt, jt1, indself, indfor;
    bool low;   // ln(p) > 4.56, decided in float64 for every precision
};

template <class R>
__device__ void sw2_layer_coef(const SwIn& a, int64_t col, int k0, SwCoef<R>& c)
{
    const int nlay = a.nlay;
    const int64_t N = a.ncol;
    const int kk0 = nlay - 1 - k0;
    auto IN = [&](const float* p, int lev) { return (R)__ldg(p + (size_t)lev * N + col); };
    const R amdw = (R)28.9644f / (R)18.0154f, amdo3 = (R)28.9644f / (R)47.9982f;
    const R tem1 = (R)100.0f * (R)9.80665f, tem2 = (R)1.0e-20f * (R)1.0e3f * (R)6.0221415e23f;
    const float pin = __ldg(a.plyr + (size_t)kk0 * N + col);
    const R pav = (R)pin, tav = IN(a.tlyr, kk0);
    const R dl = IN(a.plvl, kk0 + 1) - IN(a.plvl, kk0);
    const R qv = IN(a.qlyr, kk0), ov = IN(a.olyr, kk0);
    const R h2o = fmaxR((R)0, qv * amdw / ((R)1 - qv));
    const R o3 = fmaxR((R)0, ov * amdo3);
    const R tem0 = ((R)1 - h2o) * (R)28.9644f + h2o * (R)18.0154f;
    const R cd = tem2 * dl / (tem1 * tem0 * ((R)1 + h2o));
    const R tc = (R)1.0e-12f * cd;
    auto G = [&](int n) { return (R)__ldg(a.gasvmr + ((size_t)n * nlay + kk0) * N + col); };
    c.colamt[0] = fmaxR((R)0, cd * h2o);
    c.colamt[1] = fmaxR(tc, cd * G(0));
    c.colamt[2] = fmaxR((R)0, cd * o3);
    c.colmol = cd + c.colamt[0];
    c.colamt[3] = fmaxR(tc, cd * G(1));
    c.colamt[4] = fmaxR(tc, cd * G(2));
    c.colamt[5] = fmaxR(tc, cd * G(3));
    const R forf = pav * ((R)296.0f / (R)1013.0f) / (tav * ((R)1 + h2o));
    c.forfac = forf;
    const R plog = rlog(pav);
    const int jpk = max(1, min(58, (int)((R)36 - (R)5 * (plog + (R)0.04f))));
    const int jp1 = jpk + 1;
    const R* preflog = tab<R>(T_SW_PREFLOG);
    const R* tref = tab<R>(T_SW_TREF);
    const R fp = (R)5 * (ldt(preflog + jpk - 1) - plog);
    const R t1 = (tav - ldt(tref + jpk - 1)) / (R)15, t2 = (tav - ldt(tref + jp1 - 1)) / (R)15;
    const int jtk = max(1, min(4, (int)((R)3 + t1))), jt1k = max(1, min(4, (int)((R)3 + t2)));
    const R ft = t1 - (R)(jtk - 3), ft1 = t2 - (R)(jt1k - 3);
    c.jp = jpk; c.jt = jtk; c.jt1 = jt1k;
    const R fp1 = (R)1 - fp;
    c.fac10 = fp1 * ft;
    c.fac00 = fp1 * ((R)1 - ft);
    c.fac11 = fp * ft1;
    c.fac01 = fp * ((R)1 - ft1);
    c.low = log((double)pin) > (double)4.56f;
    if (c.low) {
        const R tem1f = ((R)332 - tav) / (R)36;
        const int indf = min(2, max(1, (int)tem1f));
        c.indfor = indf;
        c.forfrac = tem1f - (R)indf;
        const R tem2s = (tav - (R)188) / (R)7.2f;
        const int inds = min(9, max(1, (int)tem2s - 7));
        c.indself = inds;
        c.selffrac = tem2s - (R)(inds + 7);
        c.selffac = h2o * forf;
    } else {
        const R tem1f = (tav - (R)188) / (R)36;
        c.indfor = 3;
        c.forfrac = tem1f - (R)1;
        c.indself = 0;
        c.selffrac = 0;
        c.selffac = 0;
    }
}

// Cloud optics of band ib in layer k0 (phys_rrtm_sw_cldprop.cu: iswcliq = 1 with the liquid table,
// iswcice = 3, rain and snow; iswcliq = 0: optical depth, SSA and asymmetry given directly).  Besides the
// reference's tau, tau*ssa and tau*ssa*g it returns the absorption optical depth tau*(1-ssa) formed from
// the co-albedos of the tables (no 1 - ssa cancellation).
template <class R>
__device__ void sw2_cloud(const SwIn& a, int64_t col, int k0, int ib, R cf, R& tcw, R& scw, R& acw, R& tabs)
{
    const int nlay = a.nlay;
    const int64_t N = a.ncol;
    const int kk0 = nlay - 1 - k0;
    auto CLD = [&](int n) { return (R)__ldg(a.clouds + ((size_t)n * nlay + kk0) * N + col); };
    const R ftiny = (R)1.0e-12f;
    tcw = 0; scw = 1; acw = 0; tabs = 0;
    if (!(cf > ftiny)) return;
    if (!a.diagnostic) {
        const float* b0r = c_sw_rain_snow[0];
        const float* c0r = c_sw_rain_snow[1];
        const float* b0s = c_sw_rain_snow[2];
        const float* b1s = c_sw_rain_snow[3];
        const float* c0s = c_sw_rain_snow[4];
        const R cldran = CLD(5), cldsnw = CLD(7), refsnw = CLD(8);
        const R dgesnw = (R)1.0315f * refsnw;
        const R tauran = cldran * (R)3.07e-3f;
        const R tausnw = (cldsnw > 0 && refsnw > (R)10) ? cldsnw * (R)1.09087f * ((R)0 + (R)1.5f / dgesnw) : (R)0;
        const R ssaran = tauran * ((R)1 - (R)b0r[ib]);
        const R wsnw = (R)b0s[ib] + (R)b1s[ib] * dgesnw;
        const R ssasnw = tausnw * ((R)1 - wsnw);
        const R asyran = ssaran * (R)c0r[ib], asysnw = ssasnw * (R)c0s[ib];
        const R cldliq = CLD(1), refliq = CLD(2), cldice = CLD(3), refice = CLD(4);
        R tl = 0, sl = 0, al = 0, ti = 0, si = 0, ai = 0, bl = 0, bi = 0;
        // interpolated SSA and its co-albedo (1 - v0) - f (v1 - v0), both clamped to [0, 1]
        auto ssa_w = [&](const R* t, int i, R f, R& ssa, R& w) {
            const R v0 = ldt(t + i - 1), v1 = ldt(t + i), dv = v1 - v0;
            ssa = fmaxR((R)0, fminR((R)1, v0 + f * dv));
            w = fmaxR((R)0, fminR((R)1, ((R)1 - v0) - f * dv));
        };
        if (!(cldliq <= 0)) {
            const R factor = refliq - (R)1.5f;
            const int index = max(1, min(57, (int)factor));
            const R fint = factor - (R)index;
            const R *e = tab<R>(T_SW_EXTLIQ1) + ib * 58, *sv = tab<R>(T_SW_SSALIQ1) + ib * 58, *av = tab<R>(T_SW_ASYLIQ1) + ib * 58;
            const R ext = fmaxR((R)0, ldt(e + index - 1) + fint * (ldt(e + index) - ldt(e + index - 1)));
            R ssa, w;
            ssa_w(sv, index, fint, ssa, w);
            const R asy = fmaxR((R)0, fminR((R)1, ldt(av + index - 1) + fint * (ldt(av + index) - ldt(av + index - 1))));
            tl = cldliq * ext; sl = tl * ssa; al = sl * asy; bl = tl * w;
        }
        if (!(cldice <= 0)) {
            const R dge = fmaxR((R)5, fminR((R)140, (R)1.0315f * refice));
            const R factor = (dge - (R)2) / (R)3;
            const int index = max(1, min(45, (int)factor));
            const R fint = factor - (R)index;
            const R *e = tab<R>(T_SW_EXTICE3) + ib * 46, *sv = tab<R>(T_SW_SSAICE3) + ib * 46, *av = tab<R>(T_SW_ASYICE3) + ib * 46;
            const R ext = fmaxR((R)0, ldt(e + index - 1) + fint * (ldt(e + index) - ldt(e + index - 1)));
            R ssa, w;
            ssa_w(sv, index, fint, ssa, w);
            const R asy = fmaxR((R)0, fminR((R)1, ldt(av + index - 1) + fint * (ldt(av + index) - ldt(av + index - 1))));
            ti = cldice * ext; si = ti * ssa; ai = si * asy; bi = ti * w;
        }
        tcw = tl + ti + tauran + tausnw;
        scw = sl + si + ssaran + ssasnw;
        acw = al + ai + asyran + asysnw;
        tabs = bl + bi + tauran * (R)b0r[ib] + tausnw * wsnw;
    } else {
        const R t = CLD(1), w = CLD(2);
        tcw = t;
        scw = t * w;
        acw = scw * CLD(3);
        tabs = t * ((R)1 - w);
    }
}

// Layer coefficients of one layer in float64, read with the shared-memory array syntax by sw_gas.
struct SwOne {
    static constexpr bool kRatio64 = false;
    One<double> fac00, fac01, fac10, fac11, selffac, selffrac, forfac, forfrac, colmol;
    One<double> colamt[6];
    One<int> jp, jt, jt1, indself, indfor;
    int laytrop, kmin8, kminw;
};

// ------------------------------------------------------------------------------------------------------
// exp(-zb) as sw_expm evaluates it, together with its complement 1 - exp(-zb) formed without cancellation
// (below 0.06 the reference's expansion 1 - zb + zb^2/2, whose complement is zb - zb^2/2).
template <class T>
__device__ __forceinline__ T sw2_expm_c(T zb, const T* ex, T& em)
{
    if (zb <= (T)0.06f) {
        em = zb - (T)0.5f * zb * zb;
        return (T)1 - zb + (T)0.5f * zb * zb;
    }
    const T e = sw_expm(zb, ex, false);
    em = (T)1 - e;
    return e;
}

// Layer R/T (spcvrtc.cu:112-173) from (tau, absorption tau, scattering tau, scattering tau x g), equal to
// the reference's statements in exact arithmetic and accurate in float (sw2_prologue + sw2_rt_tail):
//  * co-albedo w = tau_abs / tau, so g1 - g2 = 2 w / (1 - zssaw g^2) (PIFM; sqrt(3) w / ... for the
//    discrete-ordinates mode) and g1 - k = g2^2 / (g1 + k) carry no cancellation;
//  * with e1 = exp(-k tau1), e2 = exp(-tau1 / mu0) and their complements m1 = 1 - e1, m2 = 1 - e2, the
//    reference's ze1r45 * e1 = (1 - (k mu0)^2) B with B = k (1 + e1^2) + g1 (1 - e1^2), and its
//    numerators become  rb: (1-e1^2)(a2 - k g3 k mu0) + k (g3 - a2 mu0)(m1^2 + 2 e1 m2)
//                       tb: e2 + [k (g4 + a1 mu0)(2 e1 m2 - e2 m1^2) - e2 (1-e1^2)(a1 + k g4 k mu0)] / ...
//    so thin and near-conservative layers (k tau1 -> 0) keep their accuracy;  rd = g2 (1-e1^2) / B,
//    td = 2 k e1 / B;
//  * finite for any optical depth (the reference's float form overflows 1/exp(-k tau) beyond ~88).
template <class T>
struct SwPro {   // the part of the layer R/T before the exponentials
    T ztau1, zssa1, g1, g2, g3, g4, zrk, zrp, zrpp;
};

template <class T>
__device__ __forceinline__ SwPro<T> sw2_prologue(T ztau0, T tabs, T zssa0, T zasy0, int mode, T cz)
{
    SwPro<T> p;
    const T ftiny = (T)1.0e-12f;
    const T cwmin = (T)(1.0 - ((double)1.0f - (double)1.0e-6f));   // 1 - min(oneminus, ssa) bound of FP64
    const T cw = fmaxR(cwmin, tabs / ztau0);
    const T zssaw = (T)1 - cw;
    const T zasyw = zasy0 / fmaxR(ftiny, zssa0);
    const T za2s = zssaw * (zasyw * zasyw);
    const T om = (T)1 - za2s;
    p.ztau1 = om * ztau0;
    p.zssa1 = (zssaw - za2s) / om;
    const T cw1 = cw / om;
    const T zasy1 = zasyw / ((T)1 + zasyw), zasy3 = (T)0.75f * zasy1;
    T gm, gp;
    if (mode == 2) {
        p.g1 = (T)2 - p.zssa1 * ((T)1.25f + zasy3);
        p.g2 = (T)0.75f * p.zssa1 * ((T)1 - zasy1);
        p.g3 = (T)0.5f - zasy3 * cz;
        gm = (T)2 * cw1;
        gp = (T)2 - p.zssa1 * ((T)0.5f + (T)1.5f * zasy1);
    } else if (mode == 1) {
        p.g1 = (T)1.75f - p.zssa1 * ((T)1 + zasy3);
        p.g2 = (T)-0.25f - p.zssa1 * ((T)1 - zasy3);
        p.g3 = (T)0.5f - zasy3 * cz;
        gm = p.g1 - p.g2;
        gp = p.g1 + p.g2;
    } else {
        const T zsr3 = (T)1.7320508f;
        p.g1 = zsr3 * ((T)2 - p.zssa1 * ((T)1 + zasy1)) * (T)0.5f;
        p.g2 = zsr3 * p.zssa1 * ((T)1 - zasy1) * (T)0.5f;
        p.g3 = ((T)1 - zsr3 * zasy1 * cz) * (T)0.5f;
        gm = zsr3 * cw1;
        gp = zsr3 * ((T)1 - p.zssa1 * zasy1);
    }
    p.g4 = (T)1 - p.g3;
    p.zrk = sqrtR(gm * gp);
    p.zrp = p.zrk * cz;
    p.zrpp = ((T)1 - p.zrp) * ((T)1 + p.zrp);
    return p;
}

// R/T from the prologue and the two exponentials e1 = exp(-k tau1), e2 = exp(-tau1 / mu0) with their
// complements (1 - (k mu0)^2 clamped at 1e-8 as the reference does).
template <class T>
__device__ __forceinline__ void sw2_rt_core(const SwPro<T>& p, T cz, T e1, T em1, T e2, T em2, T& rb, T& rd, T& tb,
                                            T& td)
{
    const T eps1 = (T)1.0e-8f;
    const T zrpp = fabs(p.zrpp) < eps1 ? (p.zrpp < 0 ? -eps1 : eps1) : p.zrpp;
    const T g1 = p.g1, g2 = p.g2, g3 = p.g3, g4 = p.g4, zrk = p.zrk, zrp = p.zrp;
    const T za1 = g1 * g4 + g2 * g3, za2 = g1 * g3 + g2 * g4;
    const T e11 = e1 * e1, em11 = em1 * ((T)2 - em1);
    const T B = zrk * ((T)1 + e11) + g1 * em11;
    const T D = zrpp * B;                                        // (reference ze1r45) * exp(-k tau)
    if (D >= -eps1 * e1 && D <= eps1 * e1) {
        rb = eps1;
        tb = e2;
    } else {
        const T q = p.zssa1 / D;
        const T nr = em11 * (za2 - zrk * g3 * zrp) + zrk * (g3 - za2 * cz) * (em1 * em1 + (T)2 * e1 * em2);
        const T nt = zrk * (g4 + za1 * cz) * ((T)2 * e1 * em2 - e2 * em1 * em1) - e2 * em11 * (za1 + zrk * g4 * zrp);
        rb = fmaxR((T)0, fminR((T)1, nr * q));
        tb = fmaxR((T)0, fminR((T)1, e2 + nt * q));
    }
    rd = fmaxR((T)0, fminR((T)1, g2 * em11 / B));
    td = fmaxR((T)0, fminR((T)1, (T)2 * zrk * e1 / B));
}

// R/T from the prologue, the exponentials from the reference's table (sw_expm's nearest-entry rule).
template <class T>
__device__ __forceinline__ void sw2_rt_tail(const SwPro<T>& p, T cz, T snt, const T* ex, T& rb, T& rd, T& tb, T& td)
{
    T em1, em2;
    const T e1 = sw2_expm_c(fminR(p.zrk * p.ztau1, (T)500), ex, em1);
    const T e2 = sw2_expm_c(fminR(p.ztau1 * snt, (T)500), ex, em2);
    sw2_rt_core<T>(p, cz, e1, em1, e2, em2, rb, rd, tb, td);
}

// ------------------------------------------------------------------------------------------------------
// Rayleigh optical depth per unit colmol of g-point g, as each taumol band forms taur = colmol * coefficient
// (phys_rrtm_sw_taumol16..29.cu); band 24 below laytrop interpolates in the species ratio instead (its
// depths are kept per layer).
__device__ __forceinline__ float sw2_rayl_coef(int g)
{
    int b = 0;
    while (g >= c_sw_ns[b + 1]) ++b;
    const int ig = g - c_sw_ns[b];
    switch (b + 16) {
    case 16: return ldt(tab<float>(T_SW16_RAYL));
    case 17: return 6.86e-10f;
    case 18: return ldt(tab<float>(T_SW18_RAYL));
    case 19: return 2.29e-09f;
    case 20: return ldt(tab<float>(T_SW20_RAYL));
    case 21: return 9.41e-09f;
    case 22: return 1.54e-08f;
    case 23: return ldt(tab<float>(T_SW23_RAYL) + ig);
    case 24: return ldt(tab<float>(T_SW24_RAYLB) + ig);
    case 25: return ldt(tab<float>(T_SW25_RAYL) + ig);
    case 26: return ldt(tab<float>(T_SW26_RAYL) + ig);
    case 27: return ldt(tab<float>(T_SW27_RAYL) + ig);
    case 28: return ldt(tab<float>(T_SW28_RAYL));
    default: return 9.30e-11f;
    }
}

// ------------------------------------------------------------------------------------------------------
// Shared memory of one sunlit column.  Arrays that phase C reads at [g-point or band][layer], with the lanes
// of a warp on different g-points, have a row stride of NLAY_MAX + 1 words so those lanes fall in different
// banks.
constexpr int SW2_KS = NLAY_MAX + 1;
struct SwSh2 {
    static constexpr bool kRatio64 = true;     // sw_species reads the key-species ratios from spr
    // read by the set-up and optics phases only, and the sweep phase's reduction scratch
    double fn[SW2_WARPS][NLAY_MAX + 2];        // per-warp level sums of zsolar * (down - up), passes combined
    double sc[SW2_WARPS][18];                  // per-warp scalar sums, clear (0..8) and cloudy (9..17)
    double spr[8][NLAY_MAX];                   // key-species ratio of each species-interpolating band (sw_species)
    float fac00[NLAY_MAX], fac01[NLAY_MAX], fac10[NLAY_MAX], fac11[NLAY_MAX];
    float selffac[NLAY_MAX], selffrac[NLAY_MAX], forfac[NLAY_MAX], forfrac[NLAY_MAX];
    float colamt[6][NLAY_MAX];
    int jp[NLAY_MAX], jt[NLAY_MAX], jt1[NLAY_MAX], indself[NLAY_MAX], indfor[NLAY_MAX];
    float cfrac[NLAY_MAX];
    unsigned char low[NLAY_MAX];
    int task_next;                             // phase B task counter (for_each_band_pair)
    // read by the sweep phase: from here to the end (and the aerosol block) is the column's image
    alignas(16) float colmol[NLAY_MAX];
    float cldfrc[NLAY_MAX];
    float taucw[14][SW2_KS], ssacw[14][SW2_KS], asycw[14][SW2_KS], tabsc[14][SW2_KS];
    float raylc[SW_NGPT];                      // Rayleigh optical depth per unit colmol (band 24: upper atmosphere)
    float taur24[8][SW2_KS];                   // band 24 Rayleigh optical depth below laytrop
    float sfluxzen[SW_NGPT];
    double rdelp[NLAY_MAX];                    // heatfac / delp, float64
    float cosz, sntz, ssolar, albbm[2], albdf[2], zcf0, zcf1;
    int laytrop, kmin8, kminw;
    uint32_t mcw[4][NLAY_MAX];                 // McICA route: the column's sub-column cloud words
    // last, so that the optics kernel can leave it out of shared memory (it writes it to the image directly)
    alignas(16) float taug[SW_NGPT][SW2_KS];
};
// Dynamic tail: the aerosol block (present only with aerosol inputs) and the segment checkpoints.
struct SwAer {
    float tau[14][SW2_KS], tasa[14][SW2_KS], tay[14][SW2_KS], tabs[14][SW2_KS];
};
__host__ __device__ constexpr size_t sw2_ckpt_bytes() { return (size_t)(SW2_NSEG - 1) * 4 * SW2_THREADS * sizeof(float); }
__host__ __device__ constexpr size_t sw2_smem_bytes(bool aer)
{
    return sizeof(SwSh2) + (aer ? sizeof(SwAer) : 0) + sw2_ckpt_bytes();
}

// Everything the float64 recompute of a layer needs besides the layer index and g-point, and the weights of
// the table-entry guard: wh = 1.5 zsolar 86400 / SW2_HEAT_T (times heatfac / delp of the layer: the heating
// change per unit change of the layer's R/T, relative to its limit), wf = zsolar / SW2_FLUX_T.
struct SwExactCtx {
    const SwIn* a;
    int64_t col;
    int laytrop, kmin8, kminw, mode;
    double cz, snt;
    const double* exd;
    float wh, wf;
};

// The layer's clear (cloud = false) or cloud-mixture optical properties recomputed from the column
// inputs in float64, then the reference's R/T statements in float64 (spcvrtc.cu:112-173 via sw_rt).
__device__ __noinline__ void sw2_exact(const SwExactCtx& x, int k0, int g, int ib, bool cloud, double& rb,
                                       double& rd, double& tb, double& td, double& e3, double& e4)
{
    const SwIn& a = *x.a;
    SwCoef<double> c;
    sw2_layer_coef<double>(a, x.col, k0, c);
    SwOne L;
    L.fac00.v = c.fac00; L.fac01.v = c.fac01; L.fac10.v = c.fac10; L.fac11.v = c.fac11;
    L.selffac.v = c.selffac; L.selffrac.v = c.selffrac; L.forfac.v = c.forfac; L.forfrac.v = c.forfrac;
    L.colmol.v = c.colmol;
    for (int m = 0; m < 6; ++m) L.colamt[m].v = c.colamt[m];
    L.jp.v = c.jp; L.jt.v = c.jt; L.jt1.v = c.jt1; L.indself.v = c.indself; L.indfor.v = c.indfor;
    L.laytrop = x.laytrop; L.kmin8 = x.kmin8; L.kminw = x.kminw;
    double tg, tr;
    sw_gas<double>(L, g, k0, tg, tr);
    double ta = 0, sa = 0, ya = 0;
    const int64_t N = a.ncol;
    const int kk0 = a.nlay - 1 - k0;
    if (a.faersw) {
        ta = (double)__ldg(a.faersw + (((size_t)ib) * a.nlay + kk0) * N + x.col);
        sa = (double)__ldg(a.faersw + (((size_t)(14 + ib)) * a.nlay + kk0) * N + x.col);
        ya = (double)__ldg(a.faersw + (((size_t)(28 + ib)) * a.nlay + kk0) * N + x.col);
    }
    double t0 = fmax((double)1.0e-12f, tr + tg + ta), s0 = tr + ta * sa, y0 = ya * sa * ta;
    if (cloud) {
        const double cf = (double)__ldg(a.clouds + (size_t)kk0 * N + x.col);
        double tc, sc, ac, tb_;
        sw2_cloud<double>(a, x.col, k0, ib, cf, tc, sc, ac, tb_);
        t0 = t0 + tc; s0 = s0 + sc; y0 = y0 + ac;
    }
    const double oneminus = (double)1.0f - (double)1.0e-6f, ftiny = (double)1.0e-12f;
    const double zssaw = fmin(oneminus, s0 / t0);
    const double zasyw = y0 / fmax(ftiny, s0);
    const double za1s = zasyw * zasyw, za2s = zssaw * za1s;
    const double ztau1 = (1.0 - za2s) * t0;
    const double zssa1 = (zssaw - za2s) / (1.0 - za2s);
    const double zasy1 = zasyw / (1.0 + zasyw), zasy3 = 0.75 * zasy1;
    double g1, g2, g3;
    sw_gam<double>(x.mode, zssa1, zasy1, zasy3, x.cz, g1, g2, g3);
    sw_rt<double, false>(ztau1, zssaw, zssa1, g1, g2, g3, 1.0 - g3, x.cz, x.snt, x.exd, rb, rd, tb, td);
    e3 = sw_expm(ztau1 * x.snt, x.exd, true);
    e4 = sw_expm(t0 * x.snt, x.exd, true);
}

// True when exp(-zb) takes the same entry of the reference's 10,001-entry table (or the same side of its
// 0.06 expansion switch) for every zb within the float optical properties' rounding: the float64 R/T
// below gets zb from float optics, whose relative error (~2e-6) moves the rounded table position
// 10^4 zb / (bpade + zb) + 1/2 by at most ~5e-3.
__device__ __forceinline__ bool sw2_tbl_sure(double zb)
{
    if (zb > 0.06 * (1.0 - 1.0e-5) && zb < 0.06 * (1.0 + 1.0e-5)) return false;
    if (zb <= 0.06) return true;
    const double t = 10000.0 * (zb / ((double)1.0f / (double)0.278f + zb)) + 0.5;
    const double f = t - floor(t);
    return f > SW2_TBL_MARGIN && f < 1.0 - SW2_TBL_MARGIN;
}

// Table-entry guard.  exp(-zb) comes from the reference's 10,001-entry table, entry int(10^4 zb / (bpade + zb)
// + 1/2).  A float argument that lies within its rounding (SW2_ZB_EPS relative, and the float evaluation of the
// entry position) of an entry bound may take the neighbouring entry where the float64 optics take the other.
// One entry step is ~3e-4 of the exponential; near the two-stream resonance the layer R/T amplify it by
// ~1 / |1 - (k mu0)^2|, and on a thin layer under a strong g-point one step moves the layer's heating rate by
// up to ~0.05 K/day: the reference's own outputs change that much when its optical depths change by 1e-7.
// sw2_near: the argument is that close to a bound (or to the 0.06 switch to the series).
__device__ __forceinline__ bool sw2_near(float zb)
{
    if (zb <= 0.06f * (1.0f + SW2_ZB_EPS)) return zb > 0.06f * (1.0f - SW2_ZB_EPS);
    const float ft = zb / ((float)1.0f / (float)0.278f + zb);
    const float pos = ft * (float)10000 + (float)0.5f;            // sw_expm's entry position
    const float fr = pos - floorf(pos);
    const float m = 10000.0f * ft * (SW2_ZB_EPS * (1.0f - ft) + 3.0e-7f);
    return fr < m || fr > 1.0f - m;
}
// exp(-zb) and its complement as the neighbouring entry across the nearer bound gives them (the series on the
// other side of 0.06).
__device__ __forceinline__ float sw2_expm_alt(float zb, const float* ex, float& em)
{
    const float ft = zb / ((float)1.0f / (float)0.278f + zb);
    const float pos = ft * (float)10000 + (float)0.5f;
    const int it = min(10000, (int)pos);
    if (zb <= 0.06f) {                                            // the table entry instead of the series
        em = 1.0f - __ldg(ex + it);
        return __ldg(ex + it);
    }
    if (zb <= 0.06f * (1.0f + SW2_ZB_EPS)) {                      // the series instead of the table entry
        em = zb - 0.5f * zb * zb;
        return 1.0f - zb + 0.5f * zb * zb;
    }
    const int nb = pos - (float)it < 0.5f ? max(it - 1, 0) : min(it + 1, 10000);
    em = 1.0f - __ldg(ex + nb);
    return __ldg(ex + nb);
}
// True when taking the other entry for e1 (n1) or e2 (n2) changes the layer's R/T and direct transmission
// (e3 shares e2's entry) by more than 1 / w.  Rare (arguments near a bound); the R/T are evaluated again.
__device__ __noinline__ bool sw2_flip_matters(const SwPro<float>& p, float cz, float snt, const float* ex, bool n1,
                                              bool n2, float w, float rb, float rd, float tb, float td)
{
    float em1, em2;
    const float zb1 = fminf(p.zrk * p.ztau1, 500.0f), zb2 = fminf(p.ztau1 * snt, 500.0f);
    const float e1 = sw2_expm_c(zb1, ex, em1), e2 = sw2_expm_c(zb2, ex, em2);
    float d = 0.0f;
    if (n1) {
        float a1m, rb1, rd1, tb1, td1;
        const float a1 = sw2_expm_alt(zb1, ex, a1m);
        sw2_rt_core<float>(p, cz, a1, a1m, e2, em2, rb1, rd1, tb1, td1);
        d = fabsf(rb1 - rb) + fabsf(rd1 - rd) + fabsf(tb1 - tb) + fabsf(td1 - td);
    }
    if (n2) {
        float a2m, rb2, rd2, tb2, td2;
        const float a2 = sw2_expm_alt(zb2, ex, a2m);
        sw2_rt_core<float>(p, cz, e1, em1, a2, a2m, rb2, rd2, tb2, td2);
        d = fmaxf(d, fabsf(rb2 - rb) + fabsf(rd2 - rd) + fabsf(tb2 - tb) + fabsf(td2 - td) + fabsf(a2 - e2));
    }
    return d * w > 1.0f;
}

// R/T of a layer near the two-stream resonance in float64 from its float optical properties.  Returns false
// when the result depends on more than those: a table entry of e1 = exp(-k tau1) or e2 = exp(-tau1 / mu0)
// that the float rounding could move (the resonance amplifies the neighbouring entry's 1e-4 to ~1e-2), or
// |1 - (k mu0)^2| within reach of the reference's 1e-8 clamp.
__device__ __noinline__ bool sw2_rt_double(float t0, float tabs, float s0, float y0, const SwExactCtx& x, float& rb,
                                           float& rd, float& tb, float& td)
{
    const SwPro<double> pd = sw2_prologue<double>((double)t0, (double)tabs, (double)s0, (double)y0, x.mode, x.cz);
    double a, b, c, d;
    sw2_rt_tail<double>(pd, x.cz, x.snt, x.exd, a, b, c, d);
    rb = (float)a; rd = (float)b; tb = (float)c; td = (float)d;
    return fabs(pd.zrpp) > 1.0e-5 && sw2_tbl_sure(fmin(pd.zrk * pd.ztau1, 500.0)) &&
           sw2_tbl_sure(fmin(pd.ztau1 * x.snt, 500.0));
}

// One optical-property set of a layer -> R/T and direct transmissions: float; near the resonance
// (|1 - (k mu0)^2| < SW2_RESONANCE, where the float R/T loses ~1e-7 / |1 - (k mu0)^2| of relative accuracy)
// float64 from the float optics; where even that is not decided by the float optics, the float64 recompute
// of the layer from the column inputs (sw2_exact).  The float64 recompute also replaces the float R/T where an
// exponential's argument lies within its rounding of a table-entry bound and the other entry matters: wk
// weighs the change of the R/T and of the direct transmission (the layer's heating, x.wh times its heatfac /
// delp), x.wf the step of exp(-tau0 / mu0) (the surface direct beam alone).
__device__ __forceinline__ void sw2_rt_mixed(float t0, float tabs, float s0, float y0, float cz, float snt,
                                             const float* ex, const SwExactCtx& x, int k0, int g, int ib, bool cloud,
                                             float wk, float& rb, float& rd, float& tb, float& td, float& e3, float& e4)
{
    const SwPro<float> p = sw2_prologue<float>(t0, tabs, s0, y0, x.mode, cz);
    bool exact = false;
    if (fabsf(p.zrpp) < SW2_RESONANCE) {
        exact = !sw2_rt_double(t0, tabs, s0, y0, x, rb, rd, tb, td);
    } else {
        sw2_rt_tail<float>(p, cz, snt, ex, rb, rd, tb, td);
        const bool n1 = sw2_near(fminf(p.zrk * p.ztau1, 500.0f)), n2 = sw2_near(fminf(p.ztau1 * snt, 500.0f));
        if ((n1 || n2) && wk > 0.0f) exact = sw2_flip_matters(p, cz, snt, ex, n1, n2, wk, rb, rd, tb, td);
    }
    const float zb4 = t0 * snt;
    if (!exact && x.wf * 4.0e-4f > 1.0f && sw2_near(zb4)) {
        float am;
        exact = fabsf(sw2_expm_alt(zb4, ex, am) - sw_expm(zb4, ex, true)) * x.wf > 1.0f;
    }
    if (exact) {
        double a, b, c, d, f3, f4;
        sw2_exact(x, k0, g, ib, cloud, a, b, c, d, f3, f4);
        rb = (float)a; rd = (float)b; tb = (float)c; td = (float)d; e3 = (float)f3; e4 = (float)f4;
        return;
    }
    e3 = sw_expm(p.ztau1 * snt, ex, true);
    e4 = sw_expm(zb4, ex, true);
}

// Entry int(10^4 zb / (bpade + zb) + 1/2) of the reference's exp table, exp(-bpade i / (10^4 - i)) (1e-20 for
// the last), evaluated instead of loaded (the float R/T of sw2_rt_float; within a few float ulps of the table's
// float value for the arguments that matter, ~1e-5 relative where exp is below 1e-13), with the series below
// 0.06 as sw_expm; em = its complement.
__device__ __forceinline__ float sw2_tblexp(float zb, float& em)
{
    if (zb <= 0.06f) {
        em = zb - 0.5f * zb * zb;
        return 1.0f - zb + 0.5f * zb * zb;
    }
    const float ftind = zb / ((float)1.0f / (float)0.278f + zb);
    const int it = min(10000, (int)(ftind * (float)10000 + (float)0.5f));
    const float e = it >= 10000 ? 1.0e-20f : __expf(-(3.59712230f * (float)it) / (float)(10000 - it));
    em = 1.0f - e;
    return e;
}

// The float R/T of sw2_rt_mixed alone: false (and nothing final) where sw2_rt_mixed would take any float64 step
// or test the neighbouring table entry -- the resonance, an argument near a table-entry bound with a weight.
// Where it returns true the outputs are exactly sw2_rt_mixed's.
__device__ __forceinline__ bool sw2_rt_float(float t0, float tabs, float s0, float y0, float cz, float snt,
                                             const float* ex, int mode, float wk, float wf, float& rb, float& rd,
                                             float& tb, float& td, float& e3, float& e4)
{
    const SwPro<float> p = sw2_prologue<float>(t0, tabs, s0, y0, mode, cz);
    if (fabsf(p.zrpp) < SW2_RESONANCE) return false;
    if (wk > 0.0f && (sw2_near(fminf(p.zrk * p.ztau1, 500.0f)) || sw2_near(fminf(p.ztau1 * snt, 500.0f)))) return false;
    const float zb4 = t0 * snt;
    if (wf * 4.0e-4f > 1.0f && sw2_near(zb4)) return false;
    float em1, em2, em;
    const float e1 = sw2_tblexp(fminf(p.zrk * p.ztau1, 500.0f), em1);
    const float e2 = sw2_tblexp(fminf(p.ztau1 * snt, 500.0f), em2);
    sw2_rt_core<float>(p, cz, e1, em1, e2, em2, rb, rd, tb, td);
    e3 = sw2_tblexp(p.ztau1 * snt, em);
    e4 = sw2_tblexp(zb4, em);
    return true;
}

struct SwLayerRT {
    float rb, rd, tb, td, e3, e4;
};

__device__ __forceinline__ float sw2_taur(const SwSh2& s, int g, int k0)
{
    return (g >= 66 && g < 74 && k0 < s.laytrop) ? s.taur24[g - 66][k0] : s.colmol[k0] * s.raylc[g];
}

// R/T of layer k0 for g-point g in the clear pass (c) and, for a cloudy column, the cloudy pass (o) of
// spcvrtc (spcvrtc.cu:330-460: the cloudy pass blends the clear and the cloud-mixture R/T by the layer's
// cloud fraction).  The clear R/T is computed once and serves both passes.  McICA route (mc): the second
// pass takes the cloud-mixture R/T unblended in the cloudy layers whose sub-column bit is set.
struct SwLayerRT2 {
    SwLayerRT c, o;
};
__device__ __forceinline__ bool sw2_cloud_layer(const SwSh2& s, bool mc, int g, int k0)
{
    return s.cldfrc[k0] > 1.0e-12f && (!mc || ((s.mcw[g >> 5][k0] >> (g & 31)) & 1u));
}

__device__ __noinline__ SwLayerRT2 sw2_layer(const SwSh2& s, const SwAer* aer, const SwExactCtx& x, int k0, int g,
                                             int ib, bool cloudy, bool mc, float cz, float snt, const float* ex,
                                             float tg)
{
    SwLayerRT2 r;
    SwLayerRT& c = r.c;
    SwLayerRT& o = r.o;
    if (k0 >= x.a->nlay) {   // padding above the model top: a transparent, non-reflecting layer
        c.rb = 0; c.rd = 0; c.tb = 1; c.td = 1; c.e3 = 1; c.e4 = 1;
        o = c;
        return r;
    }
    const float tr = sw2_taur(s, g, k0);
    float ta = 0, tasa = 0, tay = 0, taab = 0;
    if (aer) { ta = aer->tau[ib][k0]; tasa = aer->tasa[ib][k0]; tay = aer->tay[ib][k0]; taab = aer->tabs[ib][k0]; }
    const float ct0 = fmaxf(1.0e-12f, tr + tg + ta), cs0 = tr + tasa, cy0 = tay, cab = tg + taab;
    const float wk = x.wh * (float)s.rdelp[k0];
    sw2_rt_mixed(ct0, cab, cs0, cy0, cz, snt, ex, x, k0, g, ib, false, wk, c.rb, c.rd, c.tb, c.td, c.e3, c.e4);
    o = c;
    if (cloudy && sw2_cloud_layer(s, mc, g, k0)) {
        {
            const float zc1 = mc ? 1.0f : s.cldfrc[k0];
            const float ot0 = ct0 + s.taucw[ib][k0], os0 = cs0 + s.ssacw[ib][k0], oy0 = cy0 + s.asycw[ib][k0];
            const float oab = cab + s.tabsc[ib][k0];
            float rb2, rd2, tb2, td2, e32, e42;
            sw2_rt_mixed(ot0, oab, os0, oy0, cz, snt, ex, x, k0, g, ib, true, wk, rb2, rd2, tb2, td2, e32, e42);
            if (mc) {
                o.rb = rb2; o.rd = rd2; o.tb = tb2; o.td = td2; o.e3 = e32; o.e4 = e42;
                return r;
            }
            const float zc0 = 1.0f - zc1;
            o.rb = zc0 * c.rb + zc1 * rb2;
            o.rd = zc0 * c.rd + zc1 * rd2;
            o.tb = zc0 * c.tb + zc1 * tb2;
            o.td = zc0 * c.td + zc1 * td2;
            o.e3 = zc0 * c.e3 + zc1 * e32;
            o.e4 = zc0 * c.e4 + zc1 * e42;
        }
    }
    return r;
}

// One step of the upward (bottom-up) adding recursion through layer L (swflux.cu, zrupb / zrupd).
__device__ __forceinline__ void sw2_up(const SwLayerRT& L, float& ub, float& ud)
{
    const float den = 1.0f / (1.0f - ud * L.rd);
    const float ub1 = L.rb + (L.td * ((L.tb - L.e3) * ud + L.e3 * ub)) * den;
    ud = L.rd + L.td * L.td * ud * den;
    ub = ub1;
}
// Level fluxes from the upward (ub, ud) and downward (tdn, rdn, tdb) states (swflux.cu, zfu / zfd).
__device__ __forceinline__ void sw2_flux(float ub, float ud, float tdn, float rdn, float tdb, float& fu, float& fd)
{
    const float den = 1.0f / (1.0f - rdn * ud);
    fu = (tdb * ub + (tdn - tdb) * ud) * den;
    fd = tdb + (tdn - tdb + tdb * ub * rdn) * den;
}
// One step of the downward recursion through layer L (swflux.cu, ztdn / zrdnd / ztdbt).
__device__ __forceinline__ void sw2_down(const SwLayerRT& L, float& tdn, float& rdn, float& tdb)
{
    const float den = 1.0f / (1.0f - L.rd * rdn);
    const float tdn1 = tdb * L.tb + (L.td * ((tdn - tdb) + tdb * L.rb * rdn)) * den;
    rdn = L.rd + L.td * L.td * rdn * den;
    tdn = tdn1;
    tdb = L.e3 * tdb;
}

// Phase-C thread -> g-point: the four warps take g-points 0-27, 28-55, 56-85 (the Rayleigh-dominated bands
// 23-26) and 86-111, one per lane; each lane runs both passes of its g-point.  Idle lanes mirror the warp's
// last g-point (act = false).
__device__ __forceinline__ int sw2_lane_g(int t, bool& act)
{
    const int wq = (t >> 5) & 3, lane = t & 31;
    const int gb = wq == 0 ? 0 : (wq == 1 ? 28 : (wq == 2 ? 56 : 86));
    const int ge = wq == 0 ? 28 : (wq == 1 ? 56 : (wq == 2 ? 86 : SW_NGPT));
    act = gb + lane < ge;
    return act ? gb + lane : ge - 1;
}

// ------------------------------------------------------------------------------------------------------
// Layer R/T store of one CTA (rad_solve's SW): the upward sweep writes each layer's clear and cloudy
// rb, rd, tb, td, e3 ([layer][field][thread], coalesced) and each segment's product of the direct-beam
// transmissions e4 ([segment][pass][thread]); the downward sweep reads them back instead of recomputing the
// R/T.  The values are the ones the recompute would give, so the outputs do not change.
constexpr int SW2_RT_FIELDS = 10;
constexpr int SW2_CTAS_PER_SM = 2;                                 // the kernel's launch bound
__host__ __device__ constexpr int64_t sw2_rt_floats()
{
    return ((int64_t)NLAY_MAX * SW2_RT_FIELDS + (int64_t)SW2_NSEG * 2) * SW2_THREADS;
}
inline int64_t sw2_rt_bytes(int nsm) { return (int64_t)SW2_CTAS_PER_SM * nsm * sw2_rt_floats() * (int64_t)sizeof(float); }

// Phases A1 and A2 of one sunlit column (day index d, column col of request a) into shared memory s (aer: the
// aerosol block or null): layer coefficients, aerosol, heating factors, column scalars, cloud optics per (band,
// layer), solar source, Rayleigh coefficients.  Ends with a barrier.
template <int NT = SW2_THREADS>
__device__ __forceinline__ void sw2_setup(SwSh2& s, SwAer* aer, const SwIn& a, int64_t col, int d, int tid)
{
    const int nlay = a.nlay;
    const int64_t N = a.ncol;
    const double heatfac = 9.80665 * 1.0e-2 / 1.0046e3;
    // ---- phase A1: layer coefficients (threads = layers), aerosol, heating factors.  The coefficients are
    // formed in float64 and rounded once: the interpolation weights take a difference of logarithms, which
    // float would carry with ~1e-6 of the gas optical depths' error (and move their exp-table entries).
    for (int k0 = tid; k0 < nlay; k0 += NT) {
        SwCoef<double> c;
        sw2_layer_coef<double>(a, col, k0, c);
        s.fac00[k0] = (float)c.fac00; s.fac01[k0] = (float)c.fac01; s.fac10[k0] = (float)c.fac10;
        s.fac11[k0] = (float)c.fac11;
        s.selffac[k0] = (float)c.selffac; s.selffrac[k0] = (float)c.selffrac; s.forfac[k0] = (float)c.forfac;
        s.forfrac[k0] = (float)c.forfrac;
        s.colmol[k0] = (float)c.colmol;
        for (int m = 0; m < 6; ++m) s.colamt[m][k0] = (float)c.colamt[m];
        {   // key-species ratios x1 / (x1 + strrat x2) of bands 16-19, 21, 22, 24, 28 (sw_species slots 0..7)
            const double h = c.colamt[0], c2 = c.colamt[1], o3 = c.colamt[2], ch4 = c.colamt[4], o2 = c.colamt[5];
            auto ratio = [](double x1, double strr, double x2, bool guard) {
                const double sc = x1 + strr * x2;
                return guard ? (sc > 0 ? x1 / sc : 0.0) : x1 / sc;
            };
            s.spr[0][k0] = ratio(h, (double)ldt(tab<float>(T_SW16_STRRAT)), ch4, false);
            s.spr[1][k0] = ratio(h, (double)ldt(tab<float>(T_SW_STRRAT) + 1), c2, false);
            s.spr[2][k0] = ratio(h, (double)ldt(tab<float>(T_SW_STRRAT) + 2), ch4, true);
            s.spr[3][k0] = ratio(h, (double)5.49281e+0f, c2, false);
            s.spr[4][k0] = ratio(h, (double)4.53210e-03f, c2, false);
            s.spr[5][k0] = ratio(h, (double)3.63328e-02f, o2, true);
            s.spr[6][k0] = ratio(h, (double)1.24692e-1f, o2, false);
            s.spr[7][k0] = ratio(o3, (double)ldt(tab<float>(T_SW28_STRRAT)), o2, false);
        }
        s.jp[k0] = c.jp; s.jt[k0] = c.jt; s.jt1[k0] = c.jt1; s.indself[k0] = c.indself; s.indfor[k0] = c.indfor;
        s.low[k0] = c.low ? 1 : 0;
        const int kk0 = nlay - 1 - k0;
        s.cfrac[k0] = __ldg(a.clouds + (size_t)kk0 * N + col);
        const double dl = (double)__ldg(a.plvl + (size_t)(kk0 + 1) * N + col) - (double)__ldg(a.plvl + (size_t)kk0 * N + col);
        s.rdelp[k0] = heatfac / dl;
        if (aer) {
            for (int ib = 0; ib < 14; ++ib) {
                const float ta = __ldg(a.faersw + (((size_t)ib) * nlay + kk0) * N + col);
                const float sa = __ldg(a.faersw + (((size_t)(14 + ib)) * nlay + kk0) * N + col);
                const float ya = __ldg(a.faersw + (((size_t)(28 + ib)) * nlay + kk0) * N + col);
                aer->tau[ib][k0] = ta;
                aer->tasa[ib][k0] = ta * sa;
                aer->tay[ib][k0] = ya * sa * ta;
                aer->tabs[ib][k0] = ta * (1.0f - sa);
            }
        }
    }
    __syncthreads();
    // ---- column scalars (thread 0): sun, albedo, overlap fractions (swrad.cu:242-279), laytrop
    if (tid == 0) {
        const float cz = __ldg(a.coszen + col);
        s.cosz = cz;
        s.sntz = 1.0f / cz;
        s.ssolar = (a.solcon / 1368.22f) * cz;
        s.albbm[0] = __ldg(a.sfcalb + col);
        s.albdf[0] = __ldg(a.sfcalb + N + col);
        s.albbm[1] = __ldg(a.sfcalb + 2 * N + col);
        s.albdf[1] = __ldg(a.sfcalb + 3 * N + col);
        const float z0 = sw_zcf0<float>(s.cfrac, nlay, a.iovr);
        s.zcf0 = z0;
        s.zcf1 = 1.0f - z0;
        int lt = nlay;
        for (int k0 = 0; k0 < nlay; ++k0)
            if (s.low[k0]) lt = k0 + 1;
        s.laytrop = lt;
        s.kmin8 = a.kmin8[d];
        s.kminw = a.kminw[d];
        s.task_next = 0;
    }
    if (a.mask)
        for (int i = tid; i < 4 * nlay; i += NT)
            s.mcw[i / nlay][i % nlay] = __ldg(a.mask + ((size_t)(i / nlay) * nlay + (i % nlay)) * N + col);
    __syncthreads();
    // ---- phase A2: cloud optics per (band, layer); solar source per band
    for (int p = tid; p < 14 * nlay; p += NT) {
        const int ib = p / nlay, k0 = p - ib * nlay;
        float tcw = 0, scw = 0, acw = 0, tab_ = 0;
        if (s.zcf1 > 0) sw2_cloud<float>(a, col, k0, ib, s.cfrac[k0], tcw, scw, acw, tab_);
        s.taucw[ib][k0] = tcw; s.ssacw[ib][k0] = scw; s.asycw[ib][k0] = acw; s.tabsc[ib][k0] = tab_;
        if (ib == 0) s.cldfrc[k0] = s.zcf1 > 0 ? s.cfrac[k0] / s.zcf1 : 0.0f;
    }
    if (tid < 14) sw_sfluxzen<float>(s, tid, nlay);
    for (int g = tid; g < SW_NGPT; g += NT) s.raylc[g] = sw2_rayl_coef(g);
    __syncthreads();
}

// One sunlit column (day index d) by the CTA; STORE: rt = the CTA's R/T store, else the R/T is recomputed.
template <bool STORE>
__device__ __forceinline__ void sw2_column(const SwBatch& bt, int any_aer, const float* ex, const double* exd,
                                           int* err, int d, float* rt)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SwSh2& s = *reinterpret_cast<SwSh2*>(smem_raw);
    const int64_t gcol = bt.req[0].daycol[d];
    const int rq = bt.find(gcol);
    const SwIn& a = bt.req[rq];
    // the aerosol block is reserved when any request of the launch has aerosol; used when this one does
    SwAer* aer = a.faersw ? reinterpret_cast<SwAer*>(smem_raw + sizeof(SwSh2)) : nullptr;
    float* ckpt = reinterpret_cast<float*>(smem_raw + sizeof(SwSh2) + (any_aer ? sizeof(SwAer) : 0));
    const int nlay = a.nlay, nlp1 = nlay + 1;
    if (nlay > NLAY_MAX) {
        if (threadIdx.x == 0) atomicExch(err, RAD_DEV_NLAY);
        return;
    }
    const int64_t N = a.ncol;
    const int64_t col = gcol - bt.off[rq];
    const int tid = threadIdx.x;
    sw2_setup(s, aer, a, col, d, tid);
    // ---- phase B: gas and Rayleigh optical depths per (g, layer), band by band
    for_each_band_pair(c_sw_ns, 14, nlay, &s.task_next, tid & 31, [&](int g, int k0, int b) {
        float tg, tr;
        sw_gas<float>(s, g, k0, tg, tr, b);
        s.taug[g][k0] = tg;
        if (g >= 66 && g < 74 && k0 < s.laytrop) s.taur24[g - 66][k0] = tr;
    });
    __syncthreads();
    // ---- phase C: spcvrtc, one g-point per lane, both passes
    const int warp = tid >> 5, lane = tid & 31;
    bool act;
    const int g = sw2_lane_g(tid, act);
    int ib0 = 0;
    while (g >= c_sw_ns[ib0 + 1]) ++ib0;
    const int ibd = ib0 == 8 ? 0 : ((ib0 >= 9 && ib0 <= 12) ? 2 : 1);   // idxsfc
    const float cz = s.cosz, snt = s.sntz;
    const bool mc = a.mask != nullptr;
    const bool cloudy = mc ? s.zcf1 > 0.0f : s.zcf1 > 1.0e-6f;
    const float zsolar = act ? s.ssolar * s.sfluxzen[g] : 0.0f;
    const float ab = ibd ? s.albbm[ibd - 1] : 0.5f * (s.albbm[0] + s.albbm[1]);
    const float ad = ibd ? s.albdf[ibd - 1] : 0.5f * (s.albdf[0] + s.albdf[1]);
    SwExactCtx x{&a, col, s.laytrop, s.kmin8, s.kminw, a.iswmode, (double)__ldg(a.coszen + col),
                 1.0 / (double)__ldg(a.coszen + col), exd, zsolar * (1.5f * 86400.0f / SW2_HEAT_T),
                 zsolar * (1.0f / SW2_FLUX_T)};
    const int nseg = (nlay + SW2_SEG - 1) / SW2_SEG;
    float* ck = ckpt + tid;
    auto CK = [&](int sg, int q) -> float& { return ck[((sg - 1) * 4 + q) * SW2_THREADS]; };
    // upward sweep: reflectances of the atmosphere below each level, clear (c) and cloudy (o) passes
    float ubc = ab, udc = ad, ubo = ab, udo = ad;
    float* const rtl = STORE ? rt + tid : nullptr;
    auto RT = [&](int k0, int f) -> float& { return rtl[((size_t)k0 * SW2_RT_FIELDS + f) * SW2_THREADS]; };
    auto RS = [&](int sg, int q) -> float& {
        return rtl[((size_t)NLAY_MAX * SW2_RT_FIELDS + (size_t)sg * 2 + q) * SW2_THREADS];
    };
    for (int sg = 0; sg < nseg; ++sg) {
        if (sg > 0) { CK(sg, 0) = ubc; CK(sg, 1) = udc; CK(sg, 2) = ubo; CK(sg, 3) = udo; }
        float e4c = 1, e4o = 1;
        for (int j = 0; j < SW2_SEG; ++j) {
            const int k0 = sg * SW2_SEG + j;
            const SwLayerRT2 L = sw2_layer(s, aer, x, k0, g, ib0, cloudy, mc, cz, snt, ex, s.taug[g][k0]);
            sw2_up(L.c, ubc, udc);
            if (cloudy) sw2_up(L.o, ubo, udo);
            if (STORE) {
                e4c = e4c * L.c.e4;
                if (cloudy) e4o = e4o * L.o.e4;
                if (k0 < nlay) {
                    RT(k0, 0) = L.c.rb; RT(k0, 1) = L.c.rd; RT(k0, 2) = L.c.tb; RT(k0, 3) = L.c.td; RT(k0, 4) = L.c.e3;
                    if (cloudy) {
                        RT(k0, 5) = L.o.rb; RT(k0, 6) = L.o.rd; RT(k0, 7) = L.o.tb; RT(k0, 8) = L.o.td;
                        RT(k0, 9) = L.o.e3;
                    }
                }
            }
        }
        if (STORE) { RS(sg, 0) = e4c; RS(sg, 1) = e4o; }
    }
    // downward sweep, segment by segment from the top: recompute the segment's R/T and upward states into
    // registers from its checkpoint, then walk down through it
    const double w0 = cloudy ? (mc ? 0.0 : (double)s.zcf0) : 1.0, w1 = cloudy ? (mc ? 1.0 : (double)s.zcf1) : 0.0;
    float tdnc = 1, rdnc = 0, tdbc = 1, tdbc0 = 1, tdno = 1, rdno = 0, tdbo = 1, tdbo0 = 1;
    float toa_c = 0, toa_o = 0;
    // store path: segment sg's R/T are loaded into pf while segment sg + 1 is walked
    float pf[SW2_SEG][SW2_RT_FIELDS], pe4c = 1, pe4o = 1;
    auto fetch = [&](int sg) {
#pragma unroll
        for (int j = 0; j < SW2_SEG; ++j) {
            const int k0 = sg * SW2_SEG + j;
#pragma unroll
            for (int f = 0; f < SW2_RT_FIELDS; ++f)
                pf[j][f] = k0 < nlay && (f < 5 || cloudy) ? RT(k0, f) : 0.0f;
        }
        pe4c = RS(sg, 0);
        pe4o = RS(sg, 1);
    };
    if (STORE) fetch(nseg - 1);
    for (int sg = nseg - 1; sg >= 0; --sg) {
        SwLayerRT Lc[SW2_SEG], Lo[SW2_SEG];
        float zubc[SW2_SEG + 1], zudc[SW2_SEG + 1], zubo[SW2_SEG + 1], zudo[SW2_SEG + 1];
        zubc[0] = sg ? CK(sg, 0) : ab;
        zudc[0] = sg ? CK(sg, 1) : ad;
        zubo[0] = sg ? CK(sg, 2) : ab;
        zudo[0] = sg ? CK(sg, 3) : ad;
        float e4c = 1, e4o = 1;
        if (STORE) {
            // the segment's R/T from the store (the layers above the model top are transparent)
#pragma unroll
            for (int j = 0; j < SW2_SEG; ++j) {
                const int k0 = sg * SW2_SEG + j;
                if (k0 < nlay) {
                    Lc[j].rb = pf[j][0]; Lc[j].rd = pf[j][1]; Lc[j].tb = pf[j][2]; Lc[j].td = pf[j][3];
                    Lc[j].e3 = pf[j][4];
                    if (cloudy) {
                        Lo[j].rb = pf[j][5]; Lo[j].rd = pf[j][6]; Lo[j].tb = pf[j][7]; Lo[j].td = pf[j][8];
                        Lo[j].e3 = pf[j][9];
                    } else {
                        Lo[j] = Lc[j];
                    }
                } else {
                    Lc[j].rb = 0; Lc[j].rd = 0; Lc[j].tb = 1; Lc[j].td = 1; Lc[j].e3 = 1;
                    Lo[j] = Lc[j];
                }
                Lc[j].e4 = 1; Lo[j].e4 = 1;
            }
            e4c = pe4c;
            e4o = pe4o;
            if (sg > 0) fetch(sg - 1);
        }
#pragma unroll
        for (int j = 0; j < SW2_SEG; ++j) {
            if (!STORE) {
                const SwLayerRT2 L = sw2_layer(s, aer, x, sg * SW2_SEG + j, g, ib0, cloudy, mc, cz, snt, ex,
                                               s.taug[g][sg * SW2_SEG + j]);
                Lc[j] = L.c;
                Lo[j] = L.o;
                e4c = e4c * Lc[j].e4;
                if (cloudy) e4o = e4o * Lo[j].e4;
            }
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
                float fu, fd;
                sw2_flux(zubc[j + 1], zudc[j + 1], tdnc, rdnc, tdbc, fu, fd);
                double net = w0 * ((double)fd - (double)fu);
                if (lev == nlp1) toa_c = fu;
                if (cloudy) {
                    float fuo, fdo;
                    sw2_flux(zubo[j + 1], zudo[j + 1], tdno, rdno, tdbo, fuo, fdo);
                    net += w1 * ((double)fdo - (double)fuo);
                    if (lev == nlp1) toa_o = fuo;
                }
                const double v = warp_sum(act ? (double)zsolar * net : 0.0);
                if (lane == 0) s.fn[warp][lev - 1] = v;
            }
            sw2_down(Lc[j], tdnc, rdnc, tdbc);
            if (cloudy) sw2_down(Lo[j], tdno, rdno, tdbo);
        }
        tdbc0 = tdbc0 * e4c;
        tdbo0 = tdbo0 * e4o;
    }
    // surface level, and the per-lane scalars (zero for idle lanes)
    double scv[18];
#pragma unroll
    for (int i = 0; i < 18; ++i) scv[i] = 0;
    {
        float fu, fd, fuo = 0, fdo = 0;
        sw2_flux(ab, ad, tdnc, rdnc, tdbc, fu, fd);
        double net = w0 * ((double)fd - (double)fu);
        if (cloudy) {
            sw2_flux(ab, ad, tdno, rdno, tdbo, fuo, fdo);
            net += w1 * ((double)fdo - (double)fuo);
        }
        const double v = warp_sum(act ? (double)zsolar * net : 0.0);
        if (lane == 0) s.fn[warp][0] = v;
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
    for (int i = 0; i < 18; ++i) {
        const double v = warp_sum(scv[i]);
        if (lane == 0) s.sc[warp][i] = v;
    }
    __syncthreads();
    // ---- column end (spcvrtc.cu:493-545) and swrad_post (swrad.cu:365-403), float64
    auto tot = [&](double clr, double cld) { return cloudy ? w1 * cld + w0 * clr : clr; };
    for (int k = tid; k < nlay; k += SW2_THREADS) {
        double f0 = 0, f1 = 0;
        for (int w = 0; w < SW2_WARPS; ++w) { f0 += s.fn[w][k]; f1 += s.fn[w][k + 1]; }
        a.htsw[(size_t)(nlay - 1 - k) * N + col] = (float)((f1 - f0) * s.rdelp[k]);
    }
    if (tid == 0) {
        double c[9], t[9];
        for (int i = 0; i < 9; ++i) {
            c[i] = 0; t[i] = 0;
            for (int w = 0; w < SW2_WARPS; ++w) { c[i] += s.sc[w][i]; t[i] += s.sc[w][9 + i]; }
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
}

// STORE = false: one CTA per entry of the day list, R/T recomputed in the downward sweep (no scratch).
// STORE = true: a grid of SW2_CTAS_PER_SM CTAs per SM walks the day list; CTA b keeps its layer R/T in
// rts + b * sw2_rt_floats().
template <bool STORE>
__global__ void __launch_bounds__(SW2_THREADS, SW2_CTAS_PER_SM)
sw2_column_kernel(const __grid_constant__ SwBatch bt, int any_aer, const float* ex, const double* exd, int* err,
                  float* rts)
{
    const int nday = *bt.req[0].nday;
    if (!STORE) {
        if ((int)blockIdx.x < nday) sw2_column<false>(bt, any_aer, ex, exd, err, blockIdx.x, nullptr);
        return;
    }
    float* rt = rts + (int64_t)blockIdx.x * sw2_rt_floats();
    for (int d = blockIdx.x; d < nday; d += gridDim.x) {
        sw2_column<true>(bt, any_aer, ex, exd, err, d, rt);
        __syncthreads();                       // shared memory is reused by the next column
    }
}

}  // namespace rad
