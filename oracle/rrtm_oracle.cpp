// rrtm_oracle.cpp -- C entry points of the CPU oracle (test infrastructure only).
//
// Drives the LW and SW column restatements (rrtm_lw.hpp, rrtm_sw.hpp) over a request in the reference's
// call order: grrad cloud-path factor and lwrad (phys_rrtm_grrad_lw.cu:58-80, lw_core.seam), swrad on the
// day columns (coszen >= 1e-4, phys_rrtm_grrad_sw.cu:69) with the day list split into windows and chunks
// for the MINVAL(laytrop) groups (physics/rrtm/sw_seam.py:23-37, phys_rrtm_sw_swrad.py:340-386).
// Precision 0 runs every statement in float, precision 1 in double.  OpenMP over columns.
#include <cstdio>
#include <limits>
#include "rrtm_lw.hpp"
#include "rrtm_sw.hpp"
#include "rrtm_mcica.hpp"
#include "rrtm_aer.hpp"
#include "rrtm_solar.hpp"
#include "rrtm_grrad.hpp"
#include "rrtm_front.hpp"
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {
// Test hook: factor applied to the SW gas optical depths before the two-stream solver (orc_set_debug).
double g_sw_tau_scale = 1.0;

TableStore& tables()
{
    static TableStore s;
    return s;
}

template <class R>
static void run_lw(const Config& cfg, const Inputs& in, const Outputs& out)
{
    const int nlay = in.nlay, ncol = in.ncol, nlp1 = nlay + 1;
    const LwTables<R> tb;
    const R heatfac = (R)CON_G * (R)1.0e-2f / (R)CON_CP;
    const R fluxfac = std::is_same<R, float>::value ? (R)((double)(float)(2.0 * std::asin(1.0)) * 2.0e4)
                                                    : (R)(2.0 * std::asin(1.0) * 2.0e4);
    const int ilwcliq = cfg.diagnostic ? 0 : 1;
#pragma omp parallel for schedule(dynamic, 16)
    for (int col = 0; col < ncol; ++col) {
        std::vector<float> cl(9 * (size_t)nlay);
        for (int n = 0; n < 9; ++n)
            for (int k = 0; k < nlay; ++k) cl[n * nlay + k] = in.clouds[((size_t)n * nlay + k) * ncol + col];
        if (ilwcliq > 0) {   // grrad_lw_pre: clouds(.,.,2) and (.,.,4) scaled by the cloud-path factor
            for (int k = 0; k < nlay; ++k) {
                cl[1 * nlay + k] = cl[1 * nlay + k] * (float)cfg.cpathfac;
                cl[3 * nlay + k] = cl[3 * nlay + k] * (float)cfg.cpathfac;
            }
        }
        LwColumn<R> c(nlay);
        lw_prep(c, in, col, cl.data(), ilwcliq);
        lw_cldprop(c, cl.data(), ilwcliq);
        lw_setcoef(c);
        lw_taumol(c);
        if (cfg.route == 1) {
            lw_mcica<R>(c, cl.data(), ilwcliq, cfg, in, col, out.lw_mask);
            lw_rtrnmc(c, tb, heatfac, fluxfac);
        } else if (cfg.iovrlw <= 0) {       // lwrad's transfer dispatch (phys_rrtm_lw_lwrad.py:102-111)
            lw_rtrn(c, tb, heatfac, fluxfac);
        } else {
            lw_rtrnmr(c, tb, heatfac, fluxfac);
        }
        for (int k0 = 0; k0 < nlay; ++k0) out.htlw[(size_t)(nlay - 1 - k0) * ncol + col] = (double)c.htr[k0];
        out.topflw[0 * (size_t)ncol + col] = (double)c.totuflux[nlay];
        out.topflw[1 * (size_t)ncol + col] = (double)c.totuclfl[nlay];
        out.sfcflw[0 * (size_t)ncol + col] = (double)c.totuflux[0];
        out.sfcflw[1 * (size_t)ncol + col] = (double)c.totuclfl[0];
        out.sfcflw[2 * (size_t)ncol + col] = (double)c.totdflux[0];
        out.sfcflw[3 * (size_t)ncol + col] = (double)c.totdclfl[0];
        if (out.hlw0 || out.hlwb) {   // rtrnmr's lhlw0 / lhlwb blocks (phys_rrtm_lw_rtrnmr_body.cuh:328-362)
            for (int k = 1; k <= nlay; ++k) {
                const R rfdelp = heatfac / c.delp[k - 1];
                const size_t lev = (size_t)(nlay - k);
                if (out.hlw0) {
                    const R f0 = c.totuclfl[k - 1] - c.totdclfl[k - 1], f1 = c.totuclfl[k] - c.totdclfl[k];
                    out.hlw0[lev * ncol + col] = (double)((f0 - f1) * rfdelp);
                }
                if (out.hlwb)
                    for (int ib = 0; ib < 16; ++ib)
                        out.hlwb[((size_t)ib * nlay + lev) * ncol + col] =
                            (double)((c.fnetb[(size_t)ib * nlp1 + k - 1] - c.fnetb[(size_t)ib * nlp1 + k]) * rfdelp);
            }
        }
        if (out.lwflx) {
            for (int k = 0; k <= nlay; ++k) {
                const size_t lev = (size_t)(nlay - k);
                out.lwflx[(0 * (size_t)nlp1 + lev) * ncol + col] = (double)c.totuflux[k];
                out.lwflx[(1 * (size_t)nlp1 + lev) * ncol + col] = (double)c.totdflux[k];
                out.lwflx[(2 * (size_t)nlp1 + lev) * ncol + col] = (double)c.totuclfl[k];
                out.lwflx[(3 * (size_t)nlp1 + lev) * ncol + col] = (double)c.totdclfl[k];
            }
        }
    }
}

// Day list, windows and chunks of the SW MINVAL(laytrop) groups.  kmin8[d] is the minimum laytrop over
// the day column's group of 8 consecutive day columns of its chunk; kminw[d] over the whole chunk.
static void sw_groups(const std::vector<int>& day, const std::vector<int>& lt, const Config& cfg, int ncol,
                      std::vector<int>& kmin8, std::vector<int>& kminw)
{
    const int nday = (int)day.size();
    kmin8.assign(nday, 0);
    kminw.assign(nday, 0);
    const int wcols = cfg.window_cols > 0 ? cfg.window_cols : ncol;
    int d = 0;
    while (d < nday) {
        const int win = day[d] / wcols;
        int e = d;
        while (e < nday && day[e] / wcols == win) ++e;           // [d, e): this window's day columns
        for (int c0 = d; c0 < e; c0 += cfg.sw_chunk) {
            const int c1 = std::min(e, c0 + cfg.sw_chunk);
            int mw = std::numeric_limits<int>::max();
            for (int i = c0; i < c1; ++i) mw = std::min(mw, lt[i]);
            for (int g0 = c0; g0 < c1; g0 += 8) {
                const int g1 = std::min(c1, g0 + 8);
                int m8 = std::numeric_limits<int>::max();
                for (int i = g0; i < g1; ++i) m8 = std::min(m8, lt[i]);
                for (int i = g0; i < g1; ++i) kmin8[i] = m8;
            }
            for (int i = c0; i < c1; ++i) kminw[i] = mw;
        }
        d = e;
    }
}

template <class R>
static void run_sw(const Config& cfg, const Inputs& in, const Outputs& out)
{
    const int nlay = in.nlay, ncol = in.ncol, nlp1 = nlay + 1;
    const int iswcliq = cfg.diagnostic ? 0 : 1;
    const SwExpTable<R> tb;
    const R heatfac = std::is_same<R, float>::value ? (R)(float)(9.80665 * 1.0e-2 / 1.0046e3)
                                                    : (R)(9.80665 * 1.0e-2 / 1.0046e3);
    for (int i = 0; i < nlay * ncol; ++i) out.htsw[i] = 0;
    for (int i = 0; i < 3 * ncol; ++i) out.topfsw[i] = 0;
    for (int i = 0; i < 4 * ncol; ++i) out.sfcfsw[i] = 0;
    if (out.fdncmp)
        for (int i = 0; i < 6 * ncol; ++i) out.fdncmp[i] = 0;
    if (out.swflx)
        for (size_t i = 0; i < (size_t)4 * nlp1 * ncol; ++i) out.swflx[i] = 0;
    if (out.hsw0)
        for (size_t i = 0; i < (size_t)nlay * ncol; ++i) out.hsw0[i] = 0;
    if (out.htswb)
        for (size_t i = 0; i < (size_t)14 * nlay * ncol; ++i) out.htswb[i] = 0;
    if (cfg.route == 1 && out.sw_mask) {   // the SW generator runs over every column, as the reference's does
#pragma omp parallel for schedule(dynamic, 64)
        for (int col = 0; col < ncol; ++col) {
            std::vector<uint32_t> w;
            sw_mcica_words(cfg, in, col, w);
            for (int ww = 0; ww < 4; ++ww)
                for (int k0 = 0; k0 < nlay; ++k0) out.sw_mask[((size_t)ww * nlay + k0) * ncol + col] = w[(size_t)ww * nlay + k0];
        }
    }
    std::vector<int> day;
    for (int col = 0; col < ncol; ++col)
        if (in.coszen[col] >= 1.0e-4f) day.push_back(col);
    const int nday = (int)day.size();
    std::vector<int> lt(nday);
#pragma omp parallel for schedule(dynamic, 16)
    for (int d = 0; d < nday; ++d) {
        SwColumn<R> c(nlay);
        sw_prep(c, in, day[d], iswcliq, cfg.iovrsw);
        sw_setcoef(c);
        lt[d] = c.laytrop;
    }
    std::vector<int> kmin8, kminw;
    sw_groups(day, lt, cfg, ncol, kmin8, kminw);
#pragma omp parallel for schedule(dynamic, 16)
    for (int d = 0; d < nday; ++d) {
        const int col = day[d];
        SwColumn<R> c(nlay);
        sw_prep(c, in, col, iswcliq, cfg.iovrsw);
        sw_cldprop(c, iswcliq);
        sw_setcoef(c);
        sw_taumol(c, kmin8[d], kminw[d]);
        if (g_sw_tau_scale != 1.0)
            for (auto& v : c.taug) v = v * (R)g_sw_tau_scale;
        if (cfg.route == 1) {
            sw_mcica<R>(c, cfg, in, col, out.sw_mask);
            sw_spcvrtm(c, tb, cfg.iswmode);
        } else {
            sw_spcvrtc(c, tb, cfg.iswmode);
        }
        // swrad_post: band sums of the level fluxes, heating rates, TOA and surface fluxes
        std::vector<R> flxuc(nlp1), flxdc(nlp1), fnet(nlp1);
        for (int k = 0; k < nlp1; ++k) {
            R su = 0, sd = 0;
            for (int ib = 0; ib < 14; ++ib) {
                su = su + c.fxupc[(size_t)ib * nlp1 + k];
                sd = sd + c.fxdnc[(size_t)ib * nlp1 + k];
            }
            flxuc[k] = su; flxdc[k] = sd;
            fnet[k] = flxdc[k] - flxuc[k];
        }
        for (int k = 1; k < nlp1; ++k) {
            const R rf = heatfac / c.delp[k - 1];
            const R h = (fnet[k] - fnet[k - 1]) * rf;
            out.htsw[(size_t)(nlp1 - 1 - k) * ncol + col] = (double)h;
        }
        if (out.hsw0 || out.htswb) {   // swrad_post's lhsw0 / lhswb blocks (phys_rrtm_sw_swrad.cu:393-411)
            std::vector<R> f(nlp1);
            if (out.hsw0) {
                for (int k = 0; k < nlp1; ++k) {
                    R su0 = 0, sd0 = 0;
                    for (int ib = 0; ib < 14; ++ib) {
                        su0 = su0 + c.fxup0[(size_t)ib * nlp1 + k];
                        sd0 = sd0 + c.fxdn0[(size_t)ib * nlp1 + k];
                    }
                    f[k] = sd0 - su0;
                }
                for (int k = 1; k < nlp1; ++k)
                    out.hsw0[(size_t)(nlp1 - 1 - k) * ncol + col] = (double)((f[k] - f[k - 1]) * (heatfac / c.delp[k - 1]));
            }
            if (out.htswb)
                for (int mb = 0; mb < 14; ++mb) {
                    for (int k = 0; k < nlp1; ++k) f[k] = c.fxdnc[(size_t)mb * nlp1 + k] - c.fxupc[(size_t)mb * nlp1 + k];
                    for (int k = 1; k < nlp1; ++k)
                        out.htswb[((size_t)mb * nlay + (nlp1 - 1 - k)) * ncol + col] =
                            (double)((f[k] - f[k - 1]) * (heatfac / c.delp[k - 1]));
                }
        }
        out.topfsw[0 * (size_t)ncol + col] = (double)c.ftoauc;
        out.topfsw[1 * (size_t)ncol + col] = (double)c.ftoadc;
        out.topfsw[2 * (size_t)ncol + col] = (double)c.ftoau0;
        out.sfcfsw[0 * (size_t)ncol + col] = (double)c.fsfcuc;
        out.sfcfsw[1 * (size_t)ncol + col] = (double)c.fsfcdc;
        out.sfcfsw[2 * (size_t)ncol + col] = (double)c.fsfcu0;
        out.sfcfsw[3 * (size_t)ncol + col] = (double)c.fsfcd0;
        if (out.fdncmp) {
            out.fdncmp[0 * (size_t)ncol + col] = (double)c.suvbf0;
            out.fdncmp[1 * (size_t)ncol + col] = (double)c.suvbfc;
            out.fdncmp[2 * (size_t)ncol + col] = (double)c.sfbmc[0];
            out.fdncmp[3 * (size_t)ncol + col] = (double)c.sfdfc[0];
            out.fdncmp[4 * (size_t)ncol + col] = (double)c.sfbmc[1];
            out.fdncmp[5 * (size_t)ncol + col] = (double)c.sfdfc[1];
        }
        if (out.swflx) {
            for (int k = 0; k < nlp1; ++k) {
                R su0 = 0, sd0 = 0;
                for (int ib = 0; ib < 14; ++ib) {
                    su0 = su0 + c.fxup0[(size_t)ib * nlp1 + k];
                    sd0 = sd0 + c.fxdn0[(size_t)ib * nlp1 + k];
                }
                const size_t lev = (size_t)(nlp1 - 1 - k);
                out.swflx[(0 * (size_t)nlp1 + lev) * ncol + col] = (double)flxuc[k];
                out.swflx[(1 * (size_t)nlp1 + lev) * ncol + col] = (double)flxdc[k];
                out.swflx[(2 * (size_t)nlp1 + lev) * ncol + col] = (double)su0;
                out.swflx[(3 * (size_t)nlp1 + lev) * ncol + col] = (double)sd0;
            }
        }
    }
}
}  // namespace orc

extern "C" {

int orc_set_debug(double sw_tau_scale)
{
    orc::g_sw_tau_scale = sw_tau_scale;
    return 0;
}

// SW stage outputs (float statements) of the request's day columns; same layout as the reference
// driver's orc_sw_stages (oracle/ref_driver.cpp): one window, one chunk.
int orc_sw_stages(const int* cfg_i, int nlay, int ncol, const float* plyr, const float* plvl, const float* tlyr,
                  const float* tlvl, const float* qlyr, const float* olyr, const float* gasvmr, const float* clouds,
                  const float* sfcalb, const float* coszen, double solcon, float* taug, float* taur, float* sfluxzen,
                  float* taucw, float* ssacw, float* asycw, float* cldfrc, float* zcf, int* laytrop)
{
    try {
        using namespace orc;
        Config cfg;
        cfg.iswmode = cfg_i[0];
        cfg.diagnostic = cfg_i[1];
        cfg.iovrsw = cfg_i[2];
        cfg.sw_chunk = 1 << 30;
        Inputs in{plyr, plvl, tlyr, tlvl, qlyr, olyr, gasvmr, clouds, nullptr, nullptr, nullptr, nullptr,
                  sfcalb, coszen, nullptr, solcon, nlay, ncol};
        const int iswcliq = cfg.diagnostic ? 0 : 1;
        std::vector<int> day;
        for (int col = 0; col < ncol; ++col)
            if (coszen[col] >= 1.0e-4f) day.push_back(col);
        const int nday = (int)day.size();
        std::vector<int> lt(nday);
        for (int d = 0; d < nday; ++d) {
            SwColumn<float> c(nlay);
            sw_prep(c, in, day[d], iswcliq, cfg.iovrsw);
            sw_setcoef(c);
            lt[d] = c.laytrop;
        }
        std::vector<int> kmin8, kminw;
        sw_groups(day, lt, cfg, ncol, kmin8, kminw);
        for (int d = 0; d < nday; ++d) {
            SwColumn<float> c(nlay);
            sw_prep(c, in, day[d], iswcliq, cfg.iovrsw);
            sw_cldprop(c, iswcliq);
            sw_setcoef(c);
            sw_taumol(c, kmin8[d], kminw[d]);
            for (int k = 0; k < nlay; ++k)
                for (int g = 0; g < 112; ++g) {
                    taug[((size_t)d * nlay + k) * 112 + g] = c.TG(g, k);
                    taur[((size_t)d * nlay + k) * 112 + g] = c.TR(g, k);
                }
            for (int g = 0; g < 112; ++g) sfluxzen[(size_t)d * 112 + g] = c.sfluxzen[g];
            for (int ib = 0; ib < 14; ++ib)
                for (int k = 0; k < nlay; ++k) {
                    const size_t o = ((size_t)d * 14 + ib) * nlay + k;
                    taucw[o] = c.taucw[(size_t)ib * nlay + k];
                    ssacw[o] = c.ssacw[(size_t)ib * nlay + k];
                    asycw[o] = c.asycw[(size_t)ib * nlay + k];
                }
            for (int k = 0; k < nlay; ++k) cldfrc[(size_t)d * nlay + k] = c.cldfrc[k];
            zcf[2 * d] = c.zcf0;
            zcf[2 * d + 1] = c.zcf1;
            laytrop[d] = c.laytrop;
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return -1;
    }
    return 0;
}

// McICA sub-column masks of a request (the restatement of the generators; same layout and seeds as the
// reference driver's orc_mcica_masks).
int orc_mcica_masks(const int* cfg_i, int nlay, int ncol, const float* clouds, const int* icseed,
                    unsigned int* lw_out, unsigned int* sw_out)
{
    using namespace orc;
    Config cfg;
    cfg.iovrlw = cfg_i[5];
    cfg.iovrsw = cfg_i[6];
    cfg.lw_seed0 = cfg_i[7];
    cfg.sw_seed0 = cfg_i[8];
    Inputs in{};
    in.clouds = clouds;
    in.icseed = icseed;
    in.nlay = nlay;
    in.ncol = ncol;
#pragma omp parallel for schedule(dynamic, 64)
    for (int c = 0; c < ncol; ++c) {
        std::vector<uint32_t> w;
        if (lw_out) {
            std::vector<float> cf(nlay, 0.0f);
            bool any = false;
            for (int k0 = 0; k0 < nlay; ++k0) any = any || clouds[(size_t)(nlay - 1 - k0) * ncol + c] > 1.0e-6f;
            if (any)
                for (int k0 = 0; k0 < nlay; ++k0) cf[k0] = clouds[(size_t)(nlay - 1 - k0) * ncol + c];
            mcica_bits(cf, nlay, 140, cfg.iovrlw, icseed ? icseed[c] : cfg.lw_seed0 + c + 1, w);
            for (int ww = 0; ww < 5; ++ww)
                for (int k0 = 0; k0 < nlay; ++k0) lw_out[((size_t)ww * nlay + k0) * ncol + c] = w[(size_t)ww * nlay + k0];
        }
        if (sw_out) {
            sw_mcica_words(cfg, in, c, w);
            for (int ww = 0; ww < 4; ++ww)
                for (int k0 = 0; k0 < nlay; ++k0) sw_out[((size_t)ww * nlay + k0) * ncol + c] = w[(size_t)ww * nlay + k0];
        }
    }
    return 0;
}

int orc_clear_tables(void)
{
    orc::tables().t.clear();
    orc::tables().ti.clear();
    return 0;
}

int orc_add_table(const char* name, const double* data, long n)
{
    orc::tables().t[name] = std::vector<double>(data, data + n);
    return 0;
}

int orc_add_itable(const char* name, const int* data, long n)
{
    orc::tables().ti[name] = std::vector<int>(data, data + n);
    return 0;
}

// Solve a request.  precision: 0 float, 1 double.  cfg_i: iswmode, diagnostic, window_cols, sw_chunk,
// route, iovrlw, iovrsw, lw_seed0, sw_seed0.  Outputs are double arrays (see rrtm_common.hpp Outputs);
// fdncmp, lwflx, swflx and the masks may be null.
int orc_solve(int precision, const int* cfg_i, double cpathfac, int nlay, int ncol, const float* plyr,
              const float* plvl, const float* tlyr, const float* tlvl, const float* qlyr, const float* olyr,
              const float* gasvmr, const float* clouds, const float* faerlw, const float* faersw,
              const float* sfcemis, const float* tsfg, const float* sfcalb, const float* coszen,
              const int* icseed, double solcon, double* htlw, double* htsw, double* topflw, double* sfcflw,
              double* topfsw, double* sfcfsw, double* fdncmp, double* lwflx, double* swflx,
              unsigned int* lw_mask, unsigned int* sw_mask, int nthreads)
{
    try {
#ifdef _OPENMP
        if (nthreads > 0) omp_set_num_threads(nthreads);
#else
        (void)nthreads;
#endif
        orc::Config cfg;
        cfg.iswmode = cfg_i[0];
        cfg.diagnostic = cfg_i[1];
        cfg.window_cols = cfg_i[2];
        cfg.sw_chunk = cfg_i[3] > 0 ? cfg_i[3] : 32768;
        cfg.route = cfg_i[4];
        cfg.iovrlw = cfg_i[5];
        cfg.iovrsw = cfg_i[6];
        cfg.lw_seed0 = cfg_i[7];
        cfg.sw_seed0 = cfg_i[8];
        cfg.cpathfac = cpathfac;
        orc::Inputs in{plyr, plvl, tlyr, tlvl, qlyr, olyr, gasvmr, clouds, faerlw, faersw, sfcemis, tsfg,
                       sfcalb, coszen, icseed, solcon, nlay, ncol};
        orc::Outputs out{htlw, htsw, topflw, sfcflw, topfsw, sfcfsw, fdncmp, lwflx, swflx, lw_mask, sw_mask};
        if (precision == 0) {
            orc::run_lw<float>(cfg, in, out);
            orc::run_sw<float>(cfg, in, out);
        } else {
            orc::run_lw<double>(cfg, in, out);
            orc::run_sw<double>(cfg, in, out);
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return -1;
    }
    return 0;
}

// orc_solve with the optional outputs of lwrad / swrad (each may be null): hlw0 [nlay][ncol], hlwb
// [16][nlay][ncol], hsw0 [nlay][ncol], htswb [14][nlay][ncol], K/s, levels top first.
int orc_solve_diag(int precision, const int* cfg_i, double cpathfac, int nlay, int ncol, const float* plyr,
                   const float* plvl, const float* tlyr, const float* tlvl, const float* qlyr, const float* olyr,
                   const float* gasvmr, const float* clouds, const float* faerlw, const float* faersw,
                   const float* sfcemis, const float* tsfg, const float* sfcalb, const float* coszen,
                   const int* icseed, double solcon, double* htlw, double* htsw, double* topflw, double* sfcflw,
                   double* topfsw, double* sfcfsw, double* fdncmp, double* lwflx, double* swflx,
                   unsigned int* lw_mask, unsigned int* sw_mask, double* hlw0, double* hlwb, double* hsw0,
                   double* htswb, int nthreads)
{
    try {
#ifdef _OPENMP
        if (nthreads > 0) omp_set_num_threads(nthreads);
#else
        (void)nthreads;
#endif
        orc::Config cfg;
        cfg.iswmode = cfg_i[0];
        cfg.diagnostic = cfg_i[1];
        cfg.window_cols = cfg_i[2];
        cfg.sw_chunk = cfg_i[3] > 0 ? cfg_i[3] : 32768;
        cfg.route = cfg_i[4];
        cfg.iovrlw = cfg_i[5];
        cfg.iovrsw = cfg_i[6];
        cfg.lw_seed0 = cfg_i[7];
        cfg.sw_seed0 = cfg_i[8];
        cfg.cpathfac = cpathfac;
        orc::Inputs in{plyr, plvl, tlyr, tlvl, qlyr, olyr, gasvmr, clouds, faerlw, faersw, sfcemis, tsfg,
                       sfcalb, coszen, icseed, solcon, nlay, ncol};
        orc::Outputs out{htlw, htsw, topflw, sfcflw, topfsw, sfcfsw, fdncmp, lwflx, swflx, lw_mask, sw_mask,
                         hlw0, hlwb, hsw0, htswb};
        if (precision == 0) {
            orc::run_lw<float>(cfg, in, out);
            orc::run_sw<float>(cfg, in, out);
        } else {
            orc::run_lw<double>(cfg, in, out);
            orc::run_sw<double>(cfg, in, out);
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "oracle: %s\n", e.what());
        return -1;
    }
    return 0;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------------
// Climatological aerosol optics of a request (rrtm_aer.hpp).  Same signature as the reference driver's
// (oracle/ref_driver.cpp, the reference's kernels): the climatology as packed (rhid [4][6][61], rhdp
// [4][4][8][61], one month's records), columns top first ([level][ncol]; xlon / xlat in radians), outputs
// aerosw [3][14][nlay][ncol], aerolw [3][16][nlay][ncol] and, when tab is not null, the derived tables
// (AER_TAB_FIELDS in oracle/oracle.py).
extern "C" int orc_aerosols(const int* iendwv, const float* haer, const float* prsref, const float* rhid,
                            const float* rhdp, const float* straext0, const int* nwvns0, const float* s0intv,
                            const int* midx, const double* mcmix, const int* mkprf, const double* mdenn, int nlay,
                            int ncol, const float* plvl, const float* plyr, const float* tlyr, const float* qlyr,
                            const float* rhly, const float* xlon, const float* xlat, const float* slmsk,
                            float* aerosw, float* aerolw, float* tab)
{
    using namespace orc::aer;
    const Clim c{iendwv, haer, prsref, rhid, rhdp, straext0, nwvns0, s0intv, midx, mcmix, mkprf, mdenn};
    Tables t;
    build(c, t);
    if (tab) {
        float* o = tab;
        auto put = [&](const float* a, size_t n) { std::copy(a, a + n, o); o += n; };
        put(t.sigref, NAE * NDM);
        put(t.extrhi, NBT * NCM1); put(t.scarhi, NBT * NCM1); put(t.ssarhi, NBT * NCM1); put(t.asyrhi, NBT * NCM1);
        const size_t nd = (size_t)NBT * NCM2 * NRHLEV;
        put(t.extrhd, nd); put(t.scarhd, nd); put(t.ssarhd, nd); put(t.asyrhd, nd);
        put(t.extstra, NBT); put(t.solbnd, NSW); put(t.eirbnd, NLW);
        put(t.cmixg.data(), t.cmixg.size()); put(t.denng.data(), t.denng.size());
        for (int v : t.idxcg) *o++ = (float)v;
        for (int v : t.kprfg) *o++ = (float)v;
    }
    if (ncol <= 0) return 0;
#pragma omp parallel for schedule(dynamic, 64)
    for (int col = 0; col < ncol; ++col) {
        std::vector<float> pi(nlay + 1), pl(nlay), tl(nlay), ql(nlay), rh(nlay);
        for (int k = 0; k <= nlay; ++k) pi[k] = plvl[(size_t)k * ncol + col];
        for (int k = 0; k < nlay; ++k) {
            pl[k] = plyr[(size_t)k * ncol + col]; tl[k] = tlyr[(size_t)k * ncol + col];
            ql[k] = qlyr[(size_t)k * ncol + col]; rh[k] = rhly[(size_t)k * ncol + col];
        }
        column(t, c, nlay, pi.data(), pl.data(), tl.data(), ql.data(), rh.data(), xlon[col], xlat[col], slmsk[col],
               aerosw + col, aerolw + col, (size_t)ncol);
    }
    return 0;
}

// The volcanic stratospheric aerosol term (rrtm_aer.hpp volcanic), added in place to aerosw [3][14][nlay][ncol]
// and aerolw [3][16][nlay][ncol]: plvl [nlay + 1][ncol] mb in the order of ivflip, xlat [ncol] radians, ivolae
// [10][4][12] (year, zone, month); year mod(kyrsav, 10) + 1 as Python's modulo gives it, month kmonsav.
extern "C" int orc_setaer_volc(int nlay, int ncol, int ivflip, const float* plvl, const float* xlat,
                               const int* ivolae, int kyrsav, int kmonsav, int add_sw, int add_lw, int lw1bd,
                               float* aerosw, float* aerolw)
{
    if (nlay < 4 || ncol < 0 || kmonsav < 1 || kmonsav > 12) return 1;
    const int y = ((kyrsav % 10) + 10) % 10;
    int32_t iv[4];
    for (int z = 0; z < 4; ++z) iv[z] = ivolae[(y * 4 + z) * 12 + (kmonsav - 1)];
#pragma omp parallel for schedule(static)
    for (int col = 0; col < ncol; ++col) {
        std::vector<float> pi(nlay + 1);
        for (int k = 0; k <= nlay; ++k) pi[k] = plvl[(size_t)k * ncol + col];
        orc::aer::volcanic(nlay, ivflip, pi.data(), xlat[col], iv, add_sw != 0, add_lw != 0, lw1bd != 0,
                           aerosw + col, aerolw + col, (size_t)ncol);
    }
    return 0;
}

// Solar geometry (rrtm_solar.hpp).  Same signature as the reference driver's: date[6] = year, month, day,
// hour, minute, second; state[5] = sollag, sindec, cosdec, anginc, solcon; then coszen / coszdg of n columns.
extern "C" int orc_solar(const int* date, float deltsw, float deltim, double solc0, float* state, int* nstp, int n,
                         const float* glon, const float* glat, float solhr, float dtswav, int nrads, float* coszen,
                         float* coszdg)
{
    orc::solar::update(date[0], date[1], date[2], date[3], date[4], date[5], deltsw, deltim, solc0, state, nstp);
    for (int i = 0; i < n; ++i)
        orc::solar::coszmn(glon[i], glat[i], state[0], state[1], state[2], solhr, dtswav, nrads, coszen[i], coszdg[i]);
    return 0;
}

// grrad's radiation-layer set-up (rrtm_grrad.hpp) of n columns, [level][n] top first.  out = plvl [lm + 2],
// plyr, tlyr [lm + 1], tlvl [lm + 2], qlyr, rhly, qstl, prslk1, tvly [lm + 1] (each [..][n]) and tsfg [n],
// concatenated in that order.  Same signature as the reference driver's.
extern "C" int orc_grrad_setup(int lm, int n, const float* pint, const float* pmid, const float* prslk,
                               const float* t, const float* q, const float* tsfc, float* out)
{
    const int lmk = lm + 1, lmp = lm + 2;
    const size_t L = (size_t)lmk * n, P = (size_t)lmp * n;
    float *plvl = out, *plyr = plvl + P, *tlyr = plyr + L, *tlvl = tlyr + L, *qlyr = tlvl + P, *rhly = qlyr + L,
          *qstl = rhly + L, *prslk1 = qstl + L, *tvly = prslk1 + L, *tsfg = tvly + L;
#pragma omp parallel for schedule(static)
    for (int c = 0; c < n; ++c) {
        std::vector<float> pi(lm + 1), pm(lm), pk(lm), tt(lm), qq(lm);
        for (int k = 0; k <= lm; ++k) pi[k] = pint[(size_t)k * n + c];
        for (int k = 0; k < lm; ++k) {
            pm[k] = pmid[(size_t)k * n + c]; pk[k] = prslk[(size_t)k * n + c];
            tt[k] = t[(size_t)k * n + c]; qq[k] = q[(size_t)k * n + c];
        }
        std::vector<float> a(lmp), b(lmk), tl(lmk), tv(lmp), ql(lmk), rh(lmk), qs(lmk), p1(lmk), vy(lmk);
        float ts;
        orc::grrad::column(lm, pi.data(), pm.data(), pk.data(), tt.data(), qq.data(), tsfc[c], a.data(), b.data(),
                           tl.data(), tv.data(), ql.data(), rh.data(), qs.data(), p1.data(), vy.data(), ts);
        for (int k = 0; k < lmp; ++k) { plvl[(size_t)k * n + c] = a[k]; tlvl[(size_t)k * n + c] = tv[k]; }
        for (int k = 0; k < lmk; ++k) {
            plyr[(size_t)k * n + c] = b[k]; tlyr[(size_t)k * n + c] = tl[k]; qlyr[(size_t)k * n + c] = ql[k];
            rhly[(size_t)k * n + c] = rh[k]; qstl[(size_t)k * n + c] = qs[k]; prslk1[(size_t)k * n + c] = p1[k];
            tvly[(size_t)k * n + c] = vy[k];
        }
        tsfg[c] = ts;
    }
    return 0;
}


// ---- grrad's front end (rrtm_front.hpp).  Same signatures as the reference driver's. ----

// DAYPARTS of jm rows of im points; sol = sollag, sindec, cosdec.
extern "C" int orc_dayparts(int im, int jm, const float* xlon, const float* sinlat, const float* coslat, float solhr,
                            float dtswav, int nrads, const float* sol, float* coszen, float* coszdg, int* dp_start,
                            int* dp_len, int* dp_day, int* ndayparts)
{
    orc::front::dayparts(im, jm, xlon, sinlat, coslat, solhr, dtswav, nrads, sol[0], sol[1], sol[2], coszen, coszdg,
                         dp_start, dp_len, dp_day, ndayparts);
    return 0;
}

extern "C" int orc_getgases(int n, int lmax, const float* plvl, const float* xlon, const float* xlat, float co2_glb,
                            const float* gco2cyc, const float* co2vmr_sav, int ico2flg, int kmonsav, int ivflip,
                            float* gasvmr)
{
    orc::front::getgases(n, lmax, plvl, xlon, xlat, co2_glb, gco2cyc, co2vmr_sav, ico2flg, kmonsav, ivflip, gasvmr);
    return 0;
}

extern "C" int orc_getozn(int n, int nlev, const float* prslk, const float* xlat, const float* o3r, const float* pkstr,
                          int jmr, int loz, int k1oz, int k2oz, float facoz, float blte, float dlte, int ivflip,
                          float* o3mmr)
{
    orc::front::getozn(n, nlev, prslk, xlat, o3r, pkstr, jmr, loz, k1oz, k2oz, facoz, blte, dlte, ivflip, o3mmr);
    return 0;
}

// f = slmsk, snowf, sncovr, snoalb, zorlf, coszf, tsknf, hprif, alvsf, alnsf, alvwf, alnwf, facsf, facwf, fice,
// tisfc.
extern "C" int orc_setalb(int n, const float* const* f, int ialbflg, float* sfcalb)
{
    const orc::front::AlbIn a{f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9], f[10], f[11], f[12], f[13],
                              f[14], f[15]};
    orc::front::setalb(n, a, ialbflg, sfcalb);
    return 0;
}

// grrad's condensate: tracer [ntrac][lmk][n] -> clw [lmk][n] (rrtm_front.hpp grrad_clw).
extern "C" int orc_grrad_clw(int n, int lmk, const float* tracer, int ntcw0, int ncld, float epsq, float* clw)
{
    orc::front::grrad_clw(n, lmk, tracer, ntcw0, ncld, epsq, clw);
    return 0;
}

// grrad's IALB = 2 block: out [9][n] = sfcalbedo, smx, czmean, alvsf, alnsf, alvwf, alnwf, facsf, facwf.
extern "C" int orc_payne_albedo(int n, const float* salbedo, const float* sm, const float* coszen, const float* trn,
                                const float* za, const float* dza, const float* albd, float* out)
{
    const orc::front::PayneTab t{trn, za, dza, albd};
    for (int p = 0; p < n; ++p) {
        const float a = orc::front::payne_albedo(salbedo[p], sm[p], coszen[p], t);
        const float v[9] = {a, sm[p], coszen[p], a, a, a, a, 0.0f, 0.0f};
        for (int f = 0; f < 9; ++f) out[(size_t)f * n + p] = v[f];
    }
    return 0;
}

// f = glon, glat, sm, sice, si, sncovr, z0, stdh, tskin.
extern "C" int orc_setemis(int n, const float* const* f, const int* idxems, int ialbflg, int iemslw, float* sfcemis)
{
    const orc::front::EmisIn e{f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], idxems};
    orc::front::setemis(n, e, ialbflg, iemslw, sfcemis);
    return 0;
}

// f = plyr, plvl, tlyr, tvly, qlyr, qstl, rhly, clw, f_ice, f_rain, r_rime, cldfk1, xlat; cfg = ivflip, llyr,
// iovr, lcrick, lcnorm, lnoprec, lsashal, cld_fraction.
extern "C" int orc_progcld2(int n, int nlay, const float* const* f, const int* cfg, float* clouds, float* clds,
                            int* mtop, int* mbot)
{
    const orc::front::CldIn in{f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9], f[11], f[12]};
    const orc::front::CldCfg c{cfg[0], cfg[1], cfg[2], cfg[3], cfg[4], cfg[5], cfg[6], cfg[7]};
    orc::front::progcld2(n, nlay, in, c, clouds, clds, mtop, mbot);
    return 0;
}
