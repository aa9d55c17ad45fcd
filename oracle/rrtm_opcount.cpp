// rrtm_opcount.cpp -- operation-count table of the RRTM column path (measurement infrastructure only).
//
// Runs the oracle's restatement of the reference statements (rrtm_lw.hpp, rrtm_sw.hpp) with the counting
// type orc::CR (opcount.hpp) over a sample of columns and reports the operations per stage:
//   LW (every column):  lw_prep, lw_cldprop, lw_setcoef, lw_taumol, lw_rtrnmr (incl. heating rates)
//   SW (day columns):   sw_prep, sw_cldprop, sw_setcoef, sw_taumol, sw_spcvrtc, swrad_post
// The MINVAL(laytrop) group minima of SW bands 19/23/25/28 are taken as the column's own laytrop (they
// only move which of two equal-cost branches a layer takes).
#include "rrtm_common.hpp"
#include "opcount.hpp"
#include "rrtm_lw.hpp"
#include "rrtm_sw.hpp"

namespace orc {
OpCounts g_ops;
TableStore& tables()
{
    static TableStore s;
    return s;
}
}  // namespace orc

namespace {
using orc::CR;
void take(double* row)
{
    row[0] += (double)orc::g_ops.add;
    row[1] += (double)orc::g_ops.mul;
    row[2] += (double)orc::g_ops.div;
    row[3] += (double)orc::g_ops.func;
    row[4] += (double)orc::g_ops.other;
    orc::g_ops = orc::OpCounts();
}
}  // namespace

extern "C" {

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

// counts: [11][5] rows (5 LW stages, 6 SW stages) of (add, mul, div, func, other), summed over the
// sample; nday_out: number of day columns in the sample.
int orc_opcount(int diagnostic, int iswmode, double cpathfac, int nlay, int ncol, const float* plyr,
                const float* plvl, const float* tlyr, const float* tlvl, const float* qlyr, const float* olyr,
                const float* gasvmr, const float* clouds, const float* sfcemis, const float* tsfg,
                const float* sfcalb, const float* coszen, double solcon, double* counts, int* nday_out)
{
    using namespace orc;
    try {
        Inputs in{plyr, plvl, tlyr, tlvl, qlyr, olyr, gasvmr, clouds, nullptr, nullptr, sfcemis, tsfg,
                  sfcalb, coszen, nullptr, solcon, nlay, ncol};
        for (int i = 0; i < 55; ++i) counts[i] = 0;
        const LwTables<CR> ltb;
        const SwExpTable<CR> stb;
        const CR heatfac = (CR)CON_G * (CR)1.0e-2f / (CR)CON_CP;
        const CR fluxfac = (CR)(2.0 * std::asin(1.0) * 2.0e4);
        const int icliq = diagnostic ? 0 : 1;
        int nday = 0;
        g_ops = OpCounts();
        for (int col = 0; col < ncol; ++col) {
            std::vector<float> cl(9 * (size_t)nlay);
            for (int n = 0; n < 9; ++n)
                for (int k = 0; k < nlay; ++k) cl[n * nlay + k] = clouds[((size_t)n * nlay + k) * ncol + col];
            if (icliq)
                for (int k = 0; k < nlay; ++k) {
                    cl[1 * nlay + k] *= (float)cpathfac;
                    cl[3 * nlay + k] *= (float)cpathfac;
                }
            {
                LwColumn<CR> c(nlay);
                g_ops = OpCounts();
                lw_prep(c, in, col, cl.data(), icliq);
                take(counts + 0);
                lw_cldprop(c, cl.data(), icliq);
                take(counts + 5);
                lw_setcoef(c);
                take(counts + 10);
                lw_taumol(c);
                take(counts + 15);
                lw_rtrnmr(c, ltb, heatfac, fluxfac);
                take(counts + 20);
            }
            if (!(coszen[col] >= 1.0e-4f)) continue;
            ++nday;
            SwColumn<CR> c(nlay);
            const int nlp1 = nlay + 1;
            g_ops = OpCounts();
            sw_prep(c, in, col, icliq);
            take(counts + 25);
            sw_cldprop(c, icliq);
            take(counts + 30);
            sw_setcoef(c);
            take(counts + 35);
            sw_taumol(c, c.laytrop, c.laytrop);
            take(counts + 40);
            sw_spcvrtc(c, stb, iswmode);
            take(counts + 45);
            std::vector<CR> fnet(nlp1);
            for (int k = 0; k < nlp1; ++k) {
                CR su = 0, sd = 0;
                for (int ib = 0; ib < 14; ++ib) {
                    su = su + c.fxupc[(size_t)ib * nlp1 + k];
                    sd = sd + c.fxdnc[(size_t)ib * nlp1 + k];
                }
                fnet[k] = sd - su;
            }
            const CR hf = (CR)(9.80665 * 1.0e-2 / 1.0046e3);
            for (int k = 1; k < nlp1; ++k) {
                const CR h = (fnet[k] - fnet[k - 1]) * (hf / c.delp[k - 1]);
                (void)h;
            }
            take(counts + 50);
        }
        *nday_out = nday;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "opcount: %s\n", e.what());
        return -1;
    }
    return 0;
}

}  // extern "C"
