// ref_driver.cpp -- runs the reference's own RRTM kernels on the host (builds oracle/_ref/libref_rrtm.so).
//
// Each reference kernel source is compiled unmodified, inside its own namespace, from the reference tree
// (build_ref.sh passes -I <reference>/namgpu/kernels); nothing of it is copied here.  This file is the
// driver: it allocates the arrays in the layouts the reference's Python wrappers hand to each kernel and
// calls the kernels in the reference's order -- lwrad (physics/rrtm/phys_rrtm_lw_lwrad.py:247-290) with
// lw_core.seam (physics/rrtm/lw_core.py:217-286, bands via _bands :103-209), swrad
// (physics/rrtm/phys_rrtm_sw_swrad.py:282-386) with sw_seam (physics/rrtm/sw_seam.py) -- for one request
// seen as a single row of ncol columns (JM = 1, IM = ncol).  It exports the oracle's C entry points, so
// the tests drive it exactly like the restatement.  Test infrastructure only.
#include "ref_shim.h"

#include <cstdio>
#include <limits>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

thread_local ref_dim3 threadIdx, blockIdx, blockDim, gridDim;

// The reference's shared headers (include-once) go in the global namespace, ahead of the kernels.
#include "nmmb_common.cuh"
#include "rrtm_sw_bands.cuh"

namespace r_lwrad {
#include "phys_rrtm_lw_lwrad.cu"
}
namespace r_lwcld {
#include "phys_rrtm_lw_cldprop.cu"
}
namespace r_lwset {
#include "phys_rrtm_lw_setcoef.cu"
}
namespace r_b01 {
#include "phys_rrtm_lw_taugb01.cu"
}
namespace r_b02 {
#include "phys_rrtm_lw_taugb02.cu"
}
namespace r_b03 {
#include "phys_rrtm_lw_taugb03.cu"
}
namespace r_b04 {
#include "phys_rrtm_lw_taugb04.cu"
}
namespace r_b05 {
#include "phys_rrtm_lw_taugb05.cu"
}
namespace r_b06 {
#include "phys_rrtm_lw_taugb06.cu"
}
namespace r_b07 {
#include "phys_rrtm_lw_taugb07.cu"
}
namespace r_b08 {
#include "phys_rrtm_lw_taugb08.cu"
}
namespace r_b09 {
#include "phys_rrtm_lw_taugb09.cu"
}
namespace r_b10 {
#include "phys_rrtm_lw_taugb10.cu"
}
namespace r_b11 {
#include "phys_rrtm_lw_taugb11.cu"
}
namespace r_b12 {
#include "phys_rrtm_lw_taugb12.cu"
}
namespace r_b13 {
#include "phys_rrtm_lw_taugb13.cu"
}
namespace r_b14 {
#include "phys_rrtm_lw_taugb14.cu"
}
namespace r_b15 {
#include "phys_rrtm_lw_taugb15.cu"
}
namespace r_b16 {
#include "phys_rrtm_lw_taugb16.cu"
}
namespace r_rtrnmr {
#include "phys_rrtm_lw_rtrnmr.cu"
}
namespace r_rtrn {
#include "phys_rrtm_lw_rtrn.cu"
}
namespace r_lwmc {
#include "phys_rrtm_lw_mcica_subcol.cu"
}
#undef MCICA_NGPTLW
#undef MCICA_NWORD
namespace r_swmc {
#include "phys_rrtm_sw_mcica_subcol.cu"
}
namespace r_post {
#include "phys_rrtm_driver_post.cu"
}
namespace r_rdt {
#include "drv_rdtemp.cu"
}
namespace r_swrad {
#include "phys_rrtm_sw_swrad.cu"
}
namespace r_aeri {
#include "phys_rrtm_aer_init.cu"
}
namespace r_aerc {
#include "phys_rrtm_clim_aerinit.cu"
}
namespace r_aeru {
#include "phys_rrtm_aer_update.cu"
}
namespace r_seta {
#include "phys_rrtm_setaer.cu"
}
namespace r_aerp {
#include "phys_rrtm_aer_property.cu"
}
namespace r_solu {
#include "phys_rrtm_sol_update.cu"
}
namespace r_cosz {
#include "phys_rrtm_coszmn.cu"
}
namespace r_grs {
#include "phys_rrtm_grrad_setup.cu"
}
namespace r_grg {
#include "phys_rrtm_grrad_gases.cu"
}
namespace r_grcl {
#include "phys_rrtm_grrad_clouds.cu"
}
namespace r_swcld {
#include "phys_rrtm_sw_cldprop.cu"
}
namespace r_swset {
#include "phys_rrtm_sw_setcoef.cu"
}
namespace r_swtau {
#include "phys_rrtm_sw_taumol.cu"
}
namespace r_s16 {
#include "phys_rrtm_sw_taumol16.cu"
}
namespace r_s17 {
#include "phys_rrtm_sw_taumol17.cu"
}
namespace r_s18 {
#include "phys_rrtm_sw_taumol18.cu"
}
namespace r_s19 {
#include "phys_rrtm_sw_taumol19.cu"
}
namespace r_s20 {
#include "phys_rrtm_sw_taumol20.cu"
}
namespace r_s21 {
#include "phys_rrtm_sw_taumol21.cu"
}
namespace r_s22 {
#include "phys_rrtm_sw_taumol22.cu"
}
namespace r_s23 {
#include "phys_rrtm_sw_taumol23.cu"
}
namespace r_s24 {
#include "phys_rrtm_sw_taumol24.cu"
}
namespace r_s25 {
#include "phys_rrtm_sw_taumol25.cu"
}
namespace r_s26 {
#include "phys_rrtm_sw_taumol26.cu"
}
namespace r_s27 {
#include "phys_rrtm_sw_taumol27.cu"
}
namespace r_s28 {
#include "phys_rrtm_sw_taumol28.cu"
}
namespace r_s29 {
#include "phys_rrtm_sw_taumol29.cu"
}
namespace r_spcv {
#include "phys_rrtm_sw_spcvrtc.cu"
}

// ------------------------------------------------------------------------------------------------------
namespace r_dayp {
#include "phys_rrtm_dayparts.cu"
}
namespace r_ggas {
#include "phys_rrtm_getgases.cu"
}
namespace r_gozn {
#include "phys_rrtm_getozn.cu"
}
namespace r_salb {
#include "phys_rrtm_setalb.cu"
}
namespace r_sems {
#include "phys_rrtm_setemis.cu"
}
namespace r_pc2 {
#include "phys_rrtm_progcld2.cu"
}

namespace drv {

using FV = std::vector<float>;

// Test hooks (see orc_set_debug / orc_sw_stages): a factor applied to the SW gas optical depths before
// spcvrtc, and a capture of the SW stage outputs of the first chunk.
double g_sw_tau_scale = 1.0;
struct SwCapture {
    float *taug = nullptr, *taur = nullptr, *sfluxzen = nullptr, *taucw = nullptr, *ssacw = nullptr,
          *asycw = nullptr, *cldfrc = nullptr, *zcf = nullptr;
    int* laytrop = nullptr;
    bool stop_after_taumol = false;
} g_cap;
using IV = std::vector<int>;

std::map<std::string, std::vector<double>>& ftab()
{
    static std::map<std::string, std::vector<double>> t;
    return t;
}
std::map<std::string, std::vector<int>>& itab()
{
    static std::map<std::string, std::vector<int>> t;
    return t;
}

// A packed table ([..., g] order) as float32, optionally transposed to g-first ([g][rest]) for the kernels
// whose wrappers pass that layout.
FV T(const std::string& n)
{
    auto it = ftab().find(n);
    if (it == ftab().end()) throw std::runtime_error("ref driver: missing table " + n);
    return FV(it->second.begin(), it->second.end());
}
FV Tg(const std::string& n, int ng)
{
    FV a = T(n);
    const size_t rest = a.size() / ng;
    FV b(a.size());
    for (size_t r = 0; r < rest; ++r)
        for (int g = 0; g < ng; ++g) b[(size_t)g * rest + r] = a[r * ng + g];
    return b;
}
IV I(const std::string& n) { return itab().at(n); }

// One launch: every (block, thread) of a 1-D or 3-D grid, in parallel over blocks.
template <class F>
void launch(unsigned gx, unsigned gy, unsigned gz, unsigned bx, F&& f)
{
    const long nb = (long)gx * gy * gz;
#pragma omp parallel for schedule(dynamic, 4)
    for (long b = 0; b < nb; ++b) {
        gridDim.x = gx; gridDim.y = gy; gridDim.z = gz;
        blockDim.x = bx; blockDim.y = 1; blockDim.z = 1;
        blockIdx.x = (unsigned)(b % gx);
        blockIdx.y = (unsigned)((b / gx) % gy);
        blockIdx.z = (unsigned)(b / ((long)gx * gy));
        threadIdx.y = 0; threadIdx.z = 0;
        for (unsigned t = 0; t < bx; ++t) {
            threadIdx.x = t;
            f();
        }
    }
}
inline unsigned cdiv(long a, long b) { return (unsigned)((a + b - 1) / b); }

struct Req {
    int nlay, ncol, diag, window_cols, sw_chunk, iswmode;
    double cpathfac, solcon;
    const float *plyr, *plvl, *tlyr, *tlvl, *qlyr, *olyr, *gasvmr, *clouds, *faerlw, *faersw, *sfcemis, *tsfg,
        *sfcalb, *coszen;
    int iovrlw = 1, iovrsw = 1;   // lwrad's transfer (0: rtrn, random overlap; > 0: rtrnmr), swrad's zcf0 overlap
};

// ---------------------------------------------------------------------------------------------- LW
void run_lw(const Req& q, double* htlw, double* topflw, double* sfcflw)
{
    const int nlay = q.nlay, nlp1 = nlay + 1, n = q.ncol, IM = n, JM = 1;
    const size_t L = (size_t)nlay * n, P = (size_t)nlp1 * n;
    const int ilwcliq = q.diag ? 0 : 1;
    // grrad_lw_pre: clouds(., ., 2) and (., ., 4) times the cloud-path factor (prognostic clouds)
    FV clouds(q.clouds, q.clouds + 9 * L);
    if (ilwcliq)
        for (size_t i = 0; i < L; ++i) {
            clouds[1 * L + i] = clouds[1 * L + i] * (float)q.cpathfac;
            clouds[3 * L + i] = clouds[3 * L + i] * (float)q.cpathfac;
        }
    FV aer(q.faerlw ? FV(q.faerlw, q.faerlw + 3 * 16 * L) : FV(3 * 16 * L, 0.0f));
    IV icseed(n, 0);
    FV pavel(L), tavel(L), delp(L), tz(P), coldry(L), colbrd(L), colamt(7 * L), wx(4 * L), tauaer(16 * L),
        cldfrc((nlp1 + 1) * (size_t)n), cldin(8 * L), taucld(16 * L), cldfmc(1), secdiff(16 * (size_t)n),
        semiss(16 * (size_t)n), pwvcm(n), stemp(n);
    IV ipseed(n), lcf1(n);
    launch(cdiv(n, 128), 1, 1, 128, [&] {
        r_lwrad::lwrad_prep(q.plyr, q.plvl, q.tlyr, q.tlvl, q.qlyr, q.olyr, q.gasvmr, clouds.data(), aer.data(),
                            q.sfcemis, q.tsfg, icseed.data(), pavel.data(), tavel.data(), delp.data(), tz.data(),
                            coldry.data(), colbrd.data(), colamt.data(), wx.data(), tauaer.data(), cldfrc.data(),
                            cldin.data(), taucld.data(), cldfmc.data(), secdiff.data(), semiss.data(), pwvcm.data(),
                            stemp.data(), ipseed.data(), lcf1.data(), nlay, nlp1, JM, IM, 0, JM, 0, 1, ilwcliq, 0,
                            140);
    });
    FV absliq1 = T("lw_absliq1"), absice1 = T("lw_absice1"), absice2 = T("lw_absice2"), absice3 = T("lw_absice3");
    IV ipat = I("lw_ipat");
    FV cldf(L);
    launch(cdiv(n, 128), 1, 1, 128, [&] {
        r_lwcld::phys_rrtm_lw_cldprop(clouds.data(), absliq1.data(), absice1.data(), absice2.data(), absice3.data(),
                                      ipat.data(), taucld.data(), cldf.data(), nlay, ilwcliq, 1, 0, IM, JM);
    });
    FV h2ovmr(L);
    for (size_t i = 0; i < L; ++i) h2ovmr[i] = colamt[i] / std::max(coldry[i], 1e-30f);
    FV totplnk = T("lw_totplnk"), delwave = T("lw_delwave"), preflog = T("lw_preflog"), tref = T("lw_tref"),
       chi = T("lw_chi_mls");
    IV laytrop(n), jp(L), jt(L), jt1(L), indself(L), indfor(L), indminor(L);
    FV pklay(P * 16), pklev(P * 16), rfrate(12 * L, 0.0f), fac00(L), fac01(L), fac10(L), fac11(L), selffac(L),
        selffrac(L), forfac(L), forfrac(L), minorfrac(L), scaleminor(L), scaleminorn2(L);
    launch(cdiv(n, 128), 1, 1, 128, [&] {
        r_lwset::rrtm_lw_setcoef(pavel.data(), tavel.data(), tz.data(), stemp.data(), h2ovmr.data(), colamt.data(),
                                 coldry.data(), colbrd.data(), totplnk.data(), delwave.data(), preflog.data(),
                                 tref.data(), chi.data(), nlay, IM, JM, laytrop.data(), pklay.data(), pklev.data(),
                                 jp.data(), jt.data(), jt1.data(), rfrate.data(), fac00.data(), fac01.data(),
                                 fac10.data(), fac11.data(), selffac.data(), selffrac.data(), indself.data(),
                                 forfac.data(), forfrac.data(), indfor.data(), minorfrac.data(), scaleminor.data(),
                                 scaleminorn2.data(), indminor.data());
    });
    // taumol: the canonical pair taug/fracs [140][nlay][ncol]
    FV taug(140 * L, 0.0f), fracs(140 * L, 0.0f);
    auto put = [&](int ns, int ng, const FV& tg, const FV& fr) {   // band-local [ng][nlay][ncol]
        std::copy(tg.begin(), tg.begin() + ng * L, taug.begin() + ns * L);
        std::copy(fr.begin(), fr.begin() + ng * L, fracs.begin() + ns * L);
    };
    const int* J = jp.data();
    {   // band 1: outputs [nlay][10][ncol]
        FV a = T("lw01_absa"), b = T("lw01_absb"), s = T("lw01_selfref"), f = T("lw01_forref"),
           ka = T("lw01_ka_mn2"), kb = T("lw01_kb_mn2"), fa = T("lw01_fracrefa"), fb = T("lw01_fracrefb");
        FV tg(10 * L), fr(10 * L);
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_b01::taugb01_cols(laytrop.data(), nlay, n, pavel.data(), colamt.data(), colbrd.data(),
                                scaleminorn2.data(), selffac.data(), selffrac.data(), indself.data(), forfac.data(),
                                forfrac.data(), indfor.data(), minorfrac.data(), indminor.data(), fac00.data(),
                                fac01.data(), fac10.data(), fac11.data(), J, jt.data(), jt1.data(), a.data(),
                                b.data(), s.data(), f.data(), ka.data(), kb.data(), fa.data(), fb.data(), tg.data(),
                                fr.data());
        });
        for (int k = 0; k < nlay; ++k)
            for (int g = 0; g < 10; ++g)
                for (int c = 0; c < n; ++c) {
                    taug[((size_t)(0 + g) * nlay + k) * n + c] = tg[((size_t)k * 10 + g) * n + c];
                    fracs[((size_t)(0 + g) * nlay + k) * n + c] = fr[((size_t)k * 10 + g) * n + c];
                }
    }
    {   // band 2: g-first strides into the pair
        FV a = T("lw02_absa"), b = T("lw02_absb"), s = T("lw02_selfref"), f = T("lw02_forref"),
           fa = T("lw02_fracrefa"), fb = T("lw02_fracrefb");
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_b02::rrtm_lw_taugb02(n, nlay, laytrop.data(), J, jt.data(), jt1.data(), pavel.data(), colamt.data(),
                                   fac00.data(), fac01.data(), fac10.data(), fac11.data(), selffac.data(),
                                   selffrac.data(), indself.data(), forfac.data(), forfrac.data(), indfor.data(),
                                   a.data(), b.data(), s.data(), f.data(), fa.data(), fb.data(), taug.data(),
                                   fracs.data(), (long long)n, (long long)nlay * n);
        });
    }
    {   // band 3: rate-1 rfrate of both sides [2][nlay][ncol]; outputs [16][nlay][ncol]
        FV a = T("lw03_absa"), b = T("lw03_absb"), s = T("lw03_selfref"), f = T("lw03_forref"),
           fa = T("lw03_fracrefa"), fb = T("lw03_fracrefb"), ka = T("lw03_ka_mn2o"), kb = T("lw03_kb_mn2o");
        FV rf(2 * L);
        for (int side = 0; side < 2; ++side)
            std::copy(rfrate.begin() + ((size_t)side * 6 + 0) * L, rfrate.begin() + ((size_t)side * 6 + 1) * L,
                      rf.begin() + side * L);
        FV tg(16 * L), fr(16 * L);
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_b03::phys_rrtm_lw_taugb03(IM, JM, nlay, chi.data(), a.data(), b.data(), s.data(), f.data(), fa.data(),
                                        fb.data(), ka.data(), kb.data(), laytrop.data(), J, jt.data(), jt1.data(),
                                        colamt.data(), rf.data(), coldry.data(), fac00.data(), fac01.data(),
                                        fac10.data(), fac11.data(), selffac.data(), selffrac.data(), forfac.data(),
                                        forfrac.data(), minorfrac.data(), indself.data(), indfor.data(),
                                        indminor.data(), tg.data(), fr.data());
        });
        put(22, 16, tg, fr);
    }
    {   // band 4: per (column, layer) launch; refrats in float32 on the host (phys_rrtm_lw_taugb04.py:87-99)
        FV a = T("lw04_absa"), b = T("lw04_absb"), s = T("lw04_selfref"), f = T("lw04_forref"),
           fa = T("lw04_fracrefa"), fb = T("lw04_fracrefb");
        const float rpa = chi[10 * 7 + 0] / chi[10 * 7 + 1], rpb = chi[12 * 7 + 2] / chi[12 * 7 + 1];
        launch(cdiv(n, 128), 1, nlay, 128, [&] {
            r_b04::rrtm_lw_taugb04(laytrop.data(), colamt.data(), rfrate.data(), J, jt.data(), jt1.data(),
                                   fac00.data(), fac01.data(), fac10.data(), fac11.data(), selffac.data(),
                                   selffrac.data(), indself.data(), forfac.data(), forfrac.data(), indfor.data(),
                                   a.data(), b.data(), s.data(), f.data(), fa.data(), fb.data(), rpa, rpb, IM, JM,
                                   nlay, taug.data(), fracs.data(), (long long)n, (long long)nlay * n);
        });
    }
    {   // band 5: colamt planes 1..3, rfrate slots (r11, r12, r61, r62), wx(k,1); refrats from float64 chi
        FV a = T("lw05_absa"), b = T("lw05_absb"), s = T("lw05_selfref"), f = T("lw05_forref"),
           fa = T("lw05_fracrefa"), fb = T("lw05_fracrefb"), ka = T("lw05_ka_mo3"), cc = T("lw05_ccl4");
        const std::vector<double>& c64 = ftab().at("lw05_chi_mls_f64");   // [59][7]
        auto CH = [&](int g, int lev) { return c64[(size_t)(lev - 1) * 7 + (g - 1)]; };
        const float rpa = (float)(CH(1, 5) / CH(2, 5)), rpb = (float)(CH(3, 43) / CH(2, 43)),
                    rma = (float)(CH(1, 7) / CH(2, 7));
        FV rf(4 * L);
        std::copy(rfrate.begin() + 0 * L, rfrate.begin() + 1 * L, rf.begin() + 0 * L);
        std::copy(rfrate.begin() + 6 * L, rfrate.begin() + 7 * L, rf.begin() + 1 * L);
        std::copy(rfrate.begin() + 5 * L, rfrate.begin() + 6 * L, rf.begin() + 2 * L);
        std::copy(rfrate.begin() + 11 * L, rfrate.begin() + 12 * L, rf.begin() + 3 * L);
        FV tg(16 * L), fr(16 * L);
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_b05::phys_rrtm_lw_taugb05(colamt.data(), rf.data(), wx.data(), fac00.data(), fac01.data(), fac10.data(),
                                        fac11.data(), selffac.data(), selffrac.data(), forfac.data(), forfrac.data(),
                                        minorfrac.data(), J, jt.data(), jt1.data(), indself.data(), indfor.data(),
                                        indminor.data(), laytrop.data(), a.data(), b.data(), s.data(), f.data(),
                                        fa.data(), fb.data(), ka.data(), cc.data(), rpa, rpb, rma, IM, JM, nlay,
                                        tg.data(), fr.data());
        });
        put(52, 16, tg, fr);
    }
    FV chi_co2(59);
    for (int m = 0; m < 59; ++m) chi_co2[m] = chi[(size_t)m * 7 + 1];
    {   // band 6: writes its planes
        FV a = T("lw06_absa"), s = T("lw06_selfref"), f = T("lw06_forref"), ka = T("lw06_ka_mco2"),
           fa = T("lw06_fracrefa"), c11 = T("lw06_cfc11adj"), c12 = T("lw06_cfc12");
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_b06::phys_rrtm_lw_taugb06(nlay, n, laytrop.data(), J, jt.data(), jt1.data(), indself.data(),
                                        indfor.data(), indminor.data(), coldry.data(), colamt.data(), wx.data(),
                                        selffac.data(), selffrac.data(), forfac.data(), forfrac.data(),
                                        minorfrac.data(), fac00.data(), fac01.data(), fac10.data(), fac11.data(),
                                        chi_co2.data(), a.data(), s.data(), f.data(), ka.data(), fa.data(),
                                        c11.data(), c12.data(), taug.data() + 68 * L, fracs.data() + 68 * L);
        });
    }
    {   // band 7: column-major [ncol][nlay] inputs, padded tables, outputs [ncol][nlay][12]
        auto cl = [&](const float* a) {
            FV o(L);
            for (int k = 0; k < nlay; ++k)
                for (int c = 0; c < n; ++c) o[(size_t)c * nlay + k] = a[(size_t)k * n + c];
            return o;
        };
        auto cli = [&](const int* a) {
            IV o(L);
            for (int k = 0; k < nlay; ++k)
                for (int c = 0; c < n; ++c) o[(size_t)c * nlay + k] = a[(size_t)k * n + c];
            return o;
        };
        FV a = T("lw07_absa"), b = T("lw07_absb");
        a.resize(595 * 12, 0.0f);
        b.resize(236 * 12, 0.0f);
        FV s = T("lw07_selfref"), f = T("lw07_forref"), fa = T("lw07_fracrefa"), fb = T("lw07_fracrefb"),
           ka = T("lw07_ka_mco2"), kb = T("lw07_kb_mco2");
        FV h2o = cl(colamt.data()), co2 = cl(colamt.data() + L), o3 = cl(colamt.data() + 2 * L), cd = cl(coldry.data());
        FV rf(2 * L);
        for (int k = 0; k < nlay; ++k)
            for (int c = 0; c < n; ++c)
                for (int side = 0; side < 2; ++side)
                    rf[((size_t)c * nlay + k) * 2 + side] = rfrate[(((size_t)side * 6 + 1) * nlay + k) * n + c];
        IV jpc = cli(J), jtc = cli(jt.data()), jt1c = cli(jt1.data()), isc = cli(indself.data()),
           ifc = cli(indfor.data()), imc = cli(indminor.data());
        FV sfc = cl(selffac.data()), sfr = cl(selffrac.data()), ffc = cl(forfac.data()), ffr = cl(forfrac.data()),
           mfc = cl(minorfrac.data()), f00 = cl(fac00.data()), f01 = cl(fac01.data()), f10 = cl(fac10.data()),
           f11 = cl(fac11.data());
        FV tg(12 * L), fr(12 * L);
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_b07::phys_rrtm_lw_taugb07(h2o.data(), co2.data(), o3.data(), cd.data(), rf.data(), jpc.data(),
                                        jtc.data(), jt1c.data(), isc.data(), ifc.data(), imc.data(), sfc.data(),
                                        sfr.data(), ffc.data(), ffr.data(), mfc.data(), f00.data(), f01.data(),
                                        f10.data(), f11.data(), laytrop.data(), chi.data(), a.data(), b.data(),
                                        s.data(), f.data(), fa.data(), fb.data(), ka.data(), kb.data(), tg.data(),
                                        fr.data(), n, nlay);
        });
        for (int c = 0; c < n; ++c)
            for (int k = 0; k < nlay; ++k)
                for (int g = 0; g < 12; ++g) {
                    taug[((size_t)(76 + g) * nlay + k) * n + c] = tg[((size_t)c * nlay + k) * 12 + g];
                    fracs[((size_t)(76 + g) * nlay + k) * n + c] = fr[((size_t)c * nlay + k) * 12 + g];
                }
    }
    {   // band 8
        FV a = T("lw08_absa"), b = T("lw08_absb"), s = T("lw08_selfref"), f = T("lw08_forref"),
           kac = T("lw08_ka_mco2"), kbc = T("lw08_kb_mco2"), kao = T("lw08_ka_mo3"), kan = T("lw08_ka_mn2o"),
           kbn = T("lw08_kb_mn2o"), fa = T("lw08_fracrefa"), fb = T("lw08_fracrefb"), c12 = T("lw08_cfc12"),
           c22 = T("lw08_cfc22adj");
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_b08::phys_rrtm_lw_taugb08(laytrop.data(), J, jt.data(), jt1.data(), indself.data(), indfor.data(),
                                        indminor.data(), coldry.data(), colamt.data(), wx.data(), selffac.data(),
                                        selffrac.data(), forfac.data(), forfrac.data(), minorfrac.data(),
                                        fac00.data(), fac10.data(), fac01.data(), fac11.data(), chi_co2.data(),
                                        a.data(), b.data(), s.data(), f.data(), kac.data(), kbc.data(), kao.data(),
                                        kan.data(), kbn.data(), fa.data(), fb.data(), c12.data(), c22.data(),
                                        taug.data(), fracs.data(), nlay, n, 0, n);
        });
    }
    {   // band 9
        FV a = T("lw09_absa"), b = T("lw09_absb"), s = T("lw09_selfref"), f = T("lw09_forref"),
           ka = T("lw09_ka_mn2o"), kb = T("lw09_kb_mn2o"), fa = T("lw09_fracrefa"), fb = T("lw09_fracrefb");
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_b09::phys_rrtm_lw_taugb09(laytrop.data(), J, jt.data(), jt1.data(), indself.data(), indfor.data(),
                                        indminor.data(), coldry.data(), colamt.data(), rfrate.data(), selffac.data(),
                                        selffrac.data(), forfac.data(), forfrac.data(), minorfrac.data(),
                                        fac00.data(), fac10.data(), fac01.data(), fac11.data(), chi.data(), a.data(),
                                        b.data(), s.data(), f.data(), ka.data(), kb.data(), fa.data(), fb.data(),
                                        taug.data(), fracs.data(), nlay, n, 0, n);
        });
    }
    {   // band 10: g-first strides
        FV a = T("lw10_absa"), b = T("lw10_absb"), s = T("lw10_selfref"), f = T("lw10_forref"),
           fa = T("lw10_fracrefa"), fb = T("lw10_fracrefb");
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_b10::rrtm_lw_taugb10(IM, JM, nlay, laytrop.data(), J, jt.data(), jt1.data(), colamt.data(),
                                   fac00.data(), fac01.data(), fac10.data(), fac11.data(), selffac.data(),
                                   selffrac.data(), indself.data(), forfac.data(), forfrac.data(), indfor.data(),
                                   a.data(), b.data(), s.data(), f.data(), fa.data(), fb.data(), taug.data(),
                                   fracs.data(), (long long)n, (long long)nlay * n);
        });
    }
    {   // band 11: rows 114.. of the pair
        FV a = T("lw11_absa"), b = T("lw11_absb"), s = T("lw11_selfref"), f = T("lw11_forref"),
           fa = T("lw11_fracrefa"), fb = T("lw11_fracrefb"), ka = T("lw11_ka_mo2"), kb = T("lw11_kb_mo2");
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_b11::phys_rrtm_lw_taugb11(laytrop.data(), J, jt.data(), jt1.data(), indself.data(), indfor.data(),
                                        indminor.data(), fac00.data(), fac01.data(), fac10.data(), fac11.data(),
                                        selffac.data(), selffrac.data(), forfac.data(), forfrac.data(),
                                        minorfrac.data(), scaleminor.data(), colamt.data(), a.data(), b.data(),
                                        s.data(), f.data(), fa.data(), fb.data(), ka.data(), kb.data(), taug.data(),
                                        fracs.data(), nlay, IM, JM, 114);
        });
    }
    {   // band 12
        FV a = T("lw12_absa"), s = T("lw12_selfref"), f = T("lw12_forref"), fa = T("lw12_fracrefa");
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_b12::rrtm_lw_taugb12(colamt.data(), rfrate.data(), J, jt.data(), jt1.data(), fac00.data(), fac01.data(),
                                   fac10.data(), fac11.data(), selffac.data(), selffrac.data(), indself.data(),
                                   forfac.data(), forfrac.data(), indfor.data(), laytrop.data(), a.data(), s.data(),
                                   f.data(), fa.data(), chi.data(), nlay, IM, JM, taug.data(), fracs.data());
        });
    }
    {   // band 13: 7-gas colamt
        FV a = T("lw13_absa"), s = T("lw13_selfref"), f = T("lw13_forref"), fa = T("lw13_fracrefa"),
           fb = T("lw13_fracrefb"), kac = T("lw13_ka_mco2"), kaco = T("lw13_ka_mco"), kbo = T("lw13_kb_mo3");
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_b13::rrtm_lw_taugb13(laytrop.data(), colamt.data(), coldry.data(), J, jt.data(), jt1.data(),
                                   rfrate.data(), fac00.data(), fac01.data(), fac10.data(), fac11.data(),
                                   selffac.data(), selffrac.data(), indself.data(), forfac.data(), forfrac.data(),
                                   indfor.data(), minorfrac.data(), indminor.data(), chi.data(), a.data(), s.data(),
                                   f.data(), fa.data(), fb.data(), kac.data(), kaco.data(), kbo.data(), nlay, IM, JM,
                                   taug.data() + 130 * L, fracs.data() + 130 * L);
        });
    }
    {   // band 14
        FV a = T("lw14_absa"), b = T("lw14_absb"), s = T("lw14_selfref"), f = T("lw14_forref"),
           fa = T("lw14_fracrefa"), fb = T("lw14_fracrefb");
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_b14::phys_rrtm_lw_taugb14(nlay, n, 0, n, laytrop.data(), J, jt.data(), jt1.data(), indself.data(),
                                        indfor.data(), colamt.data(), selffac.data(), selffrac.data(), forfac.data(),
                                        forfrac.data(), fac00.data(), fac01.data(), fac10.data(), fac11.data(),
                                        a.data(), b.data(), s.data(), f.data(), fa.data(), fb.data(), taug.data(),
                                        fracs.data());
        });
    }
    {   // band 15: refrat = chi(4,1)/chi(2,1) in float32 (phys_rrtm_lw_taugb15.py:135-136)
        FV a = T("lw15_absa"), s = T("lw15_selfref"), f = T("lw15_forref"), ka = T("lw15_ka_mn2"),
           fa = T("lw15_fracrefa");
        const float refrat = chi[3] / chi[1];
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_b15::phys_rrtm_lw_taugb15(nlay, n, refrat, refrat, laytrop.data(), J, jt.data(), jt1.data(),
                                        indself.data(), indfor.data(), indminor.data(), colamt.data(), rfrate.data(),
                                        colbrd.data(), scaleminor.data(), selffac.data(), selffrac.data(),
                                        forfac.data(), forfrac.data(), minorfrac.data(), fac00.data(), fac01.data(),
                                        fac10.data(), fac11.data(), a.data(), s.data(), f.data(), ka.data(),
                                        fa.data(), taug.data() + 136 * L, fracs.data() + 136 * L);
        });
    }
    {   // band 16
        FV a = T("lw16_absa"), b = T("lw16_absb"), s = T("lw16_selfref"), f = T("lw16_forref"),
           fa = T("lw16_fracrefa"), fb = T("lw16_fracrefb");
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_b16::rrtm_lw_taugb16(colamt.data(), rfrate.data(), J, jt.data(), jt1.data(), fac00.data(), fac01.data(),
                                   fac10.data(), fac11.data(), selffac.data(), selffrac.data(), indself.data(),
                                   forfac.data(), forfrac.data(), indfor.data(), laytrop.data(), a.data(), b.data(),
                                   s.data(), f.data(), fa.data(), fb.data(), chi.data(), nlay, IM, JM, taug.data(),
                                   fracs.data());
        });
    }
    // tautot = taug + tauaer(ngb(g)) (lw_core.py:83-90)
    static const int NGB_NS[17] = {0, 10, 22, 38, 52, 68, 76, 88, 96, 108, 114, 122, 130, 134, 136, 138, 140};
    for (int b = 0; b < 16; ++b)
        for (int g = NGB_NS[b]; g < NGB_NS[b + 1]; ++g)
            for (size_t i = 0; i < L; ++i) taug[(size_t)g * L + i] = taug[(size_t)g * L + i] + tauaer[(size_t)b * L + i];
    // rlwinit tables in the float32 recipe of phys_rrtm_lw_rtrnmr.py:108-131
    const int ntbl = 10000;
    FV exp_tbl(ntbl + 1), tfn_tbl(ntbl + 1), tau_tbl(ntbl + 1);
    {
        const float bpade = 1.0f / 0.278f, expeps = 1.0e-20f;
        const float explimit = (float)std::trunc(-std::log((double)std::numeric_limits<float>::min()));
        exp_tbl[0] = 1.0f; tau_tbl[0] = 0.0f; tfn_tbl[0] = 0.0f;
        for (int i = 1; i < ntbl; ++i) {
            const float tf = (float)i / (float)(ntbl - i);
            const float ta = bpade * tf;
            const float e = ta >= explimit ? expeps : (float)std::exp(-(double)ta);
            tau_tbl[i] = ta; exp_tbl[i] = e;
            tfn_tbl[i] = ta < 0.06f ? ta / 6.0f : 1.0f - 2.0f * ((1.0f / ta) - (e / (1.0f - e)));
        }
        exp_tbl[ntbl] = expeps; tau_tbl[ntbl] = 1.0e10f; tfn_tbl[ntbl] = 1.0f;
    }
    FV totuflux(P), totdflux(P), totuclfl(P), totdclfl(P), htr(L), htrcl(L), htrb(16 * L);
    const float heatfac = 9.80665f * 1.0e-2f / 1.0046e3f;
    const float fluxfac = (float)((double)(float)(2.0 * std::asin(1.0)) * 2.0e4);
    if (q.iovrlw <= 0) {
        // rtrn (phys_rrtm_lw_rtrn.py:84-108): NAM slot order, layer k (surface first, 1-based) in slot
        // nlay - k, interface m in slot nlay - m, pklay / pklev as [16][nlay + 1][ncol]
        const int LM = nlay, LMK = nlp1;
        if (LM > 60) throw std::runtime_error("the reference's rtrn holds at most 60 layers");
        FV delp_t(L), cf_t(L), taucld_t(16 * L), taug_t(140 * L), fracs_t(140 * L), pklay_t(P * 16), pklev_t(P * 16),
            tuf_t(P), tdf_t(P), tuc_t(P), tdc_t(P), htr_t(L), htrcl_t(L), htrb_t(16 * L);
        for (int k0 = 0; k0 < LM; ++k0)
            for (int c = 0; c < n; ++c) {
                const size_t s = (size_t)(LM - 1 - k0) * n + c, f = (size_t)k0 * n + c;
                delp_t[s] = delp[f];
                cf_t[s] = cldfrc[(size_t)(k0 + 1) * n + c];
                for (int ib = 0; ib < 16; ++ib) taucld_t[(size_t)ib * L + s] = taucld[(size_t)ib * L + f];
                for (int g = 0; g < 140; ++g) {
                    taug_t[(size_t)g * L + s] = taug[(size_t)g * L + f];
                    fracs_t[(size_t)g * L + s] = fracs[(size_t)g * L + f];
                }
            }
        for (int m = 0; m <= LM; ++m)
            for (int ib = 0; ib < 16; ++ib)
                for (int c = 0; c < n; ++c) {
                    const size_t s = ((size_t)ib * LMK + (LM - m)) * n + c, f = ((size_t)m * 16 + ib) * n + c;
                    pklay_t[s] = pklay[f];
                    pklev_t[s] = pklev[f];
                }
        IV ngb(140);
        for (int b = 0; b < 16; ++b)
            for (int g = NGB_NS[b]; g < NGB_NS[b + 1]; ++g) ngb[g] = b + 1;
        launch(cdiv(n, 128), 1, 1, 128, [&] {
            r_rtrn::phys_rrtm_lw_rtrn(semiss.data(), delp_t.data(), cf_t.data(), taucld_t.data(), taug_t.data(),
                                      pklay_t.data(), pklev_t.data(), fracs_t.data(), secdiff.data(), ngb.data(),
                                      tau_tbl.data(), exp_tbl.data(), tfn_tbl.data(), tuf_t.data(), tdf_t.data(),
                                      tuc_t.data(), tdc_t.data(), htr_t.data(), htrcl_t.data(), htrb_t.data(),
                                      fluxfac, heatfac, 0, 0, IM, JM, LM);
        });
        for (int m = 0; m <= LM; ++m)
            for (int c = 0; c < n; ++c) {
                const size_t s = (size_t)(LM - m) * n + c, f = (size_t)m * n + c;
                totuflux[f] = tuf_t[s]; totdflux[f] = tdf_t[s]; totuclfl[f] = tuc_t[s]; totdclfl[f] = tdc_t[s];
            }
        for (int k0 = 0; k0 < LM; ++k0)
            for (int c = 0; c < n; ++c) htr[(size_t)k0 * n + c] = htr_t[(size_t)(LM - 1 - k0) * n + c];
    } else {
    launch(cdiv(n, 128), 1, 1, 128, [&] {
        r_rtrnmr::phys_rrtm_lw_rtrnmr_sf(IM, JM, nlay, 0, 0, heatfac, fluxfac, exp_tbl.data(), tfn_tbl.data(),
                                         tau_tbl.data(), semiss.data(), delp.data(), cldfrc.data(), taucld.data(),
                                         taug.data(), pklay.data(), pklev.data(), fracs.data(), secdiff.data(),
                                         totuflux.data(), totdflux.data(), htr.data(), totuclfl.data(),
                                         totdclfl.data(), htrcl.data(), htrb.data());
    });
    }
    // lwrad_post
    FV o_top_c(n), o_top_0(n), o_sfc_uc(n), o_sfc_u0(n), o_sfc_dc(n), o_sfc_d0(n), hlwc(L), dum(1);
    launch(cdiv(n, 128), 1, 1, 128, [&] {
        r_lwrad::lwrad_post(totuflux.data(), totdflux.data(), totuclfl.data(), totdclfl.data(), htr.data(),
                            htrcl.data(), htrb.data(), o_top_c.data(), o_top_0.data(), o_sfc_uc.data(),
                            o_sfc_u0.data(), o_sfc_dc.data(), o_sfc_d0.data(), hlwc.data(), dum.data(), dum.data(),
                            dum.data(), nlay, nlp1, JM, IM, 0, JM, 0, 0, 0, 0);
    });
    for (size_t i = 0; i < L; ++i) htlw[i] = hlwc[i];
    for (int c = 0; c < n; ++c) {
        topflw[c] = o_top_c[c]; topflw[n + c] = o_top_0[c];
        sfcflw[c] = o_sfc_uc[c]; sfcflw[n + c] = o_sfc_u0[c]; sfcflw[2 * n + c] = o_sfc_dc[c]; sfcflw[3 * n + c] = o_sfc_d0[c];
    }
}

// ---------------------------------------------------------------------------------------------- SW
void run_sw_chunk(const Req& q, const IV& idxday, int cstart, int nc, int kminw, double* htsw, double* topfsw,
                  double* sfcfsw, double* fdncmp)
{
    const int nlay = q.nlay, nlp1 = nlay + 1, im = q.ncol, jm = 1;
    const int iswcliq = q.diag ? 0 : 1;
    const size_t C = (size_t)nc * nlay;
    IV ndayp(1, (int)idxday.size());
    IV icsdsw(im, 0);
    FV faersw(q.faersw ? FV(q.faersw, q.faersw + 42 * (size_t)nlay * im) : FV(42 * (size_t)nlay * im, 0.0f));
    FV pavel(C), tavel(C), delp(C), coldry(C), colmol(C), h2ovmr(C), o3vmr(C), temcol(C), colamt(C * 6), cfrac(C),
        cliqp(C), reliq(C), cicep(C), reice(C), cdat1(C), cdat2(C), cdat3(C), cdat4(C), tauae(C * 14),
        ssaae(C * 14), asyae(C * 14), zcf0(nc), zcf1(nc), cosz1(nc), sntz1(nc), ssolar(nc), albbm(2 * nc),
        albdf(2 * nc);
    IV ipseed(nc);
    launch(cdiv(nc, 128), 1, 1, 128, [&] {
        r_swrad::swrad_prep(q.plyr, q.plvl, q.tlyr, q.qlyr, q.olyr, q.gasvmr, q.clouds, faersw.data(), q.coszen,
                            q.sfcalb, icsdsw.data(), idxday.data(), ndayp.data(), cstart, nc, nlay, nlp1, im, jm, 0, 1,
                            iswcliq, q.iovrsw, 0, 1, (float)q.solcon, pavel.data(), tavel.data(), delp.data(),
                            coldry.data(), colmol.data(), h2ovmr.data(), o3vmr.data(), temcol.data(), colamt.data(),
                            cfrac.data(), cliqp.data(), reliq.data(), cicep.data(), reice.data(), cdat1.data(),
                            cdat2.data(), cdat3.data(), cdat4.data(), tauae.data(), ssaae.data(), asyae.data(),
                            zcf0.data(), zcf1.data(), cosz1.data(), sntz1.data(), ssolar.data(), albbm.data(),
                            albdf.data(), ipseed.data());
    });
    // layer-major views ([nlay][nc]) of the chunk arrays ([nc][nlay])
    auto lm = [&](const FV& a) {
        FV o(C);
        for (int t = 0; t < nc; ++t)
            for (int k = 0; k < nlay; ++k) o[(size_t)k * nc + t] = a[(size_t)t * nlay + k];
        return o;
    };
    auto lmi = [&](const IV& a) {
        IV o(C);
        for (int t = 0; t < nc; ++t)
            for (int k = 0; k < nlay; ++k) o[(size_t)k * nc + t] = a[(size_t)t * nlay + k];
        return o;
    };
    // cldprop (sw_seam.cldprop): iswcliq 1 / iswcice 3 (or 0), outputs [14][nlay][nc]
    FV tcw(14 * C), scw(14 * C), acw(14 * C), cldfrcL(C), dummy(1);
    {
        FV a1 = lm(cfrac), a2 = lm(cliqp), a3 = lm(reliq), a4 = lm(cicep), a5 = lm(reice), a6 = lm(cdat1),
           a7 = lm(cdat2), a8 = lm(cdat3), a9 = lm(cdat4);
        FV el = T("sw_extliq1"), sl = T("sw_ssaliq1"), al = T("sw_asyliq1"), e2 = T("sw_extice2"),
           s2 = T("sw_ssaice2"), y2 = T("sw_asyice2"), e3 = T("sw_extice3"), s3 = T("sw_ssaice3"), y3 = T("sw_asyice3");
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_swcld::phys_rrtm_sw_cldprop(a1.data(), a2.data(), a3.data(), a4.data(), a5.data(), a6.data(), a7.data(),
                                          a8.data(), a9.data(), zcf1.data(), el.data(), sl.data(), al.data(),
                                          e2.data(), s2.data(), y2.data(), e3.data(), s3.data(), y3.data(),
                                          tcw.data(), scw.data(), acw.data(), cldfrcL.data(), dummy.data(), nlay,
                                          iswcliq, 3, 0, nc, 1);
        });
    }
    // setcoef (chunk form, [nc][nlay])
    FV preflog = T("sw_preflog"), tref = T("sw_tref");
    IV lt(nc), jp(C), jt(C), jt1(C), inds(C), indf(C);
    FV f00(C), f01(C), f10(C), f11(C), sfac(C), sfrac(C), ffac(C), ffrac(C);
    launch(cdiv(nc, 128), 1, 1, 128, [&] {
        r_swset::rrtm_sw_setcoef_chunk(pavel.data(), tavel.data(), h2ovmr.data(), preflog.data(), tref.data(),
                                       ndayp.data(), cstart, nc, nlay, lt.data(), jp.data(), jt.data(), jt1.data(),
                                       f00.data(), f01.data(), f10.data(), f11.data(), sfac.data(), sfrac.data(),
                                       inds.data(), ffac.data(), ffrac.data(), indf.data());
    });
    // chunk canonical taug/taur [nc][nlay][112], sfluxzen [nc][112]
    FV taug(C * 112, 0.0f), taur(C * 112, 0.0f);
    // layer-major copies (sw_seam.layer_major)
    FV Lcolmol = lm(colmol), Lf00 = lm(f00), Lf01 = lm(f01), Lf10 = lm(f10), Lf11 = lm(f11), Lsfac = lm(sfac),
       Lsfrac = lm(sfrac), Lffac = lm(ffac), Lffrac = lm(ffrac);
    IV Ljp = lmi(jp), Ljt = lmi(jt), Ljt1 = lmi(jt1), Linds = lmi(inds), Lindf = lmi(indf);
    FV Lcolamt(6 * C);
    for (int t = 0; t < nc; ++t)
        for (int k = 0; k < nlay; ++k)
            for (int m = 0; m < 6; ++m) Lcolamt[((size_t)m * nlay + k) * nc + t] = colamt[((size_t)t * nlay + k) * 6 + m];
    // sfluxzen (sw_seam.taumol)
    FV sz(112 * (size_t)nc);
    {
        FV s1 = T("sw_sfluxref01"), s2 = T("sw_sfluxref02"), s3 = T("sw_sfluxref03");
        const float scalekur = T("sw_scalekur")[0];
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_swtau::phys_rrtm_sw_taumol(Lcolamt.data(), Ljp.data(), lt.data(), s1.data(), s2.data(), s3.data(),
                                         scalekur, sz.data(), nlay, 1, nc);
        });
    }
    auto put = [&](int ns, int ng, const FV& tg, const FV& tr, bool tr_shared) {   // band [ng][nlay][nc]
        for (int g = 0; g < ng; ++g)
            for (int k = 0; k < nlay; ++k)
                for (int t = 0; t < nc; ++t) {
                    taug[((size_t)t * nlay + k) * 112 + ns + g] = tg[((size_t)g * nlay + k) * nc + t];
                    taur[((size_t)t * nlay + k) * 112 + ns + g] =
                        tr_shared ? tr[(size_t)k * nc + t] : tr[((size_t)g * nlay + k) * nc + t];
                }
    };
    const long long ca_c = (long long)nlay * 6, ca_k = 6, ca_m = 1, tg_c = (long long)nlay * 112, tg_k = 112, tg_g = 1;
    {   // 16: chunk path
        FV a = Tg("sw16_absa", 6), b = Tg("sw16_absb", 6), s = Tg("sw16_selfref", 6), f = Tg("sw16_forref", 6);
        const float rayl = T("sw16_rayl")[0], strr = T("sw16_strrat")[0];
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_s16::rrtm_sw_taumol16(colamt.data(), colmol.data(), f00.data(), f01.data(), f10.data(), f11.data(),
                                    lt.data(), ffac.data(), ffrac.data(), indf.data(), sfac.data(), sfrac.data(),
                                    inds.data(), jp.data(), jt.data(), jt1.data(), a.data(), b.data(), s.data(),
                                    f.data(), rayl, strr, ndayp.data(), 1, 0, cstart, nc, nlay, nlay, 1, ca_c, ca_k,
                                    ca_m, tg_c, tg_k, tg_g, taug.data(), taur.data());
        });
    }
    {   // 17
        FV a = T("sw17_absa"), b = T("sw17_absb"), s = T("sw17_selfref"), f = T("sw17_forref");
        FV tg(12 * C), tr(12 * C);
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_s17::phys_rrtm_sw_taumol17(nlay, nc, 0.364641f, lt.data(), Ljp.data(), Ljt.data(), Ljt1.data(),
                                         Linds.data(), Lindf.data(), Lcolamt.data(), Lcolmol.data(), Lf00.data(),
                                         Lf01.data(), Lf10.data(), Lf11.data(), Lsfac.data(), Lsfrac.data(),
                                         Lffac.data(), Lffrac.data(), a.data(), b.data(), s.data(), f.data(),
                                         tg.data(), tr.data());
        });
        put(6, 12, tg, tr, false);
    }
    {   // 18
        FV a = T("sw18_absa"), b = T("sw18_absb"), s = T("sw18_selfref"), f = T("sw18_forref");
        const float rayl = T("sw18_rayl")[0];
        FV tg(8 * C), tr(C);
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_s18::phys_rrtm_sw_taumol18(Lcolamt.data(), Lcolmol.data(), lt.data(), Ljp.data(), Ljt.data(),
                                         Ljt1.data(), Lf00.data(), Lf01.data(), Lf10.data(), Lf11.data(),
                                         Lsfac.data(), Lsfrac.data(), Linds.data(), Lffac.data(), Lffrac.data(),
                                         Lindf.data(), a.data(), b.data(), s.data(), f.data(), rayl, 3.89589e+1f,
                                         tg.data(), tr.data(), nlay, 1, nc);
        });
        put(18, 8, tg, tr, true);
    }
    {   // 19: chunk path, 8-column groups formed in the kernel
        FV a = T("sw19_absa"), b = T("sw19_absb"), s = T("sw19_selfref"), f = T("sw19_forref");
        IV dummyi(1);
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_s19::rrtm_sw_taumol19(colamt.data(), colmol.data(), f00.data(), f01.data(), f10.data(), f11.data(),
                                    sfac.data(), sfrac.data(), ffac.data(), ffrac.data(), inds.data(), indf.data(),
                                    jp.data(), jt.data(), jt1.data(), lt.data(), a.data(), b.data(), s.data(),
                                    f.data(), ndayp.data(), 1, 0, cstart, nc, nlay, nlay, 1, ca_c, ca_k, ca_m, tg_c,
                                    tg_k, tg_g, taug.data(), taur.data(), dummyi.data(), 0);
        });
    }
    {   // 20: chunk path, planes from NS20
        FV a = Tg("sw20_absa", 10), b = Tg("sw20_absb", 10), s = Tg("sw20_selfref", 10), f = Tg("sw20_forref", 10),
           ch4 = T("sw20_absch4"), sfl(10, 0.0f);
        const float rayl = T("sw20_rayl")[0];
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_s20::rrtm_sw_taumol20(colamt.data(), colmol.data(), lt.data(), jp.data(), jt.data(), jt1.data(),
                                    f00.data(), f01.data(), f10.data(), f11.data(), sfac.data(), sfrac.data(),
                                    inds.data(), ffac.data(), ffrac.data(), indf.data(), a.data(), b.data(), s.data(),
                                    f.data(), ch4.data(), sfl.data(), rayl, ndayp.data(), 1, 0, cstart, nc, nlay, nlay,
                                    1, ca_c, ca_k, ca_m, tg_c, tg_k, tg_g, 0, 0, 0, taug.data() + 34,
                                    taur.data() + 34, dummy.data());
        });
    }
    {   // 21: plane0 = 0 band-local
        FV a = T("sw21_absa"), b = T("sw21_absb"), s = T("sw21_selfref"), f = T("sw21_forref");
        FV tg(10 * C), tr(10 * C);
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_s21::rrtm_sw_taumol21(Lcolmol.data(), Lcolamt.data(), Lf00.data(), Lf01.data(), Lf10.data(),
                                    Lf11.data(), Ljp.data(), Ljt.data(), Ljt1.data(), lt.data(), Lsfac.data(),
                                    Lsfrac.data(), Linds.data(), Lffac.data(), Lffrac.data(), Lindf.data(), a.data(),
                                    b.data(), s.data(), f.data(), nlay, nc, 1, 0, tg.data(), tr.data());
        });
        put(44, 10, tg, tr, false);
    }
    {   // 22: chunk path; tables in Fortran column-major order ([g][ms])
        FV a = Tg("sw22_absa", 2), b = Tg("sw22_absb", 2), s = Tg("sw22_selfref", 2), f = Tg("sw22_forref", 2);
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_s22::rrtm_sw_taumol22(colmol.data(), colamt.data(), lt.data(), f00.data(), f01.data(), f10.data(),
                                    f11.data(), sfac.data(), sfrac.data(), inds.data(), ffac.data(), ffrac.data(),
                                    indf.data(), jp.data(), jt.data(), jt1.data(), a.data(), b.data(), s.data(),
                                    f.data(), ndayp.data(), cstart, nc, nlay, nlay, 1, ca_c, ca_k, ca_m, tg_c, tg_k,
                                    tg_g, taug.data(), taur.data());
        });
    }
    {   // 23: MINVAL(laytrop) per 8-column tile of the chunk (sw_seam.band23)
        FV a = T("sw23_absa"), s = T("sw23_selfref"), f = T("sw23_forref"), ray = T("sw23_rayl");
        const int tpr = (nc + 7) / 8;
        IV kmin(tpr, std::numeric_limits<int>::max());
        for (int t = 0; t < nc; ++t) kmin[t / 8] = std::min(kmin[t / 8], lt[t]);
        FV tg(10 * C, 0.0f), tr(10 * C, 0.0f);
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_s23::rrtm_sw_taumol23(Lcolamt.data(), Lcolmol.data(), Lf00.data(), Lf01.data(), Lf10.data(),
                                    Lf11.data(), Ljp.data(), Ljt.data(), Ljt1.data(), lt.data(), kmin.data(),
                                    Lffac.data(), Lffrac.data(), Lindf.data(), Lsfac.data(), Lsfrac.data(),
                                    Linds.data(), a.data(), f.data(), s.data(), ray.data(), tg.data(), tr.data(), nlay,
                                    nc, 1, 6, 0, nc, tpr);
        });
        put(56, 10, tg, tr, false);
    }
    {   // 24: writes planes 66..73 of a 112-plane output
        FV a = Tg("sw24_absa", 8), b = Tg("sw24_absb", 8), s = Tg("sw24_selfref", 8), f = Tg("sw24_forref", 8),
           rla = T("sw24_rayla"), rlb = T("sw24_raylb"), o3a = T("sw24_abso3a"), o3b = T("sw24_abso3b");
        FV tg(112 * C, 0.0f), tr(112 * C, 0.0f);
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_s24::phys_rrtm_sw_taumol24(Lcolamt.data(), Lcolmol.data(), Ljp.data(), Ljt.data(), Ljt1.data(),
                                         Lf00.data(), Lf01.data(), Lf10.data(), Lf11.data(), Lsfac.data(),
                                         Lsfrac.data(), Linds.data(), Lffac.data(), Lffrac.data(), Lindf.data(),
                                         lt.data(), a.data(), b.data(), s.data(), f.data(), rla.data(), rlb.data(),
                                         o3a.data(), o3b.data(), tg.data(), tr.data(), nlay, 1, nc);
        });
        FV tg2(tg.begin() + 66 * C, tg.begin() + 74 * C), tr2(tr.begin() + 66 * C, tr.begin() + 74 * C);
        put(66, 8, tg2, tr2, false);
    }
    IV kminv(1, kminw);
    {   // 25: chunk minimum
        FV a = Tg("sw25_absa", 6), o3a = T("sw25_abso3a"), o3b = T("sw25_abso3b"), ray = T("sw25_rayl");
        FV tg(6 * C, 0.0f), tr(6 * C, 0.0f);
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_s25::rrtm_sw_taumol25(Lcolamt.data(), Lcolmol.data(), Lf00.data(), Lf01.data(), Lf10.data(),
                                    Lf11.data(), lt.data(), Ljp.data(), Ljt.data(), Ljt1.data(), kminv.data(),
                                    a.data(), o3a.data(), o3b.data(), ray.data(), nlay, nc, 1, tg.data(), tr.data(), 0);
        });
        put(74, 6, tg, tr, false);
    }
    {   // 26
        FV ray = T("sw26_rayl");
        FV tg(6 * C), tr(6 * C);
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_s26::rrtm_sw_taumol26(Lcolmol.data(), ray.data(), nlay, nc, 1, tg.data(), tr.data());
        });
        put(80, 6, tg, tr, false);
    }
    {   // 27
        FV a = T("sw27_absa"), b = T("sw27_absb"), ray = T("sw27_rayl");
        FV tg(8 * C, 0.0f), tr(8 * C, 0.0f);
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_s27::rrtm_sw_taumol27(Lcolmol.data(), Lcolamt.data(), Lf00.data(), Lf01.data(), Lf10.data(),
                                    Lf11.data(), Ljp.data(), Ljt.data(), Ljt1.data(), lt.data(), a.data(), b.data(),
                                    ray.data(), nlay, nc, 1, 0, tg.data(), tr.data());
        });
        put(86, 8, tg, tr, false);
    }
    {   // 28: chunk minimum
        FV a = Tg("sw28_absa", 6), b = Tg("sw28_absb", 6);
        const float rayl = T("sw28_rayl")[0], strr = T("sw28_strrat")[0];
        FV tg(6 * C, 0.0f), tr(6 * C, 0.0f);
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_s28::rrtm_sw_taumol28(Lcolamt.data(), Lcolmol.data(), Lf00.data(), Lf01.data(), Lf10.data(),
                                    Lf11.data(), lt.data(), Ljp.data(), Ljt.data(), Ljt1.data(), kminv.data(),
                                    a.data(), b.data(), rayl, strr, nlay, nc, 1, tg.data(), tr.data(), 0);
        });
        put(94, 6, tg, tr, false);
    }
    {   // 29: id0/id1 from the dispatcher (sw_seam.band29)
        FV a = Tg("sw29_absa", 12), b = Tg("sw29_absb", 12), s = Tg("sw29_selfref", 12), f = Tg("sw29_forref", 12),
           h2o = T("sw29_absh2o"), co2 = T("sw29_absco2");
        IV id0(C), id1(C);
        for (int k = 0; k < nlay; ++k)
            for (int t = 0; t < nc; ++t) {
                const size_t i = (size_t)k * nc + t;
                const bool low = k + 1 <= lt[t];
                id0[i] = low ? (Ljp[i] - 1) * 5 + (Ljt[i] - 1) : (Ljp[i] - 13) * 5 + (Ljt[i] - 1);
                id1[i] = low ? Ljp[i] * 5 + (Ljt1[i] - 1) : (Ljp[i] - 12) * 5 + (Ljt1[i] - 1);
            }
        FV tg(12 * C), tr(C);
        launch(cdiv(nc, 128), 1, 1, 128, [&] {
            r_s29::rrtm_sw_taumol29(Lcolmol.data(), Lcolamt.data(), lt.data(), Lf00.data(), Lf01.data(), Lf10.data(),
                                    Lf11.data(), Lsfac.data(), Lsfrac.data(), Linds.data(), Lffac.data(),
                                    Lffrac.data(), Lindf.data(), id0.data(), id1.data(), a.data(), b.data(), s.data(),
                                    f.data(), h2o.data(), co2.data(), nlay, nc, 1, tg.data(), tr.data());
        });
        put(100, 12, tg, tr, true);
    }
    if (g_cap.taug && cstart == 0) {
        for (int t = 0; t < nc; ++t) {
            for (size_t i = 0; i < (size_t)nlay * 112; ++i) {
                g_cap.taug[(size_t)t * nlay * 112 + i] = taug[(size_t)t * nlay * 112 + i];
                g_cap.taur[(size_t)t * nlay * 112 + i] = taur[(size_t)t * nlay * 112 + i];
            }
            for (int gg = 0; gg < 112; ++gg) g_cap.sfluxzen[(size_t)t * 112 + gg] = sz[(size_t)gg * nc + t];
            for (int ib = 0; ib < 14; ++ib)
                for (int k = 0; k < nlay; ++k) {
                    const size_t o = ((size_t)t * 14 + ib) * nlay + k, i = ((size_t)ib * nlay + k) * nc + t;
                    g_cap.taucw[o] = tcw[i]; g_cap.ssacw[o] = scw[i]; g_cap.asycw[o] = acw[i];
                }
            for (int k = 0; k < nlay; ++k) g_cap.cldfrc[(size_t)t * nlay + k] = cldfrcL[(size_t)k * nc + t];
            g_cap.zcf[2 * t] = zcf0[t]; g_cap.zcf[2 * t + 1] = zcf1[t];
            g_cap.laytrop[t] = lt[t];
        }
    }
    if (g_cap.stop_after_taumol) return;
    if (g_sw_tau_scale != 1.0)
        for (auto& v : taug) v = v * (float)g_sw_tau_scale;
    // spcvrtc: 112 launches in g order (sw_seam.spcvrtc)
    FV ex(10001);
    {
        ex[0] = 1.0f;
        const double bpade = 1.0 / 0.278;
        for (int i = 1; i < 10000; ++i) ex[i] = (float)std::exp(-bpade * ((double)i / (10000.0 - i)));
        ex[10000] = 1.0e-20f;
    }
    const size_t P = (size_t)nlp1 * nc;
    FV fxupc(14 * P), fxdnc(14 * P), fxup0(14 * P), fxdn0(14 * P), ftoadc(nc), ftoauc(nc), ftoau0(nc), fsfcuc(nc),
        fsfcu0(nc), fsfcdc(nc), fsfcd0(nc), sfbmc(2 * nc), sfdfc(2 * nc), sfbm0(2 * nc), sfdf0(2 * nc), suvbfc(nc),
        suvbf0(nc);
    FV albbmL(2 * nc), albdfL(2 * nc);
    for (int t = 0; t < nc; ++t)
        for (int j = 0; j < 2; ++j) { albbmL[(size_t)j * nc + t] = albbm[2 * t + j]; albdfL[(size_t)j * nc + t] = albdf[2 * t + j]; }
    FV szL(112 * (size_t)nc);
    for (int t = 0; t < nc; ++t)
        for (int g = 0; g < 112; ++g) szL[(size_t)g * nc + t] = sz[(size_t)g * nc + t];
    static const int NGB[14] = {6, 12, 8, 8, 10, 10, 2, 10, 8, 6, 6, 8, 6, 12};
    static const int IDXSFC[14] = {1, 1, 1, 1, 1, 1, 1, 1, 0, 2, 2, 2, 2, 1};
    FV tgg(C), trg(C), ta(C), sa(C), ya(C), tc(C), sc(C), yc(C);
    int jg = 1;
    for (int ib = 1; ib <= 14; ++ib) {
        for (int k = 0; k < nlay; ++k)
            for (int t = 0; t < nc; ++t) {
                const size_t i = (size_t)k * nc + t, s = ((size_t)t * nlay + k) * 14 + (ib - 1);
                ta[i] = tauae[s]; sa[i] = ssaae[s]; ya[i] = asyae[s];
                tc[i] = tcw[((size_t)(ib - 1) * nlay + k) * nc + t];
                sc[i] = scw[((size_t)(ib - 1) * nlay + k) * nc + t];
                yc[i] = acw[((size_t)(ib - 1) * nlay + k) * nc + t];
            }
        for (int j = 0; j < NGB[ib - 1]; ++j, ++jg) {
            for (int k = 0; k < nlay; ++k)
                for (int t = 0; t < nc; ++t) {
                    tgg[(size_t)k * nc + t] = taug[((size_t)t * nlay + k) * 112 + jg - 1];
                    trg[(size_t)k * nc + t] = taur[((size_t)t * nlay + k) * 112 + jg - 1];
                }
            launch(cdiv(nc, 128), 1, 1, 128, [&] {
                r_spcv::phys_rrtm_sw_spcvrtc(ssolar.data(), cosz1.data(), sntz1.data(), albbmL.data(), albdfL.data(),
                                             cldfrcL.data(), zcf1.data(), zcf0.data(), tgg.data(), trg.data(),
                                             ta.data(), sa.data(), ya.data(), tc.data(), sc.data(), yc.data(),
                                             ex.data(), fxupc.data(), fxdnc.data(), fxup0.data(), fxdn0.data(),
                                             ftoadc.data(), ftoauc.data(), ftoau0.data(), fsfcuc.data(),
                                             fsfcu0.data(), fsfcdc.data(), fsfcd0.data(), sfbmc.data(), sfdfc.data(),
                                             sfbm0.data(), sfdf0.data(), suvbfc.data(), suvbf0.data(), szL.data(), jg,
                                             ib, IDXSFC[ib - 1], jg == 1, jg == 112, nlay, nlp1, 1, nc, q.iswmode);
            });
        }
    }
    // swrad_post on the chunk layout ([nc][nlp1][14], [nc][2])
    auto ch3 = [&](const FV& a) {
        FV o(14 * P);
        for (int ib = 0; ib < 14; ++ib)
            for (int k = 0; k < nlp1; ++k)
                for (int t = 0; t < nc; ++t) o[((size_t)t * nlp1 + k) * 14 + ib] = a[((size_t)ib * nlp1 + k) * nc + t];
        return o;
    };
    auto ch2 = [&](const FV& a) {
        FV o(2 * nc);
        for (int t = 0; t < nc; ++t) { o[2 * t] = a[t]; o[2 * t + 1] = a[nc + t]; }
        return o;
    };
    FV cu = ch3(fxupc), cd = ch3(fxdnc), cu0 = ch3(fxup0), cd0 = ch3(fxdn0), sbm = ch2(sfbmc), sdf = ch2(sfdfc);
    const size_t Lfull = (size_t)nlay * im;
    FV htswc(Lfull, 0.0f), topflx(3 * (size_t)im, 0.0f), sfcflx(4 * (size_t)im, 0.0f), fdn(6 * (size_t)im, 0.0f), d1(1);
    const float heatfac = (float)(9.80665 * 1.0e-2 / 1.0046e3);
    launch(cdiv(nc, 128), 1, 1, 128, [&] {
        r_swrad::swrad_post(delp.data(), cu.data(), cd.data(), cu0.data(), cd0.data(), ftoauc.data(), ftoau0.data(),
                            ftoadc.data(), fsfcuc.data(), fsfcu0.data(), fsfcdc.data(), fsfcd0.data(), suvbfc.data(),
                            suvbf0.data(), sbm.data(), sdf.data(), idxday.data(), ndayp.data(), cstart, nc, nlay,
                            nlp1, im, jm, 0, heatfac, 0, 0, 0, 1, htswc.data(), topflx.data(), sfcflx.data(),
                            d1.data(), d1.data(), d1.data(), fdn.data());
    });
    for (int t = 0; t < nc; ++t) {
        const int c = idxday[cstart + t];
        for (int k = 0; k < nlay; ++k) htsw[(size_t)k * im + c] = htswc[(size_t)k * im + c];
        for (int m = 0; m < 3; ++m) topfsw[(size_t)m * im + c] = topflx[(size_t)m * im + c];
        for (int m = 0; m < 4; ++m) sfcfsw[(size_t)m * im + c] = sfcflx[(size_t)m * im + c];
        if (fdncmp)
            for (int m = 0; m < 6; ++m) fdncmp[(size_t)m * im + c] = fdn[(size_t)m * im + c];
    }
}

void run_sw(const Req& q, double* htsw, double* topfsw, double* sfcfsw, double* fdncmp)
{
    const int n = q.ncol, nlay = q.nlay;
    for (size_t i = 0; i < (size_t)nlay * n; ++i) htsw[i] = 0;
    for (int i = 0; i < 3 * n; ++i) topfsw[i] = 0;
    for (int i = 0; i < 4 * n; ++i) sfcfsw[i] = 0;
    if (fdncmp)
        for (int i = 0; i < 6 * n; ++i) fdncmp[i] = 0;
    // windows of window_cols columns, each window's day columns in chunks of sw_chunk (the reference runs
    // swrad per row window and chunks its day list, phys_rrtm_sw_swrad.py:340-386)
    const int wcols = q.window_cols > 0 ? q.window_cols : n;
    for (int w0 = 0; w0 < n; w0 += wcols) {
        IV day;
        for (int c = w0; c < std::min(n, w0 + wcols); ++c)
            if (q.coszen[c] >= 1.0e-4f) day.push_back(c);
        const int nday = (int)day.size();
        for (int c0 = 0; c0 < nday; c0 += q.sw_chunk) {
            const int nc = std::min(q.sw_chunk, nday - c0);
            // the chunk minimum of laytrop for bands 25/28 (taumol25.py:89-90) needs setcoef first: run
            // the prep + setcoef part of the chunk once on the host statements to find it
            FV pav((size_t)nc * nlay), tav((size_t)nc * nlay), h2o((size_t)nc * nlay);
            int kminw = std::numeric_limits<int>::max();
            for (int t = 0; t < nc; ++t) {
                const int c = day[c0 + t];
                int lt = nlay;
                for (int k0 = 0; k0 < nlay; ++k0) {
                    const int kk0 = nlay - 1 - k0;
                    const float p = q.plyr[(size_t)kk0 * n + c];
                    if (logf(p) > 4.56f) lt = k0 + 1;
                }
                kminw = std::min(kminw, lt);
            }
            // cstart is relative to the window's own day list
            IV idx(day.begin(), day.end());
            run_sw_chunk(q, idx, c0, nc, kminw, htsw, topfsw, sfcfsw, fdncmp);
        }
    }
}

}  // namespace drv

extern "C" {

// McICA sub-column masks of a request from the reference's generator kernels: LW words [5][nlay][ncol]
// from the LW cloud fraction (cldprop: the input cloud fraction, zero for a column with no layer above
// 1e-6), SW words [4][nlay][ncol] from the input cloud fraction (the kernel applies the 1e-12 step);
// layers surface first.  Seeds: icseed [2][ncol] (LW row, SW row) or seed0 + column + 1.
int orc_mcica_masks(const int* cfg_i, int nlay, int ncol, const float* clouds, const int* icseed,
                    unsigned int* lw_out, unsigned int* sw_out)
{
    const int iovrlw = cfg_i[5], iovrsw = cfg_i[6], lw_seed0 = cfg_i[7], sw_seed0 = cfg_i[8];
    std::vector<float> cf((size_t)nlay * ncol), cfl((size_t)nlay * ncol, 0.0f);
    std::vector<int> slw(ncol), ssw(ncol);
    for (int c = 0; c < ncol; ++c) {
        bool any = false;
        for (int k0 = 0; k0 < nlay; ++k0) {
            const float x = clouds[(size_t)(nlay - 1 - k0) * ncol + c];
            cf[(size_t)k0 * ncol + c] = x;
            any = any || x > 1.0e-6f;
        }
        if (any)
            for (int k0 = 0; k0 < nlay; ++k0) cfl[(size_t)k0 * ncol + c] = cf[(size_t)k0 * ncol + c];
        slw[c] = icseed ? icseed[c] : lw_seed0 + c + 1;
        ssw[c] = icseed ? icseed[(size_t)ncol + c] : sw_seed0 + c + 1;
    }
    if (lw_out)
        drv::launch(drv::cdiv(ncol, 128), 1, 1, 128, [&] {
            r_lwmc::phys_rrtm_lw_mcica_subcol(cfl.data(), slw.data(), lw_out, nlay, 1, ncol, iovrlw);
        });
    if (sw_out)
        drv::launch(drv::cdiv(ncol, 128), 1, 1, 128, [&] {
            r_swmc::phys_rrtm_sw_mcica_subcol(cf.data(), ssw.data(), sw_out, nlay, 1, ncol, iovrsw);
        });
    return 0;
}

int orc_set_debug(double sw_tau_scale)
{
    drv::g_sw_tau_scale = sw_tau_scale;
    return 0;
}

// SW stage outputs of the day columns of the first chunk (window 0): taug/taur [nday][nlay][112],
// sfluxzen [nday][112], taucw/ssacw/asycw [nday][14][nlay], cldfrc [nday][nlay], zcf [nday][2] (zcf0, zcf1),
// laytrop [nday]; layers surface first.
int orc_sw_stages(const int* cfg_i, int nlay, int ncol, const float* plyr, const float* plvl, const float* tlyr,
                  const float* tlvl, const float* qlyr, const float* olyr, const float* gasvmr, const float* clouds,
                  const float* sfcalb, const float* coszen, double solcon, float* taug, float* taur, float* sfluxzen,
                  float* taucw, float* ssacw, float* asycw, float* cldfrc, float* zcf, int* laytrop)
{
    try {
        drv::Req q{nlay, ncol, cfg_i[1], 0, 1 << 30, cfg_i[0], 1.5, solcon, plyr, plvl, tlyr, tlvl, qlyr, olyr,
                   gasvmr, clouds, nullptr, nullptr, nullptr, nullptr, sfcalb, coszen, 1, cfg_i[2]};
        drv::g_cap = drv::SwCapture{taug, taur, sfluxzen, taucw, ssacw, asycw, cldfrc, zcf, laytrop, true};
        std::vector<double> h((size_t)nlay * ncol), t3(3 * (size_t)ncol), s4(4 * (size_t)ncol);
        drv::run_sw(q, h.data(), t3.data(), s4.data(), nullptr);
        drv::g_cap = drv::SwCapture{};
    } catch (const std::exception& e) {
        drv::g_cap = drv::SwCapture{};
        std::fprintf(stderr, "reference driver: %s\n", e.what());
        return -1;
    }
    return 0;
}

int orc_clear_tables(void)
{
    drv::ftab().clear();
    drv::itab().clear();
    return 0;
}
int orc_add_table(const char* name, const double* data, long n)
{
    drv::ftab()[name] = std::vector<double>(data, data + n);
    return 0;
}
int orc_add_itable(const char* name, const int* data, long n)
{
    drv::itab()[name] = std::vector<int>(data, data + n);
    return 0;
}

// Same entry as the restatement's (oracle/rrtm_oracle.cpp); the reference kernels are float32 only, the
// McICA route and the optional profiles are not driven here.  iovrlw <= 0 runs the reference's rtrn, which
// holds at most 60 layers (phys_rrtm_lw_rtrn.py:60).
int orc_solve(int precision, const int* cfg_i, double cpathfac, int nlay, int ncol, const float* plyr,
              const float* plvl, const float* tlyr, const float* tlvl, const float* qlyr, const float* olyr,
              const float* gasvmr, const float* clouds, const float* faerlw, const float* faersw,
              const float* sfcemis, const float* tsfg, const float* sfcalb, const float* coszen,
              const int* icseed, double solcon, double* htlw, double* htsw, double* topflw, double* sfcflw,
              double* topfsw, double* sfcfsw, double* fdncmp, double* lwflx, double* swflx,
              unsigned int* lw_mask, unsigned int* sw_mask, int nthreads)
{
    (void)precision; (void)icseed; (void)lwflx; (void)swflx; (void)lw_mask; (void)sw_mask; (void)nthreads;
    try {
        if (cfg_i[4] != 0) throw std::runtime_error("the reference driver runs the NAM route only");
        drv::Req q{nlay, ncol, cfg_i[1], cfg_i[2], cfg_i[3] > 0 ? cfg_i[3] : 32768, cfg_i[0], cpathfac, solcon,
                   plyr, plvl, tlyr, tlvl, qlyr, olyr, gasvmr, clouds, faerlw, faersw, sfcemis, tsfg, sfcalb, coszen,
                   cfg_i[5], cfg_i[6]};
        drv::run_lw(q, htlw, topflw, sfcflw);
        drv::run_sw(q, htsw, topfsw, sfcfsw, fdncmp);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "reference driver: %s\n", e.what());
        return -1;
    }
    return 0;
}

// The radiation call's post step from the reference kernel rrtm_post_outputs (phys_rrtm_driver_post.cu:71-145),
// columns flattened (IM = ncol, JM = 1), so every [l, JM, IM] array is [l][ncol].  lssav is 1 (the
// reference refuses anything else).
int ref_post_outputs(int ncol, int lm, int icwp, int lw_step, const float* hlw, const float* swh,
                     const float* coszdg_v, const float* coszen_v, const float* sfcflw_dnfxc,
                     const float* sfcfsw_dnfxc, const float* sfcfsw_upfxc, const float* sfcfsw_dnfx0,
                     const float* topflw_upfxc, const float* topfsw_upfxc, float* cldcov, float* cldsa,
                     const float* cw, const float* t, const int* cu_cloud, float* rlwtt, float* rswtt,
                     float* cldfra, float* csmid, float* rlwin, float* rswin, float* rswinc, float* rswout,
                     float* rlwtoa, float* rswtoa, float* czmean, float* sigt4, float* coszdg, float* cfracl,
                     float* cfracm, float* cfrach, float* acfrst, float* acfrcv, int* ncfrst, int* ncfrcv)
{
    drv::launch(drv::cdiv(ncol, 128), 1, 1, 128, [&] {
        r_post::rrtm_post_outputs(ncol, 1, lm, icwp, 1, lw_step, hlw, swh, coszdg_v, coszen_v, sfcflw_dnfxc,
                                  sfcfsw_dnfxc, sfcfsw_upfxc, sfcfsw_dnfx0, topflw_upfxc, topfsw_upfxc, cldcov,
                                  cldsa, cw, t, cu_cloud, rlwtt, rswtt, cldfra, csmid, rlwin, rswin, rswinc,
                                  rswout, rlwtoa, rswtoa, czmean, sigt4, coszdg, cfracl, cfracm, cfrach, acfrst,
                                  acfrcv, ncfrst, ncfrcv);
    });
    return 0;
}

// RDTEMP from the reference kernel rdtemp_apply (drv_rdtemp.cu:140-198) on the host; lim is the
// loop-limit table (1-based values at the DL_* slots), one row slab (JOFF = 0).
int ref_rdtemp(int ntsd, float dt, int julday, int julyr, int ihrst, int leap_seen, const float* glat,
               const float* glon, float* czen, const float* czmean, float* t, const float* rswtt,
               const float* rlwtt, int im, int jm, int lm, const int* lim)
{
    drv::launch(drv::cdiv((long)im * jm, 128), 1, 1, 128, [&] {
        r_rdt::rdtemp_apply(ntsd, dt, julday, julyr, ihrst, leap_seen, glat, glon, czen, czmean, t, rswtt, rlwtt,
                            im, jm, lm, lim, 0);
    });
    return 0;
}

// Climatological aerosol optics from the reference's kernels, in the reference's order: aer_init
// (phys_rrtm_aer_init.py: flags, set_spectrum), clim_aerinit (phys_rrtm_clim_aerinit.py:196-235: bands, then
// optavg), aer_update's month fill (phys_rrtm_aer_update.py:139-165), setaer (phys_rrtm_setaer.py: zero, prep,
// then aer_property as phys_rrtm_aer_property.py:176-200 binds it, cmixg / denng cast to float), for the NAM
// settings iaer 11 (SW and LW on, volcanic off), one row of ncol columns, levels top first (ivflip 0) or surface
// first (ivflip 1, the reference's other orientation).
int orc_aerosols_iv(const int* iendwv, const float* haer, const float* prsref, const float* rhid, const float* rhdp,
                    const float* straext0, const int* nwvns0, const float* s0intv, const int* midx, const double* mcmix,
                    const int* mkprf, const double* mdenn, int nlay, int ncol, const float* plvl, const float* plyr,
                    const float* tlyr, const float* qlyr, const float* rhly, const float* xlon, const float* xlat,
                    const float* slmsk, float* aerosw, float* aerolw, float* tab, int ivflip)
{
    (void)nwvns0; (void)s0intv;   // the reference kernel carries the solar spectrum itself
    using FV = std::vector<float>;
    using IV = std::vector<int>;
    const int kNAER = 61, kNSW = 14, kNLW = 16, kNBT = 30, kNCM1 = 6, kNCM2 = 4, kNRH = 8, kNDM = 5, kNAE = 7;
    const int kNCELL = 37 * 72, kNXC = 5;
    int rip[16] = {0};
    rip[4] = 11; rip[5] = 1; rip[6] = 1; rip[7] = 0; rip[8] = 0;     // iaerflg, laswflg, lalwflg, lavoflg, iaermdl
    IV aflags(16, 0);
    drv::launch(1, 1, 1, 1, [&] { r_aeri::aer_init_flags(rip, aflags.data()); });
    FV solfwv(57600), eirfwv(4000);
    drv::launch(drv::cdiv(57600, 128), 1, 1, 128, [&] { r_aeri::aer_init_solfwv(solfwv.data(), aflags.data()); });
    drv::launch(drv::cdiv(4000, 128), 1, 1, 128, [&] { r_aeri::aer_init_eirfwv(eirfwv.data(), aflags.data()); });
    FV wsw1(r_seta::SA_WVNSW1, r_seta::SA_WVNSW1 + kNSW), wsw2(r_seta::SA_WVNSW2, r_seta::SA_WVNSW2 + kNSW),
        wlw1(r_seta::SA_WVNLW1, r_seta::SA_WVNLW1 + kNLW), wlw2(r_seta::SA_WVNLW2, r_seta::SA_WVNLW2 + kNLW);
    FV sigref(kNAE * kNDM), solbnd(kNSW), solwaer(kNAER * kNSW), eirbnd(kNLW), eirwaer(kNAER * kNLW);
    IV nv1(kNSW), nv2(kNSW), nr1(kNLW), nr2(kNLW);
    const int nb1 = kNSW + kNLW + kNAE * kNDM;
    drv::launch(drv::cdiv(nb1, 128), 1, 1, 128, [&] {
        r_aerc::clim_aerinit_bands(solfwv.data(), eirfwv.data(), iendwv, wsw1.data(), wsw2.data(), wlw1.data(),
                                   wlw2.data(), prsref, sigref.data(), solbnd.data(), solwaer.data(), nv1.data(),
                                   nv2.data(), eirbnd.data(), eirwaer.data(), nr1.data(), nr2.data(), kNSW, kNLW, 1, 1);
    });
    const size_t R1 = (size_t)kNCM1 * kNAER, R2 = (size_t)kNCM2 * kNRH * kNAER, ND = (size_t)kNBT * kNCM2 * kNRH;
    FV extrhi(kNBT * kNCM1), scarhi(kNBT * kNCM1), ssarhi(kNBT * kNCM1), asyrhi(kNBT * kNCM1), extrhd(ND), scarhd(ND),
        ssarhd(ND), asyrhd(ND), extstra(kNBT);
    const int nb2 = kNBT * (kNCM1 + kNCM2 * kNRH + 1);
    drv::launch(drv::cdiv(nb2, 128), 1, 1, 128, [&] {
        r_aerc::clim_aerinit_optavg(rhid, rhid + R1, rhid + 2 * R1, rhid + 3 * R1, rhdp, rhdp + R2, rhdp + 2 * R2,
                                    rhdp + 3 * R2, straext0, solbnd.data(), solwaer.data(), nv1.data(), nv2.data(),
                                    eirbnd.data(), eirwaer.data(), nr1.data(), nr2.data(), extrhi.data(),
                                    scarhi.data(), ssarhi.data(), asyrhi.data(), extrhd.data(), scarhd.data(),
                                    ssarhd.data(), asyrhd.data(), extstra.data(), kNSW, kNLW, 1, 1);
    });
    IV idxcg(kNCELL * kNXC), kprfg(kNCELL);
    std::vector<double> cmixd(kNCELL * kNXC), denngd(kNCELL * 2);
    drv::launch(drv::cdiv(kNCELL, 128), 1, 1, 128, [&] {
        r_aeru::aer_trop_fill(midx, mcmix, mkprf, mdenn, idxcg.data(), cmixd.data(), denngd.data(), kprfg.data());
    });
    FV cmixg(cmixd.begin(), cmixd.end()), denng(denngd.begin(), denngd.end());
    if (tab) {
        float* o = tab;
        auto put = [&](const FV& a) { std::copy(a.begin(), a.end(), o); o += a.size(); };
        put(sigref); put(extrhi); put(scarhi); put(ssarhi); put(asyrhi); put(extrhd); put(scarhd); put(ssarhd);
        put(asyrhd); put(extstra); put(solbnd); put(eirbnd); put(cmixg); put(denng);
        for (int v : idxcg) *o++ = (float)v;
        for (int v : kprfg) *o++ = (float)v;
    }
    if (ncol <= 0) return 0;
    const int nlp1 = nlay + 1;
    FV alon(ncol), alat(ncol), dz((size_t)nlay * ncol), hz((size_t)nlp1 * ncol);
    drv::launch(drv::cdiv(ncol, 128), 1, 1, 128, [&] {
        r_seta::phys_rrtm_setaer_prep(plvl, plyr, tlyr, qlyr, xlon, xlat, alon.data(), alat.data(), dz.data(),
                                      hz.data(), ncol, nlay, nlp1, ivflip, 1);
    });
    const size_t nsw = (size_t)3 * kNSW * nlay * ncol, nlw = (size_t)3 * kNLW * nlay * ncol;
    drv::launch(1, 1, 1, 1, [&] { r_seta::phys_rrtm_setaer_zero(aerosw, aerolw, nsw, nlw); });
    const float rhlev[8] = {0.0f, 0.5f, 0.7f, 0.8f, 0.9f, 0.95f, 0.98f, 0.99f};
    drv::launch(drv::cdiv(ncol, 128), 1, 1, 128, [&] {
        r_aerp::phys_rrtm_aer_property_column(plvl, dz.data(), hz.data(), rhly, alon.data(), alat.data(), slmsk, haer,
                                              prsref, sigref.data(), rhlev, extrhi.data(), scarhi.data(),
                                              ssarhi.data(), asyrhi.data(), extrhd.data(), scarhd.data(),
                                              ssarhd.data(), asyrhd.data(), extstra.data(), cmixg.data(),
                                              denng.data(), idxcg.data(), kprfg.data(), aerosw, aerolw, ncol, 1, nlay,
                                              1, 1, ivflip, kNSW, kNLW, kNBT);
    });
    return 0;
}

// The NAM orientation (ivflip 0, levels top first) of orc_aerosols_iv; same signature as the oracle's orc_aerosols.
int orc_aerosols(const int* iendwv, const float* haer, const float* prsref, const float* rhid, const float* rhdp,
                 const float* straext0, const int* nwvns0, const float* s0intv, const int* midx, const double* mcmix,
                 const int* mkprf, const double* mdenn, int nlay, int ncol, const float* plvl, const float* plyr,
                 const float* tlyr, const float* qlyr, const float* rhly, const float* xlon, const float* xlat,
                 const float* slmsk, float* aerosw, float* aerolw, float* tab)
{
    return orc_aerosols_iv(iendwv, haer, prsref, rhid, rhdp, straext0, nwvns0, s0intv, midx, mcmix, mkprf, mdenn, nlay,
                           ncol, plvl, plyr, tlyr, qlyr, rhly, xlon, xlat, slmsk, aerosw, aerolw, tab, 0);
}

// The volcanic term from the reference's kernels: phys_rrtm_setaer_prep for alat (do_dz 0), then
// phys_rrtm_setaer_volc with year mod(kyrsav, 10) + 1 and month kmonsav as phys_rrtm_setaer.py:178-192 passes
// them.  Same signature as the oracle's orc_setaer_volc.
int orc_setaer_volc(int nlay, int ncol, int ivflip, const float* plvl, const float* xlat, const int* ivolae,
                    int kyrsav, int kmonsav, int add_sw, int add_lw, int lw1bd, float* aerosw, float* aerolw)
{
    if (nlay < 4 || ncol < 0 || kmonsav < 1 || kmonsav > 12) return 1;
    if (ncol == 0) return 0;
    const int year1 = ((kyrsav % 10) + 10) % 10 + 1;
    std::vector<float> zero((size_t)(nlay + 1) * ncol, 0.0f), xlon(ncol, 0.0f), alon(ncol), alat(ncol);
    drv::launch(drv::cdiv(ncol, 128), 1, 1, 128, [&] {
        r_seta::phys_rrtm_setaer_prep(plvl, zero.data(), zero.data(), zero.data(), xlon.data(), xlat, alon.data(),
                                      alat.data(), nullptr, nullptr, ncol, nlay, nlay + 1, ivflip, 0);
    });
    drv::launch(drv::cdiv(ncol, 128), 1, 1, 128, [&] {
        r_seta::phys_rrtm_setaer_volc(aerosw, aerolw, plvl, alat.data(), ivolae, ncol, nlay, ivflip, year1, kmonsav,
                                      add_sw, add_lw, lw1bd);
    });
    return 0;
}

// grrad's condensate from the reference's kernel grrad_clouds_clw (phys_rrtm_grrad_clouds.py:183-193), one row of n
// columns.  Same signature as the oracle's orc_grrad_clw.
int orc_grrad_clw(int n, int lmk, const float* tracer, int ntcw0, int ncld, float epsq, float* clw)
{
    if (n <= 0) return 0;
    drv::launch(drv::cdiv(n, 128), 1, lmk, 128, [&] {
        r_grcl::grrad_clouds_clw(tracer, clw, n, 1, lmk, ntcw0, ncld, epsq);
    });
    return 0;
}

// grrad's IALB = 2 block from the reference's kernel grrad_clouds_albedo (phys_rrtm_grrad_clouds.py:230-245), with
// its own built-in tables (the table arguments are not read).  Same signature as the oracle's orc_payne_albedo.
int orc_payne_albedo(int n, const float* salbedo, const float* sm, const float* coszen, const float* trn,
                     const float* za, const float* dza, const float* albd, float* out)
{
    (void)trn; (void)za; (void)dza; (void)albd;
    if (n <= 0) return 0;
    float* o[9];
    for (int f = 0; f < 9; ++f) o[f] = out + (size_t)f * n;
    drv::launch(drv::cdiv(n, 128), 1, 1, 128, [&] {
        r_grcl::grrad_clouds_albedo(salbedo, sm, coszen, o[0], o[1], o[2], o[3], o[4], o[5], o[6], o[7], o[8], n, 1);
    });
    return 0;
}

// Solar geometry from the reference's kernels sol_update_nmmb (phys_rrtm_sol_update.py: one thread) and
// phys_rrtm_coszmn (phys_rrtm_coszmn.py:51-67, one row of n columns).  Same signature as the oracle's.
int orc_solar(const int* date, float deltsw, float deltim, double solc0, float* state, int* nstp, int n,
              const float* glon, const float* glat, float solhr, float dtswav, int nrads, float* coszen, float* coszdg)
{
    float out[4], st[4];
    drv::launch(1, 1, 1, 1, [&] {
        r_solu::sol_update_nmmb(date[0], date[1], date[2], date[3], date[4], date[5], deltsw, deltim, &solc0, out, st,
                                nstp);
    });
    state[0] = st[0]; state[1] = st[1]; state[2] = st[2]; state[3] = st[3]; state[4] = out[3];
    if (n > 0)
        drv::launch(drv::cdiv(n, 128), 1, 1, 128, [&] {
            r_cosz::phys_rrtm_coszmn(glon, glat, coszen, coszdg, solhr, dtswav, nrads, st, n, 1);
        });
    return 0;
}

// grrad's radiation-layer set-up from the reference's kernels rrtm_grrad_setup (phys_rrtm_grrad_setup.py: one
// tracer, np3d 0, ntoz 0, ivflip 0) then phys_rrtm_grrad_gases (ivflip 0), one row of n columns.  Same
// signature as the oracle's orc_grrad_setup.
int orc_grrad_setup(int lm, int n, const float* pint, const float* pmid, const float* prslk, const float* t,
                    const float* q, const float* tsfc, float* out)
{
    const int lmk = lm + 1, lmp = lm + 2;
    const size_t L = (size_t)lmk * n, P = (size_t)lmp * n, M = (size_t)lm * n;
    float *plvl = out, *plyr = plvl + P, *tlyr = plyr + L, *tlvl = tlyr + L, *qlyr = tlvl + P, *rhly = qlyr + L,
          *qstl = rhly + L, *prslk1 = qstl + L, *tvly = prslk1 + L, *tsfg = tvly + L;
    std::vector<float> tracer(M, 0.0f), cldf(M, 0.0f), dum(M, 0.0f), cldfk1(L), tracer1(L), gdum(L), olyr(L), tskn(n),
        tem2da(L), tem2db(P), tsfa(n);
    drv::launch(drv::cdiv(n, 128), 1, 1, 128, [&] {
        r_grs::rrtm_grrad_setup(pint, pmid, prslk, t, q, tracer.data(), cldf.data(), dum.data(), dum.data(), dum.data(),
                                tsfc, plvl, plyr, tlyr, prslk1, rhly, qstl, cldfk1.data(), tracer1.data(), gdum.data(),
                                gdum.data(), gdum.data(), olyr.data(), tskn.data(), tsfg, qlyr, tvly, n, 1, lm, 1, 0, 0,
                                0);
    });
    drv::launch(drv::cdiv(n, 128), 1, 1, 128, [&] {
        r_grg::phys_rrtm_grrad_gases(plyr, plvl, tlyr, tskn.data(), t, q, tlvl, tvly, qlyr, tem2da.data(),
                                     tem2db.data(), tsfa.data(), n, 1, lm, 0);
    });
    return 0;
}

// ---- grrad's front end from the reference's kernels, one row of n columns (jm = 1, im = n) except DAYPARTS,
// which takes its rows as they are.  Same signatures as the oracle's. ----

// DAYPARTS (phys_rrtm_dayparts.py:67-105): the per-point kernel, the inclusive scan of the run starts (a library
// cumsum in the reference, a host prefix sum here), then the scatter and length kernels.
int orc_dayparts(int im, int jm, const float* xlon, const float* sinlat, const float* coslat, float solhr, float dtswav,
                 int nrads, const float* sol, float* coszen, float* coszdg, int* dp_start, int* dp_len, int* dp_day,
                 int* ndayparts)
{
    const int n = im * jm;
    std::vector<int> day(n), start(n), scan(n);
    const float st[4] = {sol[0], sol[1], sol[2], 0.0f};
    drv::launch(drv::cdiv(n, 128), 1, 1, 128, [&] {
        r_dayp::phys_rrtm_dayparts_cosz(xlon, sinlat, coslat, solhr, dtswav, nrads, st, n, im, coszen, coszdg,
                                        day.data(), start.data());
    });
    int acc = 0;
    for (int p = 0; p < n; ++p) scan[p] = (acc += start[p]);
    drv::launch(drv::cdiv(n, 128), 1, 1, 128, [&] {
        r_dayp::phys_rrtm_dayparts_scatter(start.data(), scan.data(), day.data(), n, im, dp_start, dp_day);
    });
    drv::launch(drv::cdiv(n, 128), 1, 1, 128, [&] {
        r_dayp::phys_rrtm_dayparts_len(dp_start, scan.data(), n, im, dp_len, ndayparts);
    });
    return 0;
}

int orc_getgases(int n, int lmax, const float* plvl, const float* xlon, const float* xlat, float co2_glb,
                 const float* gco2cyc, const float* co2vmr_sav, int ico2flg, int kmonsav, int ivflip, float* gasvmr)
{
    drv::launch(drv::cdiv(n, 128), 1, 1, 128, [&] {
        r_ggas::phys_rrtm_getgases(plvl, xlon, xlat, &co2_glb, gco2cyc, co2vmr_sav, gasvmr, n, 1, lmax, ico2flg,
                                   kmonsav, ivflip);
    });
    return 0;
}

int orc_getozn(int n, int nlev, const float* prslk, const float* xlat, const float* o3r, const float* pkstr, int jmr,
               int loz, int k1oz, int k2oz, float facoz, float blte, float dlte, int ivflip, float* o3mmr)
{
    drv::launch(drv::cdiv(n, 128), 1, 1, 128, [&] {
        r_gozn::phys_rrtm_getozn(prslk, xlat, o3r, pkstr, o3mmr, n, 1, nlev, jmr, loz, k1oz, k2oz, facoz, blte, dlte,
                                 ivflip);
    });
    return 0;
}

int orc_setalb(int n, const float* const* f, int ialbflg, float* sfcalb)
{
    drv::launch(drv::cdiv(n, 128), 1, 1, 128, [&] {
        r_salb::phys_rrtm_setalb(f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9], f[10], f[11], f[12], f[13],
                                 f[14], f[15], ialbflg, n, 1, sfcalb);
    });
    return 0;
}

int orc_setemis(int n, const float* const* f, const int* idxems, int ialbflg, int iemslw, float* sfcemis)
{
    const int flags[3] = {ialbflg, iemslw, iemslw};
    drv::launch(drv::cdiv(n, 128), 1, 1, 128, [&] {
        r_sems::phys_rrtm_setemis(f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], idxems, flags, sfcemis, n, 1);
    });
    return 0;
}

int orc_progcld2(int n, int nlay, const float* const* f, const int* cfg, float* clouds, float* clds, int* mtop,
                 int* mbot)
{
    drv::launch(drv::cdiv(n, 128), 1, 1, 128, [&] {
        r_pc2::phys_rrtm_progcld2_column(n, 1, nlay, cfg[0], cfg[1], cfg[2], cfg[3], cfg[4], cfg[5], cfg[6], cfg[7],
                                         f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8], f[9], f[10], f[11], f[12],
                                         clouds, clds, mtop, mbot);
    });
    return 0;
}
}
