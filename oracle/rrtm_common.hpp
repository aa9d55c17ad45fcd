// rrtm_common.hpp -- shared pieces of the CPU oracle (test infrastructure only).
//
// The oracle is a plain, serial, one-column-at-a-time restatement of the reference's RRTM LW/SW column
// radiation (WOOF-NAM namgpu/kernels/phys_rrtm_*.cu), templated on the arithmetic type so that the same
// statements run in float (to pin against the reference's own kernels compiled for the host) and in
// double (the FP64 error oracle).  It is never linked into the product library.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>
#include <algorithm>
#include <cstdio>
#include <limits>
#include <type_traits>

namespace orc {

// Named table store: every table is held as double (exact promotion of the float32 values the
// reference uses) and read as the arithmetic type R.
struct TableStore {
    std::map<std::string, std::vector<double>> t;
    std::map<std::string, std::vector<int>> ti;
    const double* f(const std::string& name) const {
        auto it = t.find(name);
        if (it == t.end()) throw std::runtime_error("oracle: missing table " + name);
        return it->second.data();
    }
    bool has(const std::string& name) const { return t.count(name) != 0; }
    const int* i(const std::string& name) const {
        auto it = ti.find(name);
        if (it == ti.end()) throw std::runtime_error("oracle: missing int table " + name);
        return it->second.data();
    }
};

TableStore& tables();

// Reference constants (physcons.f values as the reference kernels carry them).
constexpr double CON_G = 9.80665;
constexpr double CON_AVGD = 6.0221415e23;
constexpr double CON_AMD = 28.9644;
constexpr double CON_AMW = 18.0154;
constexpr double CON_AMO3 = 47.9982;
constexpr double CON_CP = 1.0046e3;

constexpr int NBDLW = 16, NGPTLW = 140;
constexpr int NBDSW = 14, NGPTSW = 112;
constexpr int LW_NG[16] = {10, 12, 16, 14, 16, 8, 12, 8, 12, 6, 8, 8, 4, 2, 2, 2};
constexpr int LW_NS[16] = {0, 10, 22, 38, 52, 68, 76, 88, 96, 108, 114, 122, 130, 134, 136, 138};
constexpr int SW_NG[14] = {6, 12, 8, 8, 10, 10, 2, 10, 8, 6, 6, 8, 6, 12};
constexpr int SW_NS[14] = {0, 6, 18, 26, 34, 44, 54, 56, 66, 74, 80, 86, 94, 100};

// fmin/fmax with the IEEE minNum/maxNum rule of CUDA's fminf/fmaxf (a NaN operand yields the other one).
template <class R> inline R fminR(R a, R b) { return std::fmin(a, b); }
template <class R> inline R fmaxR(R a, R b) { return std::fmax(a, b); }
inline int imin(int a, int b) { return a < b ? a : b; }
inline int imax(int a, int b) { return a > b ? a : b; }

// Fortran mod(a, 1.0) for a >= 0.
template <class R> inline R fmod1(R a) { return std::fmod(a, R(1)); }

// Elementary functions of the arithmetic type (the operation counter overloads them for its type).
template <class R> inline R mexp(R a) { return std::exp(a); }
template <class R> inline R mlog(R a) { return std::log(a); }
template <class R> inline R msqrt(R a) { return std::sqrt(a); }
template <class R> inline R mfabs(R a) { return std::fabs(a); }
template <class R> inline R mpow(R a, R b) { return std::pow(a, b); }

// Solve configuration (the reference's NAM runtime switches unless stated).
struct Config {
    int iswmode = 2;          // SW two-stream: 1 delta-Eddington, 2 PIFM (NAM), 3 discrete ordinates
    int diagnostic = 0;       // 1: cloud optics given directly (ilwcliq = iswcliq = 0)
    double cpathfac = 1.5;    // LW cloud-path factor applied before lwrad (prognostic clouds only)
    int window_cols = 0;      // SW MINVAL(laytrop) window in columns (0 = the whole request)
    int sw_chunk = 32768;     // SW day-column chunk (groups restart at each chunk)
    int route = 0;            // 0 NAM (rtrnmr + spcvrtc), 1 McICA
    int iovrlw = 1, iovrsw = 1;
    int lw_seed0 = 140, sw_seed0 = 1;   // McICA permutation seed offsets (ipsdlw0 / ipsdsw0)
};

// Column inputs in the reference's [field][level][ncol] float32 layout, level 0 = model top.
struct Inputs {
    const float *plyr, *plvl, *tlyr, *tlvl, *qlyr, *olyr, *gasvmr, *clouds;
    const float *faerlw, *faersw;     // may be null: no aerosol
    const float *sfcemis, *tsfg, *sfcalb, *coszen;
    const int* icseed;                // may be null
    double solcon;
    int nlay, ncol;
};

// Outputs in double, [field][level][ncol] or [field][ncol].
struct Outputs {
    double *htlw, *htsw;              // [nlay][ncol] K/s, level 0 = model top
    double *topflw;                   // [2][ncol] upfxc, upfx0
    double *sfcflw;                   // [4][ncol] upfxc, upfx0, dnfxc, dnfx0
    double *topfsw;                   // [3][ncol] upfxc, dnfxc, upfx0
    double *sfcfsw;                   // [4][ncol] upfxc, dnfxc, upfx0, dnfx0
    double *fdncmp;                   // [6][ncol] uvbf0, uvbfc, nirbm, nirdf, visbm, visdf (may be null)
    double *lwflx;                    // optional [4][nlay+1][ncol] up/dn total, up/dn clear (top first)
    double *swflx;                    // optional [4][nlay+1][ncol] up/dn total, up/dn clear (top first)
    unsigned int* lw_mask;            // optional McICA masks [5][nlay][ncol]
    unsigned int* sw_mask;            // optional McICA masks [4][nlay][ncol]
    double* hlw0 = nullptr;           // optional [nlay][ncol] LW clear-sky heating, K/s (lhlw0)
    double* hlwb = nullptr;           // optional [16][nlay][ncol] LW heating per band (lhlwb)
    double* hsw0 = nullptr;           // optional [nlay][ncol] SW clear-sky heating (lhsw0)
    double* htswb = nullptr;          // optional [14][nlay][ncol] SW heating per band (lhswb)
};

}  // namespace orc
