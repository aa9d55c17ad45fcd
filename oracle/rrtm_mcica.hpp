// rrtm_mcica.hpp -- CPU oracle: McICA route (sub-column cloud generators and the per-g-point solvers).
// Filled in with the McICA restatement; the NAM route does not use it.
#pragma once
#include "rrtm_lw.hpp"
#include "rrtm_sw.hpp"

namespace orc {
template <class R>
void lw_mcica(LwColumn<R>&, const float*, int, const Config&, const Inputs&, int, unsigned int*)
{
    throw std::runtime_error("oracle: McICA route not built");
}
template <class R>
void lw_rtrnmc(LwColumn<R>&, const LwTables<R>&, R, R) { throw std::runtime_error("oracle: McICA route not built"); }
template <class R>
void sw_mcica(SwColumn<R>&, const Config&, const Inputs&, int, unsigned int*)
{
    throw std::runtime_error("oracle: McICA route not built");
}
template <class R>
void sw_spcvrtm(SwColumn<R>&, const SwExpTable<R>&, int) { throw std::runtime_error("oracle: McICA route not built"); }
}  // namespace orc
