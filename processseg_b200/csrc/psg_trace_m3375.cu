// psg_trace_m3375.cu — trace-kernel builds for m = 3375 (nfft 6750): traces
// of up to 6750 samples, e.g. 50000 × 6001 at 1 ms with a band-pass, a 250 ms
// AGC (w = 251, E = 9) and a per-trace p99 normalization. The reference's
// stages 3, 3, 3, 5, 5, 5 grouped into passes; every build rounds as those
// stages do (same bits). The row (24 KB) and the two transform buffers
// (54 KB) leave two CTAs per SM, so the builds ask for two: 128 registers.
#include "psg_trace.cuh"

namespace psg {
namespace {

using tk::Grp;
// 3·3 | 3·5 | 5·5
using A = tk::RPlan<3375, 256, 2, Grp<3, 3>, Grp<3, 5>, Grp<5, 5>>;
// 3·3 | 3 | 5·5 | 5
using B = tk::RPlan<3375, 256, 2, Grp<3, 3>, Grp<3>, Grp<5, 5>, Grp<5>>;

// A with 85 registers: three CTAs per SM when the row shares the first
// transform buffer (the launch shape that has no row buffer of its own)
using C = tk::RPlan<3375, 256, 3, Grp<3, 3>, Grp<3, 5>, Grp<5, 5>>;

const TracePlanInfo a = tk::info_served<A, 9>();
const TracePlanInfo b = tk::info<B, 9>();
const TracePlanInfo c = tk::info<C, 9>();
const TracePlanInfo* const builds[] = {&a, &b, &c, nullptr};

}  // namespace

const TracePlanInfo* const* trace_builds_m3375_e9() { return builds; }

}  // namespace psg
