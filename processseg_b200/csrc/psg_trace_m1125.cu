// psg_trace_m1125.cu — trace-kernel builds for m = 1125 (nfft 2250): traces
// of up to 2250 samples, e.g. 48 × 2001 at 2 ms with a band-pass and a 500 ms
// AGC (w = 251, E = 9). The reference's stages 3, 3, 5, 5, 5 grouped into
// passes; every build rounds as those stages do (same bits).
#include "psg_trace.cuh"

namespace psg {
namespace {

using tk::Grp;
// 3·3 | 5·5 | 5: three passes, few butterflies per pass (throughput form)
using A = tk::RPlan<1125, 256, 3, Grp<3, 3>, Grp<5, 5>, Grp<5>>;
// one stage per pass over 512 threads: 375 or 225 butterflies a pass, each
// thread one at most (the latency form for panels of a few dozen traces;
// demean, filter, AGC only)
using B = tk::RPlan<1125, 512, 1, Grp<3>, Grp<3>, Grp<5>, Grp<5>, Grp<5>>;
// 3·3 | 5 | 5 | 5 over 256 threads
using C = tk::RPlan<1125, 256, 3, Grp<3, 3>, Grp<5>, Grp<5>, Grp<5>>;

const TracePlanInfo a = tk::info_served<A, 9>();
const TracePlanInfo b = tk::info<B, 9>();
const TracePlanInfo c = tk::info<C, 9>();
const TracePlanInfo* const builds[] = {&a, &b, &c, nullptr};

}  // namespace

const TracePlanInfo* const* trace_builds_m1125_e9() { return builds; }

}  // namespace psg
