// psg_trace_m1944.cu — trace-kernel builds for m = 1944 (nfft 3888): traces
// of 2001..3888 samples, e.g. 2000 × 3001 at 2 ms with a band-pass + notch and
// a 300 ms AGC (w = 151, E = 5). The reference's stages 4, 2, 3, 3, 3, 3, 3
// (fft/plan.nim:120-132) grouped into passes three ways; every build rounds
// as those stages do, so they give the same bits and the tuner picks by time.
#include "psg_trace.cuh"

namespace psg {
namespace {

using tk::Grp;
// 4 | 2·3 | 3·3 | 3·3: more butterflies in the first pass, four CTAs per SM
// (64 registers); the fastest on a 2000 × 3001 panel, so the first (untuned)
// build and the request loop's
using A = tk::RPlan<1944, 256, 4, Grp<4>, Grp<2, 3>, Grp<3, 3>, Grp<3, 3>>;
// 4·2 | 3·3 | 3·3 | 3, four CTAs per SM
using B = tk::RPlan<1944, 256, 4, Grp<4, 2>, Grp<3, 3>, Grp<3, 3>, Grp<3>>;
// the same passes with 85 registers (three CTAs per SM, no spills)
using C = tk::RPlan<1944, 256, 3, Grp<4, 2>, Grp<3, 3>, Grp<3, 3>, Grp<3>>;
// over 512 threads, two CTAs per SM (64 registers): half the latency of a
// trace for the last rows of a panel and for small panels (demean, filter,
// AGC only); 4 | 2·3 | 3·3 | 3·3, and 4 | 2 | 3·3 | 3·3 | 3 with more
// butterflies in the later passes
using D = tk::RPlan<1944, 512, 2, Grp<4>, Grp<2, 3>, Grp<3, 3>, Grp<3, 3>>;
using F = tk::RPlan<1944, 512, 2, Grp<4>, Grp<2>, Grp<3, 3>, Grp<3, 3>, Grp<3>>;

// A with 48 registers: five CTAs per SM when the row shares the first
// transform buffer
using G = tk::RPlan<1944, 256, 5, Grp<4>, Grp<2, 3>, Grp<3, 3>, Grp<3, 3>>;

const TracePlanInfo a = tk::info_served<A, 5>();
const TracePlanInfo b = tk::info<B, 5>();
const TracePlanInfo c = tk::info<C, 5>();
const TracePlanInfo d = tk::info<D, 5>();
const TracePlanInfo f = tk::info<F, 5>();
const TracePlanInfo g = tk::info<G, 5>();
const TracePlanInfo* const builds[] = {&a, &b, &c, &d, &f, &g, nullptr};

}  // namespace

const TracePlanInfo* const* trace_builds_m1944_e5() { return builds; }

}  // namespace psg
