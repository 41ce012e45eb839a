// psg_trace_f32.cu — the float32 trace kernels (psg_trace.cuh) for the
// transform lengths of the benchmarked panels, each with the radices and
// AGC lane width its panels use, and the host's table of them.
//   m = 1944 (nfft 3888): 2000 × 3001 at 2 ms, band-pass 3/6/70/90 + notch,
//     AGC 300 ms (w = 151, E = 5)
//   m = 1125 (nfft 2250): 48 × 2001 at 2 ms, band-pass 4/8/60/80, AGC 500 ms
//     (w = 251, E = 9)
//   m = 3375 (nfft 6750): 50000 × 6001 at 1 ms, band-pass 2/5/120/150,
//     AGC 250 ms (w = 251, E = 9), then a per-trace p99 normalization
// and the float32 correlation kernel for m = 8100 (nfft 16200: records of
// 10001 samples at 2 ms against a 12 s sweep).
#include "psg_trace.cuh"

namespace psg {
namespace {

template <class P, int E> TracePlanInfo info() {
  TracePlanInfo t{};
  t.m = P::M;
  t.nt = P::NT;
  t.np = P::NP;
  for (int i = 0; i < P::NP; i++) {
    t.radix[i] = P::radix(i);
    t.g1[i] = P::G1[i];
    t.g2[i] = P::G2[i];
  }
  t.agc_e = E;
  t.min_blocks = P::MINB;
  t.buf = P::BUF;
  t.kernel[0][0] = (const void*)tk::trace_kernel<P, RC_DFA, false, E>;
  t.kernel[0][1] = (const void*)tk::trace_kernel<P, RC_DFA, true, E>;
  t.kernel[1][0] = (const void*)tk::trace_kernel<P, RC_DFAN, false, E>;
  t.kernel[1][1] = (const void*)tk::trace_kernel<P, RC_DFAN, true, E>;
  return t;
}

template <class P> TracePlanInfo corr_info() {
  TracePlanInfo t{};
  t.m = P::M;
  t.nt = P::NT;
  t.np = P::NP;
  for (int i = 0; i < P::NP; i++) {
    t.radix[i] = P::radix(i);
    t.g1[i] = P::radix(i);
  }
  t.min_blocks = P::MINB;
  t.buf = P::M;
  t.kernel[0][0] = (const void*)tk::corr_trace_kernel<P>;
  return t;
}

// the reference's stages (4s, a 2, 3s, 5s), two per pass
using tk::Grp;
using P1944 = tk::RPlan<1944, 256, 4, Grp<4, 2>, Grp<3, 3>, Grp<3, 3>, Grp<3>>;
// correlation: nfft 16200 (20 s records at 2 ms with a 12 s sweep); the two
// transform buffers (129.6 KB) leave one CTA per SM
using P8100 = tk::FPlan<8100, 512, 1, 9, 9, 10, 10>;
const TracePlanInfo k8100 = corr_info<P8100>();
const TracePlanInfo* const c8100[] = {&k8100, nullptr};
using P1125 = tk::RPlan<1125, 256, 3, Grp<3, 3>, Grp<5, 5>, Grp<5>>;
using P3375 = tk::RPlan<3375, 256, 3, Grp<3, 3>, Grp<3, 5>, Grp<5, 5>>;

const TracePlanInfo k1944e5 = info<P1944, 5>();
const TracePlanInfo k1125e9 = info<P1125, 9>();
const TracePlanInfo k3375e9 = info<P3375, 9>();

const TracePlanInfo* const t1944e5[] = {&k1944e5, nullptr};
const TracePlanInfo* const t1125e9[] = {&k1125e9, nullptr};
const TracePlanInfo* const t3375e9[] = {&k3375e9, nullptr};
const TracePlanInfo* const none[] = {nullptr};

}  // namespace

const TracePlanInfo* const* trace_plans_for(int m, int w) {
  const int e = agc_lane_samples(w);
  if (w > 32 * e) return none;
  if (m == 1944 && e == 5) return t1944e5;
  if (m == 1125 && e == 9) return t1125e9;
  if (m == 3375 && e == 9) return t3375e9;
  return none;
}

const TracePlanInfo* const* corr_plans_for(int m) { return m == 8100 ? c8100 : none; }

}  // namespace psg
