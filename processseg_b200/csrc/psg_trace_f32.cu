// psg_trace_f32.cu — the host's table of the float32 trace kernels
// (psg_trace.cuh) by transform length and AGC lane width, the builds of each
// length in their own units (psg_trace_m*.cu) so they compile in parallel:
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

const TracePlanInfo* const* trace_builds_m1944_e5();
const TracePlanInfo* const* trace_builds_m1125_e9();
const TracePlanInfo* const* trace_builds_m3375_e9();

namespace {

// correlation: nfft 16200 (20 s records at 2 ms with a 12 s sweep); the two
// transform buffers (129.6 KB) leave one CTA per SM
using P8100 = tk::FPlan<8100, 512, 1, 9, 9, 10, 10>;
const TracePlanInfo k8100 = tk::corr_info<P8100>();
const TracePlanInfo* const c8100[] = {&k8100, nullptr};
const TracePlanInfo* const none[] = {nullptr};

}  // namespace

const TracePlanInfo* const* trace_plans_for(int m, int w) {
  const int e = agc_lane_samples(w);
  if (w > 32 * e) return none;
  if (m == 1944 && e == 5) return trace_builds_m1944_e5();
  if (m == 1125 && e == 9) return trace_builds_m1125_e9();
  if (m == 3375 && e == 9) return trace_builds_m3375_e9();
  return none;
}

const TracePlanInfo* const* corr_plans_for(int m) { return m == 8100 ? c8100 : none; }

}  // namespace psg
