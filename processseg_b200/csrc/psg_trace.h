// psg_trace.h — what the host side of libpsgcuda.so needs of the float32
// trace kernels (psg_trace.cuh, instantiated in psg_trace_f32.cu): the
// compile-time transform plans they are built for.
#pragma once

namespace psg {

// A trace-kernel build: the transform length m (complex points), the CTA
// width, the radices in pass order, the AGC's samples per lane E (it takes
// windows w ≤ 32·E with pipeline_kernel's choice of E), and the kernels by
// recipe (0: demean, filter, AGC; 1: then a per-trace normalization) and by
// the next-row prefetch.
struct TracePlanInfo {
  int m, nt, np;
  int radix[8];
  // the trace kernels' passes as the reference's stages: pass i runs stage
  // g1[i] then, when g2[i] > 0, stage g2[i] (radix[i] = g1[i]·max(g2[i], 1))
  int g1[8], g2[8];
  int agc_e;
  int min_blocks;            // the CTAs per SM its launch bounds ask for
  int buf;                   // complex elements of each of its two transform buffers
  const void* kernel[2][2];  // [recipe][prefetch]; nullptr where not built
  // [recipe]: the request loop's kernel over many requests' rows (the
  // prefetch form; nullptr where not built)
  const void* batch[2];
};

// The builds for transform length m whose E serves AGC window w, in the
// order the tuner tries them (nullptr-terminated; empty when none).
const TracePlanInfo* const* trace_plans_for(int m, int w);
// The float32 correlation kernels for transform length m (kernel[0][0];
// nullptr-terminated; empty when none).
const TracePlanInfo* const* corr_plans_for(int m);

// pipeline_kernel's AGC samples per lane for window w (1, 3, 5 or 9; beyond
// 288 samples its block sums run in chunks, which the trace kernel does not).
inline int agc_lane_samples(int w) { return w <= 32 ? 1 : w <= 96 ? 3 : w <= 160 ? 5 : 9; }

}  // namespace psg
