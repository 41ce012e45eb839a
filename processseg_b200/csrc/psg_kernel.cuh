// psg_kernel.cuh — the fused pipeline kernel of libpsgcuda.so and its steps.
//
// One kernel per plan part (pipeline_kernel): each CTA takes a trace, loads
// its live samples from HBM into shared memory once, runs every step of the
// part on it there (demean/detrend/scale/clip/polarity, the zero-phase FFT
// filter with its trend removal, padding and trend add-back, AGC with block
// prefix/suffix sums in float64, per-trace normalization with an exact radix
// selection, gain curves), and writes the trace back once. src → dst copies
// of dead rows and of samples past the live length ride in the same kernel.
//
// The kernel's instantiations live in psg_pipe_f32.cu and psg_pipe_f64.cu
// (compiled in parallel); the host side reaches them through
// pipe_kernel_f32 / pipe_kernel_f64.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "psg_device.cuh"
#include "psg_internal.h"

namespace psg {
using namespace psgd;

// The pipeline kernels' CTA width (every launch of them uses it), a
// compile-time constant so that the trace loops' strides and offsets are too.
constexpr int kNT = 256;

// ============================================================ device plan
struct DevStep {
  int kind, trend, reflect, zero_dc;
  int agc_mode, stat, pad, nfft;
  int half, table_len, need, need_next;
  double factor, lo, hi, dc_gain, target, epsilon, norm_target, percentile, t_min_ms, dt_ms;
  FftDesc fft;
  const void* bridge;  // Quad<T>[m]: the split · gain · unsplit map of each bin pair
  const void* fall;
  const void* tw;
  // the trace kernel's split twiddles (float4 per bin pair: bins c and m − c)
  // and bin gains (float2 per bin pair), and 1/nfft in float32
  const void* ref_split;
  const void* ref_gain;
  float ref_scale, _pad3;
  const void* table;
  psg_gain_curve curve;
  // mutes: the curve (knots: |offset| knots then their times) and the taper
  int mute_kind, n_knots;
  double mute_t, ms_per_dist, mute_t0, mute_pad, taper_ms;
  const double* knots;
  // IIR filter: sections (b0, b1, b2, a1, a2, g each), zero phase or
  // minimum, the pads before and after the data, G'(1) (trend, reflect and
  // dc_gain as the FFT filter's)
  int n_sec, iir_zero, lead, tail;
  double dc_slope;
  const double* sec;
  // per section and chunk length L = 1 .. pw_len: (M^L)^k, k = 1 .. 32,
  // 2×2 in double-double (kIirTab doubles)
  const double* pw;
  int pw_len, _pad2;
};

// One apply: a block of rows and the plan steps of one part.
struct Job {
  const void* src;  // NULL or == dst: in place
  void* dst;
  const int* live;
  const double* start_ms;
  const DevStep* steps;
  long long rows;
  int cols, first, last;
  int first_sample;        // the block's first sample of the trace (mutes)
  const double* offset;    // per row: the trace's offset (mutes; NULL: NaN)
  const double* t0_ms;     // per row: the trace's t0Ms (mutes; NULL: NaN)
  double dt_ms;            // the rows' sample interval
};

struct PipeArgs {
  Job job;                     // the apply (single-job launches)
  const Job* jobs;             // batched launches: the jobs, and the first
  const long long* row_begin;  // global row of each (ascending)
  int njobs;
  long long total_rows;
  const double* factor;  // the part's panel factor (NaN: none) or NULL
  int work_off;          // byte offset of the work area
  int x_bytes;           // bytes of one row buffer (two of them with the bulk prefetch)
  int* status;           // set to 1 when a bounded wait gives up
  // Traces whose FFT buffers do not fit beside the row in shared memory:
  // each CTA's work area is its own slice of global memory (mostly
  // L2-resident), gwork + blockIdx.x · gwork_stride.
  unsigned char* gwork;
  long long gwork_stride;
  // the trace kernel's twiddles, pass by pass, for the build launched
  // (psg_trace.cuh; its passes group the stages their own way)
  const void* tw_pass;
};

// ----------------------------------------------------------- device helpers
__device__ __forceinline__ bool fin_pos_d(double x) { return isfinite(x) && x > 0; }
template <class T> __device__ __forceinline__ bool fits_d(double x) {
  if (!fin_pos_d(x)) return false;
  double y = (double)(T)x;
  return isfinite(y) && y > 0;
}

// The k-th smallest |x| (0-based) as its bits, by an 8-bit radix selection
// over the bit patterns in shared memory.
template <class T>
__device__ unsigned long long select_kth(const T* X, int n, int k, unsigned* hist, int* sh) {
  unsigned long long prefix = 0, mask = 0;
  int kk = k;
  for (int shift = (int)sizeof(T) * 8 - 8; shift >= 0; shift -= 8) {
    for (int i = threadIdx.x; i < 256; i += kNT) hist[i] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += kNT) {
      unsigned long long key = abs_bits(X[i]);
      if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      int lane = threadIdx.x;
      unsigned c[8], tot = 0;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        c[j] = hist[lane * 8 + j];
        tot += c[j];
      }
      unsigned incl = tot;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        unsigned u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
      }
      unsigned excl = incl - tot;
      if ((unsigned)kk >= excl && (unsigned)kk < incl) {
        unsigned below = excl;
        int d = 0;
        for (; d < 8; d++) {
          if ((unsigned)kk < below + c[d]) break;
          below += c[d];
        }
        sh[0] = lane * 8 + d;
        sh[1] = kk - (int)below;
        sh[2] = (int)(c[d] - (unsigned)(kk - (int)below));  // this bucket's keys at rank k and above
      }
    }
    __syncthreads();
    prefix |= (unsigned long long)sh[0] << shift;
    mask |= 255ull << shift;
    kk = sh[1];
    __syncthreads();
  }
  return prefix;
}

// ------------------------------------------------------------------ steps
// Statistics a step needs of its input, accumulated in the loop that wrote
// that input (the load, or the previous step's output loop), so that no step
// makes a pass of its own for them.
enum { NEED_S1 = 1, NEED_SI = 2, NEED_S2 = 4, NEED_MX = 8 };

// The CTA's static shared memory: two sets of per-warp reduction slots (a
// reduction fills one set while threads may still read the other set of the
// reduction before it), and the radix selection's histogram.
struct SharedMem {
  double red[2][4][32];
  unsigned long long redu[2][32];
  unsigned hist[256];
  int sh[4];
};
// A thread's handle on its CTA's SharedMem: `flip` picks the reduction slot
// set, and every thread flips it at every reduction (all threads run the
// same reductions in the same order, so they agree on it).
struct Shared {
  SharedMem* m;
  int flip;
};

struct Stats {
  double s1, si, s2, mx;
};

// Per-thread partial sums Σx, Σi·x, Σx² and the largest |x| bits, for the
// statistics NEED asks for (a compile-time set, so the loops carry no
// per-sample branch on it). The partials are kept in T: a thread sums a few
// tens of samples (a trace over the CTA's threads), so a float32 partial is
// within ~25 ulp of its exact sum, and reduce_stats folds the partials in
// float64 — the reference's float64 sums (core/sums.nim) to ~1e-6 of the
// row's Σ|x|, without a float32 → float64 conversion per sample (a
// conversion issues at an eighth of the float32 rate). The index enters as
// T (ti), carried by the loops rather than converted per sample.
template <class T> struct Acc {
  T s1 = 0, si = 0, s2 = 0;
  unsigned long long mx = 0;
  template <int NEED> __device__ __forceinline__ void add_t(T v, T ti) {
    if (NEED & NEED_S1) s1 += v;
    if (NEED & NEED_SI) si = fma(ti, v, si);
    if (NEED & NEED_S2) s2 = fma(v, v, s2);
    if (NEED & NEED_MX) {
      unsigned long long b = abs_bits(v);
      mx = b > mx ? b : mx;
    }
  }
  template <int NEED> __device__ __forceinline__ void add(T v, int i) {
    add_t<NEED>(v, (NEED & NEED_SI) ? (T)i : (T)0);
  }
};

// Calls f with the statistics set `need` as a compile-time constant.
template <int K> struct NeedC { static constexpr int value = K; };
template <class F> __device__ __forceinline__ auto with_need(int need, F&& f) {
  switch (need) {
    case 0: return f(NeedC<0>());
    case NEED_S1: return f(NeedC<NEED_S1>());
    case NEED_S1 | NEED_SI: return f(NeedC<NEED_S1 | NEED_SI>());
    case NEED_S2: return f(NeedC<NEED_S2>());
    case NEED_MX: return f(NeedC<NEED_MX>());
    default: return f(NeedC<NEED_S1 | NEED_SI | NEED_S2 | NEED_MX>());
  }
}

// f(NeedC<NEED>) when the set is known at compile time (NEED ≥ 0), else the
// run-time dispatch.
template <int NEED, class F> __device__ __forceinline__ auto with_need_k(int need, F&& f) {
  if constexpr (NEED >= 0) {
    (void)need;
    return f(NeedC<NEED>());
  } else {
    return with_need(need, f);
  }
}

// Folds the partial sums over the block with one barrier: each warp's lane 0
// writes its warp's sums, and after the barrier every thread adds the warps'
// sums itself, in warp order (the same order, so the same result, in every
// thread). The barrier also orders the loop's writes to the trace before the
// next step reads them. Consecutive reductions use alternate slot sets
// (Shared::flip), so a warp that runs ahead into the next reduction never
// writes slots another thread is still reading: the reduction after that
// reuses them only past the next reduction's barrier.
template <class T> __device__ __forceinline__ Stats reduce_stats(const Acc<T>& a, int need, Shared& S) {
  Stats r{0, 0, 0, 0};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (kNT + 31) >> 5;
  double v0 = (double)a.s1, v1 = (double)a.si, v2 = (double)a.s2;
  unsigned long long m = a.mx;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    if (need & NEED_S1) v0 += __shfl_xor_sync(0xffffffffu, v0, o);
    if (need & NEED_SI) v1 += __shfl_xor_sync(0xffffffffu, v1, o);
    if (need & NEED_S2) v2 += __shfl_xor_sync(0xffffffffu, v2, o);
    if (need & NEED_MX) {
      unsigned long long u = __shfl_xor_sync(0xffffffffu, m, o);
      m = u > m ? u : m;
    }
  }
  double(*red)[32] = S.m->red[S.flip];
  unsigned long long* redu = S.m->redu[S.flip];
  S.flip ^= 1;
  if (need && lane == 0) {
    if (need & NEED_S1) red[0][warp] = v0;
    if (need & NEED_SI) red[1][warp] = v1;
    if (need & NEED_S2) red[2][warp] = v2;
    if (need & NEED_MX) redu[warp] = m;
  }
  __syncthreads();
  if (need == 0) return r;
  v0 = v1 = v2 = 0;
  m = 0;
  for (int w = 0; w < nw; w++) {
    if (need & NEED_S1) v0 += red[0][w];
    if (need & NEED_SI) v1 += red[1][w];
    if (need & NEED_S2) v2 += red[2][w];
    if (need & NEED_MX) {
      const unsigned long long u = redu[w];
      m = u > m ? u : m;
    }
  }
  r.s1 = v0;
  r.si = v1;
  r.s2 = v2;
  r.mx = bits_value(m, (T)0);
  return r;
}

// The elementwise loop of a step: X[i] = op(X[i], i) over the live samples,
// accumulating what the next step needs.
template <int NEED_K = -1, class T, class Op>
__device__ __forceinline__ Stats map_trace(T* X, int n, int need, Shared& S, Op op) {
  return with_need_k<NEED_K>(need, [&](auto K) {
    constexpr int NEED = decltype(K)::value;
    Acc<T> acc;
    T ti = (T)threadIdx.x;
    const T tstep = (T)kNT;
    for (int i = threadIdx.x; i < n; i += kNT, ti += tstep) {
      const T o = op(X[i], i);
      X[i] = o;
      acc.template add_t<NEED>(o, ti);
    }
    return reduce_stats(acc, NEED, S);
  });
}

// A pass over the unchanged trace when a step left it as it was.
template <int NEED_K = -1, class T>
__device__ __forceinline__ Stats stats_pass(const T* X, int n, int need, Shared& S) {
  return with_need_k<NEED_K>(need, [&](auto K) {
    constexpr int NEED = decltype(K)::value;
    Acc<T> acc;
    if (NEED) {
      T ti = (T)threadIdx.x;
      const T tstep = (T)kNT;
      for (int i = threadIdx.x; i < n; i += kNT, ti += tstep) acc.template add_t<NEED>(X[i], ti);
    }
    return reduce_stats(acc, NEED, S);
  });
}

// filter/edges.nim:16-30, from the sums of the step's input.
__device__ __forceinline__ void trend_from(int trend, const Stats& st, int n, double& a, double& b) {
  a = 0;
  b = 0;
  if (trend == PSG_TR_NONE) return;
  double nf = (double)n, mean = st.s1 / nf;
  if (trend == PSG_TR_MEAN || n == 1) {
    a = mean;
    return;
  }
  double c = (nf - 1) / 2;
  double slope = (st.si - c * st.s1) / (nf * (nf * nf - 1) / 12);
  a = mean - slope * c;
  b = slope;
}

// The zero-phase FFT filter with the reference's edge handling
// (filter/apply.nim:194-231, 340-363) on the trace in shared memory.
// `pre` is subtracted (in T) from every sample as it is read: a demean fused
// into the filter (the caller passes the statistics of the demeaned samples).
// NEED_K: the next step's statistics when known at compile time. The two
// transform buffers are at byte `work_off` of `mem` (shared memory, or a
// CTA's slice of global memory for traces too long for it).
// packInto's value of complex input c of the forward transform (real
// samples 2c and 2c + 1 of the padded trace) for zero pads: the detrended
// sample x[k − p] − (a + b·(k − p)) in float64 rounded to T inside the trace,
// 0 in the pads.
template <class T> struct PackLoad {
  typedef typename C2<T>::type V;
  const T* X;
  int n, p;
  T pre;
  double a, b;
  __device__ __forceinline__ T at(int k) const {
    const int i = k - p;
    return (unsigned)i < (unsigned)n ? (T)((double)(X[i] - pre) - (a + b * (double)i)) : (T)0;
  }
  __device__ __forceinline__ V operator()(int c, bool) const { return V{at(2 * c), at(2 * c + 1)}; }
};

template <class T, int MAXR, int NEED_K = -1, class M = InShared>
__device__ __forceinline__ Stats step_filter(const DevStep& st, const Stats& in, T* X, int n, int work_off, Shared& S,
                                             T pre = (T)0, const M& mem = M()) {
  typedef typename C2<T>::type V;
  const int p = st.pad, nfft = st.nfft, m = nfft / 2;
  const int ao = work_off / (int)sizeof(V), bo = ao + m;  // offsets of the two buffers
  V* A = reinterpret_cast<V*>(mem.base()) + ao;
  double a, b;
  trend_from(st.trend, in, n, a, b);
  const V* tw = reinterpret_cast<const V*>(st.tw);
  int zo;
  if (!st.reflect) {
    // packInto with zero pads: each value is computed where the forward
    // transform's first pass reads it (PackLoad) rather than stored first
    const PackLoad<T> pack{X, n, p, pre, a, b};
    zo = cfft_forward_loaded<T, MAXR, kNT>(mem, bo, ao, st.fft, tw, pack);
  } else {
    // packInto with reflected pads: the detrended samples at p .. p+n (a loop
    // of its own, so that the pads' arithmetic is not evaluated for them),
    // then the odd reflections tapered by `fall`, and zeros to nfft
    const T* fall = reinterpret_cast<const T*>(st.fall);
    T* Ar = reinterpret_cast<T*>(A);
    for (int i = threadIdx.x; i < n; i += kNT) Ar[p + i] = (T)((double)(X[i] - pre) - (a + b * (double)i));
    const int rest = nfft - n;  // [0, p) and [p + n, nfft)
    const T d0 = (T)((double)(X[0] - pre) - a);
    const T dn = (T)((double)(X[n - 1] - pre) - (a + b * (double)(n - 1)));
    for (int t = threadIdx.x; t < rest; t += kNT) {
      const int j = t < p ? t : t + n, i = j - p;
      T v = (T)0;
      if (i < 0) {
        const int k = -i, ii = min(k, n - 1);
        const T r = (T)((double)(X[ii] - pre) - (a + b * (double)ii));
        v = (d0 + d0 - r) * __ldg(&fall[k - 1]);
      } else if (i < n + p) {
        const int k = i - (n - 1), ii = n - 1 - min(k, n - 1);
        const T r = (T)((double)(X[ii] - pre) - (a + b * (double)ii));
        v = (dn + dn - r) * __ldg(&fall[k - 1]);
      }
      Ar[j] = v;
    }
    __syncthreads();
    zo = cfft_forward<T, MAXR, kNT>(mem, ao, bo, st.fft, tw);
  }
  // the real-FFT bridge fused into the inverse transform's first pass
  const BridgeLoad<T, M> bridge{mem, zo, m, reinterpret_cast<const Quad<T>*>(st.bridge)};
  const int yo = cfft_forward_loaded<T, MAXR, kNT>(mem, zo == ao ? bo : ao, zo, st.fft, tw, bridge);
  // unpackFrom: the output is swap(y): sample 2k is y[k].im and 2k + 1 is
  // y[k].re, so sample j of the real view is Yr[j ^ 1].
  const T* Yr = reinterpret_cast<const T*>(reinterpret_cast<const V*>(mem.base()) + yo);
  const double gb = b * st.dc_gain;
  const double ga = st.zero_dc ? -gb * (double)(n - 1) / 2 : a * st.dc_gain;
  if (ga == 0 && gb == 0) return map_trace<NEED_K>(X, n, st.need_next, S, [&](T, int i) { return Yr[(p + i) ^ 1]; });
  return map_trace<NEED_K>(X, n, st.need_next, S,
                   [&](T, int i) { return (T)((double)Yr[(p + i) ^ 1] + (ga + gb * (double)i)); });
}

// Σx² of a trace for a step that divides by it: the folded partials, or,
// where float32 partials may have overflowed (|x| ≳ 1e19) or dropped samples
// below the float32 range of squares, the float64 sum of a pass of its own.
template <class T> __device__ __forceinline__ double trace_s2(const Stats& in, const T* X, int n, Shared& S) {
  if (sizeof(T) == 8 || (isfinite(in.s2) && in.s2 >= 1e-30)) return in.s2;
  Acc<double> acc;
  for (int i = threadIdx.x; i < n; i += kNT) acc.template add_t<NEED_S2>((double)X[i], 0.0);
  return reduce_stats(acc, NEED_S2, S).s2;
}

// Warp scans of one value per lane: the sum over the lanes below (or above)
// this one.
template <class A> __device__ __forceinline__ A warp_excl_prefix(A v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const A u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  const A e = __shfl_up_sync(0xffffffffu, v, 1);
  return lane == 0 ? (A)0 : e;
}
template <class A> __device__ __forceinline__ A warp_excl_suffix(A v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const A u = __shfl_down_sync(0xffffffffu, v, o);
    if (lane + o < 32) v += u;
  }
  const A e = __shfl_down_sync(0xffffffffu, v, 1);
  return lane == 31 ? (A)0 : e;
}

// The AGC's block sums (gain/gain.nim:351-390): per block of w samples,
// P[e] the sum of the terms from the block's start to e − 1 (0 at a block
// start; P[n] the last block's sum unless n starts a block) and S[i] the sum
// from i to the block's end (or n − 1) — sums of non-negative terms without
// subtraction, so each keeps its relative precision however quiet its part
// of the trace. The terms are normalized by the trace level r = 1/rms
// ((x·r)² or |x|·r, so they are near 1 and their squares in range) and summed
// in T: one warp per block, a lane holding E consecutive terms (E odd, so
// the strided shared-memory reads are free of bank conflicts) that it scans
// locally both ways, the lanes' totals below (prefix) and above (suffix) from
// warp scans — a float32 sum within (E + 5) ulp, against the reference's
// float64 chains. Blocks longer than 32·E run in chunks: forwards for P,
// then backwards for S.
template <class T, int E>
__device__ __forceinline__ void agc_block_sums(const T* X, int n, int w, bool rms_mode, T r, T* P, T* Sx) {
  constexpr int CH = 32 * E;
  const int lane = threadIdx.x & 31, nw = (int)(kNT >> 5);
  const int j0 = lane * E;
  const int nb = (n + w - 1) / w;
  auto term = [&](int g) {
    const T v = X[g] * r;
    return rms_mode ? v * v : fabs(v);
  };
  for (int b = (int)(threadIdx.x >> 5); b < nb; b += nw) {
    const int base = b * w, L = min(w, n - base);
    if (lane == 0) P[base] = (T)0;
    // P[base + j + 1] for j < L: the next block's start (0) when the block is whole
    auto put_p = [&](int j, T v) { P[base + j + 1] = (j + 1 < L || L < w) ? v : (T)0; };
    if (L <= CH) {
      T t[E];
#pragma unroll
      for (int e = 0; e < E; e++) t[e] = j0 + e < L ? term(base + j0 + e) : (T)0;
      T inc[E], run = 0;
#pragma unroll
      for (int e = 0; e < E; e++) {
        run += t[e];
        inc[e] = run;
      }
      const T below = warp_excl_prefix(run);
#pragma unroll
      for (int e = 0; e < E; e++)
        if (j0 + e < L) put_p(j0 + e, below + inc[e]);
      run = 0;
#pragma unroll
      for (int e = E - 1; e >= 0; e--) {
        run += t[e];
        inc[e] = run;
      }
      const T above = warp_excl_suffix(run);
#pragma unroll
      for (int e = 0; e < E; e++)
        if (j0 + e < L) Sx[base + j0 + e] = above + inc[e];
    } else {
      T carry = 0;
      for (int c0 = 0; c0 < L; c0 += CH) {
        T inc[E], run = 0;
#pragma unroll
        for (int e = 0; e < E; e++) {
          const int j = c0 + j0 + e;
          run += j < L ? term(base + j) : (T)0;
          inc[e] = run;
        }
        const T below = warp_excl_prefix(run);
#pragma unroll
        for (int e = 0; e < E; e++) {
          const int j = c0 + j0 + e;
          if (j < L) put_p(j, (carry + below) + inc[e]);
        }
        carry += __shfl_sync(0xffffffffu, below + run, 31);
      }
      carry = 0;
      for (int c0 = (L - 1) / CH * CH; c0 >= 0; c0 -= CH) {
        T inc[E], run = 0;
#pragma unroll
        for (int e = E - 1; e >= 0; e--) {
          const int j = c0 + j0 + e;
          run += j < L ? term(base + j) : (T)0;
          inc[e] = run;
        }
        const T above = warp_excl_suffix(run);
#pragma unroll
        for (int e = 0; e < E; e++) {
          const int j = c0 + j0 + e;
          if (j < L) Sx[base + j] = (carry + above) + inc[e];
        }
        carry += __shfl_sync(0xffffffffu, above + run, 0);
      }
    }
  }
}

// The gain step of the AGC, g = k / (level + ε) with level = sqrt(mean) (rms)
// or the mean (mean-abs) (gain/gain.nim:392-402, :429-431). float32 uses the
// hardware's approximate square root and division (within 2 ulp of the
// correctly rounded ones); float64 keeps both correctly rounded.
// The AGC's gain k / (sqrt(mean) + ε) (rms mode; mean itself otherwise) with
// every operation correctly rounded, as the reference forms it in T
// (gain/gain.nim:399-401).
__device__ __forceinline__ float agc_gain(float mean, float k, float eps, bool rms_mode) {
  const float lv = rms_mode ? __fsqrt_rn(mean) : mean;
  return __fdiv_rn(k, __fadd_rn(lv, eps));
}
__device__ __forceinline__ double agc_gain(double mean, double k, double eps, bool rms_mode) {
  const double lv = rms_mode ? sqrt(mean) : mean;
  return k / (lv + eps);
}
__device__ __forceinline__ float recip(float c) { return __frcp_rn(c); }
__device__ __forceinline__ double recip(double c) { return __drcp_rn(c); }

// AGC (gain/gain.nim:351-461): the block sums into the work area, then one
// pass forms each window mean — s[i − h] + p[i + h + 1] over w for whole
// windows, the head, whole-trace and tail forms at the ends — and scales the
// sample by the gain, all in T.
template <class T, int NEED_K = -1, class M = InShared>
__device__ __forceinline__ Stats step_agc(const DevStep& st, const Stats& in, T* X, int n, int work_off, Shared& S,
                                          const M& mem = M()) {
  const int need = st.need_next;
  const bool rms_mode = st.agc_mode == PSG_AGC_RMS;
  const double rms = sqrt(trace_s2(in, X, n, S) / (double)n);
  if (rms == 0 || !fits_d<T>(st.target / rms / st.epsilon)) return stats_pass<NEED_K>(X, n, need, S);
  const int h = st.half, w = 2 * h + 1;
  T* P = reinterpret_cast<T*>(mem.base() + work_off);  // n + 1 values
  T* Sx = P + ((n + 1 + 3) & ~3);                          // n values
  const T r = (T)(1 / rms);
  if (w <= 32) agc_block_sums<T, 1>(X, n, w, rms_mode, r, P, Sx);
  else if (w <= 96) agc_block_sums<T, 3>(X, n, w, rms_mode, r, P, Sx);
  else if (w <= 160) agc_block_sums<T, 5>(X, n, w, rms_mode, r, P, Sx);
  else agc_block_sums<T, 9>(X, n, w, rms_mode, r, P, Sx);
  __syncthreads();
  const T k = (T)(st.target / rms), eps = (T)st.epsilon;
  const int first = min(h, n), last = max(first, n - h);
  const int headCut = min(max(n - h, 0), first);
  const int lastBlock = (n - 1) / w * w;
  const int tailCut = min(max(lastBlock + h, last), n);
  const T pn = P[n];
  const T invW = recip((T)w);
  const T headWhole = pn * recip((T)n);
  // The five ranges of i (gain/gain.nim:433-461), each a loop of its own so
  // that the whole windows run without the ends' arithmetic.
  return with_need_k<NEED_K>(need, [&](auto K) {
    constexpr int NEED = decltype(K)::value;
    Acc<T> acc;
    auto put = [&](int i, T mean) {
      const T y = X[i] * agc_gain(mean, k, eps, rms_mode);
      X[i] = y;
      acc.template add<NEED>(y, i);
    };
    for (int i = first + (int)threadIdx.x; i < last; i += kNT) put(i, (Sx[i - h] + P[i + h + 1]) * invW);
    for (int i = threadIdx.x; i < headCut; i += kNT) put(i, P[i + h + 1] * recip((T)(i + h + 1)));
    for (int i = headCut + (int)threadIdx.x; i < first; i += kNT) put(i, headWhole);
    for (int i = last + (int)threadIdx.x; i < tailCut; i += kNT)
      put(i, (Sx[i - h] + pn) * recip((T)(n - (i - h))));
    for (int i = tailCut + (int)threadIdx.x; i < n; i += kNT) put(i, Sx[i - h] * recip((T)(n - (i - h))));
    return reduce_stats(acc, NEED, S);
  });
}

// Per-trace normalization (gain/gain.nim:198-219; stats.nim:129-182).
template <class T, int NEED_K = -1>
__device__ __forceinline__ Stats step_norm_trace(const DevStep& st, const Stats& in, T* X, int n, Shared& S) {
  const int need = st.need_next;
  double level;
  if (st.stat == PSG_NORM_MAX) {
    level = in.mx;
  } else if (st.stat == PSG_NORM_RMS) {
    level = sqrt(trace_s2(in, X, n, S) / (double)n);
  } else if (isnan(in.mx)) {
    level = in.mx;
  } else {
    double hr = (double)(n - 1) * st.percentile / 100;
    int k = min((int)floor(hr), n - 1);
    const unsigned long long lb = select_kth(X, n, k, S.m->hist, S.m->sh);
    const int same = S.m->sh[2];  // keys equal to the k-th at ranks k and above
    double lower = bits_value(lb, (T)0);
    if (k + 1 >= n) {
      level = lower;
    } else {
      // the (k+1)-th: the k-th again when it repeats, else the least key
      // above it (the largest complement), one pass instead of a selection
      unsigned long long ub = lb;
      if (same < 2) {
        unsigned long long best = 0;
        for (int i = threadIdx.x; i < n; i += kNT) {
          const unsigned long long key = abs_bits(X[i]);
          if (key > lb && ~key > best) best = ~key;
        }
        best = block_max_u64(best, S.m->redu[S.flip]);
        S.flip ^= 1;
        ub = ~best;
      }
      double upper = bits_value(ub, (T)0);
      double f = hr - (double)k;
      level = f == 0 ? lower : lower + f * (upper - lower);
    }
  }
  if (!(fin_pos_d(level) && fits_d<T>(st.norm_target / level))) return stats_pass<NEED_K>(X, n, need, S);
  const T kf = (T)(st.norm_target / level);
  return map_trace<NEED_K>(X, n, need, S, [&](T x, int) { return x * kf; });
}

// gain/curves.nim:132-160 on the device, in float64.
__device__ inline double factor_at_d(const psg_gain_curve& c, double t) {
  if (isnan(t)) return t;
  if (c.kind == PSG_GC_POWER) return pow(fmax(t, c.min_ms) / c.ref_ms, c.power);
  double db;
  if (c.kind == PSG_GC_KNOTS) {
    int nk = c.n_knots;
    if (t <= c.knots[0].t_ms) db = c.knots[0].db;
    else if (t >= c.knots[nk - 1].t_ms) db = c.knots[nk - 1].db;
    else {
      int lo = 0, hi = nk - 1;
      while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (c.knots[mid].t_ms <= t) lo = mid; else hi = mid;
      }
      double f = (t - c.knots[lo].t_ms) / (c.knots[hi].t_ms - c.knots[lo].t_ms);
      db = c.knots[lo].db + f * (c.knots[hi].db - c.knots[lo].db);
    }
  } else {
    db = c.db_per_s * t / 1000;
  }
  return pow(10.0, db / 20);
}

// The gain curve on one row (gain/curves.nim:316-350 and the workspace form
// :383-418): the table where the row's times fall on it (as it is on the
// grid, linearly interpolated off it), the curve itself elsewhere.
template <class T, int NEED_K = -1>
__device__ __forceinline__ Stats step_gain_curve(const DevStep& st, T* X, int n, double start, Shared& S) {
  const int need = st.need_next;
  if (isnan(start)) return stats_pass<NEED_K>(X, n, need, S);
  const T* tab = reinterpret_cast<const T*>(st.table);
  double u = (start - st.t_min_ms) / st.dt_ms;
  long long s = 0, j0 = n, j1 = n;
  double f = 0;
  bool on = false;
  if (isfinite(u) && fabs(u) <= 1e15) {
    double r = round(u);
    on = fabs(u - r) <= 1e-9 * fmax(1.0, fabs(u));
    s = (long long)(on ? r : floor(u));
    f = u - (double)s;
    long long last = (long long)st.table_len - (on ? 1 : 2);
    j0 = min(max(-s, 0ll), (long long)n);
    j1 = min(max(last - s + 1, j0), (long long)n);
  }
  const T tf = (T)f;
  return map_trace<NEED_K>(X, n, need, S, [&](T v, int j) {
    if (j >= j0 && j < j1) {
      T a = __ldg(&tab[s + j]);
      return on ? v * a : v * (a + tf * (__ldg(&tab[s + j + 1]) - a));
    }
    if (v != (T)0) return v * (T)factor_at_d(st.curve, start + (double)j * st.dt_ms);
    return v;
  });
}

// ------------------------------------------------------------ IIR filters
// Double-double numbers (an unevaluated sum hi + lo, |lo| ≤ ulp(hi)/2) by
// the error-free transformations of Dekker and Knuth: the carried states of
// the chunked recurrence below keep about 106 bits, so that its result is
// as close to the exact recurrence as the serial float64 one is.
struct DD {
  double hi, lo;
};
__device__ __forceinline__ DD dd_quick(double a, double b) {
  const double s = __dadd_rn(a, b);
  return DD{s, __dsub_rn(b, __dsub_rn(s, a))};
}
__device__ __forceinline__ DD dd_two_sum(double a, double b) {
  const double s = __dadd_rn(a, b), bb = __dsub_rn(s, a);
  return DD{s, __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb))};
}
__device__ __forceinline__ DD dd_add(DD x, DD y) {
  DD s = dd_two_sum(x.hi, y.hi);
  const DD t = dd_two_sum(x.lo, y.lo);
  s = dd_quick(s.hi, __dadd_rn(s.lo, t.hi));
  return dd_quick(s.hi, __dadd_rn(s.lo, t.lo));
}
__device__ __forceinline__ DD dd_mul(DD x, DD y) {
  const double p = __dmul_rn(x.hi, y.hi);
  double e = __fma_rn(x.hi, y.hi, -p);
  e = __dadd_rn(e, __dadd_rn(__dmul_rn(x.hi, y.lo), __dmul_rn(x.lo, y.hi)));
  return dd_quick(p, e);
}
// A 2×2 matrix of the biquad state map, row-major, in double-double.
struct M2 {
  DD a, b, c, d;
};
__device__ __forceinline__ M2 m2_mul(const M2& x, const M2& y) {
  return M2{dd_add(dd_mul(x.a, y.a), dd_mul(x.b, y.c)), dd_add(dd_mul(x.a, y.b), dd_mul(x.b, y.d)),
            dd_add(dd_mul(x.c, y.a), dd_mul(x.d, y.c)), dd_add(dd_mul(x.c, y.b), dd_mul(x.d, y.d))};
}
__device__ __forceinline__ M2 m2_load(const double* t) {
  return M2{DD{t[0], t[1]}, DD{t[2], t[3]}, DD{t[4], t[5]}, DD{t[6], t[7]}};
}
// y += Q·u
__device__ __forceinline__ void m2_madd(const M2& Q, DD u1, DD u2, DD& y1, DD& y2) {
  y1 = dd_add(y1, dd_add(dd_mul(Q.a, u1), dd_mul(Q.b, u2)));
  y2 = dd_add(y2, dd_add(dd_mul(Q.c, u1), dd_mul(Q.d, u2)));
}
__device__ __forceinline__ DD dd_shfl_up(DD v, int d) {
  return DD{__shfl_up_sync(0xffffffffu, v.hi, d), __shfl_up_sync(0xffffffffu, v.lo, d)};
}

// Doubles per chunk length in a section's IIR scan table: P^k, k = 1 .. 32,
// then P^64 and P^128, 2×2 in double-double.
constexpr int kIirTab = 34 * 8;

// One pass of one section (filter/iir.nim:319-351) over the m padded samples
// of B (float64, in place), forwards or backwards, from rest or from the
// steady state of its first input sample. A section in transposed direct
// form II is a linear map of its state (s1, s2) per sample,
//   y = b0·x + s1,  s1' = b1·x − a1·y + s2,  s2' = b2·x − a2·y,
// so the pass runs in parallel over the CTA: thread t takes the L = ⌈m/256⌉
// samples of chunk t, (1) runs them from a zero state (thread 0 from the
// pass's start state) to the chunk's end state Z_t, (2) a scan over the
// threads gives each chunk's true start state, E_t = P·E_{t−1} + Z_t with
// P = M^L the state map over L zero samples (warp scans with the powers
// P^(2^i); then the eight warps' totals scanned by eight lanes with P^32,
// P^64 and P^128; every power read from the host's double-double table
// `pw` for this L), and (3) each thread reruns its chunk from its start
// state and writes the outputs. A start state below 1e-250 is set to 0, so a
// decay after the input stops ends in exact zeros (filter/iir.nim:311-317).
__device__ __forceinline__ void iir_pass(double* B, int m, const double* c, const double* pw, bool steady,
                                         bool backward) {
  __shared__ double w_end[kNT / 32][4];
  __shared__ double w_carry[kNT / 32][4];  // the true end state of the chunk before each warp's first
  const double b0 = c[0], b1 = c[1], b2 = c[2], a1 = c[3], a2 = c[4], g = c[5];
  const int L = (m + kNT - 1) / kNT;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int j0 = min(t * L, m), j1 = min(j0 + L, m);
  const double* tab = pw + (size_t)(L - 1) * kIirTab;  // P^k at tab + 8·(k − 1)
  auto at = [&](int j) -> double& { return B[backward ? m - 1 - j : j]; };
  __syncthreads();  // the previous pass's outputs
  double i1 = 0, i2 = 0;  // the pass's start state
  if (steady && m > 0) {
    const double u = at(0);
    const double y = __dmul_rn(g, u);
    i2 = __dsub_rn(__dmul_rn(b2, u), __dmul_rn(a2, y));
    i1 = __dsub_rn(y, __dmul_rn(b0, u));
  }
  auto step = [&](double x, double& s1, double& s2) {
    const double y = __dadd_rn(__dmul_rn(b0, x), s1);
    s1 = __dadd_rn(__dsub_rn(__dmul_rn(b1, x), __dmul_rn(a1, y)), s2);
    s2 = __dsub_rn(__dmul_rn(b2, x), __dmul_rn(a2, y));
    return y;
  };
  // (1) the chunk from rest (chunk 0 from the start state)
  double z1 = t == 0 ? i1 : 0.0, z2 = t == 0 ? i2 : 0.0;
  for (int j = j0; j < j1; j++) step(at(j), z1, z2);
  // (2) warp scan: e_t = Σ_k P^(t−k)·Z_k over the warp's lanes
  DD e1{z1, 0}, e2{z2, 0};
  for (int i = 0; i < 5; i++) {
    const DD u1 = dd_shfl_up(e1, 1 << i), u2 = dd_shfl_up(e2, 1 << i);
    if (lane >= (1 << i)) m2_madd(m2_load(tab + 8 * ((1 << i) - 1)), u1, u2, e1, e2);
  }
  if (lane == 31) {
    w_end[warp][0] = e1.hi;
    w_end[warp][1] = e1.lo;
    w_end[warp][2] = e2.hi;
    w_end[warp][3] = e2.lo;
  }
  __syncthreads();
  // the warps' carries: an inclusive scan of the warp totals with P^32
  // between neighbours (warp 0, eight lanes, three doubling steps)
  constexpr int kW = kNT / 32;
  static_assert(kW == 8, "the carry scan takes three steps over eight warps");
  if (warp == 0) {
    const int l = lane < kW ? lane : kW - 1;
    DD v1{w_end[l][0], w_end[l][1]}, v2{w_end[l][2], w_end[l][3]};
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const int d = 1 << i;
      const DD u1 = dd_shfl_up(v1, d), u2 = dd_shfl_up(v2, d);
      if (lane >= d && lane < kW) m2_madd(m2_load(tab + 8 * (31 + i)), u1, u2, v1, v2);  // P^(32·d)
    }
    if (lane + 1 < kW) {
      w_carry[lane + 1][0] = v1.hi;
      w_carry[lane + 1][1] = v1.lo;
      w_carry[lane + 1][2] = v2.hi;
      w_carry[lane + 1][3] = v2.lo;
    }
  }
  __syncthreads();
  // the carry into this warp: the true end state of the previous warp's last chunk
  DD c1{0, 0}, c2{0, 0};
  if (warp > 0) {
    c1 = DD{w_carry[warp][0], w_carry[warp][1]};
    c2 = DD{w_carry[warp][2], w_carry[warp][3]};
    // E_t = e_t + P^(lane+1)·carry
    m2_madd(m2_load(tab + 8 * lane), c1, c2, e1, e2);
  }
  // this chunk starts from the previous chunk's end
  const DD p1 = dd_shfl_up(e1, 1), p2 = dd_shfl_up(e2, 1);
  double s1 = __dadd_rn(p1.hi, p1.lo), s2 = __dadd_rn(p2.hi, p2.lo);
  if (lane == 0) {
    s1 = __dadd_rn(c1.hi, c1.lo);
    s2 = __dadd_rn(c2.hi, c2.lo);
  }
  if (t == 0) {
    s1 = i1;
    s2 = i2;
  }
  if (fabs(s1) < 1e-250) s1 = 0;
  if (fabs(s2) < 1e-250) s2 = 0;
  // (3) the chunk from its true start
  for (int j = j0; j < j1; j++) {
    double& x = at(j);
    x = step(x, s1, s2);
  }
}

// The IIR filter (filter/iir.nim:363-433) on one trace: the detrended live
// samples with their pads (odd reflections, or zeros after the data) in a
// float64 work area of lead + n + tail values, every section forwards (then
// backwards for zero phase), and the trend added back as the cascade's
// steady-state response to it, G(1)·(a + b·i) − b·G'(1).
template <class T, int NEED_K = -1, class M = InShared>
__device__ __noinline__ Stats step_iir(const DevStep& st, const Stats& in, T* X, int n, int work_off, Shared& S,
                                          const M& mem = M()) {
  double* B = reinterpret_cast<double*>(mem.base() + work_off);
  double a, b;
  trend_from(st.trend, in, n, a, b);
  const int p = st.lead, tail = st.tail, m = p + n + tail;
  for (int i = threadIdx.x; i < n; i += kNT)
    B[p + i] = __dsub_rn((double)X[i], __dadd_rn(a, __dmul_rn(b, (double)i)));
  __syncthreads();
  if (st.reflect) {
    const double d0 = B[p], dn = B[p + n - 1];
    for (int k = threadIdx.x + 1; k <= p; k += kNT) B[p - k] = __dsub_rn(2 * d0, B[p + min(k, n - 1)]);
    for (int k = threadIdx.x + 1; k <= tail; k += kNT) B[p + n - 1 + k] = __dsub_rn(2 * dn, B[p + n - 1 - min(k, n - 1)]);
  } else {
    for (int k = threadIdx.x + 1; k <= tail; k += kNT) B[p + n - 1 + k] = 0;
  }
  const int lmax = st.pw_len;
  for (int i = 0; i < st.n_sec; i++)
    iir_pass(B, m, st.sec + 6 * i, st.pw + (size_t)i * lmax * kIirTab, st.reflect, false);
  if (st.iir_zero)
    for (int i = 0; i < st.n_sec; i++)
      iir_pass(B, m, st.sec + 6 * i, st.pw + (size_t)i * lmax * kIirTab, st.reflect, true);
  __syncthreads();
  const double ga = __dsub_rn(__dmul_rn(a, st.dc_gain), __dmul_rn(b, st.dc_slope)), gb = __dmul_rn(b, st.dc_gain);
  return map_trace<NEED_K>(X, n, st.need_next, S,
                           [&](T, int i) { return (T)__dadd_rn(B[p + i], __dadd_rn(ga, __dmul_rn(gb, (double)i))); });
}

// ------------------------------------------------------------ mutes
// muteTimeMs (core/mute.nim:103-123) in the reference's order of operations
// (no contraction into fused multiply-adds).
__device__ __forceinline__ double mute_time_d(const DevStep& st, double offset) {
  if (st.mute_kind == PSG_MK_TIME) return st.mute_t;
  const double x = fabs(offset);
  if (st.mute_kind == PSG_MK_LMO) return __dadd_rn(__dadd_rn(st.mute_t0, __dmul_rn(x, st.ms_per_dist)), st.mute_pad);
  if (isnan(x)) return x;
  const double* off = st.knots;
  const double* tm = st.knots + st.n_knots;
  const int last = st.n_knots - 1;
  if (x <= off[0]) return tm[0];
  if (x >= off[last]) return tm[last];
  int lo = 0, hi = last;  // the last knot ≤ x
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= x) lo = mid;
    else hi = mid;
  }
  const double u = __ddiv_rn(__dsub_rn(x, off[lo]), __dsub_rn(off[hi], off[lo]));
  return __dadd_rn(tm[lo], __dmul_rn(u, __dsub_rn(tm[hi], tm[lo])));
}
// firstAtOrAfter / firstAfter (core/mute.nim:127-137): the first column ≥ c
// (> c), clamped to 0 .. n, 0 for NaN.
__device__ __forceinline__ int first_at_or_after(double c, int n) {
  if (!(c > 0)) return 0;
  if (c >= (double)n) return n;
  return (int)ceil(c);
}
__device__ __forceinline__ int first_after(double c, int n) {
  if (!(c >= 0)) return 0;
  if (c >= (double)n) return n;
  return (int)floor(c) + 1;
}
// muteTop / muteBottom of one row (core/mute.nim:139-200) at the column of
// the row's keys, (t − t0Ms)/dtMs − firstSample (core/mute.nim:209-214),
// with a taper of taperMs/dtMs columns on the muted side: sin² weights in
// float64, zeros beyond. A NaN column leaves the row alone.
template <class T, int NEED_K = -1>
__device__ __forceinline__ Stats step_mute(const DevStep& st, const Job* J, long long r, T* X, int n, Shared& S) {
  const int need = st.need_next;
  const double offset = J->offset ? J->offset[r] : (double)NAN;
  const double t0 = J->t0_ms ? J->t0_ms[r] : (double)NAN;
  const double c = __dsub_rn(__ddiv_rn(__dsub_rn(mute_time_d(st, offset), t0), J->dt_ms), (double)J->first_sample);
  if (isnan(c)) return stats_pass<NEED_K>(X, n, need, S);
  double taper = __ddiv_rn(st.taper_ms, J->dt_ms);
  if (!(taper < INFINITY)) taper = 0;
  const double half_pi = 3.141592653589793 / 2;
  if (st.kind == ST_MUTE_TOP) {
    const double ramp = __dsub_rn(c, taper);
    const int zero_end = first_at_or_after(ramp, n);
    const int keep = taper > 0 ? first_at_or_after(c, n) : zero_end;
    return map_trace<NEED_K>(X, n, need, S, [&](T v, int j) {
      if (j < zero_end) return (T)0;
      if (j < keep) {
        const double w = sin(__ddiv_rn(__dmul_rn(half_pi, __dsub_rn((double)j, ramp)), taper));
        return (T)((double)v * __dmul_rn(w, w));
      }
      return v;
    });
  }
  const double ramp = __dadd_rn(c, taper);
  const int zero_start = first_after(ramp, n);
  const int keep = taper > 0 ? first_after(c, n) : zero_start;
  return map_trace<NEED_K>(X, n, need, S, [&](T v, int j) {
    if (j >= zero_start) return (T)0;
    if (j >= keep) {
      const double w = sin(__ddiv_rn(__dmul_rn(half_pi, __dsub_rn(ramp, (double)j)), taper));
      return (T)((double)v * __dmul_rn(w, w));
    }
    return v;
  });
}

// ------------------------------------------------------------ the kernel
// Stores a row from shared memory, 16-byte vectors where the row allows.
template <class T> __device__ __forceinline__ void store_out(const T* s, T* __restrict__ g, int n) {
  if (sizeof(T) == 4) {
    const int head = min((int)((4 - (((uintptr_t)g >> 2) & 3)) & 3), n);
    const int nv = (n - head) >> 2;
    for (int i = threadIdx.x; i < head; i += kNT) g[i] = s[i];
    float4* gv = reinterpret_cast<float4*>(g + head);
    const float* sf = reinterpret_cast<const float*>(s) + head;
    for (int v = threadIdx.x; v < nv; v += kNT)
      __stcs(gv + v, make_float4(sf[4 * v], sf[4 * v + 1], sf[4 * v + 2], sf[4 * v + 3]));
    for (int i = head + 4 * nv + threadIdx.x; i < n; i += kNT) g[i] = s[i];
  } else {
    for (int i = threadIdx.x; i < n; i += kNT) g[i] = s[i];
  }
}

// A row's place in its buffer: X starts `off` bytes in (the row's address
// mod 16); elements [head, tail) arrive by the bulk copy of `body` bytes,
// the rest of [0, len) by direct loads.
struct RowSlot {
  int head, tail, body, len, off;
};

// What one row of a launch needs: its job's pointers and plan, and its live
// length. Batched launches find the job by a binary search of row_begin.
template <class T> struct RowCtx {
  const T* from;  // the row to read (src, or dst in place)
  T* to;          // the row to write
  const T* blk_lo;  // the block `from` lies in: [blk_lo, blk_hi)
  const T* blk_hi;
  const DevStep* steps;
  const Job* job;
  long long r;  // the row within its job
  double start;
  int n, cols, first, last;
  bool copy;
};
template <class T, bool BATCH>
__device__ __forceinline__ RowCtx<T> row_ctx(const PipeArgs& a, long long t) {
  long long r = t;
  const Job* J = &a.job;
  if (BATCH) {
    int lo = 0, hi = a.njobs - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (a.row_begin[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    J = &a.jobs[lo];
    r = t - a.row_begin[lo];
  }
  RowCtx<T> c;
  const T* src = reinterpret_cast<const T*>(J->src);
  T* dst = reinterpret_cast<T*>(J->dst);
  c.copy = src != nullptr && src != dst;
  c.cols = J->cols;
  c.blk_lo = c.copy ? src : dst;
  c.blk_hi = c.blk_lo + J->rows * (long long)c.cols;
  c.from = c.blk_lo + r * (long long)c.cols;
  c.to = dst + r * (long long)c.cols;
  c.n = min(max(J->live[r], 0), c.cols);
  c.start = J->start_ms ? J->start_ms[r] : (double)NAN;
  c.steps = J->steps;
  c.job = J;
  c.r = r;
  c.first = J->first;
  c.last = J->last;
  return c;
}

// Recipes: step sequences that run as straight-line code with their
// statistics sets known at compile time (recipe 0 runs any sequence by a
// switch over the steps). A demean followed by the filter is fused into the
// filter's pack: one statistics pass over the raw samples gives Σx and Σi·x,
// from which follow the mean and the sums of the demeaned samples the
// trend needs (Σx' = Σx − n·m, Σi·x' = Σi·x − m·n(n − 1)/2, exact up to the
// float64 rounding and the T rounding of each x − m, far below a sample's
// unit in the last place).
enum Recipe : int {
  RC_GENERIC = 0,
  RC_DFA = 1,   // demean, filter, AGC
  RC_DFAN = 2,  // demean, filter, AGC, per-trace normalization
  RC_FN = 3,    // filter, per-trace normalization
  RC_FG = 4,    // filter, gain curve
  RC_COUNT = 5
};
constexpr int NEED_NORM = NEED_S2 | NEED_MX;  // any per-trace normalization's input statistics
constexpr int NEED_FILTER = NEED_S1 | NEED_SI;
template <int RECIPE> constexpr int recipe_need0() {
  return RECIPE == RC_DFA || RECIPE == RC_DFAN ? NEED_S1 | NEED_SI : NEED_FILTER;
}

template <class T, int MAXR, int RECIPE>
__device__ __forceinline__ void run_recipe(const DevStep* d, Stats st, T* X, int n, int work_off, double start,
                                           Shared& S) {
  if constexpr (RECIPE == RC_DFA || RECIPE == RC_DFAN) {
    const T mean = (T)(st.s1 / (double)n);
    Stats sd = st;
    sd.s1 = st.s1 - (double)n * (double)mean;
    sd.si = st.si - (double)mean * ((double)n * (double)(n - 1) / 2);
    st = step_filter<T, MAXR, NEED_S2>(d[1], sd, X, n, work_off, S, mean);
    if constexpr (RECIPE == RC_DFA) {
      step_agc<T, 0>(d[2], st, X, n, work_off, S);
    } else {
      st = step_agc<T, NEED_NORM>(d[2], st, X, n, work_off, S);
      step_norm_trace<T, 0>(d[3], st, X, n, S);
    }
  } else if constexpr (RECIPE == RC_FN) {
    st = step_filter<T, MAXR, NEED_NORM>(d[0], st, X, n, work_off, S);
    step_norm_trace<T, 0>(d[1], st, X, n, S);
  } else if constexpr (RECIPE == RC_FG) {
    st = step_filter<T, MAXR, 0>(d[0], st, X, n, work_off, S);
    step_gain_curve<T, 0>(d[1], X, n, start, S);
  }
}

// PF: prefetch the next row into the second buffer while this one is
// processed (when the second buffer costs no occupancy); otherwise one buffer,
// loaded at the top of each row. BATCH: the rows of several jobs (several
// plans, widths and blocks) in one launch. GW: the FFT and AGC work areas in
// global memory (a.gwork), for traces whose work does not fit beside the row
// in shared memory.
template <class T, int MAXR, bool PF, bool BATCH, int RECIPE, bool GW = false>
__global__ void __launch_bounds__(kNT, (GW || sizeof(T) == 8 ? 2 : 4)) pipeline_kernel(PipeArgs a) {
  __shared__ SharedMem smem;
  Shared S{&smem, 0};
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ RowSlot slot[2];
  __shared__ int s_ok;
  const double pf = a.factor ? *a.factor : (double)NAN;
  const bool scale = !isnan(pf);
  const T kf = scale ? (T)pf : (T)1;
  const long long total = BATCH ? a.total_rows : a.job.rows;
  constexpr int esz = (int)sizeof(T);
  // Thread 0 starts the bulk copy of row t into buffer b: the part we need
  // (the whole row for src → dst, the live samples in place), widened to
  // 16-byte boundaries where those stay inside the block (the bytes of the
  // neighbouring rows are read and left unused), so that only a row at
  // either end of an unaligned block has a few ragged elements, read
  // directly.
  auto issue = [&](long long t, int b) {
    const RowCtx<T> c = row_ctx<T, BATCH>(a, t);
    const int len = c.copy ? c.cols : c.n;
    const uintptr_t ga = (uintptr_t)c.from, ge = ga + (uintptr_t)len * esz;
    const int off = (int)(ga & 15);
    uintptr_t lo = ga & ~(uintptr_t)15, hi = (ge + 15) & ~(uintptr_t)15;
    if (lo < (uintptr_t)c.blk_lo) lo += 16;
    if (hi > (uintptr_t)c.blk_hi) hi -= 16;
    unsigned char* xb = psg_dyn_smem + b * a.x_bytes;
    if (len > 0 && hi > lo) {
      const int head = lo > ga ? (int)((lo - ga) / esz) : 0;
      const int tail = hi < ge ? (int)((hi - ga) / esz) : len;
      const uint32_t body = (uint32_t)(hi - lo);
      slot[b] = RowSlot{head, tail, (int)body, len, off};
      mbar_arrive_expect_tx(&bars[b], body);
      // lo − ga is −off or 16 − off: the copy lands at xb or xb + 16
      bulk_load(xb + off + ((long long)lo - (long long)ga), reinterpret_cast<const void*>(lo), body, &bars[b]);
    } else {
      slot[b] = RowSlot{len, len, 0, len, off};
      mbar_arrive(&bars[b]);
    }
  };
  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    mbar_init_fence();
    if (PF && blockIdx.x < total) issue(blockIdx.x, 0);
  }
  __syncthreads();
  uint32_t phase[2] = {0, 0};
  int cur = 0;
  for (long long t = blockIdx.x; t < total; t += gridDim.x, cur = PF ? cur ^ 1 : 0) {
    const long long tn = t + gridDim.x;
    if (threadIdx.x == 0) {
      // the buffer's last reads (the previous row's store) come before the copy into it
      if (PF && tn < total) {
        fence_proxy_async();
        issue(tn, cur ^ 1);
      } else if (!PF) {
        fence_proxy_async();
        issue(t, 0);
      }
    }
    // One warp polls the row's barrier while the others wait at the CTA
    // barrier (no issue slots spent); then every thread takes the completed
    // phase itself, which returns at once and orders its reads after the copy.
    if (threadIdx.x < 32) {
      const bool ok = mbar_wait(&bars[cur], phase[cur], 1ll << 26);
      if (threadIdx.x == 0) s_ok = ok ? 1 : 0;
    }
    __syncthreads();
    if (!s_ok) {
      if (threadIdx.x == 0) {
        atomicExch(a.status, 1);
        mbar_wait(&bars[cur], phase[cur], 1ll << 26);  // the copy still in flight lands before the CTA exits
      }
      return;
    }
    mbar_try_wait(&bars[cur], phase[cur]);
    phase[cur] ^= 1;
    const RowCtx<T> c = row_ctx<T, BATCH>(a, t);
    const RowSlot sl = slot[cur];
    T* X = reinterpret_cast<T*>(psg_dyn_smem + cur * a.x_bytes + sl.off);
    for (int i = threadIdx.x; i < sl.head; i += kNT) X[i] = c.from[i];
    for (int i = sl.tail + threadIdx.x; i < sl.len; i += kNT) X[i] = c.from[i];
    if (sl.head > 0 || sl.tail < sl.len) __syncthreads();  // the ragged ends are read by other threads below
    const int n = c.n;
    if constexpr (RECIPE != RC_GENERIC) {
      if (n > 0) {
        // the panel factor of a part that starts with one, and the first
        // step's statistics
        constexpr int N0 = recipe_need0<RECIPE>();
        Stats st = scale ? map_trace<N0>(X, n, N0, S, [&](T x, int) { return x * kf; }) : stats_pass<N0>(X, n, N0, S);
        run_recipe<T, MAXR, RECIPE>(c.steps + c.first, st, X, n, a.work_off, c.start, S);
      }
    } else {
      const int need0 = c.first < c.last ? c.steps[c.first].need : 0;
      Stats st{0, 0, 0, 0};
      if (n > 0) {
        if (scale) st = map_trace(X, n, need0, S, [&](T x, int) { return x * kf; });
        else st = stats_pass(X, n, need0, S);
      } else {
        __syncthreads();
      }
      for (int si = c.first; n > 0 && si < c.last; si++) {
        const DevStep& d = c.steps[si];
        const int need = d.need_next;
        switch (d.kind) {
          case ST_DEMEAN: {
            const T mean = (T)(st.s1 / (double)n);
            st = map_trace(X, n, need, S, [&](T x, int) { return x - mean; });
            break;
          }
          case ST_DETREND: {
            double nf = (double)n, cc = (nf - 1) / 2, mean = st.s1 / nf;
            double stt = nf * (nf * nf - 1) / 12;
            double slope = n > 1 ? (st.si - cc * st.s1) / stt : 0.0;
            const T ta = (T)(mean - slope * cc), tb = (T)slope;
            st = map_trace(X, n, need, S, [&](T x, int i) { return x - (ta + tb * (T)i); });
            break;
          }
          case ST_SCALE: {
            const T k = (T)d.factor;
            st = map_trace(X, n, need, S, [&](T x, int) { return x * k; });
            break;
          }
          case ST_CLIP: {
            const T lo = (T)d.lo, hi = (T)d.hi;
            st = map_trace(X, n, need, S, [&](T v, int) { return v > hi ? hi : (v < lo ? lo : v); });
            break;
          }
          case ST_POLARITY:
            st = map_trace(X, n, need, S, [&](T x, int) { return -x; });
            break;
          case ST_FILTER:
            if constexpr (GW)
              st = step_filter<T, MAXR, -1, InGlobal>(d, st, X, n, 0, S, (T)0,
                                                      InGlobal{a.gwork + (size_t)blockIdx.x * a.gwork_stride});
            else
              st = step_filter<T, MAXR>(d, st, X, n, a.work_off, S);
            break;
          case ST_AGC:
            if constexpr (GW)
              st = step_agc<T, -1, InGlobal>(d, st, X, n, 0, S, InGlobal{a.gwork + (size_t)blockIdx.x * a.gwork_stride});
            else
              st = step_agc(d, st, X, n, a.work_off, S);
            break;
          case ST_NORM_TRACE: st = step_norm_trace(d, st, X, n, S); break;
          case ST_GAIN_CURVE: st = step_gain_curve(d, X, n, c.start, S); break;
          // mutes and IIR filters: single-job launches only (the request
          // loop, which batches, refuses plans with them)
          case ST_MUTE_TOP:
          case ST_MUTE_BOTTOM:
            if constexpr (!BATCH) st = step_mute(d, c.job, c.r, X, n, S);
            break;
          case ST_IIR:
            if constexpr (GW)
              st = step_iir<T, -1, InGlobal>(d, st, X, n, 0, S, InGlobal{a.gwork + (size_t)blockIdx.x * a.gwork_stride});
            else if constexpr (!BATCH)
              st = step_iir(d, st, X, n, a.work_off, S);
            break;
          default: break;
        }
      }
    }
    if (c.copy || n > 0) store_out(X, c.to, c.copy ? c.cols : n);
    __syncthreads();
  }
}

// ============================================================ correlation
// One launch of correlateInto (psg_cuda.cu corr_kernel, psg_trace.cuh
// corr_trace_kernel).
struct CorrArgs {
  const void* src;
  void* dst;
  long long rows;
  int cols, out, nfft, shift, pilot_len, record;
  const int* live;
  const void* bridge;  // Quad<T>[m]: the split · multiplier · unsplit map of each bin pair
  const void* tw;
  const void* tw_pass;  // the compile-time transform's twiddles, pass by pass (corr_trace_kernel)
  FftDesc fft;
  void* gwork;        // per-CTA global scratch when shared memory is too small (else NULL)
  // stack epilogue
  double* num;
  int* cnt;
  int stack_samples;
  long long stack_rows;
  const int* row_map;
  const int* stack_live;
  int stack_on;
};

// Complex input c of a record's forward transform: samples 2c and 2c + 1
// of the record (read-only global memory), 0 past its n samples.
template <class T> struct RecordLoad {
  typedef typename C2<T>::type V;
  const T* x;
  int n;
  __device__ __forceinline__ V operator()(int c, bool) const {
    const int k = 2 * c;
    return V{k < n ? __ldg(x + k) : (T)0, k + 1 < n ? __ldg(x + k + 1) : (T)0};
  }
};

// The kernel instantiations: a pointer for cudaLaunchKernel, the occupancy
// query and the shared-memory attribute. BATCH is float32 only.
const void* pipe_kernel_f32(int recipe, bool pf, bool batch);
const void* pipe_kernel_f64(int recipe, bool pf);
// GW: the step switch with its work areas in global memory (single job, no prefetch)
const void* wide_kernel_f32();
const void* wide_kernel_f64();
const void* recipe_kernel_f32(int recipe, bool pf);
const void* recipe_kernel_f64(int recipe, bool pf);

}  // namespace psg
