// psg_cuda.cu — the device side of libpsgcuda.so and its C ABI (include/psg.h).
//
// The hot path is one fused kernel per plan part (pipeline_kernel): each CTA
// takes a trace, loads its live samples from HBM into shared memory once,
// runs every step of the part on it there (demean/detrend/scale/clip/
// polarity, the zero-phase FFT filter with its trend removal, padding and
// trend add-back, AGC with block prefix/suffix sums in float64, per-trace
// normalization with an exact radix selection, gain curves), and writes the
// trace back once. src → dst copies of dead rows and of samples past the live
// length ride in the same kernel. A per-panel normalization splits the plan
// into parts; its factor is computed on the device by the panel-statistics
// kernels and read by the next part's kernel (no host round trip).

#include <cuda_runtime.h>

#include <algorithm>
#include <complex>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include <type_traits>

#include "psg_device.cuh"
#include "psg_internal.h"

using namespace psgd;

namespace psg {

static thread_local std::string t_err;
void set_error(const std::string& m) { t_err = m; }

#define CUDA_OK(x)                                                                         \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess) throw CudaError(std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

}  // namespace psg

#include "psg_kernel.cuh"
#include "psg_trace.h"

namespace psg {

// ======================================================= panel statistics
// gain/stats.nim:253-304: per row Σx² and max |x| (pass 1), then one CTA
// folds the usable rows, and for a percentile counts a 65536-bin histogram
// of the float32 bits of |x| >> 15 and reads the order statistics from it.
template <class T>
__global__ void __launch_bounds__(256) row_stats_kernel(const T* __restrict__ b, long long rows, int cols,
                                                        const int* __restrict__ live, double* __restrict__ ss,
                                                        double* __restrict__ mx) {
  __shared__ SharedMem S;
  for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
    int n = min(max(live[r], 0), cols);
    const T* x = b + r * (long long)cols;
    double s = 0;
    unsigned long long m = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double v = (double)x[i];
      s += v * v;
      unsigned long long bb = abs_bits(x[i]);
      m = bb > m ? bb : m;
    }
    s = block_sum(s, S.red[0][0]);
    m = block_max_u64(m, S.redu[0]);
    if (threadIdx.x == 0) {
      ss[r] = s;
      mx[r] = n > 0 ? bits_value(m, (T)0) : (double)NAN;
    }
    __syncthreads();
  }
}

struct PanelOut {
  double rms, maxAbs, clip, rows, samples;
  double factor;
  double k_rank;
  double sum_sq;  // Σx² of the usable rows
};

__device__ __forceinline__ bool usable_d(double ssr, double mxr, int n) {
  return n > 0 && !isnan(mxr) && !isinf(mxr) && !(ssr == INFINITY);
}

// One CTA: fold the rows; for `stat` < 0 no factor is computed.
// signed_live: live[r] < 0 marks a row that is not live and live[r] == 0 a
// live row with no live samples, which panelStats counts among its rows
// (gain/stats.nim:267-276: sumSqMaxAbs of no samples is (0, 0), usable);
// otherwise (the pipeline's flattening) live[r] == 0 is a row not processed.
__global__ void __launch_bounds__(1024) panel_fold_kernel(long long rows, int cols, const int* __restrict__ live,
                                                          const double* __restrict__ ss, const double* __restrict__ mx,
                                                          PanelOut* out, int signed_live = 0) {
  __shared__ SharedMem S;
  double sum = 0, cnt = 0, nr = 0;
  unsigned long long mb = 0;
  for (long long r = threadIdx.x; r < rows; r += blockDim.x) {
    int n = min(max(live[r], 0), cols);
    if (signed_live && live[r] == 0) {
      nr += 1;
      continue;
    }
    if (!usable_d(ss[r], mx[r], n)) continue;
    sum += ss[r];
    cnt += (double)n;
    nr += 1;
    unsigned long long b = (unsigned long long)__double_as_longlong(mx[r]);
    mb = b > mb ? b : mb;
  }
  sum = block_sum(sum, S.red[0][0]);
  cnt = block_sum(cnt, S.red[0][0]);
  nr = block_sum(nr, S.red[0][0]);
  mb = block_max_u64(mb, S.redu[0]);
  if (threadIdx.x == 0) {
    out->rows = nr;
    out->samples = cnt;
    out->clip = NAN;
    out->rms = cnt > 0 ? sqrt(sum / cnt) : 0.0;
    out->maxAbs = cnt > 0 ? __longlong_as_double((long long)mb) : 0.0;
    out->sum_sq = sum;
  }
}

// The 65536-bin histogram of |x| (float32 bits >> 15, capped at 0xFEFF) over
// the usable rows' live samples (gain/stats.nim:208-235), added into `hist`.
// Each CTA counts its rows' samples in shared memory, the counts of bins 2k
// and 2k + 1 as the two 16-bit halves of word k (128 KB), and adds them to
// the global histogram before any count could pass 65535 (every 65535
// samples it takes) and at its end: shared-memory atomics where a filtered
// panel's samples pile onto a few hundred bins, instead of global ones.
constexpr int kHistWords = 65536 / 2;
template <class T>
__global__ void __launch_bounds__(512) panel_hist_kernel(const T* __restrict__ b, long long rows, int cols,
                                                         const int* __restrict__ live, const double* __restrict__ ss,
                                                         const double* __restrict__ mx, unsigned* __restrict__ hist) {
  extern __shared__ unsigned h2[];
  for (int k = threadIdx.x; k < kHistWords; k += blockDim.x) h2[k] = 0;
  __syncthreads();
  auto flush = [&]() {
    __syncthreads();
    for (int k = threadIdx.x; k < kHistWords; k += blockDim.x) {
      const unsigned w = h2[k];
      if (w) {
        if (w & 0xFFFFu) atomicAdd(&hist[2 * k], w & 0xFFFFu);
        if (w >> 16) atomicAdd(&hist[2 * k + 1], w >> 16);
        h2[k] = 0;
      }
    }
    __syncthreads();
  };
  int pending = 0;  // samples counted since the last flush (the same in every thread)
  for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
    const int n = min(max(live[r], 0), cols);
    if (!usable_d(ss[r], mx[r], n)) continue;
    const T* x = b + r * (long long)cols;
    for (int i0 = 0; i0 < n; i0 += 65535) {
      const int m = min(n - i0, 65535);
      if (pending + m > 65535) {
        flush();
        pending = 0;
      }
      for (int i = i0 + (int)threadIdx.x; i < i0 + m; i += blockDim.x) {
        const float a = (float)fabs((double)x[i]);
        const unsigned key = min(__float_as_uint(a) >> 15, 0xFEFFu);
        atomicAdd(&h2[key >> 1], (key & 1u) ? 0x10000u : 1u);
      }
      pending += m;
    }
  }
  flush();
}

// orderStat (gain/stats.nim:237-251) for ranks j0 and j0 + 1, one CTA of
// 1024. The counts are uint32 (one device's histogram) or float64 (the
// merged histogram of several shards, exact integers).
template <class C>
__device__ double order_stat_from(const C* hist, long long j, double mxv, int bin, long long below) {
  if (bin == 0) return 0;
  double c = (double)hist[bin];
  double lo = (double)__uint_as_float((unsigned)bin << 15);
  double hi = fmin((double)__uint_as_float((unsigned)(bin + 1) << 15), mxv);
  return fmin(fmax(lo + ((double)(j - below) + 0.5) / c * (hi - lo), lo), mxv);
}

template <class C>
__global__ void __launch_bounds__(1024) panel_clip_kernel(const C* __restrict__ hist, PanelOut* out,
                                                          double clipP, int stat, double target, int dtype) {
  // warp w owns the bins [2048·w, 2048·w + 2048), read 32 at a time by its
  // lanes (coalesced): their count, then the warps' exclusive prefix
  __shared__ long long seg[32], segbase[32];
  __shared__ long long found_below[2];
  __shared__ int found_bin[2];
  const int maxKey = 0xFEFF;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  auto count = [&](int bin) -> long long { return bin <= maxKey ? (long long)hist[bin] : 0; };
  long long tot = 0;
  for (int c = 0; c < 64; c++) tot += count(warp * 2048 + c * 32 + lane);
  for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
  if (lane == 0) seg[warp] = tot;
  __syncthreads();
  if (warp == 0) {
    long long v = seg[lane], incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const long long u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    segbase[lane] = incl - v;
  }
  double samples = out->samples, mxv = out->maxAbs;
  bool have = samples > 0 && !isnan(clipP);
  double rank = have ? (samples - 1) * clipP / 100 : 0;
  long long k0 = have ? (long long)fmin(floor(rank), samples - 1) : 0;
  if (threadIdx.x < 2) {
    found_bin[threadIdx.x] = -1;
    found_below[threadIdx.x] = 0;
  }
  __syncthreads();
  if (have) {
    for (int q = 0; q < 2; q++) {
      const long long j = k0 + q;
      // the warp whose bins hold rank j walks them 32 at a time
      if (j >= segbase[warp] && j < segbase[warp] + seg[warp]) {
        long long below = segbase[warp];
        for (int c = 0; c < 64; c++) {
          const int bin = warp * 2048 + c * 32 + lane;
          const long long v = count(bin);
          long long incl = v;
          for (int o = 1; o < 32; o <<= 1) {
            const long long u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
          }
          const unsigned hit = __ballot_sync(0xffffffffu, below + incl > j);
          if (hit) {
            const int l = __ffs(hit) - 1;
            if (lane == l) {
              found_bin[q] = bin;
              found_below[q] = below + incl - v;
            }
            break;
          }
          below += __shfl_sync(0xffffffffu, incl, 31);
        }
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double clip = NAN;
    if (have) {
      if (clipP == 100) {
        clip = mxv;
      } else {
        double lower = found_bin[0] < 0 ? mxv : order_stat_from(hist, k0, mxv, found_bin[0], found_below[0]);
        double f = rank - (double)k0;
        if (f == 0 || (double)(k0 + 1) >= samples) clip = lower;
        else {
          double upper = found_bin[1] < 0 ? mxv : order_stat_from(hist, k0 + 1, mxv, found_bin[1], found_below[1]);
          clip = lower + f * (upper - lower);
        }
      }
    }
    out->clip = clip;
    double factor = NAN;
    if (stat >= 0) {
      double level = stat == PSG_NORM_MAX ? out->maxAbs : (stat == PSG_NORM_RMS ? out->rms : clip);
      bool ok = dtype == PSG_F32 ? fits_d<float>(target / level) : fits_d<double>(target / level);
      if (fin_pos_d(level) && ok) factor = target / level;
    }
    out->factor = factor;
  }
}


// Mergeable statistics of a shard of a panel: {Σx², samples, rows, maxAbs}
// of its usable rows, then the 65536 histogram counts as float64 (exact).
// Shards merge by summing every entry but maxAbs, which takes the maximum.
__global__ void panel_partial_head_kernel(const PanelOut* fold, double* partial) {
  partial[0] = fold->sum_sq;
  partial[1] = fold->samples;
  partial[2] = fold->rows;
  partial[3] = fold->maxAbs;
}

__global__ void hist_to_f64_kernel(const unsigned* __restrict__ hist, double* __restrict__ out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < 65536) out[k] = (double)hist[k];
}

// The panel output of merged partials: rms, maxAbs, rows and samples.
__global__ void partial_to_out_kernel(const double* __restrict__ partial, PanelOut* out) {
  double cnt = partial[1];
  out->samples = cnt;
  out->rows = partial[2];
  out->rms = cnt > 0 ? sqrt(partial[0] / cnt) : 0.0;
  out->maxAbs = cnt > 0 ? partial[3] : 0.0;
  out->clip = NAN;
}

// ============================================================ correlation
// CorrArgs and RecordLoad: psg_kernel.cuh.

// correlateInto (vibroseis/correlate.nim:205-300, 421-464) one record per CTA
// pass, with the vertical-stack add (vstack.nim:186-202) fused after it.
template <class T, class M>
__device__ __forceinline__ void corr_rows(const CorrArgs& a, const M& mem, SharedMem& S) {
  typedef typename C2<T>::type V;
  const int m = a.nfft / 2;
  V* buf = reinterpret_cast<V*>(mem.base());
  const T* src = reinterpret_cast<const T*>(a.src);
  T* dst = reinterpret_cast<T*>(a.dst);
  const V* tw = reinterpret_cast<const V*>(a.tw);
  const int wrapped = min(max(1 - a.pilot_len - a.shift, 0), a.out);
  const int direct = min(max(-a.shift, wrapped), a.out);
  const int last = min(max(a.record - a.shift, direct), a.out);
  for (long long r = blockIdx.x; r < a.rows; r += gridDim.x) {
    int n = min(max(a.live[r], 0), a.cols);
    const V* y = nullptr;
    if (n > 0) {
      const T* x = src + r * (long long)a.cols;
      // the record, zero-padded to nfft, read by the forward transform's
      // first pass straight from global memory (RecordLoad)
      constexpr int MAXR = sizeof(T) == 4 ? 16 : 8;
      const RecordLoad<T> rec{x, n};
      const int zo = cfft_forward_loaded<T, MAXR, 0>(mem, m, 0, a.fft, tw, rec);
      const BridgeLoad<T, M> bridge{mem, zo, m, reinterpret_cast<const Quad<T>*>(a.bridge)};
      y = buf + cfft_forward_loaded<T, MAXR, 0>(mem, zo == 0 ? m : 0, zo, a.fft, tw, bridge);
    }
    // lagSpans / scatter: the output at column c reads lag c + shift
    // (wrapped by nfft for negative lags).
    auto value = [&](int c) -> T {
      if (!y || c < wrapped || c >= last) return (T)0;
      int idx = c < direct ? c + a.shift + a.nfft : c + a.shift;
      V v = y[idx >> 1];
      return (idx & 1) ? v.x : v.y;
    };
    if (dst) {
      T* d = dst + r * (long long)a.out;
      for (int c = threadIdx.x; c < a.out; c += blockDim.x) d[c] = value(c);
    }
    if (a.stack_on) {
      int o = a.row_map ? a.row_map[r] : (int)r;
      int sn = a.stack_live ? min(max(a.stack_live[r], 0), a.stack_samples) : min(a.out, a.stack_samples);
      if (o >= 0 && o < a.stack_rows && sn > 0) {
        double bad = 0;
        for (int c = threadIdx.x; c < sn; c += blockDim.x) {
          double v = (double)value(c);
          bad += v - v;  // allFinite: x − x is 0 for finite x
        }
        bad = block_sum(bad, S.red[0][0]);
        if (bad == 0) {
          double* nm = a.num + (long long)o * a.stack_samples;
          int* ct = a.cnt + (long long)o * a.stack_samples;
          for (int c = threadIdx.x; c < sn; c += blockDim.x) {
            atomicAdd(nm + c, (double)value(c));
            atomicAdd(ct + c, 1);
          }
        }
      }
    }
    __syncthreads();
  }
}

// correlateInto (vibroseis/correlate.nim:205-300, 421-464) one record per CTA
// pass, with the vertical-stack add (vstack.nim:186-202) fused after it. A
// record's two transform buffers fill most of an SM's shared memory (one CTA
// per SM at nfft 16200), so the CTA is 512 threads wide: 16 warps per SM to
// hide the latency of the record's loads and of the passes.
constexpr int kCorrThreads = 512;
template <class T>
__global__ void __launch_bounds__(kCorrThreads) corr_kernel(CorrArgs a) {
  __shared__ SharedMem S;
  if (a.gwork) {
    typedef typename C2<T>::type V;
    InGlobal g{reinterpret_cast<unsigned char*>(a.gwork) + (size_t)blockIdx.x * a.nfft * sizeof(V)};
    corr_rows<T>(a, g, S);
  } else {
    corr_rows<T>(a, InShared(), S);
  }
}

// RecordStack.addRecord for a block already in memory.
template <class T>
__global__ void __launch_bounds__(256) stack_add_kernel(const T* __restrict__ b, long long rows, int cols,
                                                        const int* __restrict__ live, const int* __restrict__ row_map,
                                                        double* num, int* cnt, int samples, long long out_rows) {
  __shared__ SharedMem S;
  for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
    int o = row_map ? row_map[r] : (int)r;
    int n = min(max(live[r], 0), min(cols, samples));
    if (o < 0 || o >= out_rows || n == 0) continue;
    const T* x = b + r * (long long)cols;
    double bad = 0;
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
      double v = (double)x[c];
      bad += v - v;
    }
    bad = block_sum(bad, S.red[0][0]);
    if (bad == 0) {
      for (int c = threadIdx.x; c < n; c += blockDim.x) {
        num[(long long)o * samples + c] += (double)x[c];
        cnt[(long long)o * samples + c] += 1;
      }
    }
    __syncthreads();
  }
}

template <class T>
__global__ void stack_result_kernel(const double* __restrict__ num, const int* __restrict__ cnt, long long total,
                                    int norm, T* __restrict__ d) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    double c = (double)cnt[i];
    T v;
    if (c == 0) v = (T)0;
    else if (norm == PSG_FN_NONE) v = (T)num[i];
    else if (norm == PSG_FN_FOLD) v = (T)(num[i] / c);
    else v = (T)(num[i] / sqrt(c));
    d[i] = v;
  }
}

// ============================================================ spectra
struct SpecArgs {
  const void* src;
  long long row0, row1;  // the rows taken (inclusive)
  int cols, first_col;
  const int* live;
  int window, nfft, bins, odd, demean;
  const void* taper;  // T[window]
  double taper_sum;
  const void* tw;     // ω_m^e of the complex FFT
  const void* split;  // exp(−2πik/nfft), k = 0 .. nfft/2 (even nfft)
  FftDesc fft;
  void* gwork;        // per-CTA transform buffers in global memory (else NULL)
  long long gstride;
  double* acc;        // average: per CTA, Σ over its rows of |X[k]|²/Σw²
  int* used;          // average: per CTA, its rows
  void* amp;          // amplitude: rows × bins of T (the block's rows)
  void* phase;
};

// The windowed spectrum of rows row0 .. row1 (fft/spectrum.nim:232-416), one
// CTA per row: the window's samples (up to its live end) demeaned in T and
// tapered (a short window with its own end ramp and Σw), the forward
// transform in the CTA's buffers, and per bin either the scaled power added
// to this CTA's accumulator (AVG; rows in order, so the sums are the same on
// every run) or the scaled amplitude and the phase of the row.
// Complex input c of a window's forward transform: (x[j] − mean)·w[j] for
// j < n (w the window's taper, min(w[j], w[n − 1 − j]) for a short window),
// 0 up to nfft; samples 2c and 2c + 1 for an even nfft, sample c (real) for
// an odd one.
template <class T> struct WindowLoad {
  typedef typename C2<T>::type V;
  const T* x;
  const T* taper;
  int n, W;
  T mean;
  bool odd;
  __device__ __forceinline__ T at(int j) const {
    if (j >= n) return (T)0;
    const T w = n == W ? __ldg(taper + j) : min(__ldg(taper + j), __ldg(taper + n - 1 - j));
    return (__ldg(x + j) - mean) * w;
  }
  __device__ __forceinline__ V operator()(int c, bool) const {
    return odd ? V{at(c), (T)0} : V{at(2 * c), at(2 * c + 1)};
  }
};

template <class T, bool AVG, class M>
__device__ __forceinline__ void spectrum_rows(const SpecArgs& a, const M& mem, SharedMem& S) {
  typedef typename C2<T>::type V;
  const T* src = reinterpret_cast<const T*>(a.src);
  const T* taper = reinterpret_cast<const T*>(a.taper);
  const V* tw = reinterpret_cast<const V*>(a.tw);
  const V* split = reinterpret_cast<const V*>(a.split);
  const int W = a.window, n2 = a.nfft, mc = a.odd ? n2 : n2 / 2;  // complex points
  V* buf = reinterpret_cast<V*>(mem.base());
  double* acc = AVG ? a.acc + (size_t)blockIdx.x * a.bins : nullptr;
  int used = 0;
  for (long long r = a.row0 + blockIdx.x; r <= a.row1; r += gridDim.x) {
    const int live = min(max(a.live[r], 0), a.cols);
    if (AVG && live <= a.first_col) continue;
    const int n = max(0, min(live, a.first_col + W) - a.first_col);
    const T* x = src + r * (long long)a.cols + a.first_col;
    double sum = 0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) sum += (double)x[j];
    sum = block_sum(sum, S.red[0][0]);
    const bool finite = sum - sum == 0;
    const T mean = a.demean && n > 0 && finite ? (T)(sum / (double)n) : (T)0;
    double sw = a.taper_sum;
    if (n != W) {
      // a short window: its own taper, min(w[j], w[n − 1 − j]), and its sum
      sw = 0;
      for (int j = threadIdx.x; j < n; j += blockDim.x) sw += (double)min(taper[j], taper[n - 1 - j]);
      sw = block_sum(sw, S.red[1][0]);
    }
    if (!finite) sw = NAN;
    if (AVG && !(sw > 0)) continue;  // a NaN or infinite sample: the row is left out
    // the demeaned, tapered window, zero-padded to nfft, read by the forward
    // transform's first pass straight from global memory (WindowLoad)
    constexpr int MAXR = sizeof(T) == 4 ? 16 : 8;
    const WindowLoad<T> win{x, taper, n, W, mean, (bool)a.odd};
    const V* z = buf + cfft_forward_loaded<T, MAXR, 0>(mem, mc, 0, a.fft, tw, win);
    const double sc = AVG ? 1 / (sw * sw) : 0.0;
    for (int k = threadIdx.x; k < a.bins; k += blockDim.x) {
      T re, im;
      if (a.odd) {
        re = z[k].x;
        im = z[k].y;
      } else if (k == 0 || k == mc) {
        // the real DC and Nyquist bins: Re z0 ± Im z0
        re = k == 0 ? z[0].x + z[0].y : z[0].x - z[0].y;
        im = (T)0;
      } else {
        // X[k] = E − i·ω^k·O, E = (z[k] + conj z[m−k])/2, O = (z[k] − conj z[m−k])/2
        const V p = z[k], q = z[mc - k], w = split[k];
        const T er = (p.x + q.x) * (T)0.5, ei = (p.y - q.y) * (T)0.5;
        const T orr = (p.x - q.x) * (T)0.5, oi = (p.y + q.y) * (T)0.5;
        const T tr = w.x * orr - w.y * oi, ti = w.x * oi + w.y * orr;  // ω^k·O
        re = er + ti;
        im = ei - tr;
      }
      if (AVG) {
        const double dr = (double)re, di = (double)im;
        acc[k] += (dr * dr + di * di) * sc;
      } else {
        const double side = (k == 0 || 2 * k == n2) ? 1.0 : 2.0;
        reinterpret_cast<T*>(a.amp)[r * (long long)a.bins + k] = (T)(hypot((double)re, (double)im) * side / sw);
        reinterpret_cast<T*>(a.phase)[r * (long long)a.bins + k] = (T)atan2((double)im, (double)re);
      }
    }
    used++;
    __syncthreads();  // the buffers are refilled for the next row
  }
  if (AVG && threadIdx.x == 0) a.used[blockIdx.x] = used;
}

template <class T, bool AVG>
__global__ void __launch_bounds__(256) spectrum_kernel(SpecArgs a) {
  __shared__ SharedMem S;
  if (AVG)
    for (int k = threadIdx.x; k < a.bins; k += blockDim.x) a.acc[(size_t)blockIdx.x * a.bins + k] = 0;
  __syncthreads();
  if (a.gwork) {
    spectrum_rows<T, AVG>(a, InGlobal{reinterpret_cast<unsigned char*>(a.gwork) + (size_t)blockIdx.x * a.gstride}, S);
  } else {
    spectrum_rows<T, AVG>(a, InShared(), S);
  }
}

// averageAmplitudeInto's last step, one CTA per bin: the CTAs' sums of the
// bin (each thread a fixed set of CTAs, then a fixed reduction tree, so the
// bits repeat), sqrt(mean power)·sides, and the rows averaged.
__global__ void __launch_bounds__(256) spectrum_finish(const double* __restrict__ acc, const int* __restrict__ used,
                                                       int ctas, int bins, int nfft, double* __restrict__ amp,
                                                       long long* __restrict__ used_out) {
  __shared__ double red_t[32], red_u[32];
  const int k = blockIdx.x;
  double t = 0, u = 0;
  for (int b = threadIdx.x; b < ctas; b += blockDim.x) {
    t += acc[(size_t)b * bins + k];
    u += (double)used[b];
  }
  t = block_sum(t, red_t);
  u = block_sum(u, red_u);
  if (threadIdx.x == 0) {
    const double side = (k == 0 || 2 * k == nfft) ? 1.0 : 2.0;
    amp[k] = u > 0 ? sqrt(t / u) * side : 0.0;
    if (k == 0 && used_out) *used_out = (long long)u;
  }
}

// ============================================================ SEG-Y decode
// The sample formats of SEG-Y rev 2 (data sample format code, binary header
// bytes 3225-3226): 1 IBM hexadecimal float, 2 int32, 3 int16, 5 IEEE
// float32, 6 IEEE float64, 7 int24, 8 int8, 10 uint32, 11 uint16, 15
// uint24, 16 uint8; big-endian unless the file is little-endian.
__host__ __device__ inline int segy_sample_bytes(int format) {
  switch (format) {
    case 1: case 2: case 5: case 10: return 4;
    case 3: case 11: return 2;
    case 6: return 8;
    case 7: case 15: return 3;
    case 8: case 16: return 1;
    default: return 0;
  }
}
// An unsigned big- (or little-) endian integer of `n` bytes at p.
__device__ __forceinline__ unsigned long long segy_uint(const unsigned char* __restrict__ p, int n, bool little) {
  unsigned long long v = 0;
  for (int i = 0; i < n; i++) v = (v << 8) | (unsigned long long)__ldg(p + (little ? n - 1 - i : i));
  return v;
}
// One sample as a double: exact for every format (an IBM float's 24-bit
// fraction times 16^(e − 64) is a double).
__device__ __forceinline__ double segy_value(unsigned long long u, int format) {
  switch (format) {
    case 1: {  // IBM: sign, 7-bit excess-64 base-16 exponent, 24-bit fraction
      // fraction · 2^(4e − 280), the power of two built as a double (exact:
      // 4e − 280 lies in −280 .. 228)
      const int e2 = 4 * (int)((u >> 24) & 0x7f) - 280;
      const double f = (double)(unsigned)(u & 0xffffffu) * __hiloint2double((e2 + 1023) << 20, 0);
      return (u >> 31) ? -f : f;
    }
    case 2: return (double)(int)(unsigned)u;
    case 3: return (double)(short)(unsigned short)u;
    case 5: return (double)__uint_as_float((unsigned)u);
    case 6: return __longlong_as_double((long long)u);
    case 7: return (double)((int)((unsigned)u << 8) >> 8);
    case 8: return (double)(signed char)(unsigned char)u;
    default: return (double)u;  // 10, 11, 15, 16: unsigned
  }
}
// Rows of raw trace records (a header of `header_bytes`, then `samples`
// samples) into a block of T, `out_cols` wide (zeros past the record's
// samples). One CTA per row; a warp reads consecutive samples.
// 4- and 2-byte samples on their own alignment (every row's samples start
// aligned when the records' base, header and length are) are read one word
// per sample, four words in flight per thread, and byte-swapped with a
// permute; other layouts byte by byte.
template <class T, class W>
__device__ __forceinline__ void segy_words(const W* __restrict__ w, T* __restrict__ o, int samples, int out_cols,
                                           int format, bool le) {
  constexpr int U = 4;
  for (int j0 = threadIdx.x; j0 < out_cols; j0 += U * blockDim.x) {
    unsigned u[U];
#pragma unroll
    for (int q = 0; q < U; q++) {
      const int j = j0 + q * (int)blockDim.x;
      u[q] = j < samples ? (unsigned)__ldg(w + j) : 0u;
    }
#pragma unroll
    for (int q = 0; q < U; q++) {
      const int j = j0 + q * (int)blockDim.x;
      if (j < out_cols) {
        unsigned v = u[q];
        if (!le) v = sizeof(W) == 4 ? __byte_perm(v, 0, 0x0123) : (__byte_perm(v, 0, 0x3201) & 0xffffu);
        o[j] = j < samples ? (T)segy_value(v, format) : (T)0;
      }
    }
  }
}
template <class T>
__global__ void __launch_bounds__(256) segy_decode_kernel(const unsigned char* __restrict__ rec, long long rows,
                                                          long long record_bytes, int header_bytes, int samples,
                                                          int format, int little, T* __restrict__ out, int out_cols) {
  const int sz = segy_sample_bytes(format);
  const bool le = little != 0;
  const bool words = (sz == 4 || sz == 2) && (((uintptr_t)rec | (uintptr_t)header_bytes | (uintptr_t)record_bytes) % sz) == 0;
  for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
    const unsigned char* p = rec + r * record_bytes + header_bytes;
    T* o = out + r * (long long)out_cols;
    if (words && sz == 4) {
      segy_words<T>(reinterpret_cast<const unsigned*>(p), o, samples, out_cols, format, le);
    } else if (words) {
      segy_words<T>(reinterpret_cast<const unsigned short*>(p), o, samples, out_cols, format, le);
    } else {
      for (int j = threadIdx.x; j < out_cols; j += blockDim.x)
        o[j] = j < samples ? (T)segy_value(segy_uint(p + (long long)j * sz, sz, le), format) : (T)0;
    }
  }
}
// The trace-header keys a meta needs, one thread per row (SEG-Y rev 2 trace
// header, 1-based byte positions): the trace identification code (29-30:
// 1 live, 2 dead, 0 unknown, others auxiliary), the offset (37-40, int32),
// the delay recording time (109-110, int16 ms), the number of samples
// (115-116, uint16) and the sample interval (117-118, uint16 µs).
__global__ void segy_keys_kernel(const unsigned char* __restrict__ rec, long long rows, long long record_bytes,
                                 int little, int* __restrict__ status, int* __restrict__ num_samples,
                                 double* __restrict__ interval_us, double* __restrict__ offset,
                                 double* __restrict__ t0_ms) {
  const bool le = little != 0;
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < rows; r += (long long)gridDim.x * blockDim.x) {
    const unsigned char* h = rec + r * record_bytes;
    const int code = (short)(unsigned short)segy_uint(h + 28, 2, le);
    if (status) status[r] = code == 1 ? PSG_TS_LIVE : (code == 2 ? PSG_TS_DEAD : (code == 0 ? PSG_TS_UNKNOWN : PSG_TS_AUX));
    if (offset) offset[r] = (double)(int)(unsigned)segy_uint(h + 36, 4, le);
    if (t0_ms) t0_ms[r] = (double)(short)(unsigned short)segy_uint(h + 108, 2, le);
    if (num_samples) num_samples[r] = (int)segy_uint(h + 114, 2, le);
    if (interval_us) interval_us[r] = (double)segy_uint(h + 116, 2, le);
  }
}

// ============================================================ per-row scale
// scaleRows / scaleRowsInto (core/calibrate.nim:562-612): row r times T(k[r])
// over its first n[r] samples, the rest (and rows with n = 0) copied from
// src when it is another block. One CTA per row, four samples in flight per
// thread.
template <class T>
__global__ void __launch_bounds__(256) scale_rows_kernel(const T* __restrict__ src, T* __restrict__ dst, long long rows,
                                                         int cols, const int* __restrict__ live,
                                                         const double* __restrict__ k) {
  for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
    const int n = min(max(live[r], 0), cols);
    const T f = (T)k[r];
    const T* x = src + r * (long long)cols;
    T* y = dst + r * (long long)cols;
    const bool copy = src != dst;
    if (!copy && n == 0) continue;
    const int end = copy ? cols : n;
    for (int j0 = threadIdx.x; j0 < end; j0 += 4 * blockDim.x) {
      T v[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int j = j0 + q * (int)blockDim.x;
        v[q] = j < end ? x[j] : (T)0;
      }
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int j = j0 + q * (int)blockDim.x;
        if (j < end) y[j] = j < n ? v[q] * f : v[q];
      }
    }
  }
}

// ======================================================== host plumbing
static int g_sm_count = 0, g_max_smem = 0, g_device = -1;

static void ensure_device() {
  int dev;
  CUDA_OK(cudaGetDevice(&dev));
  if (dev != g_device) {
    cudaDeviceProp p;
    CUDA_OK(cudaGetDeviceProperties(&p, dev));
    if (p.major < 10) throw CudaError("libpsgcuda.so needs an sm_100 device, found sm_" + std::to_string(p.major * 10 + p.minor));
    g_sm_count = p.multiProcessorCount;
    g_max_smem = (int)p.sharedMemPerBlockOptin;
    g_device = dev;
  }
}

static void allow_smem(const void* kernel) {
  CUDA_OK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, g_max_smem - (int)sizeof(SharedMem) - 1024));
}

struct DeviceBuf {
  void* p = nullptr;
  ~DeviceBuf() {
    if (p) cudaFree(p);
  }
};

template <class T> static void* upload(std::vector<std::unique_ptr<DeviceBuf>>& keep, const std::vector<T>& v) {
  if (v.empty()) return nullptr;
  auto b = std::make_unique<DeviceBuf>();
  CUDA_OK(cudaMalloc(&b->p, v.size() * sizeof(T)));
  CUDA_OK(cudaMemcpy(b->p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  void* p = b->p;
  keep.push_back(std::move(b));
  return p;
}
template <class T> static std::vector<T> as_t(const std::vector<double>& v) {
  return std::vector<T>(v.begin(), v.end());
}
template <class T>
static std::vector<typename C2<T>::type> as_c(const std::vector<double>& re, const std::vector<double>& im) {
  std::vector<typename C2<T>::type> o(re.size());
  for (size_t i = 0; i < re.size(); i++) o[i] = {(T)re[i], (T)im[i]};
  return o;
}
// The split · multiplier · unsplit map of each pair of bins (BridgeLoad):
// for k ≥ 1, with ω = exp(−2πik/n), c1 = 1 + i·conj ω, c2 = 1 − i·conj ω,
// a1 = (1 − iω)/2, a2 = (1 + iω)/2 and j = m − k:
//   A = c1·a1·M[k] + c2·conj(c2)/2·conj M[j],  B = c1·a2·M[k] + c2·conj(c1)/2·conj M[j],
//   A' = i·conj(A)/n,  B' = i·conj(B)/n;
// bin 0 holds (Re M[0]/n, Re M[m]/n). Computed in float64, rounded to T.
template <class T>
static std::vector<Quad<T>> bridge_table(const FftTables& f, const std::vector<double>& mre, const std::vector<double>& mim) {
  typedef std::complex<double> cd;
  const int64_t m = f.m;
  const double scale = 1.0 / (double)f.n;
  if ((int64_t)mre.size() < m + 1 || (int64_t)mim.size() < m + 1) throw InvalidArg("a bin multiplier shorter than m + 1");
  std::vector<Quad<T>> ab((size_t)m);
  ab[0] = Quad<T>{(T)(mre[0] * scale), (T)(mre[m] * scale), (T)0, (T)0};
  const cd I(0, 1);
  for (int64_t k = 1; k < m; k++) {
    const int64_t j = m - k;
    const cd w(f.split_re[k], f.split_im[k]);
    const cd c1 = 1.0 + I * std::conj(w), c2 = 1.0 - I * std::conj(w);
    const cd a1 = (1.0 - I * w) / 2.0, a2 = (1.0 + I * w) / 2.0;
    const cd Mk(mre[k], mim[k]), Mj(mre[j], mim[j]);
    const cd A = c1 * a1 * Mk + c2 * std::conj(c2) / 2.0 * std::conj(Mj);
    const cd B = c1 * a2 * Mk + c2 * std::conj(c1) / 2.0 * std::conj(Mj);
    const cd Ap = I * std::conj(A) * scale, Bp = I * std::conj(B) * scale;
    ab[k] = Quad<T>{(T)Ap.real(), (T)Ap.imag(), (T)Bp.real(), (T)Bp.imag()};
  }
  return ab;
}

static FftDesc fft_desc(const FftTables& t) {
  FftDesc d{};
  d.m = (int)t.m;
  d.npass = (int)t.radices.size();
  if (d.npass > 24) throw InvalidArg("an FFT of more than 24 passes");
  unsigned long long st = 1;  // the product of the earlier radices
  for (int i = 0; i < d.npass; i++) {
    d.radix[i] = t.radices[i];
    d.magic[i] = st == 1 ? 0u : (unsigned)((1ull << 32) / st + ((1ull << 32) % st != 0));  // ⌈2^32 / s⌉
    st *= (unsigned long long)t.radices[i];
  }
  return d;
}

}  // namespace psg

using namespace psg;

__global__ void trace_stats_finish(double* rms, double* mx, const int* live, long long rows, int cols);

// =================================================================== plans
// A launch shape of a trace-kernel build: the build, the next row's bulk
// copy in flight (pf), one CTA per row (the block scheduler balancing
// ragged rows) or a persistent grid of per_sm CTAs per SM, the row
// buffers' size before the transform buffers (work_off), the dynamic
// shared memory, and the build's twiddles pass by pass.
struct TraceCand {
  const TracePlanInfo* tp = nullptr;
  bool pf = false, per_row = false;
  bool row_in_buffer = false;  // the row lives in the first transform buffer (work_off 0)
  int per_sm = 0, work_off = 0;
  size_t smem = 0;
  const void* tw = nullptr;
};
// What the tuner measured for one (part, row-count class): each launch
// shape's time per launch (µs) and the one it chose.
struct TraceTuning {
  int choice = 0;
  int64_t rows = 0;
  std::vector<float> us;
};

struct psg_plan {
  PlanHost host;
  std::vector<std::unique_ptr<DeviceBuf>> keep;
  DevStep* d_steps = nullptr;
  int device = 0;
  int threads = kNT;
  int max_radix = 12;  // the largest FFT radix compiled into the plan's kernel
  std::vector<int> recipe;  // per part: the recipe kernel that runs it (RC_GENERIC: the step switch)
  int x_elems = 0, work_off = 0, x_bytes = 0;
  bool prefetch = false;
  size_t smem = 0;
  int grid = 1;
  bool needs_panel = false;
  // Traces whose FFT and AGC work does not fit beside the row in shared
  // memory: the work areas are per-CTA slices of the workspace's global
  // scratch (gwork_stride bytes each, gwork_bytes for the plan's grid).
  bool wide = false;
  int64_t gwork_stride = 0, gwork_bytes = 0;
  bool needs_keys = false;  // a mute reads each row's offset and t0Ms
  // Per part: the float32 trace kernel's first build (psg_trace.cuh), or
  // nullptr for pipeline_kernel; its recipe slot (0: demean, filter, AGC;
  // 1: then a per-trace normalization); the launch shapes of its builds
  // (the first one the untuned choice).
  std::vector<const TracePlanInfo*> trace;
  std::vector<int> trace_recipe;
  std::vector<std::vector<TraceCand>> trace_cands;
  // The tuner's choices by (part, bit length of the row count), with the
  // times it measured; a part's pinned choice (−1: none) overrides them.
  bool tune = true;
  mutable std::mutex tune_mu;
  mutable std::map<std::pair<int, int>, TraceTuning> tuned;
  mutable std::vector<int> pinned;
};

struct psg_workspace {
  int device = -1;
  void* d = nullptr;
  int64_t bytes = 0;
  void* g = nullptr;  // the work areas of plans with long traces (psg_plan::wide)
  int64_t g_bytes = 0;
  void* sp = nullptr;  // spectra: per-CTA sums and transform buffers
  int64_t sp_bytes = 0;
  // Streams and events of the chunked host-memory apply (created on first use).
  static const int kLanes = 4;
  cudaStream_t lane[kLanes] = {};
  cudaEvent_t start_ev = nullptr, done_ev[kLanes] = {};
  // Asynchronous host applies alternate two slots of staged row metadata;
  // slot_ev[s][i]: lane i is done with the last call that used slot s.
  cudaEvent_t slot_ev[2][kLanes] = {};
  unsigned long long calls = 0;
  // pinned host staging of each slot's metadata (a copy from pageable memory
  // would wait for the stream)
  void* hmeta[2] = {nullptr, nullptr};
  int64_t hmeta_bytes = 0;
  // the staging layout of the last host apply (-1: whole block; else the
  // bytes of a lane's chunk buffer), and its lanes
  int64_t last_layout = 0;
  int last_lanes = 0;
  bool lanes_ready = false;
};

struct psg_corr_plan {
  CorrHost host;
  int dtype = 0;
  std::vector<std::unique_ptr<DeviceBuf>> keep;
  void* bridge = nullptr;
  void* tw = nullptr;
  void* gwork = nullptr;
  size_t smem = 0;
  int grid = 1;
  FftDesc fft{};
  // the compile-time correlation kernel (float32, a transform length it is
  // built for), its twiddles pass by pass and its grid; else corr_kernel
  const TracePlanInfo* trace = nullptr;
  void* tw_pass = nullptr;
  int trace_grid = 1;
};

struct psg_spectrum_plan {
  SpectrumHost host;
  std::vector<std::unique_ptr<DeviceBuf>> keep;
  void* taper = nullptr;
  void* tw = nullptr;
  void* split = nullptr;
  FftDesc fft{};
  size_t smem = 0;   // dynamic shared memory per CTA (0: global buffers)
  int grid = 1;
  int64_t gstride = 0;
};

struct psg_stack {
  int64_t rows = 0;
  int32_t samples = 0;
  double dt_ms = 0;
  double* num = nullptr;
  int* cnt = nullptr;
};

template <class F> static int guarded(F&& f) {
  try {
    f();
    t_err.clear();
    return PSG_OK;
  } catch (const InvalidArg& e) {
    t_err = e.what();
    return PSG_EINVAL;
  } catch (const WorkspaceError& e) {
    t_err = e.what();
    return PSG_EWORKSPACE;
  } catch (const NoMemory& e) {
    t_err = e.what();
    return PSG_ENOMEM;
  } catch (const CudaError& e) {
    t_err = e.what();
    std::string w = e.what();
    if (w.find("out of memory") != std::string::npos) return PSG_ENOMEM;
    if (w.find("needs an sm_100") != std::string::npos || w.find("no CUDA-capable") != std::string::npos) return PSG_ENODEV;
    return PSG_ECUDA;
  } catch (const std::bad_alloc&) {
    t_err = "host allocation failed";
    return PSG_ENOMEM;
  } catch (const std::exception& e) {
    t_err = e.what();
    return PSG_EINVAL;
  }
}

// Workspace layout (bytes): [0, 512) panel outputs and factors, then
// rows × 16 B of per-row statistics, then the 65536-bin histogram, then the
// host-path staging (live, start_ms, samples).
// Launches panel_hist_kernel: one CTA of 512 per SM (its 128 KB of counts).
template <class T>
static void launch_hist(const T* blk, long long rows, int cols, const int* live, const double* ss, const double* mx,
                        unsigned* hist, cudaStream_t s) {
  if (rows <= 0) return;
  const size_t sm = (size_t)kHistWords * sizeof(unsigned);
  CUDA_OK(cudaFuncSetAttribute((const void*)panel_hist_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const int g = (int)std::min<long long>(rows, (long long)g_sm_count);
  panel_hist_kernel<T><<<g, 512, sm, s>>>(blk, rows, cols, live, ss, mx, hist);
}

static const int64_t kHist = 65536 * 4;
static int64_t align256(int64_t x) { return (x + 255) / 256 * 256; }
static int64_t ws_device_bytes(int64_t rows) { return 512 + align256(rows * 16) + kHist; }
// The host path streams a block through the device in chunks, one staging
// buffer per lane stream, so that a block larger than the device's memory
// still runs; a plan with a per-panel normalization stages the whole block
// (its factor reads every row). Chunks of about 4 MiB for a call that
// waits (short fill and drain of its own pipeline) and 8 MiB for queued
// calls, whose pipelines follow one another (fewer, longer copies: measured
// 9.2 against 7.9 Gsamples/s on the 2000×3001 panel);
// PSG_HOST_CHUNK_BYTES sets both.
static int64_t chunk_bytes(bool queued) {
  static const int64_t env = [] {
    const char* e = getenv("PSG_HOST_CHUNK_BYTES");
    int64_t v = e ? atoll(e) : 0;
    return v >= (64 << 10) ? v : (int64_t)0;
  }();
  return env ? env : (int64_t)(queued ? 8 << 20 : 4 << 20);
}
static int64_t host_chunk_rows(int64_t rows, int32_t cols, int64_t esz, bool queued) {
  return std::max<int64_t>(16, std::min<int64_t>(rows, chunk_bytes(queued) / std::max<int64_t>(1, cols * esz)));
}
static bool host_whole_block(bool needs_panel, int64_t rows, int32_t cols, int64_t esz, bool queued) {
  return needs_panel || rows <= host_chunk_rows(rows, cols, esz, queued);
}
// One slot of staged row metadata: live, startMs, offset, t0Ms.
static int64_t ws_meta_bytes(int64_t rows) { return align256(rows * 4) + 3 * align256(rows * 8); }
static int64_t ws_host_bytes(bool needs_panel, int64_t rows, int32_t cols, int dtype) {
  int64_t esz = dtype == PSG_F32 ? 4 : 8;
  int64_t stage_rows = 0;  // the larger staging of the two kinds of call
  for (bool queued : {false, true})
    stage_rows = std::max<int64_t>(stage_rows, host_whole_block(needs_panel, rows, cols, esz, queued)
                                                   ? rows
                                                   : psg_workspace::kLanes * host_chunk_rows(rows, cols, esz, queued));
  return ws_device_bytes(rows) + 2 * ws_meta_bytes(rows) + align256(stage_rows * (int64_t)cols * esz);
}

// The pipeline kernel of a sample type and largest radix (psg_pipe_f32.cu,
// psg_pipe_f64.cu).
template <class T> static const void* pipe_kernel_for(int recipe, bool pf) {
  return sizeof(T) == 4 ? pipe_kernel_f32(recipe, pf, false) : pipe_kernel_f64(recipe, pf);
}
template <class T> static const void* wide_kernel_for() { return sizeof(T) == 4 ? wide_kernel_f32() : wide_kernel_f64(); }
// The batched form (float32 plans, any step sequence).
static const void* batch_kernel_for(bool pf) { return pipe_kernel_f32(RC_GENERIC, pf, true); }

// The recipe that runs steps [first, last) of a plan, by their kinds;
// PSG_RECIPES=0 in the environment (read at compile time) keeps every plan on
// the step switch.
static int recipe_of(const PlanHost& h, int first, int last) {
  if (const char* e = getenv("PSG_RECIPES"))
    if (atoi(e) == 0) return RC_GENERIC;
  std::vector<int> k;
  for (int i = first; i < last; i++) k.push_back(h.steps[i].kind);
  if (k == std::vector<int>{ST_DEMEAN, ST_FILTER, ST_AGC}) return RC_DFA;
  if (k == std::vector<int>{ST_DEMEAN, ST_FILTER, ST_AGC, ST_NORM_TRACE}) return RC_DFAN;
  if (k == std::vector<int>{ST_FILTER, ST_NORM_TRACE}) return RC_FN;
  if (k == std::vector<int>{ST_FILTER, ST_GAIN_CURVE}) return RC_FG;
  return RC_GENERIC;
}
static void launch_pipe(const void* kernel, int grid, int threads, size_t smem, cudaStream_t stream, PipeArgs& a) {
  void* args[] = {&a};
  CUDA_OK(cudaLaunchKernel(kernel, dim3(grid), dim3(threads), args, smem, stream));
}

// Double-double on the host (Dekker's and Knuth's error-free sums and
// products), for the IIR scan tables.
namespace hdd {
struct DD {
  double hi, lo;
};
static DD quick(double a, double b) {
  double s = a + b;
  return DD{s, b - (s - a)};
}
static DD two_sum(double a, double b) {
  double s = a + b, bb = s - a;
  return DD{s, (a - (s - bb)) + (b - bb)};
}
static DD add(DD x, DD y) {
  DD s = two_sum(x.hi, y.hi), t = two_sum(x.lo, y.lo);
  s = quick(s.hi, s.lo + t.hi);
  return quick(s.hi, s.lo + t.lo);
}
static DD mul(DD x, DD y) {
  double p = x.hi * y.hi;
  double e = std::fma(x.hi, y.hi, -p) + (x.hi * y.lo + x.lo * y.hi);
  return quick(p, e);
}
struct M2 {
  DD a, b, c, d;
};
static M2 mul(const M2& x, const M2& y) {
  return M2{add(mul(x.a, y.a), mul(x.b, y.c)), add(mul(x.a, y.b), mul(x.b, y.d)), add(mul(x.c, y.a), mul(x.d, y.c)),
            add(mul(x.c, y.b), mul(x.d, y.d))};
}
}  // namespace hdd

// The IIR scan table of a section: for each chunk length L = 1 .. lmax the
// powers P^k, k = 1 .. 32, then P^64 and P^128, of P = M^L,
// M = [[−a1, 1], [−a2, 0]] its state map, as 2×2 double-double matrices
// (kIirTab doubles per L).
static void iir_scan_table(const Biquad& q, int lmax, std::vector<double>& out) {
  const hdd::M2 m{hdd::DD{-q.a1, 0}, hdd::DD{1, 0}, hdd::DD{-q.a2, 0}, hdd::DD{0, 0}};
  hdd::M2 pl{hdd::DD{1, 0}, hdd::DD{0, 0}, hdd::DD{0, 0}, hdd::DD{1, 0}};
  auto put = [&](const hdd::M2& w) {
    out.insert(out.end(), {w.a.hi, w.a.lo, w.b.hi, w.b.lo, w.c.hi, w.c.lo, w.d.hi, w.d.lo});
  };
  for (int L = 1; L <= lmax; L++) {
    pl = hdd::mul(pl, m);
    hdd::M2 w = pl, p32 = pl;
    for (int k = 1; k <= 32; k++) {
      put(w);
      p32 = w;
      w = hdd::mul(w, pl);
    }
    const hdd::M2 p64 = hdd::mul(p32, p32);
    put(p64);
    put(hdd::mul(p64, p64));
  }
}

// The trace kernel's twiddles, pass by pass: pass i (all but the last) of
// radix R after radices of product S holds, for each of its m/(S·R)
// butterflies p, the R − 1 twiddles ω_m^{p·k·S} (k = 1 .. R − 1, padded to
// an even count): the values of the transform's one table ω_m^e, e = p·k·S,
// laid out in the order a butterfly reads them.
static std::vector<float2> trace_twiddles(const TracePlanInfo& t) {
  std::vector<float2> out;
  int64_t S = 1;
  for (int i = 0; i + 1 < t.np; i++) {
    const int R = t.radix[i], tws = (R - 1 + 1) & ~1;
    const int64_t sub = t.m / (S * R);
    for (int64_t pp = 0; pp < sub; pp++)
      for (int k = 1; k <= tws; k++) {
        float2 v{0.f, 0.f};
        if (k < R) {
          const int64_t e = pp * k * S;
          const double a = -2 * 3.141592653589793 * (double)e / (double)t.m;
          v = float2{(float)std::cos(a), (float)std::sin(a)};
        }
        out.push_back(v);
      }
    S *= R;
  }
  return out;
}

// The reference's stages of an m-point transform (fft/plan.nim:120-132): 4s
// first, then a 2, then 3s and 5s.
static std::vector<int> reference_stages(int64_t m) {
  std::vector<int> r;
  while (m % 4 == 0) {
    r.push_back(4);
    m /= 4;
  }
  if (m % 2 == 0) {
    r.push_back(2);
    m /= 2;
  }
  for (int q : {3, 5})
    while (m % q == 0) {
      r.push_back(q);
      m /= q;
    }
  return r;
}
static bool runs_reference_stages(const TracePlanInfo& t) {
  std::vector<int> st;
  for (int i = 0; i < t.np; i++) {
    st.push_back(t.g1[i]);
    if (t.g2[i]) st.push_back(t.g2[i]);
  }
  return st == reference_stages(t.m);
}
// A twiddle as the reference tabulates it (fft/plan.nim:146-155): angle
// −2π·e/cur in float64, its cosine and sine rounded to float32.
static float2 ref_twiddle(int64_t e, int64_t cur) {
  const double a = -2 * 3.14159265358979323846 * (double)e / (double)cur;
  return float2{(float)std::cos(a), (float)std::sin(a)};
}
// The trace kernel's twiddles, pass by pass (psg_trace.cuh ref_pass): for
// each butterfly p of pass i (stride S, radix R, m/(S·R) butterflies), the
// first stage's R2·(R1 − 1) twiddles ω_cur^{((p + jB·m/(S·R))·kA) mod cur}
// (cur = m/S), then the second stage's R2 − 1 twiddles
// ω_{cur/R1}^{(p·kB) mod (cur/R1)}, padded to an even count.
static std::vector<float2> ref_twiddles(const TracePlanInfo& t) {
  std::vector<float2> out;
  int64_t S = 1;
  for (int i = 0; i < t.np; i++) {
    const int R = t.radix[i], r1 = t.g1[i], r2 = t.g2[i], tws = (R - 1 + 1) & ~1;
    const int64_t curA = t.m / S, sub = t.m / (S * R);
    for (int64_t pp = 0; pp < sub; pp++) {
      size_t n0 = out.size();
      if (r2) {
        for (int jB = 0; jB < r2; jB++) {
          const int64_t pA = pp + jB * sub;
          for (int kA = 1; kA < r1; kA++) out.push_back(ref_twiddle((pA * kA) % curA, curA));
        }
        const int64_t curB = curA / r1;
        for (int kB = 1; kB < r2; kB++) out.push_back(ref_twiddle((pp * kB) % curB, curB));
      } else {
        for (int k = 1; k < r1; k++) out.push_back(ref_twiddle((pp * k) % curA, curA));
      }
      while (out.size() - n0 < (size_t)tws) out.push_back(float2{0.f, 0.f});
    }
    S *= R;
  }
  return out;
}

// The trace kernel for part `part` of a float32 plan, or nullptr: a part of
// exactly demean, filter (zero pads), AGC (and a per-trace normalization)
// whose transform length and AGC window one of its builds serves, with the
// row fitting the transform's buffers. PSG_TRACE=0 in the environment (read
// at compile time) keeps every plan on pipeline_kernel.
static const TracePlanInfo* trace_plan_of(const psg_plan* p, int part) {
  if (const char* e = getenv("PSG_TRACE"))
    if (atoi(e) == 0) return nullptr;
  if (p->host.dtype != PSG_F32) return nullptr;
  const int rc = p->recipe[part];
  if (rc != RC_DFA && rc != RC_DFAN) return nullptr;
  const int first = p->host.parts[part].first;
  const StepHost& f = p->host.steps[first + 1];
  const StepHost& ag = p->host.steps[first + 2];
  if (f.kind != ST_FILTER || ag.kind != ST_AGC || f.filter.reflect) return nullptr;
  const int64_t m = f.filter.fft.m;
  if (2 * m < p->host.samples) return nullptr;  // the filtered row lives in one transform buffer
  const TracePlanInfo* const* c = trace_plans_for((int)m, (int)(2 * ag.half + 1));
  return c[0] && runs_reference_stages(*c[0]) ? c[0] : nullptr;
}

template <class T> static void build_device_steps(psg_plan* p) {
  typedef typename C2<T>::type V;
  std::vector<DevStep> ds;
  int64_t work = 0;
  for (auto& s : p->host.steps) {
    DevStep d{};
    d.kind = s.kind;
    d.factor = s.factor;
    d.lo = s.lo;
    d.hi = s.hi;
    d.dt_ms = p->host.dt_ms;
    if (s.kind == ST_FILTER) {
      const FilterHost& f = s.filter;
      if (f.nfft > (1 << 24)) throw InvalidArg("the filter's FFT is too long for the device");
      d.trend = f.trend;
      d.reflect = f.reflect;
      d.zero_dc = f.spec.zero_dc;
      d.pad = (int)f.pad;
      d.nfft = (int)f.nfft;
      d.dc_gain = f.dc_gain;
      d.fft = fft_desc(f.fft);
      d.bridge = upload(p->keep, bridge_table<T>(f.fft, f.gain, std::vector<double>(f.gain.size(), 0.0)));
      d.fall = upload(p->keep, as_t<T>(f.fall));
      d.tw = upload(p->keep, as_c<T>(f.fft.tw_re, f.fft.tw_im));
      for (size_t part = 0; part < p->trace.size(); part++)
        if (p->trace[part] && &p->host.steps[p->host.parts[part].first + 1] == &s) {
          // the trace kernel's tables: twiddles pass by pass, and the split
          // twiddles and gains of each bin pair (c, m − c) as the reference
          // rounds them to float32 (fft/plan.nim:156-159, filter/apply.nim:141)
          const int64_t m = f.fft.m, nf = f.fft.n;
          std::vector<float4> sp((size_t)m);
          std::vector<float2> gg((size_t)m);
          auto split = [&](int64_t k) { return ref_twiddle(k, nf); };
          for (int64_t c = 0; c < m; c++) {
            const float2 a = split(c), b = split(m - c);
            sp[(size_t)c] = float4{a.x, a.y, b.x, b.y};
            gg[(size_t)c] = c == 0 ? float2{(float)f.gain[0], (float)f.gain[m]}
                                   : float2{(float)f.gain[c], (float)f.gain[m - c]};
          }
          d.ref_split = upload(p->keep, sp);
          d.ref_gain = upload(p->keep, gg);
          d.ref_scale = 1.0f / (float)nf;
        }
      work = std::max<int64_t>(work, 2 * f.fft.m * (int64_t)sizeof(V));
    } else if (s.kind == ST_AGC) {
      d.half = (int)s.half;
      d.agc_mode = s.agc_mode;
      d.target = s.target;
      d.epsilon = s.epsilon;
      int64_t n = p->host.samples;
      work = std::max<int64_t>(work, (((n + 1 + 3) & ~3LL) + n) * (int64_t)sizeof(T));
    } else if (s.kind == ST_NORM_TRACE || s.kind == ST_NORM_PANEL) {
      d.stat = s.stat;
      d.norm_target = s.norm_target;
      d.percentile = s.percentile;
    } else if (s.kind == ST_GAIN_CURVE) {
      d.curve = s.curve;
      d.t_min_ms = s.t_min_ms;
      d.table_len = (int)s.table.size();
      d.table = upload(p->keep, as_t<T>(s.table));
    } else if (s.kind == ST_MUTE_TOP || s.kind == ST_MUTE_BOTTOM) {
      d.mute_kind = s.mute.kind;
      d.mute_t = s.mute.t_ms;
      d.ms_per_dist = s.ms_per_dist;
      d.mute_t0 = s.mute.t0_ms;
      d.mute_pad = s.mute.pad_ms;
      d.taper_ms = s.taper_ms;
      if (s.mute.kind == PSG_MK_TABLE) {
        d.n_knots = s.mute.n_knots;
        std::vector<double> k(s.mute.offsets, s.mute.offsets + s.mute.n_knots);
        k.insert(k.end(), s.mute.times_ms, s.mute.times_ms + s.mute.n_knots);
        d.knots = (const double*)upload(p->keep, k);
      }
      p->needs_keys = true;
    } else if (s.kind == ST_IIR) {
      const IirHost& f = s.iir;
      d.trend = f.trend;
      d.reflect = f.reflect;
      d.dc_gain = f.dc_gain;
      d.dc_slope = f.dc_slope;
      d.n_sec = (int)f.sections.size();
      d.iir_zero = f.phase == PSG_IP_ZERO;
      d.lead = (int)f.lead;
      d.tail = (int)f.tail;
      if (f.lead + f.tail > (1 << 24)) throw InvalidArg("the IIR filter's pads are too long for the device");
      std::vector<double> sec, pw;
      const int lmax = (int)((f.lead + p->host.samples + f.tail + kNT - 1) / kNT);
      for (const Biquad& b : f.sections) {
        sec.insert(sec.end(), {b.b0, b.b1, b.b2, b.a1, b.a2, b.g});
        iir_scan_table(b, lmax, pw);
      }
      d.pw_len = lmax;
      if (!sec.empty()) {
        d.sec = (const double*)upload(p->keep, sec);
        d.pw = (const double*)upload(p->keep, pw);
        static_assert(kIirTab == 34 * 8, "the IIR scan table holds P^1 .. P^32, P^64, P^128 per chunk length");
      }
      work = std::max<int64_t>(work, (f.lead + p->host.samples + f.tail) * 8);
    }
    if (s.kind == ST_NORM_PANEL) p->needs_panel = true;
    // what the step needs of its input (accumulated by the loop before it)
    switch (s.kind) {
      case ST_DEMEAN: d.need = NEED_S1; break;
      case ST_DETREND: d.need = NEED_S1 | NEED_SI; break;
      case ST_FILTER:
        d.need = s.filter.trend == PSG_TR_LINEAR ? (NEED_S1 | NEED_SI) : (s.filter.trend == PSG_TR_MEAN ? NEED_S1 : 0);
        break;
      case ST_IIR:
        d.need = s.iir.trend == PSG_TR_LINEAR ? (NEED_S1 | NEED_SI) : (s.iir.trend == PSG_TR_MEAN ? NEED_S1 : 0);
        break;
      case ST_AGC: d.need = NEED_S2; break;
      case ST_NORM_TRACE: d.need = s.stat == PSG_NORM_RMS ? NEED_S2 : NEED_MX; break;
      default: d.need = 0;
    }
    ds.push_back(d);
  }
  for (size_t i = 0; i < ds.size(); i++)
    ds[i].need_next = (i + 1 < ds.size() && ds[i + 1].kind != ST_NORM_PANEL) ? ds[i + 1].need : 0;
  // Each part's panel statistics live in a 64-byte slot of the workspace's
  // first 448 bytes.
  if (p->host.parts.size() > 6) throw InvalidArg("a plan takes at most 5 per-panel normalizations after its first op");
  p->x_elems = (int)((p->host.samples + 3) & ~3LL);
  // Row buffers with room for the 16-byte alignment of a row's body: two
  // (the next row's bulk load lands in the other) when that keeps as many
  // CTAs on an SM as one does, else one.
  p->x_bytes = (int)align256((p->host.samples + 8) * (int64_t)sizeof(T));
  auto occupancy = [&](bool pf) {
    size_t sm = (size_t)((pf ? 2 : 1) * p->x_bytes + work);
    auto k = pipe_kernel_for<T>(RC_GENERIC, pf);
    allow_smem(k);
    int per_sm = 0;
    CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, p->threads, sm));
    return per_sm;
  };
  int limit = g_max_smem - (int)sizeof(SharedMem) - 1024;
  // PSG_WIDE=1 in the environment (read at compile time) puts every plan's
  // work areas in global memory: the layout of long traces, for any plan.
  const char* wide_env = getenv("PSG_WIDE");
  const bool force_wide = wide_env && atoi(wide_env) != 0;
  if (!force_wide && (int64_t)p->x_bytes + work <= limit) {
    int one = occupancy(false), two = occupancy(true);
    p->prefetch = two > 0 && two >= one;
    if (const char* e = getenv("PSG_PREFETCH")) p->prefetch = atoi(e) != 0 && two > 0;
    p->work_off = (p->prefetch ? 2 : 1) * p->x_bytes;
    p->smem = (size_t)(p->work_off + work);
  } else {
    // The row alone in shared memory; the FFT and AGC work areas in global
    // memory, one slice per CTA of the grid.
    if (p->x_bytes > limit)
      throw InvalidArg("a trace of " + std::to_string(p->host.samples) + " samples needs " +
                       std::to_string(p->x_bytes) + " bytes of shared memory; the device gives " + std::to_string(limit));
    p->wide = true;
    p->prefetch = false;
    p->work_off = p->x_bytes;
    p->smem = (size_t)p->x_bytes;
    p->gwork_stride = align256(work);
  }
  if (!ds.empty()) {
    DeviceBuf* b = new DeviceBuf();
    p->keep.emplace_back(b);
    CUDA_OK(cudaMalloc(&b->p, ds.size() * sizeof(DevStep)));
    CUDA_OK(cudaMemcpy(b->p, ds.data(), ds.size() * sizeof(DevStep), cudaMemcpyHostToDevice));
    p->d_steps = (DevStep*)b->p;
  }
  auto kern = p->wide ? wide_kernel_for<T>() : pipe_kernel_for<T>(RC_GENERIC, p->prefetch);
  allow_smem(kern);
  int per_sm = 0;
  CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, p->threads, p->smem));
  p->grid = std::max(1, per_sm) * g_sm_count;
  if (p->wide) p->gwork_bytes = p->gwork_stride * p->grid;
  // The trace kernel's launch shapes, part by part: each build of the part's
  // transform length, with the row buffer and its two transform buffers,
  // with the next row's copy in flight or not, on a persistent grid or one
  // CTA per row. The first shape is the untuned choice: the first build, the
  // prefetch when it keeps as many CTAs on an SM, the persistent grid.
  p->trace_cands.assign(p->trace.size(), {});
  p->pinned.assign(p->trace.size(), -1);
  const char* pf_env = getenv("PSG_PREFETCH");
  for (size_t part = 0; part < p->trace.size(); part++) {
    if (!p->trace[part] || p->wide) {
      p->trace[part] = nullptr;
      continue;
    }
    const int rc = p->trace_recipe[part];
    const StepHost& ag = p->host.steps[p->host.parts[part].first + 2];
    const TracePlanInfo* const* builds = trace_plans_for(p->trace[part]->m, (int)(2 * ag.half + 1));
    std::vector<TraceCand>& cs = p->trace_cands[part];
    for (int bi = 0; builds[bi]; bi++) {
      const TracePlanInfo* tb = builds[bi];
      if (!tb->kernel[rc][0] || !runs_reference_stages(*tb)) continue;
      const void* tw = upload(p->keep, ref_twiddles(*tb));
      const int64_t fw = 2 * (int64_t)tb->buf * 8;
      int per[2] = {0, 0};
      for (int pf = 0; pf < 2; pf++) {
        const void* k = tb->kernel[rc][pf];
        allow_smem(k);
        CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[pf], k, tb->nt, (size_t)(p->x_bytes + fw)));
      }
      bool pf_first = per[1] > 0 && per[1] >= per[0];
      if (pf_env) pf_first = atoi(pf_env) != 0 && per[1] > 0;
      for (int o = 0; o < 2; o++) {
        const int pf = o == 0 ? (int)pf_first : (int)!pf_first;
        if (per[pf] <= 0 || (pf_env && pf != (int)pf_first)) continue;
        for (int per_row = 0; per_row < 2; per_row++) {
          if (pf && per_row) continue;  // one row per CTA: nothing to prefetch
          TraceCand c;
          c.tp = tb;
          c.pf = pf != 0;
          c.per_row = per_row != 0;
          c.per_sm = per[pf];
          c.work_off = p->x_bytes;
          c.smem = (size_t)(c.work_off + fw);
          c.tw = tw;
          cs.push_back(c);
        }
      }
      // The row in the first transform buffer: only the forward transform's
      // first pass reads it, and that pass writes the other buffer. With no
      // row buffer of its own, more CTAs fit where shared memory sets the
      // count (the row's copy then waits for the row before it: no copy in
      // flight); offered only when it adds CTAs per SM.
      if ((!pf_env || atoi(pf_env) == 0) && (int64_t)p->x_bytes <= (int64_t)tb->buf * 8) {
        int px = 0;
        CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&px, tb->kernel[rc][0], tb->nt, (size_t)fw));
        if (px > std::max(per[0], per[1])) {
          for (int per_row = 0; per_row < 2; per_row++) {
            TraceCand c;
            c.tp = tb;
            c.pf = false;
            c.per_row = per_row != 0;
            c.per_sm = px;
            c.work_off = 0;
            c.smem = (size_t)fw;
            c.tw = tw;
            c.row_in_buffer = true;
            cs.push_back(c);
          }
        }
      }
    }
    if (cs.empty()) p->trace[part] = nullptr;
    else p->trace[part] = cs[0].tp;
  }
  if (const char* e = getenv("PSG_TUNE")) p->tune = atoi(e) != 0;
}

// The per-panel factor of part `part` (which starts with a per-panel
// normalization) over the whole block, left in the part's workspace slot;
// returns its device address.
template <class T>
static const double* panel_factor_dev(const psg_plan* p, psg_workspace* ws, int part, const T* blk, int64_t rows,
                                      int32_t cols, const int* live, cudaStream_t stream) {
  const StepHost& ns = p->host.steps[p->host.parts[part].first];
  char* base = (char*)ws->d;
  PanelOut* out = reinterpret_cast<PanelOut*>(base + 64 * part);
  double* ss = reinterpret_cast<double*>(base + 512);
  double* mx = ss + rows;
  unsigned* hist = reinterpret_cast<unsigned*>(base + 512 + align256(rows * 16));
  int g = (int)std::max<int64_t>(1, std::min<int64_t>(rows, (int64_t)g_sm_count * 8));
  if (rows > 0) row_stats_kernel<T><<<g, 256, 0, stream>>>(blk, rows, cols, live, ss, mx);
  panel_fold_kernel<<<1, 1024, 0, stream>>>(rows, cols, live, ss, mx, out);
  double clipP = ns.stat == PSG_NORM_PERCENTILE ? ns.percentile : NAN;
  if (!std::isnan(clipP)) {
    CUDA_OK(cudaMemsetAsync(hist, 0, kHist, stream));
    launch_hist<T>(blk, rows, cols, live, ss, mx, hist, stream);
  }
  panel_clip_kernel<unsigned><<<1, 1024, 0, stream>>>(hist, out, clipP, ns.stat, ns.norm_target, p->host.dtype);
  return &out->factor;
}

static bool part_needs_panel(const psg_plan* p, int part) {
  auto range = p->host.parts[part];
  return range.first < range.second && p->host.steps[range.first].kind == ST_NORM_PANEL;
}

// Launches launch shape c of part `part`'s trace kernel.
static void launch_trace(const psg_plan* p, int part, const TraceCand& c, PipeArgs a, int64_t rows,
                         cudaStream_t stream) {
  const void* k = c.tp->kernel[p->trace_recipe[part]][c.pf ? 1 : 0];
  a.work_off = c.work_off;
  a.tw_pass = c.tw;
  allow_smem(k);
  const int64_t grid = c.per_row ? rows : std::min<int64_t>(rows, (int64_t)c.per_sm * g_sm_count);
  launch_pipe(k, (int)std::min<int64_t>(grid, 1 << 30), c.tp->nt, c.smem, stream, a);
}

// The launch shape of part `part`'s trace kernel for a call of `rows` rows:
// its pinned choice, else the tuner's for the row count's class (its bit
// length), else, tuning now: every shape runs on the call's own input into
// a scratch block on `stream`, each timed launch with events after a write
// of twice the L2's size has flushed the input from it (the panel comes
// from HBM, as a fresh one does); one warm-up launch per shape, then the
// least mean time of six launches (three rounds over the shapes) wins, and
// the choice is kept for the class. The shapes give the same bits, so the choice
// never changes a result. No tuning under stream capture, with tuning off
// (PSG_TUNE=0), or when the scratch block cannot be had: the first shape.
static int trace_choice(const psg_plan* p, int part, const PipeArgs& a, int64_t rows, int32_t cols, size_t esz,
                        cudaStream_t stream) {
  const std::vector<TraceCand>& cs = p->trace_cands[part];
  std::lock_guard<std::mutex> lk(p->tune_mu);
  if (p->pinned[part] >= 0 && p->pinned[part] < (int)cs.size()) return p->pinned[part];
  if (cs.size() < 2 || !p->tune || rows <= 0) return 0;
  int cls = 0;
  for (int64_t r = rows; r; r >>= 1) cls++;
  auto it = p->tuned.find({part, cls});
  if (it != p->tuned.end()) return it->second.choice;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CUDA_OK(cudaStreamIsCapturing(stream, &cap));
  if (cap != cudaStreamCaptureStatusNone) return 0;
  // at most 1 GiB of scratch: the first rows of a larger call
  const int64_t row_bytes = (int64_t)cols * (int64_t)esz;
  const int64_t trows = std::max<int64_t>(1, std::min<int64_t>(rows, (int64_t(1) << 30) / std::max<int64_t>(row_bytes, 1)));
  int dev = 0, l2 = 0;
  CUDA_OK(cudaGetDevice(&dev));
  CUDA_OK(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
  const size_t flush_bytes = 2 * (size_t)std::max(l2, 1 << 20);
  void* scratch = nullptr;
  void* flush = nullptr;
  if (cudaMalloc(&scratch, (size_t)(trows * row_bytes)) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  if (cudaMalloc(&flush, flush_bytes) != cudaSuccess) {
    cudaGetLastError();
    flush = nullptr;
  }
  PipeArgs t = a;
  t.job.src = a.job.src ? a.job.src : a.job.dst;
  t.job.dst = scratch;
  t.job.rows = trows;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  TraceTuning res;
  res.rows = trows;
  res.us.assign(cs.size(), INFINITY);
  auto done = [&] {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(scratch);
    if (flush) cudaFree(flush);
  };
  try {
    CUDA_OK(cudaEventCreate(&e0));
    CUDA_OK(cudaEventCreate(&e1));
    std::vector<float> sum(cs.size(), 0.f);
    constexpr int kRounds = 3, kPer = 2;
    for (int round = 0; round < kRounds; round++)
      for (size_t i = 0; i < cs.size(); i++) {
        if (round == 0) launch_trace(p, part, cs[i], t, trows, stream);
        for (int k = 0; k < kPer; k++) {
          if (flush) CUDA_OK(cudaMemsetAsync(flush, kPer * round + k, flush_bytes, stream));
          CUDA_OK(cudaEventRecord(e0, stream));
          launch_trace(p, part, cs[i], t, trows, stream);
          CUDA_OK(cudaEventRecord(e1, stream));
          CUDA_OK(cudaEventSynchronize(e1));
          float ms = 0;
          CUDA_OK(cudaEventElapsedTime(&ms, e0, e1));
          sum[i] += ms * 1000.f;
        }
      }
    // the mean of the samples: the event clock ticks in steps of a few
    // microseconds at these durations, which a minimum would keep
    for (size_t i = 0; i < cs.size(); i++) res.us[i] = sum[i] / (kRounds * kPer);
  } catch (...) {
    done();
    throw;
  }
  done();
  res.choice = (int)(std::min_element(res.us.begin(), res.us.end()) - res.us.begin());
  p->tuned[{part, cls}] = res;
  return res.choice;
}

// runPart (pipeline.nim:690-723): the steps of part `part` after its
// per-panel normalization, if any, whose factor (a device double, NaN: the
// rows are left alone) scales the live rows first; `src` (first part only)
// is copied in.
template <class T>
static void run_part(const psg_plan* p, psg_workspace* ws, int part, const void* src, void* dst, int64_t rows,
                     int32_t cols, const int* live, const double* start, const double* factor, cudaStream_t stream,
                     const psg_keys* keys = nullptr, double dt_ms = 0) {
  auto range = p->host.parts[part];
  bool panel = part_needs_panel(p, part);
  PipeArgs a{};
  a.job.offset = keys ? keys->offset : nullptr;
  a.job.t0_ms = keys ? keys->t0_ms : nullptr;
  a.job.first_sample = keys ? keys->first_sample : 0;
  a.job.dt_ms = dt_ms > 0 ? dt_ms : p->host.dt_ms;
  a.job.src = src;
  a.job.dst = dst;
  a.job.rows = rows;
  a.job.cols = cols;
  a.job.first = panel ? range.first + 1 : range.first;
  a.job.last = range.second;
  a.job.live = live;
  a.job.start_ms = start;
  a.job.steps = p->d_steps;
  a.work_off = p->work_off;
  a.factor = factor;
  a.x_bytes = p->x_bytes;
  a.status = reinterpret_cast<int*>((char*)ws->d + 504);
  bool nothing = a.job.first >= a.job.last && !factor && (src == nullptr || src == dst);
  if (nothing || rows == 0) return;
  int grid = (int)std::min<int64_t>(rows, p->grid);
  if (p->wide) {
    if (ws->g_bytes < p->gwork_bytes) throw WorkspaceError("reserve the workspace for the plan first");
    a.gwork = (unsigned char*)ws->g;
    a.gwork_stride = p->gwork_stride;
  }
  if (part < (int)p->trace.size() && p->trace[part] && !factor) {
    const int k = trace_choice(p, part, a, rows, cols, sizeof(T), stream);
    launch_trace(p, part, p->trace_cands[part][k], a, rows, stream);
    return;
  }
  const void* kern = p->wide ? wide_kernel_for<T>() : pipe_kernel_for<T>(p->recipe[part], p->prefetch);
  allow_smem(kern);
  launch_pipe(kern, grid, p->threads, p->smem, stream, a);
}

template <class T>
static void launch_part(const psg_plan* p, psg_workspace* ws, int part, const void* src, void* dst, int64_t rows,
                        int32_t cols, const int* live, const double* start, cudaStream_t stream,
                        const psg_keys* keys = nullptr, double dt_ms = 0) {
  const double* factor = nullptr;
  if (part_needs_panel(p, part))
    factor = panel_factor_dev<T>(p, ws, part, reinterpret_cast<const T*>(src ? src : dst), rows, cols, live, stream);
  run_part<T>(p, ws, part, src, dst, rows, cols, live, start, factor, stream, keys, dt_ms);
}

template <class T> static void corr_upload(psg_corr_plan* p) {
  typedef typename C2<T>::type V;
  p->bridge = upload(p->keep, bridge_table<T>(p->host.fft, p->host.mul_re, p->host.mul_im));
  p->tw = upload(p->keep, as_c<T>(p->host.fft.tw_re, p->host.fft.tw_im));
  p->fft = fft_desc(p->host.fft);
  size_t need = (size_t)(2 * p->host.fft.m * sizeof(V));
  int limit = g_max_smem - (int)sizeof(SharedMem) - 1024;
  // PSG_TRACE=0 in the environment (read at plan creation) keeps corr_kernel
  const char* te = getenv("PSG_TRACE");
  if (sizeof(T) == 4 && !(te && atoi(te) == 0) && (int64_t)need <= limit) {
    if (const TracePlanInfo* tp = corr_plans_for((int)p->host.fft.m)[0]) {
      allow_smem(tp->kernel[0][0]);
      int per = 0;
      CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, tp->kernel[0][0], tp->nt, need));
      if (per > 0) {
        p->trace = tp;
        p->tw_pass = upload(p->keep, trace_twiddles(*tp));
        p->trace_grid = per * g_sm_count;
      }
    }
  }
  allow_smem((const void*)corr_kernel<T>);
  if ((int64_t)need <= limit) {
    p->smem = need;
    int per_sm = 0;
    CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, corr_kernel<T>, kCorrThreads, p->smem));
    p->grid = std::max(1, per_sm) * g_sm_count;
  } else {
    // Too long for shared memory: each CTA works in its own slice of global
    // memory (mostly L2-resident at these lengths).
    p->smem = 0;
    p->grid = g_sm_count * 2;
    auto b = std::make_unique<DeviceBuf>();
    CUDA_OK(cudaMalloc(&b->p, need * p->grid));
    p->gwork = b->p;
    p->keep.push_back(std::move(b));
  }
}

extern "C" {

const char* psg_last_error(void) { return t_err.c_str(); }
const char* psg_version(void) { return "processseg_b200 0.1 (sm_100a)"; }

int psg_init(int device) {
  return guarded([&] {
    CUDA_OK(cudaSetDevice(device));
    ensure_device();
  });
}

int psg_is_fast_len(int64_t n) { return fast_len(n) ? 1 : 0; }
int64_t psg_next_fast_len(int64_t n, int even) { return next_fast(n, even != 0); }

int psg_impulse_length(const psg_filter_spec* spec, double dt_ms, int32_t* out) {
  return guarded([&] {
    if (!spec || !out) throw InvalidArg("null argument");
    *out = (int32_t)spec_impulse_length(*spec, dt_ms);
  });
}
int psg_response(const psg_filter_spec* spec, double f_hz, double dt_ms, double* out) {
  return guarded([&] {
    if (!spec || !out) throw InvalidArg("null argument");
    *out = spec_response(*spec, f_hz, dt_ms);
  });
}
int psg_iir_design(const psg_filter_spec* spec, double dt_ms, int32_t samples, int32_t phase, int32_t trend,
                   int32_t* order, int32_t* margin, double* dc_gain) {
  return guarded([&] {
    if (!spec) throw InvalidArg("null argument");
    IirHost p = iir_plan(*spec, dt_ms, samples, phase, trend);
    if (order) *order = iir_order(p);
    if (margin) *margin = (int32_t)p.pad;
    if (dc_gain) *dc_gain = p.dc_gain;
  });
}
int psg_iir_magnitude(const psg_filter_spec* spec, double dt_ms, int32_t phase, const double* f_hz, int32_t n,
                      double* out) {
  return guarded([&] {
    if (!spec || (n > 0 && (!f_hz || !out)) || n < 0) throw InvalidArg("null argument");
    IirHost p = iir_plan(*spec, dt_ms, 1, phase, PSG_TR_NONE);
    for (int32_t i = 0; i < n; i++) out[i] = iir_magnitude(p, f_hz[i], dt_ms);
  });
}
int psg_required_margin(const psg_op* ops, int32_t n_ops, double dt_ms, int32_t* out) {
  return guarded([&] {
    if (!out || (n_ops > 0 && !ops)) throw InvalidArg("null argument");
    *out = (int32_t)required_margin(ops, n_ops, dt_ms);
  });
}
void psg_decode_window(int64_t a, int64_t b, int64_t margin, int64_t trace_len, int64_t* out) {
  int64_t m = std::min(std::max<int64_t>(margin, 0), std::max<int64_t>(trace_len, 0));
  out[0] = std::max<int64_t>(0, a - m);
  out[1] = std::min(trace_len - 1, b + m);
}

}  // extern "C"

// compile (pipeline.nim:466-523): the host plan, its recipes, its device tables.
static std::unique_ptr<psg_plan> make_plan(const psg_op* ops, int32_t n_ops, int32_t dtype, double dt_ms,
                                           int32_t samples, int32_t record_samples) {
  std::unique_ptr<psg_plan> p(new psg_plan());
  p->max_radix = dtype == PSG_F32 ? 12 : 8;
  p->host = compile_plan(ops, n_ops, dtype, dt_ms, samples, record_samples, p->max_radix);
  for (auto& r : p->host.parts) {
    const bool panel = r.first < r.second && p->host.steps[r.first].kind == ST_NORM_PANEL;
    p->recipe.push_back(recipe_of(p->host, panel ? r.first + 1 : r.first, r.second));
  }
  ensure_device();
  CUDA_OK(cudaGetDevice(&p->device));
  for (size_t part = 0; part < p->host.parts.size(); part++) {
    p->trace.push_back(trace_plan_of(p.get(), (int)part));
    p->trace_recipe.push_back(p->recipe[part] == RC_DFAN ? 1 : 0);
  }
  if (dtype == PSG_F32) build_device_steps<float>(p.get());
  else build_device_steps<double>(p.get());
  if (p->wide) std::fill(p->recipe.begin(), p->recipe.end(), (int)RC_GENERIC);
  return p;
}

extern "C" {

int psg_plan_compile(const psg_op* ops, int32_t n_ops, int32_t dtype, double dt_ms, int32_t samples,
                     int32_t record_samples, psg_plan** out) {
  return guarded([&] {
    if (!out) throw InvalidArg("null argument");
    *out = nullptr;
    *out = make_plan(ops, n_ops, dtype, dt_ms, samples, record_samples).release();
  });
}
void psg_plan_destroy(psg_plan* plan) { delete plan; }
int32_t psg_plan_margin(const psg_plan* p) { return p ? (int32_t)p->host.margin : 0; }
uint64_t psg_plan_generation(const psg_plan* p) { return p ? p->host.generation : 0; }
int32_t psg_plan_samples(const psg_plan* p) { return p ? (int32_t)p->host.samples : 0; }
int32_t psg_plan_record_samples(const psg_plan* p) { return p ? (int32_t)p->host.record_samples : 0; }
int32_t psg_plan_part_count(const psg_plan* p) { return p ? (int32_t)p->host.parts.size() : 0; }
int32_t psg_plan_len(const psg_plan* p) { return p ? (int32_t)p->host.steps.size() : 0; }
int32_t psg_plan_step_nfft(const psg_plan* p, int32_t i) {
  if (!p || i < 0 || i >= (int)p->host.steps.size()) return 0;
  return p->host.steps[i].kind == ST_FILTER ? (int32_t)p->host.steps[i].filter.nfft : 0;
}

int32_t psg_plan_needs_keys(const psg_plan* plan) { return plan && plan->needs_keys ? 1 : 0; }
int32_t psg_plan_trace_shapes(const psg_plan* plan, int32_t part) {
  if (!plan || part < 0 || part >= (int)plan->trace_cands.size() || !plan->trace[part]) return 0;
  return (int32_t)plan->trace_cands[part].size();
}
int psg_plan_pin_trace(psg_plan* plan, int32_t part, int32_t shape) {
  return guarded([&] {
    const int n = psg_plan_trace_shapes(plan, part);
    if (n == 0) throw InvalidArg("the part has no trace-kernel launch shapes");
    if (shape < -1 || shape >= n) throw InvalidArg("launch shape out of range");
    std::lock_guard<std::mutex> lk(plan->tune_mu);
    plan->pinned[part] = shape;
  });
}
int psg_plan_tuning(const psg_plan* plan, char* buf, int64_t cap, int64_t* needed) {
  return guarded([&] {
    if (!plan || (!buf && cap > 0)) throw InvalidArg("null argument");
    std::string j = "{\"parts\": [";
    char tmp[256];
    std::lock_guard<std::mutex> lk(plan->tune_mu);
    bool first = true;
    for (size_t part = 0; part < plan->trace_cands.size(); part++) {
      if (!plan->trace[part]) continue;
      snprintf(tmp, sizeof tmp, "%s{\"part\": %d, \"pinned\": %d, \"shapes\": [", first ? "" : ", ", (int)part,
               plan->pinned[part]);
      j += tmp;
      first = false;
      const auto& cs = plan->trace_cands[part];
      for (size_t i = 0; i < cs.size(); i++) {
        const TracePlanInfo& t = *cs[i].tp;
        std::string passes;
        for (int k = 0; k < t.np; k++) {
          passes += (k ? " " : "") + std::to_string(t.g1[k]);
          if (t.g2[k]) passes += "x" + std::to_string(t.g2[k]);
        }
        snprintf(tmp, sizeof tmp,
                 "%s{\"m\": %d, \"threads\": %d, \"min_blocks\": %d, \"passes\": \"%s\", \"prefetch\": %s, "
                 "\"grid\": \"%s\", \"row\": \"%s\", \"ctas_per_sm\": %d, \"smem\": %lld}",
                 i ? ", " : "", t.m, t.nt, t.min_blocks, passes.c_str(), cs[i].pf ? "true" : "false",
                 cs[i].per_row ? "per_row" : "persistent", cs[i].row_in_buffer ? "transform buffer" : "own buffer",
                 cs[i].per_sm, (long long)cs[i].smem);
        j += tmp;
      }
      j += "]}";
    }
    j += "], \"tuned\": [";
    first = true;
    for (const auto& kv : plan->tuned) {
      snprintf(tmp, sizeof tmp, "%s{\"part\": %d, \"class\": %d, \"rows\": %lld, \"choice\": %d, \"us\": [",
               first ? "" : ", ", kv.first.first, kv.first.second, (long long)kv.second.rows, kv.second.choice);
      j += tmp;
      first = false;
      for (size_t i = 0; i < kv.second.us.size(); i++) {
        snprintf(tmp, sizeof tmp, "%s%.3f", i ? ", " : "", kv.second.us[i]);
        j += tmp;
      }
      j += "]}";
    }
    j += "]}";
    if (needed) *needed = (int64_t)j.size() + 1;
    if (cap > 0) {
      const size_t n = std::min<size_t>(j.size(), (size_t)cap - 1);
      memcpy(buf, j.data(), n);
      buf[n] = 0;
    }
  });
}
int32_t psg_plan_part_needs_panel(const psg_plan* plan, int32_t part) {
  if (!plan || part < 0 || part >= (int)plan->host.parts.size()) return 0;
  return part_needs_panel(plan, part) ? 1 : 0;
}
int32_t psg_plan_step_margin(const psg_plan* p, int32_t i) {
  if (!p || i < 0 || i >= (int)p->host.steps.size()) return 0;
  return (int32_t)p->host.steps[i].margin();
}
int64_t psg_plan_workspace_bytes(const psg_plan* p, int64_t rows, int32_t cols) {
  return p ? ws_host_bytes(p->needs_panel, rows, cols, p->host.dtype) + p->gwork_bytes : 0;
}

int psg_workspace_create(psg_workspace** out) {
  return guarded([&] {
    if (!out) throw InvalidArg("null argument");
    *out = new psg_workspace();
  });
}
void psg_workspace_destroy(psg_workspace* ws) {
  if (!ws) return;
  if (ws->lanes_ready) {
    // work still queued (an asynchronous apply) finishes before its buffers go
    for (int i = 0; i < psg_workspace::kLanes; i++) cudaStreamSynchronize(ws->lane[i]);
    for (int i = 0; i < psg_workspace::kLanes; i++) {
      cudaStreamDestroy(ws->lane[i]);
      cudaEventDestroy(ws->done_ev[i]);
      cudaEventDestroy(ws->slot_ev[0][i]);
      cudaEventDestroy(ws->slot_ev[1][i]);
    }
    cudaEventDestroy(ws->start_ev);
  }
  if (ws->d) cudaFree(ws->d);
  if (ws->g) cudaFree(ws->g);
  if (ws->sp) cudaFree(ws->sp);
  for (void* h : ws->hmeta)
    if (h) cudaFreeHost(h);
  delete ws;
}
static void ws_grow(psg_workspace* ws, int64_t need) {
  int dev;
  CUDA_OK(cudaGetDevice(&dev));
  if (ws->d && ws->device != dev) throw InvalidArg("the workspace belongs to another device");
  if (ws->bytes >= need) return;
  if (ws->d) {
    CUDA_OK(cudaDeviceSynchronize());
    CUDA_OK(cudaFree(ws->d));
    ws->d = nullptr;
    ws->bytes = 0;
  }
  CUDA_OK(cudaMalloc(&ws->d, (size_t)need));
  CUDA_OK(cudaMemset(ws->d, 0, 512));  // panel slots and the kernels' status word
  ws->bytes = need;
  ws->device = dev;
}
// The arena and, for a plan with long traces, its global work areas.
static void ws_grow_for(psg_workspace* ws, const psg_plan* p, int64_t rows, int32_t cols) {
  ws_grow(ws, ws_host_bytes(p->needs_panel, rows, cols, p->host.dtype));
  if (ws->g_bytes >= p->gwork_bytes) return;
  if (ws->g) {
    CUDA_OK(cudaDeviceSynchronize());
    CUDA_OK(cudaFree(ws->g));
    ws->g = nullptr;
    ws->g_bytes = 0;
  }
  CUDA_OK(cudaMalloc(&ws->g, (size_t)p->gwork_bytes));
  ws->g_bytes = p->gwork_bytes;
}
int psg_workspace_reserve(psg_workspace* ws, const psg_plan* plan, int64_t rows, int32_t cols) {
  return guarded([&] {
    if (!ws) throw InvalidArg("null argument");
    if (rows < 0 || cols < 0) throw InvalidArg("rows and cols must be ≥ 0");
    if (!plan) {
      // no plan: the statistics' scratch for `rows` rows (panelStatsWorkspace)
      ensure_device();
      ws_grow(ws, ws_device_bytes(rows));
      return;
    }
    ws_grow_for(ws, plan, rows, cols);
  });
}
int64_t psg_workspace_bytes(const psg_workspace* ws) { return ws ? ws->bytes + ws->g_bytes : 0; }

int psg_rows_flatten(const int32_t* status, const int32_t* num_samples, const double* t0_ms, int64_t rows,
                     int32_t first_sample, double dt_ms, const int64_t* failed, int64_t n_failed, int32_t cols,
                     int32_t mode, int32_t* live_out, double* start_ms_out) {
  return guarded([&] {
    if (rows < 0 || (rows > 0 && (!status || !num_samples || !live_out))) throw InvalidArg("null argument");
    if (!(std::isfinite(dt_ms) && dt_ms > 0)) throw InvalidArg("dtMs must be finite and positive");
    if (first_sample < 0) throw InvalidArg("firstSample must be ≥ 0");
    // ChunkMeta's failed list is ascending and unique (core/types.nim:106-113).
    for (int64_t i = 0; i < n_failed; i++) {
      if (failed[i] < 0 || failed[i] >= rows) throw InvalidArg("failed row " + std::to_string(failed[i]) + " is outside 0 ..< " + std::to_string(rows));
      if (i > 0 && failed[i] <= failed[i - 1]) throw InvalidArg("failed rows must be ascending and unique");
    }
    int64_t fi = 0;
    for (int64_t r = 0; r < rows; r++) {
      bool is_failed = false;
      while (fi < n_failed && failed[fi] < r) fi++;
      if (fi < n_failed && failed[fi] == r) is_failed = true;
      int32_t st = status[r];
      bool use = mode == 0 || mode == 3 ? ((st == PSG_TS_LIVE || st == PSG_TS_UNKNOWN) && !is_failed)
                 : mode == 1 ? (st != PSG_TS_DEAD && !is_failed)
                             : !is_failed;
      int64_t n = std::min<int64_t>(std::max<int64_t>((int64_t)num_samples[r] - first_sample, 0), cols);
      live_out[r] = use ? (int32_t)n : (mode == 3 ? -1 : 0);
      if (start_ms_out) start_ms_out[r] = (t0_ms ? t0_ms[r] : NAN) + (double)first_sample * dt_ms;
    }
  });
}

static void check_apply(const psg_plan* plan, psg_workspace* ws, const void* src, void* dst, int64_t rows, int32_t cols,
                        const int32_t* live, double dt_ms, bool need_ws, const psg_keys* keys = nullptr) {
  if (!plan) throw InvalidArg("a PipelinePlan must come from compile");
  if (plan->needs_keys && !keys)
    throw InvalidArg("the plan mutes: each row's offset and t0Ms are needed (apply it with its keys, psg_apply_keyed)");
  if (keys && keys->first_sample < 0) throw InvalidArg("firstSample must be ≥ 0");
  if (rows < 0 || cols < 0) throw InvalidArg("rows and cols must be ≥ 0");
  if (rows > 0 && (!dst || !live)) throw InvalidArg("dst and live are required");
  int64_t esz = plan->host.dtype == PSG_F32 ? 4 : 8;
  if (src && src != dst) {
    uintptr_t s0 = (uintptr_t)src, d0 = (uintptr_t)dst, bytes = (uintptr_t)(rows * cols * esz);
    if (s0 < d0 + bytes && d0 < s0 + bytes) throw InvalidArg("src and dst overlap without being the same block");
  }
  if (!same_interval(dt_ms, plan->host.dt_ms))
    throw InvalidArg("the plan is for dtMs = " + std::to_string(plan->host.dt_ms) + ", the rows have " + std::to_string(dt_ms));
  if (cols > plan->host.samples)
    throw InvalidArg("the block has " + std::to_string(cols) + " columns, the plan takes " + std::to_string(plan->host.samples) + " samples");
  if (need_ws) {
    if (!ws) throw WorkspaceError("reserve the workspace for the plan first");
    int64_t need = plan->needs_panel ? ws_device_bytes(rows) : 512;
    if (ws->bytes < need || ws->g_bytes < plan->gwork_bytes) throw WorkspaceError("reserve the workspace for the plan first");
  }
}

int psg_check_apply(const psg_plan* plan, const void* src, const void* dst, int64_t rows, int32_t cols, double dt_ms) {
  return guarded([&] {
    // the checks apply makes before any sample changes; the rows' liveness
    // and keys are the caller's, so stand-ins pass their presence checks
    const int32_t live = 0;
    const psg_keys keys{};
    check_apply(plan, nullptr, src, const_cast<void*>(dst), rows, cols, &live, dt_ms, false,
                plan && plan->needs_keys ? &keys : nullptr);
  });
}

int psg_apply(const psg_plan* plan, psg_workspace* ws, const void* src, void* dst, int64_t rows, int32_t cols,
              const int32_t* live, const double* start_ms, double dt_ms, void* stream) {
  return psg_apply_keyed(plan, ws, src, dst, rows, cols, live, start_ms, nullptr, dt_ms, stream);
}

int psg_apply_keyed(const psg_plan* plan, psg_workspace* ws, const void* src, void* dst, int64_t rows, int32_t cols,
                    const int32_t* live, const double* start_ms, const psg_keys* keys, double dt_ms, void* stream) {
  return guarded([&] {
    check_apply(plan, ws, src, dst, rows, cols, live, dt_ms, true, keys);
    ensure_device();
    cudaStream_t s = (cudaStream_t)stream;
    for (int part = 0; part < (int)plan->host.parts.size(); part++) {
      const void* from = part == 0 ? src : nullptr;
      if (plan->host.dtype == PSG_F32) launch_part<float>(plan, ws, part, from, dst, rows, cols, live, start_ms, s, keys, dt_ms);
      else launch_part<double>(plan, ws, part, from, dst, rows, cols, live, start_ms, s, keys, dt_ms);
    }
    CUDA_OK(cudaGetLastError());
  });
}

// ------------------------------------------------------------ graph replay
// One psg_apply_keyed captured into a CUDA graph on a stream of its own, for
// replay: a launch then costs the host one call (no checks, no per-part
// launches). The graph holds the call's pointers: the plan's tables, the
// workspace's slots, the blocks and the row arrays.
}  // extern "C"
struct psg_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = 0;
};
extern "C" {

int psg_graph_capture(const psg_plan* plan, psg_workspace* ws, const void* src, void* dst, int64_t rows, int32_t cols,
                      const int32_t* live, const double* start_ms, const psg_keys* keys, double dt_ms,
                      psg_graph** out) {
  cudaStream_t s = nullptr;
  std::unique_ptr<psg_graph> g(new psg_graph());
  int st = guarded([&] {
    if (!out) throw InvalidArg("null argument");
    *out = nullptr;
    check_apply(plan, ws, src, dst, rows, cols, live, dt_ms, true, keys);
    ensure_device();
    CUDA_OK(cudaGetDevice(&g->device));
    // the kernels' shared-memory attributes are set before the capture
    for (int part = 0; part < (int)plan->host.parts.size(); part++) {
      if (part < (int)plan->trace.size() && plan->trace[part])
        for (const TraceCand& c : plan->trace_cands[part])
          allow_smem(c.tp->kernel[plan->trace_recipe[part]][c.pf ? 1 : 0]);
      allow_smem(plan->wide ? (plan->host.dtype == PSG_F32 ? wide_kernel_for<float>() : wide_kernel_for<double>())
                            : (plan->host.dtype == PSG_F32 ? pipe_kernel_for<float>(plan->recipe[part], plan->prefetch)
                                                           : pipe_kernel_for<double>(plan->recipe[part], plan->prefetch)));
    }
    CUDA_OK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    CUDA_OK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      for (int part = 0; part < (int)plan->host.parts.size(); part++) {
        const void* from = part == 0 ? src : nullptr;
        if (plan->host.dtype == PSG_F32)
          launch_part<float>(plan, ws, part, from, dst, rows, cols, live, start_ms, s, keys, dt_ms);
        else
          launch_part<double>(plan, ws, part, from, dst, rows, cols, live, start_ms, s, keys, dt_ms);
      }
    } catch (...) {
      cudaGraph_t dead = nullptr;
      cudaStreamEndCapture(s, &dead);
      if (dead) cudaGraphDestroy(dead);
      throw;
    }
    CUDA_OK(cudaStreamEndCapture(s, &g->graph));
    CUDA_OK(cudaGraphInstantiate(&g->exec, g->graph, 0));
  });
  if (s) cudaStreamDestroy(s);
  if (st == PSG_OK) *out = g.release();
  else if (g->graph) cudaGraphDestroy(g->graph);
  return st;
}

int psg_graph_launch(psg_graph* g, void* stream) {
  return guarded([&] {
    if (!g || !g->exec) throw InvalidArg("null argument");
    CUDA_OK(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
  });
}

void psg_graph_destroy(psg_graph* g) {
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
}

int psg_apply_host(const psg_plan* plan, psg_workspace* ws, const void* src_host, void* dst_host, int64_t rows,
                   int32_t cols, const int32_t* live_host, const double* start_ms_host, double dt_ms, void* stream) {
  return psg_apply_host_keyed(plan, ws, src_host, dst_host, rows, cols, live_host, start_ms_host, nullptr, dt_ms, stream);
}

static void ensure_lanes(psg_workspace* ws) {
  if (ws->lanes_ready) return;
  for (int i = 0; i < psg_workspace::kLanes; i++) {
    CUDA_OK(cudaStreamCreateWithFlags(&ws->lane[i], cudaStreamNonBlocking));
    CUDA_OK(cudaEventCreateWithFlags(&ws->done_ev[i], cudaEventDisableTiming));
    CUDA_OK(cudaEventCreateWithFlags(&ws->slot_ev[0][i], cudaEventDisableTiming));
    CUDA_OK(cudaEventCreateWithFlags(&ws->slot_ev[1][i], cudaEventDisableTiming));
  }
  CUDA_OK(cudaEventCreateWithFlags(&ws->start_ev, cudaEventDisableTiming));
  ws->lanes_ready = true;
}

// The host-memory apply. A plan without per-panel normalizations runs chunk
// by chunk of rows on the workspace's lane streams, so that the copy in of
// one chunk, the kernel of the one before and the copy out of the one
// before that overlap (the device's two copy engines and its SMs). A plan
// with one needs the whole block on the device before its factor: copy in,
// apply, copy out. `async`: the lanes are not joined back into `stream` and
// the call returns once everything is queued (psg_workspace_sync waits);
// consecutive calls then overlap, each staging its row metadata in the slot
// the call before the last one used, once that call's lanes are done with it.
static void apply_host(const psg_plan* plan, psg_workspace* ws, const void* src_host, void* dst_host, int64_t rows,
                       int32_t cols, const int32_t* live_host, const double* start_ms_host, const psg_keys* keys_host,
                       double dt_ms, cudaStream_t s, bool async) {
  check_apply(plan, ws, src_host, dst_host, rows, cols, live_host, dt_ms, false, keys_host);
  if (!ws) throw WorkspaceError("reserve the workspace for the plan first");
  if (ws->bytes < ws_host_bytes(plan->needs_panel, rows, cols, plan->host.dtype) || ws->g_bytes < plan->gwork_bytes)
    throw WorkspaceError("reserve the workspace for the plan first");
  if (rows == 0) return;
  ensure_device();
  ensure_lanes(ws);
  const int slot = async ? (int)(ws->calls++ & 1) : 0;
  int64_t esz = plan->host.dtype == PSG_F32 ? 4 : 8;
  char* base = (char*)ws->d + ws_device_bytes(rows) + slot * ws_meta_bytes(rows);
  int32_t* d_live = (int32_t*)base;
  double* d_start = (double*)(base + align256(rows * 4));
  double* d_offset = (double*)(base + align256(rows * 4) + align256(rows * 8));
  double* d_t0 = (double*)(base + align256(rows * 4) + 2 * align256(rows * 8));
  char* d_data = (char*)ws->d + ws_device_bytes(rows) + 2 * ws_meta_bytes(rows);
  const char* from = (const char*)(src_host ? src_host : dst_host);
  const double* dstart = start_ms_host ? d_start : nullptr;
  const bool koff = keys_host && keys_host->offset, kt0 = keys_host && keys_host->t0_ms;
  auto run_parts = [&](void* blk, int64_t r0, int64_t nr, cudaStream_t st) {
    psg_keys k{};
    if (keys_host) {
      k.offset = koff ? d_offset + r0 : nullptr;
      k.t0_ms = kt0 ? d_t0 + r0 : nullptr;
      k.first_sample = keys_host->first_sample;
    }
    const psg_keys* kp = keys_host ? &k : nullptr;
    for (int part = 0; part < (int)plan->host.parts.size(); part++) {
      if (plan->host.dtype == PSG_F32)
        launch_part<float>(plan, ws, part, nullptr, blk, nr, cols, d_live + r0, dstart ? dstart + r0 : nullptr, st, kp,
                           dt_ms);
      else
        launch_part<double>(plan, ws, part, nullptr, blk, nr, cols, d_live + r0, dstart ? dstart + r0 : nullptr, st, kp,
                            dt_ms);
    }
  };
  auto copy_meta = [&](cudaStream_t st) {
    if (!async) {
      CUDA_OK(cudaMemcpyAsync(d_live, live_host, rows * 4, cudaMemcpyHostToDevice, st));
      if (start_ms_host) CUDA_OK(cudaMemcpyAsync(d_start, start_ms_host, rows * 8, cudaMemcpyHostToDevice, st));
      if (koff) CUDA_OK(cudaMemcpyAsync(d_offset, keys_host->offset, rows * 8, cudaMemcpyHostToDevice, st));
      if (kt0) CUDA_OK(cudaMemcpyAsync(d_t0, keys_host->t0_ms, rows * 8, cudaMemcpyHostToDevice, st));
      return;
    }
    // through the slot's pinned staging, free once the slot's last user is
    const int64_t mb = ws_meta_bytes(rows);
    for (int i = 0; i < psg_workspace::kLanes; i++) CUDA_OK(cudaEventSynchronize(ws->slot_ev[slot][i]));
    if (ws->hmeta_bytes < mb) {
      for (int i = 0; i < psg_workspace::kLanes; i++) CUDA_OK(cudaStreamSynchronize(ws->lane[i]));
      for (void*& h : ws->hmeta) {
        if (h) CUDA_OK(cudaFreeHost(h));
        h = nullptr;
      }
      ws->hmeta_bytes = 0;
      for (void*& h : ws->hmeta) CUDA_OK(cudaHostAlloc(&h, (size_t)mb, cudaHostAllocDefault));
      ws->hmeta_bytes = mb;
    }
    char* hb = (char*)ws->hmeta[slot];
    std::memcpy(hb, live_host, (size_t)rows * 4);
    if (start_ms_host) std::memcpy(hb + align256(rows * 4), start_ms_host, (size_t)rows * 8);
    if (koff) std::memcpy(hb + align256(rows * 4) + align256(rows * 8), keys_host->offset, (size_t)rows * 8);
    if (kt0) std::memcpy(hb + align256(rows * 4) + 2 * align256(rows * 8), keys_host->t0_ms, (size_t)rows * 8);
    CUDA_OK(cudaMemcpyAsync(base, hb, (size_t)mb, cudaMemcpyHostToDevice, st));
  };
  const int64_t row_bytes = (int64_t)cols * esz;
  const int64_t chunk = host_chunk_rows(rows, cols, esz, async);
  const bool whole = host_whole_block(plan->needs_panel, rows, cols, esz, async);
  // A plan with long traces keeps its kernels on one lane: their global work
  // areas are one set per workspace.
  const int nl = plan->wide ? 1 : psg_workspace::kLanes;
  // The lanes start after what the caller queued on its stream.
  CUDA_OK(cudaEventRecord(ws->start_ev, s));
  for (int i = 0; i < psg_workspace::kLanes; i++) CUDA_OK(cudaStreamWaitEvent(ws->lane[i], ws->start_ev, 0));
  // A lane reuses its own staging after its own last call; when the staging
  // is laid out otherwise than in the last call (another width, whole
  // block or chunks, another lane count), every lane first waits for all
  // of that call's lanes.
  const int64_t layout = whole ? -1 : chunk * row_bytes;
  if (layout != ws->last_layout || nl != ws->last_lanes)
    for (int i = 0; i < psg_workspace::kLanes; i++)
      for (int j = 0; j < psg_workspace::kLanes; j++) CUDA_OK(cudaStreamWaitEvent(ws->lane[i], ws->done_ev[j], 0));
  ws->last_layout = layout;
  ws->last_lanes = nl;
  // the metadata slot's last user is done with it (for a waiting call, the
  // last call of either kind)
  for (int i = 0; i < psg_workspace::kLanes; i++)
    CUDA_OK(cudaStreamWaitEvent(ws->lane[0], async ? ws->slot_ev[slot][i] : ws->done_ev[i], 0));
  auto finish = [&]() {
    for (int i = 0; i < psg_workspace::kLanes; i++) {
      CUDA_OK(cudaEventRecord(ws->done_ev[i], ws->lane[i]));
      if (async) CUDA_OK(cudaEventRecord(ws->slot_ev[slot][i], ws->lane[i]));
      else CUDA_OK(cudaStreamWaitEvent(s, ws->done_ev[i], 0));
    }
    if (!async) CUDA_OK(cudaStreamSynchronize(s));
  };
  if (whole) {
    cudaStream_t st = ws->lane[0];
    copy_meta(st);
    CUDA_OK(cudaMemcpyAsync(d_data, from, (size_t)(rows * row_bytes), cudaMemcpyHostToDevice, st));
    run_parts(d_data, 0, rows, st);
    CUDA_OK(cudaMemcpyAsync(dst_host, d_data, (size_t)(rows * row_bytes), cudaMemcpyDeviceToHost, st));
    finish();
    return;
  }
  copy_meta(ws->lane[0]);
  CUDA_OK(cudaEventRecord(ws->done_ev[0], ws->lane[0]));
  for (int i = 1; i < psg_workspace::kLanes; i++) CUDA_OK(cudaStreamWaitEvent(ws->lane[i], ws->done_ev[0], 0));
  int k = 0;
  // Lane k % kLanes reuses its own staging buffer: on its stream the copy
  // in of a chunk queues after the copy out of that lane's previous one.
  for (int64_t r0 = 0; r0 < rows; r0 += chunk, k++) {
    int64_t nr = std::min(chunk, rows - r0);
    int lane = k % nl;
    cudaStream_t st = ws->lane[lane];
    char* buf = d_data + (size_t)lane * (size_t)(chunk * row_bytes);
    size_t off = (size_t)(r0 * row_bytes), nb = (size_t)(nr * row_bytes);
    CUDA_OK(cudaMemcpyAsync(buf, from + off, nb, cudaMemcpyHostToDevice, st));
    run_parts(buf, r0, nr, st);
    CUDA_OK(cudaMemcpyAsync((char*)dst_host + off, buf, nb, cudaMemcpyDeviceToHost, st));
  }
  finish();
}

int psg_apply_host_keyed(const psg_plan* plan, psg_workspace* ws, const void* src_host, void* dst_host, int64_t rows,
                         int32_t cols, const int32_t* live_host, const double* start_ms_host, const psg_keys* keys_host,
                         double dt_ms, void* stream) {
  return guarded([&] {
    apply_host(plan, ws, src_host, dst_host, rows, cols, live_host, start_ms_host, keys_host, dt_ms,
               (cudaStream_t)stream, false);
  });
}
int psg_apply_host_async(const psg_plan* plan, psg_workspace* ws, const void* src_host, void* dst_host, int64_t rows,
                         int32_t cols, const int32_t* live_host, const double* start_ms_host, const psg_keys* keys_host,
                         double dt_ms, void* stream) {
  return guarded([&] {
    apply_host(plan, ws, src_host, dst_host, rows, cols, live_host, start_ms_host, keys_host, dt_ms,
               (cudaStream_t)stream, true);
  });
}
int psg_workspace_sync(psg_workspace* ws) {
  return guarded([&] {
    if (!ws) throw InvalidArg("null argument");
    if (!ws->lanes_ready) return;
    for (int i = 0; i < psg_workspace::kLanes; i++) CUDA_OK(cudaStreamSynchronize(ws->lane[i]));
  });
}

static void check_panel_part(const psg_plan* plan, int32_t part) {
  if (!plan) throw InvalidArg("a PipelinePlan must come from compile");
  if (part < 0 || part >= (int)plan->host.parts.size()) throw WorkspaceError("no part " + std::to_string(part));
  if (!part_needs_panel(plan, part))
    throw WorkspaceError("part " + std::to_string(part) + " has no per-panel normalization");
}

int psg_panel_factor(const psg_plan* plan, psg_workspace* ws, int32_t part, const void* block, int64_t rows, int32_t cols,
                     const int32_t* live, double* factor_out, void* stream) {
  return guarded([&] {
    check_panel_part(plan, part);
    if (!ws || ws->bytes < ws_device_bytes(rows)) throw WorkspaceError("reserve the workspace for the plan first");
    if (!factor_out) throw InvalidArg("null argument");
    ensure_device();
    cudaStream_t s = (cudaStream_t)stream;
    const double* f = plan->host.dtype == PSG_F32
                          ? panel_factor_dev<float>(plan, ws, part, (const float*)block, rows, cols, live, s)
                          : panel_factor_dev<double>(plan, ws, part, (const double*)block, rows, cols, live, s);
    CUDA_OK(cudaMemcpyAsync(factor_out, f, 8, cudaMemcpyDeviceToDevice, s));
    CUDA_OK(cudaGetLastError());
  });
}

int psg_run_part(const psg_plan* plan, psg_workspace* ws, int32_t part, const void* src, void* dst, int64_t rows,
                 int32_t cols, const int32_t* live, const double* start_ms, double dt_ms, const double* factor,
                 void* stream) {
  return psg_run_part_keyed(plan, ws, part, src, dst, rows, cols, live, start_ms, nullptr, dt_ms, factor, stream);
}

int psg_run_part_keyed(const psg_plan* plan, psg_workspace* ws, int32_t part, const void* src, void* dst, int64_t rows,
                       int32_t cols, const int32_t* live, const double* start_ms, const psg_keys* keys, double dt_ms,
                       const double* factor, void* stream) {
  return guarded([&] {
    check_apply(plan, ws, src, dst, rows, cols, live, dt_ms, false, keys);
    if (part < 0 || part >= (int)plan->host.parts.size()) throw WorkspaceError("no part " + std::to_string(part));
    if (!ws || ws->bytes < 512) throw WorkspaceError("reserve the workspace for the plan first");
    ensure_device();
    cudaStream_t s = (cudaStream_t)stream;
    const double* f = part_needs_panel(plan, part) ? factor : nullptr;
    if (plan->host.dtype == PSG_F32) run_part<float>(plan, ws, part, src, dst, rows, cols, live, start_ms, f, s, keys, dt_ms);
    else run_part<double>(plan, ws, part, src, dst, rows, cols, live, start_ms, f, s, keys, dt_ms);
  });
}

int psg_panel_partials(const psg_plan* plan, psg_workspace* ws, int32_t part, const void* block, int64_t rows,
                       int32_t cols, const int32_t* live, double* partial, void* stream) {
  return guarded([&] {
    check_panel_part(plan, part);
    if (!ws || ws->bytes < ws_device_bytes(rows)) throw WorkspaceError("reserve the workspace for the plan first");
    if (!partial) throw InvalidArg("null argument");
    ensure_device();
    cudaStream_t s = (cudaStream_t)stream;
    const StepHost& ns = plan->host.steps[plan->host.parts[part].first];
    char* base = (char*)ws->d;
    PanelOut* out = reinterpret_cast<PanelOut*>(base + 64 * part);
    double* ss = reinterpret_cast<double*>(base + 512);
    double* mx = ss + rows;
    unsigned* hist = reinterpret_cast<unsigned*>(base + 512 + align256(rows * 16));
    int g = (int)std::max<int64_t>(1, std::min<int64_t>(rows, (int64_t)g_sm_count * 8));
    bool f32 = plan->host.dtype == PSG_F32;
    if (rows > 0) {
      if (f32) row_stats_kernel<float><<<g, 256, 0, s>>>((const float*)block, rows, cols, live, ss, mx);
      else row_stats_kernel<double><<<g, 256, 0, s>>>((const double*)block, rows, cols, live, ss, mx);
    }
    panel_fold_kernel<<<1, 1024, 0, s>>>(rows, cols, live, ss, mx, out);
    panel_partial_head_kernel<<<1, 1, 0, s>>>(out, partial);
    if (ns.stat == PSG_NORM_PERCENTILE) {
      CUDA_OK(cudaMemsetAsync(hist, 0, kHist, s));
      if (f32) launch_hist<float>((const float*)block, rows, cols, live, ss, mx, hist, s);
      else launch_hist<double>((const double*)block, rows, cols, live, ss, mx, hist, s);
      hist_to_f64_kernel<<<256, 256, 0, s>>>(hist, partial + PSG_PANEL_PARTIAL_HEAD);
    } else {
      CUDA_OK(cudaMemsetAsync(partial + PSG_PANEL_PARTIAL_HEAD, 0, 65536 * sizeof(double), s));
    }
    CUDA_OK(cudaGetLastError());
  });
}

int psg_panel_factor_from(const psg_plan* plan, psg_workspace* ws, int32_t part, const double* partial,
                          double* factor_out, void* stream) {
  return guarded([&] {
    check_panel_part(plan, part);
    if (!ws || ws->bytes < 512) throw WorkspaceError("reserve the workspace for the plan first");
    if (!partial || !factor_out) throw InvalidArg("null argument");
    ensure_device();
    cudaStream_t s = (cudaStream_t)stream;
    const StepHost& ns = plan->host.steps[plan->host.parts[part].first];
    PanelOut* out = reinterpret_cast<PanelOut*>((char*)ws->d + 64 * part);
    double clipP = ns.stat == PSG_NORM_PERCENTILE ? ns.percentile : NAN;
    partial_to_out_kernel<<<1, 1, 0, s>>>(partial, out);
    panel_clip_kernel<double><<<1, 1024, 0, s>>>(partial + PSG_PANEL_PARTIAL_HEAD, out, clipP, ns.stat,
                                                 ns.norm_target, plan->host.dtype);
    CUDA_OK(cudaMemcpyAsync(factor_out, &out->factor, 8, cudaMemcpyDeviceToDevice, s));
    CUDA_OK(cudaGetLastError());
  });
}

}  // extern "C"

// responseModuli (pipeline.nim:774-838): |Σ_j x[j]·exp(−2πi·f·j·dt)| at each
// frequency, one warp per frequency. Each lane sums every 32nd sample in
// float64 at the angle ((−2π·f)·j)·dt, rounded as the reference forms it
// (its phasor is snapped onto that angle every sample); the sine and cosine
// are taken at each sample instead of stepping a phasor, and the lanes' sums
// fold by shuffles.
template <class T>
__global__ void __launch_bounds__(256) response_moduli_kernel(const T* __restrict__ x, int n,
                                                              const double* __restrict__ hz, int m, double dt_s,
                                                              double* __restrict__ gain) {
  const int lane = threadIdx.x & 31;
  const int warps = (int)((gridDim.x * blockDim.x) >> 5);
  for (int k = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); k < m; k += warps) {
    const double a = (-2.0 * 3.141592653589793) * hz[k];
    double re = 0, im = 0;
    for (int j = lane; j < n; j += 32) {
      const double v = (double)x[j];
      double sn, cs;
      sincos(__dmul_rn(a, (double)j) * dt_s, &sn, &cs);
      re += v * cs;
      im += v * sn;
    }
    re = warp_sum(re);
    im = warp_sum(im);
    if (lane == 0) gain[k] = hypot(re, im);
  }
}

template <class T>
static void applied_response(const psg_plan* p, psg_workspace* ws, int32_t samples, const double* hz, int32_t n_hz,
                             double* gain) {
  // the workspace's queued host applies finish first; then a stream of its
  // own, so that nothing else on the device waits for this call
  if (ws->lanes_ready)
    for (int i = 0; i < psg_workspace::kLanes; i++) CUDA_OK(cudaStreamSynchronize(ws->lane[i]));
  struct Stream {
    cudaStream_t s = nullptr;
    ~Stream() {
      if (s) cudaStreamDestroy(s);
    }
  } own;
  CUDA_OK(cudaStreamCreateWithFlags(&own.s, cudaStreamNonBlocking));
  cudaStream_t st = own.s;
  const size_t xb = align256((int64_t)samples * (int64_t)sizeof(T));
  DeviceBuf buf;
  CUDA_OK(cudaMalloc(&buf.p, xb + 256 + 256 + align256((int64_t)n_hz * 16)));
  char* base = (char*)buf.p;
  T* x = reinterpret_cast<T*>(base);
  int* live = reinterpret_cast<int*>(base + xb);
  double* start = reinterpret_cast<double*>(base + xb + 256);  // startMs, t0Ms, offset: all 0
  double* dhz = reinterpret_cast<double*>(base + xb + 512);
  double* dg = dhz + n_hz;
  // a unit impulse at samples / 2 on one live row at t0 = 0 and offset 0
  const T one = (T)1;
  const double zeros[3] = {0, 0, 0};
  CUDA_OK(cudaMemsetAsync(x, 0, (size_t)samples * sizeof(T), st));
  CUDA_OK(cudaMemcpyAsync(x + samples / 2, &one, sizeof(T), cudaMemcpyHostToDevice, st));
  CUDA_OK(cudaMemcpyAsync(live, &samples, sizeof(int), cudaMemcpyHostToDevice, st));
  CUDA_OK(cudaMemcpyAsync(start, zeros, sizeof(zeros), cudaMemcpyHostToDevice, st));
  if (n_hz > 0) CUDA_OK(cudaMemcpyAsync(dhz, hz, (size_t)n_hz * sizeof(double), cudaMemcpyHostToDevice, st));
  const psg_keys keys{start + 2, start + 1, 0, 0};
  for (int part = 0; part < (int)p->host.parts.size(); part++)
    launch_part<T>(p, ws, part, nullptr, x, 1, samples, live, start, st, &keys, p->host.dt_ms);
  if (n_hz > 0) {
    const int grid = (int)std::min<int64_t>(((int64_t)n_hz + 7) / 8, (int64_t)g_sm_count * 8);
    response_moduli_kernel<T><<<grid, 256, 0, st>>>(x, samples, dhz, n_hz, p->host.dt_ms / 1000, dg);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaMemcpyAsync(gain, dg, (size_t)n_hz * sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  CUDA_OK(cudaStreamSynchronize(st));
}

extern "C" {

int psg_applied_response(const psg_op* ops, int32_t n_ops, int32_t dtype, double dt_ms, int32_t samples,
                         const double* hz, int32_t n_hz, double* gain, psg_workspace* ws) {
  return guarded([&] {
    if (n_ops < 0 || (n_ops > 0 && !ops) || n_hz < 0 || (n_hz > 0 && (!hz || !gain)) || !ws)
      throw InvalidArg("null argument");
    // the filters without their trend removal, so that it does not bend the impulse
    std::vector<psg_op> copy(ops, ops + n_ops);
    for (auto& o : copy)
      if (o.kind == PSG_OP_FILTER || o.kind == PSG_OP_IIR) o.trend = PSG_TR_NONE;
    std::unique_ptr<psg_plan> p = make_plan(copy.data(), n_ops, dtype, dt_ms, samples, 0);
    ws_grow_for(ws, p.get(), 1, samples);
    if (dtype == PSG_F32) applied_response<float>(p.get(), ws, samples, hz, n_hz, gain);
    else applied_response<double>(p.get(), ws, samples, hz, n_hz, gain);
  });
}

// The sample types the statistics kernels are built for; anything else is
// refused before a launch (a float32 block read as float64 would be read
// past its end).
static void check_dtype(int32_t dtype) {
  if (dtype != PSG_F32 && dtype != PSG_F64) throw InvalidArg("dtype must be PSG_F32 or PSG_F64, got " + std::to_string(dtype));
}

int psg_trace_stats(const void* block, int32_t dtype, int64_t rows, int32_t cols, const int32_t* live, double* rms_out,
                    double* max_abs_out, void* stream) {
  return guarded([&] {
    check_dtype(dtype);
    if (rows < 0 || cols < 0) throw InvalidArg("rows and cols must be ≥ 0");
    if (rows == 0) return;
    if (!block || !live || !rms_out || !max_abs_out) throw InvalidArg("null argument");
    ensure_device();
    cudaStream_t s = (cudaStream_t)stream;
    int g = (int)std::min<int64_t>(rows, (int64_t)g_sm_count * 8);
    // Σx² into rms_out, max into max_abs_out, then rms = sqrt(Σx²/n) per row
    if (dtype == PSG_F32) row_stats_kernel<float><<<g, 256, 0, s>>>((const float*)block, rows, cols, live, rms_out, max_abs_out);
    else row_stats_kernel<double><<<g, 256, 0, s>>>((const double*)block, rows, cols, live, rms_out, max_abs_out);
    trace_stats_finish<<<(int)((rows + 255) / 256), 256, 0, s>>>(rms_out, max_abs_out, live, rows, cols);
    CUDA_OK(cudaGetLastError());
  });
}

int psg_panel_stats(psg_workspace* ws, const void* block, int32_t dtype, int64_t rows, int32_t cols, const int32_t* live,
                    double clip_percentile, double* out, void* stream) {
  return guarded([&] {
    check_dtype(dtype);
    if (!std::isnan(clip_percentile) && !(clip_percentile >= 0 && clip_percentile <= 100))
      throw InvalidArg("a percentile must be in 0 .. 100, got " + std::to_string(clip_percentile));
    if (rows < 0 || cols < 0) throw InvalidArg("rows and cols must be ≥ 0");
    if ((rows > 0 && (!block || !live)) || !out) throw InvalidArg("null argument");
    if (!ws || ws->bytes < ws_device_bytes(rows)) throw WorkspaceError("reserve the workspace first (psg_workspace_reserve)");
    ensure_device();
    cudaStream_t s = (cudaStream_t)stream;
    char* base = (char*)ws->d;
    PanelOut* po = reinterpret_cast<PanelOut*>(base + 448);
    double* ss = reinterpret_cast<double*>(base + 512);
    double* mx = ss + rows;
    unsigned* hist = reinterpret_cast<unsigned*>(base + 512 + align256(rows * 16));
    int g = (int)std::max<int64_t>(1, std::min<int64_t>(rows, (int64_t)g_sm_count * 8));
    if (rows > 0) {
      if (dtype == PSG_F32) row_stats_kernel<float><<<g, 256, 0, s>>>((const float*)block, rows, cols, live, ss, mx);
      else row_stats_kernel<double><<<g, 256, 0, s>>>((const double*)block, rows, cols, live, ss, mx);
    }
    panel_fold_kernel<<<1, 1024, 0, s>>>(rows, cols, live, ss, mx, po, 1);
    if (!std::isnan(clip_percentile)) {
      CUDA_OK(cudaMemsetAsync(hist, 0, kHist, s));
      if (dtype == PSG_F32) launch_hist<float>((const float*)block, rows, cols, live, ss, mx, hist, s);
      else launch_hist<double>((const double*)block, rows, cols, live, ss, mx, hist, s);
    }
    panel_clip_kernel<unsigned><<<1, 1024, 0, s>>>(hist, po, clip_percentile, -1, 1.0, dtype);
    CUDA_OK(cudaMemcpyAsync(out, po, 5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CUDA_OK(cudaGetLastError());
  });
}

// ------------------------------------------------- panel stats, no allocation
// psg_panel_stats for callers that cannot allocate device memory: its scratch
// (the panel output, per-row Σx² and max |x|, and the 65536-bin histogram)
// is a fixed array of this file, sized for PSG_STATIC_MAX_ROWS rows, that
// every GPU which loads the library holds until the process exits. Host code
// must not pass the array's name to a kernel (on the host it is a stand-in,
// not a device address): the device address is looked up once per device
// with cudaGetSymbolAddress and cached.
}  // extern "C"
static const int64_t kStaticBytes = 512 + (int64_t)PSG_STATIC_MAX_ROWS * 16 + kHist;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];
static std::mutex g_static_mu;
// The array's device address per device, looked up on the first call on that
// device. A device reset (cudaDeviceReset) unloads the module and with it the
// array: after one, the cached address is stale, so a process that resets a
// device must not call psg_panel_stats_static on it again.
static void* g_static_addr[128];
extern "C" {

int psg_panel_stats_static(const void* block, int32_t dtype, int64_t rows, int32_t cols, const int32_t* live,
                           double clip_percentile, double* out, void* stream) {
  return guarded([&] {
    check_dtype(dtype);
    if (!std::isnan(clip_percentile) && !(clip_percentile >= 0 && clip_percentile <= 100))
      throw InvalidArg("a percentile must be in 0 .. 100, got " + std::to_string(clip_percentile));
    if (rows < 0 || cols < 0) throw InvalidArg("rows and cols must be ≥ 0");
    if (rows > PSG_STATIC_MAX_ROWS)
      throw InvalidArg("psg_panel_stats_static takes at most " + std::to_string(PSG_STATIC_MAX_ROWS) +
                       " rows, got " + std::to_string(rows) + " (use psg_panel_stats with a workspace)");
    if (rows > 0 && (!block || !live)) throw InvalidArg("null argument");
    if (!out) throw InvalidArg("null argument");
    ensure_device();
    int dev;
    CUDA_OK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) throw InvalidArg("device ordinal out of range");
    char* base;
    {
      std::lock_guard<std::mutex> g(g_static_mu);
      if (!g_static_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) throw CudaError(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_static_addr[dev] = p;
      }
      base = (char*)g_static_addr[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    PanelOut* po = reinterpret_cast<PanelOut*>(base + 448);
    double* ss = reinterpret_cast<double*>(base + 512);
    double* mx = ss + rows;
    unsigned* hist = reinterpret_cast<unsigned*>(base + 512 + (int64_t)PSG_STATIC_MAX_ROWS * 16);
    int g = (int)std::max<int64_t>(1, std::min<int64_t>(rows, (int64_t)g_sm_count * 8));
    if (rows > 0) {
      if (dtype == PSG_F32) row_stats_kernel<float><<<g, 256, 0, s>>>((const float*)block, rows, cols, live, ss, mx);
      else row_stats_kernel<double><<<g, 256, 0, s>>>((const double*)block, rows, cols, live, ss, mx);
    }
    panel_fold_kernel<<<1, 1024, 0, s>>>(rows, cols, live, ss, mx, po, 1);
    if (!std::isnan(clip_percentile)) {
      // The array keeps the previous call's counts: the histogram starts at zero.
      CUDA_OK(cudaMemsetAsync(hist, 0, kHist, s));
      if (dtype == PSG_F32) launch_hist<float>((const float*)block, rows, cols, live, ss, mx, hist, s);
      else launch_hist<double>((const double*)block, rows, cols, live, ss, mx, hist, s);
    }
    panel_clip_kernel<unsigned><<<1, 1024, 0, s>>>(hist, po, clip_percentile, -1, 1.0, dtype);
    CUDA_OK(cudaMemcpyAsync(out, po, 5 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CUDA_OK(cudaGetLastError());
  });
}

// ------------------------------------------------------------- vibroseis
namespace {
SweepHost sweep_host(const psg_sweep* p) {
  if (!p) throw InvalidArg("null argument");
  SweepHost s;
  s.law = p->law;
  s.f1 = p->f1_hz;
  s.f2 = p->f2_hz;
  s.length_ms = p->length_ms;
  s.dt_ms = p->dt_ms;
  s.boost_db = p->boost_db;
  if (p->law == PSG_SL_TABLE) {
    if (p->n_table < 0 || p->n_table > (1 << 24) || (p->n_table > 0 && !p->table))
      throw InvalidArg("a sweep table needs 0 .. 2²⁴ points and a pointer to them");
    s.table.assign(p->table, p->table + p->n_table);
  }
  s.phase_deg = p->start_phase_deg;
  s.amplitude = p->amplitude;
  s.taper_start = p->taper_start_ms;
  s.taper_end = p->taper_end_ms;
  s.taper_shape = p->taper_shape;
  s.taper_param = p->taper_param;
  s.max_nyq = p->max_nyquist_fraction;
  return s;
}
void put_samples(const std::vector<double>& x, int32_t dtype, void* out) {
  if (dtype == PSG_F32)
    for (size_t i = 0; i < x.size(); i++) ((float*)out)[i] = (float)x[i];
  else
    std::memcpy(out, x.data(), x.size() * 8);
}
}  // namespace

int psg_sweep_validate(const psg_sweep* spec) {
  return guarded([&] { sweep_validate(sweep_host(spec)); });
}

int psg_sweep_len(const psg_sweep* spec, int64_t* n) {
  return guarded([&] {
    if (!n) throw InvalidArg("null argument");
    *n = sweep_len(sweep_host(spec));
  });
}

int psg_sweep_frequency_at(const psg_sweep* spec, double t_ms, double* out) {
  return guarded([&] {
    if (!out) throw InvalidArg("null argument");
    SweepHost s = sweep_host(spec);
    sweep_validate(s);
    *out = sweep_frequency_at(s, t_ms);
  });
}

int psg_sweep_phase_at(const psg_sweep* spec, double t_ms, double* out) {
  return guarded([&] {
    if (!out) throw InvalidArg("null argument");
    SweepHost s = sweep_host(spec);
    sweep_validate(s);
    *out = sweep_phase_at(s, t_ms);
  });
}

int psg_sweep_samples(const psg_sweep* spec, const psg_sweep_harmonic* harmonics, int32_t n_harmonics, int32_t dtype,
                      void* out, int64_t n, int32_t* segy_type) {
  return guarded([&] {
    if (dtype != PSG_F32 && dtype != PSG_F64) throw InvalidArg("dtype must be float32 or float64");
    if (!out || n_harmonics < 0 || (n_harmonics > 0 && !harmonics)) throw InvalidArg("null argument");
    SweepHost s = sweep_host(spec);
    std::vector<psg_sweep_harmonic> hs(harmonics, harmonics + n_harmonics);
    std::vector<double> x = sweep_samples(s, hs, n, dtype);
    put_samples(x, dtype, out);
    if (segy_type) *segy_type = sweep_segy_type(s);
  });
}

int psg_linear_sweep(double f1, double f2, double length_ms, double dt_ms, double ts, double te, int32_t shape,
                     double taper_param, double phase_deg, double amplitude, double max_nyq, int32_t dtype,
                     void* out, int64_t* n_out) {
  return guarded([&] {
    if (!n_out) throw InvalidArg("null argument");
    if (dtype != PSG_F32 && dtype != PSG_F64) throw InvalidArg("dtype must be float32 or float64");
    SweepHost s;
    s.law = PSG_SL_LINEAR;
    s.f1 = f1;
    s.f2 = f2;
    s.length_ms = length_ms;
    s.dt_ms = dt_ms;
    s.phase_deg = phase_deg;
    s.amplitude = amplitude;
    s.taper_start = ts;
    s.taper_end = te;
    s.taper_shape = shape;
    s.taper_param = taper_param;
    s.max_nyq = max_nyq;
    sweep_validate(s);
    *n_out = sweep_len(s);
    if (out) put_samples(sweep_samples(s, {}, *n_out, dtype), dtype, out);
  });
}

int psg_taper_weight(int32_t shape, double x, double param, double* out) {
  return guarded([&] {
    if (!out) throw InvalidArg("null argument");
    *out = taper_weight(shape, x, param);
  });
}

int psg_apply_taper(int32_t dtype, void* x, int64_t n, double dt_ms, double start_ms, double end_ms, int32_t shape,
                    double param) {
  return guarded([&] {
    if (dtype != PSG_F32 && dtype != PSG_F64) throw InvalidArg("dtype must be float32 or float64");
    if (n < 0 || (n > 0 && !x)) throw InvalidArg("null argument or a negative length");
    std::vector<double> v((size_t)n);
    for (int64_t i = 0; i < n; i++) v[i] = dtype == PSG_F32 ? (double)((float*)x)[i] : ((double*)x)[i];
    apply_taper(dtype, v.data(), n, dt_ms, start_ms, end_ms, shape, param);  // raises before any write
    for (int64_t i = 0; i < n; i++) {
      if (dtype == PSG_F32) ((float*)x)[i] = (float)v[i];
      else ((double*)x)[i] = v[i];
    }
  });
}

int psg_corr_plan_create(const void* pilot, int32_t pilot_dtype, int64_t pilot_len, double pilot_dt_ms, double pilot_t0_ms,
                         int32_t dtype, double dt_ms, int32_t record_samples, int32_t out_samples, int32_t mode,
                         double eps_percent, int32_t normalize, psg_corr_plan** out) {
  return guarded([&] {
    if (!out || !pilot) throw InvalidArg("null argument");
    if (dtype != PSG_F32 && dtype != PSG_F64) throw InvalidArg("dtype must be float32 or float64");
    std::vector<double> pv(pilot_len > 0 ? pilot_len : 0);
    for (int64_t i = 0; i < pilot_len; i++)
      pv[i] = pilot_dtype == PSG_F32 ? (double)((const float*)pilot)[i] : ((const double*)pilot)[i];
    std::unique_ptr<psg_corr_plan> p(new psg_corr_plan());
    p->host = corr_plan(pv.data(), pilot_len, pilot_dt_ms, pilot_t0_ms, dt_ms, record_samples, out_samples, mode,
                        eps_percent, normalize != 0, dtype == PSG_F32 ? 16 : 8);
    p->dtype = dtype;
    ensure_device();
    if (dtype == PSG_F32) corr_upload<float>(p.get());
    else corr_upload<double>(p.get());
    *out = p.release();
  });
}
void psg_corr_plan_destroy(psg_corr_plan* p) { delete p; }
int32_t psg_corr_plan_nfft(const psg_corr_plan* p) { return p ? (int32_t)p->host.n : 0; }
int32_t psg_corr_plan_out_samples(const psg_corr_plan* p) { return p ? (int32_t)p->host.out : 0; }
double psg_corr_plan_scale(const psg_corr_plan* p) { return p ? p->host.scale : 0; }

static int corr_launch(const psg_corr_plan* plan, psg_stack* st, const void* src, void* dst, int64_t rows, int32_t cols,
                       const int32_t* live, const int32_t* stack_live, const int32_t* row_map, double dt_ms, void* stream) {
  return guarded([&] {
    if (!plan) throw InvalidArg("a CorrelationPlan must come from initCorrelationPlan");
    if (rows < 0 || cols < 0) throw InvalidArg("rows and cols must be ≥ 0");
    if (cols > plan->host.record)
      throw InvalidArg("the records are " + std::to_string(cols) + " samples, the plan takes " + std::to_string(plan->host.record));
    if (!same_interval(dt_ms, plan->host.dt_ms))
      throw InvalidArg("the records are at " + std::to_string(dt_ms) + " ms, the plan at " + std::to_string(plan->host.dt_ms) + " ms");
    if (st && !same_interval(st->dt_ms, dt_ms)) throw InvalidArg("the stack is at another interval");
    if (st && !row_map && rows > st->rows) throw InvalidArg("a record of " + std::to_string(rows) + " rows into a stack of " + std::to_string(st->rows) + " (pass a rowMap)");
    if (rows == 0) return;
    if (!src || !live || (!dst && !st)) throw InvalidArg("null argument");
    ensure_device();
    CorrArgs a{};
    a.src = src;
    a.dst = dst;
    a.rows = rows;
    a.cols = cols;
    a.out = (int)plan->host.out;
    a.nfft = (int)plan->host.n;
    a.shift = (int)plan->host.shift;
    a.pilot_len = (int)plan->host.pilot_len;
    a.record = (int)plan->host.record;
    a.live = live;
    a.bridge = plan->bridge;
    a.tw = plan->tw;
    a.fft = plan->fft;
    a.gwork = plan->gwork;
    if (st) {
      a.stack_on = 1;
      a.num = st->num;
      a.cnt = st->cnt;
      a.stack_samples = st->samples;
      a.stack_rows = st->rows;
      a.row_map = row_map;
      a.stack_live = stack_live;
    }
    int grid = (int)std::min<int64_t>(rows, plan->grid);
    cudaStream_t s = (cudaStream_t)stream;
    if (plan->trace) {
      a.tw_pass = plan->tw_pass;
      void* args[] = {&a};
      CUDA_OK(cudaLaunchKernel(plan->trace->kernel[0][0], dim3((int)std::min<int64_t>(rows, plan->trace_grid)),
                               dim3(plan->trace->nt), args, plan->smem, s));
    } else if (plan->dtype == PSG_F32) {
      corr_kernel<float><<<grid, kCorrThreads, plan->smem, s>>>(a);
    } else {
      corr_kernel<double><<<grid, kCorrThreads, plan->smem, s>>>(a);
    }
    CUDA_OK(cudaGetLastError());
  });
}

int psg_correlate(const psg_corr_plan* plan, const void* src, void* dst, int64_t rows, int32_t cols, const int32_t* live,
                  double dt_ms, void* stream) {
  if (!dst && rows > 0) {
    t_err = "dst is required";
    return PSG_EINVAL;
  }
  return corr_launch(plan, nullptr, src, dst, rows, cols, live, nullptr, nullptr, dt_ms, stream);
}

int psg_stack_create(int64_t rows, int32_t samples, double dt_ms, psg_stack** out) {
  return guarded([&] {
    if (!out) throw InvalidArg("null argument");
    if (rows < 0 || samples < 0) throw InvalidArg("rows and samples must be ≥ 0");
    if (!(std::isfinite(dt_ms) && dt_ms > 0)) throw InvalidArg("dtMs must be finite and positive");
    ensure_device();
    std::unique_ptr<psg_stack> s(new psg_stack());
    s->rows = rows;
    s->samples = samples;
    s->dt_ms = dt_ms;
    size_t n = (size_t)(rows * samples);
    if (n) {
      CUDA_OK(cudaMalloc(&s->num, n * 8));
      CUDA_OK(cudaMalloc(&s->cnt, n * 4));
      CUDA_OK(cudaMemset(s->num, 0, n * 8));
      CUDA_OK(cudaMemset(s->cnt, 0, n * 4));
    }
    *out = s.release();
  });
}
void psg_stack_destroy(psg_stack* s) {
  if (!s) return;
  if (s->num) cudaFree(s->num);
  if (s->cnt) cudaFree(s->cnt);
  delete s;
}
int psg_stack_clear(psg_stack* st, void* stream) {
  return guarded([&] {
    if (!st) throw InvalidArg("null argument");
    size_t n = (size_t)(st->rows * st->samples);
    if (n) {
      CUDA_OK(cudaMemsetAsync(st->num, 0, n * 8, (cudaStream_t)stream));
      CUDA_OK(cudaMemsetAsync(st->cnt, 0, n * 4, (cudaStream_t)stream));
    }
  });
}
int psg_stack_add(psg_stack* st, const void* block, int32_t dtype, int64_t rows, int32_t cols, const int32_t* live,
                  const int32_t* row_map, void* stream) {
  return guarded([&] {
    if (!st) throw InvalidArg("null argument");
    if (cols > st->samples) throw InvalidArg("the record has " + std::to_string(cols) + " samples, the stack " + std::to_string(st->samples));
    if (!row_map && rows > st->rows) throw InvalidArg("a record of " + std::to_string(rows) + " rows into a stack of " + std::to_string(st->rows) + " (pass a rowMap)");
    if (rows == 0) return;
    ensure_device();
    int g = (int)std::min<int64_t>(rows, (int64_t)g_sm_count * 8);
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == PSG_F32) stack_add_kernel<float><<<g, 256, 0, s>>>((const float*)block, rows, cols, live, row_map, st->num, st->cnt, st->samples, st->rows);
    else stack_add_kernel<double><<<g, 256, 0, s>>>((const double*)block, rows, cols, live, row_map, st->num, st->cnt, st->samples, st->rows);
    CUDA_OK(cudaGetLastError());
  });
}
int psg_correlate_stack(const psg_corr_plan* plan, psg_stack* st, const void* src, void* dst, int64_t rows, int32_t cols,
                        const int32_t* live, const int32_t* stack_live, const int32_t* row_map, double dt_ms, void* stream) {
  if (!st) {
    t_err = "a stack is required";
    return PSG_EINVAL;
  }
  return corr_launch(plan, st, src, dst, rows, cols, live, stack_live, row_map, dt_ms, stream);
}

// ------------------------------------------------------------- spectra
int psg_spectrum_plan_create(int32_t dtype, double dt_ms, int32_t window_len, double taper_fraction, int32_t nfft,
                             int32_t demean, psg_spectrum_plan** out) {
  return guarded([&] {
    if (!out) throw InvalidArg("null argument");
    *out = nullptr;
    std::unique_ptr<psg_spectrum_plan> p(new psg_spectrum_plan());
    p->host = spectrum_plan(dtype, dt_ms, window_len, taper_fraction, nfft, demean != 0, dtype == PSG_F32 ? 12 : 8);
    ensure_device();
    const SpectrumHost& h = p->host;
    const int limit = g_max_smem - (int)sizeof(SharedMem) - 1024;
    auto setup = [&](auto tag) {
      typedef decltype(tag) T;
      typedef typename C2<T>::type V;
      p->taper = upload(p->keep, as_t<T>(h.taper));
      p->tw = upload(p->keep, as_c<T>(h.fft.tw_re, h.fft.tw_im));
      p->split = upload(p->keep, as_c<T>(h.fft.split_re, h.fft.split_im));
      p->fft = fft_desc(h.fft);
      const int64_t need = 2 * h.fft.m * (int64_t)sizeof(V);
      const void* k0 = (const void*)spectrum_kernel<T, true>;
      const void* k1 = (const void*)spectrum_kernel<T, false>;
      if (need <= limit) {
        p->smem = (size_t)need;
        allow_smem(k0);
        allow_smem(k1);
        int per_sm = 0;
        CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k0, 256, p->smem));
        p->grid = std::max(1, per_sm) * g_sm_count;
      } else {
        p->smem = 0;
        p->gstride = align256(need);
        p->grid = 2 * g_sm_count;
      }
    };
    if (dtype == PSG_F32) setup(float());
    else setup(double());
    *out = p.release();
  });
}
void psg_spectrum_plan_destroy(psg_spectrum_plan* p) { delete p; }
int psg_spectrum_plan_info(const psg_spectrum_plan* p, int32_t* nfft, int32_t* bins, int32_t* window_len,
                           double* taper_sum) {
  return guarded([&] {
    if (!p) throw InvalidArg("a SpectrumPlan must come from initSpectrumPlan");
    if (nfft) *nfft = (int32_t)p->host.nfft;
    if (bins) *bins = (int32_t)p->host.bins;
    if (window_len) *window_len = (int32_t)p->host.window;
    if (taper_sum) *taper_sum = p->host.taper_sum;
  });
}

static void sp_grow(psg_workspace* ws, int64_t need) {
  int dev;
  CUDA_OK(cudaGetDevice(&dev));
  if ((ws->d || ws->sp) && ws->device >= 0 && ws->device != dev) throw InvalidArg("the workspace belongs to another device");
  ws->device = dev;
  if (ws->sp_bytes >= need) return;
  if (ws->sp) {
    CUDA_OK(cudaDeviceSynchronize());
    CUDA_OK(cudaFree(ws->sp));
    ws->sp = nullptr;
    ws->sp_bytes = 0;
  }
  CUDA_OK(cudaMalloc(&ws->sp, (size_t)need));
  ws->sp_bytes = need;
}

static void spectrum_launch(const psg_spectrum_plan* p, psg_workspace* ws, const void* block, int64_t rows, int32_t cols,
                            const int32_t* live, double dt_ms, int32_t first_col, int64_t row0, int64_t row1, bool avg,
                            double* amp, int64_t* used, void* amp_t, void* phase_t, cudaStream_t stream) {
  if (!p) throw InvalidArg("a SpectrumPlan must come from initSpectrumPlan");
  if (!ws) throw InvalidArg("a workspace is required");
  if (rows < 0 || cols < 0) throw InvalidArg("rows and cols must be ≥ 0");
  if (rows > 0 && (!block || !live)) throw InvalidArg("block and live are required");
  if (!same_interval(dt_ms, p->host.dt_ms))
    throw InvalidArg("the rows' interval " + std::to_string(dt_ms) + " ms is not the plan's " + std::to_string(p->host.dt_ms) + " ms");
  if (first_col < 0) throw InvalidArg("firstCol must be ≥ 0, got " + std::to_string(first_col));
  if (avg && !amp) throw InvalidArg("amp is required");
  if (!avg && rows > 0 && (!amp_t || !phase_t)) throw InvalidArg("amp and phase are required");
  ensure_device();
  const int64_t lo = std::max<int64_t>(row0, 0), hi = std::min<int64_t>(row1, rows - 1);
  const int64_t nr = hi >= lo ? hi - lo + 1 : 0;
  const int bins = (int)p->host.bins;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(nr, p->grid));
  const int64_t acc_b = avg ? align256((int64_t)grid * bins * 8) + align256((int64_t)grid * 4) : 0;
  sp_grow(ws, acc_b + p->gstride * grid + 256);
  SpecArgs a{};
  a.src = block;
  a.row0 = lo;
  a.row1 = hi;
  a.cols = cols;
  a.first_col = first_col;
  a.live = live;
  a.window = (int)p->host.window;
  a.nfft = (int)p->host.nfft;
  a.bins = bins;
  a.odd = p->host.odd;
  a.demean = p->host.demean;
  a.taper = p->taper;
  a.taper_sum = p->host.taper_sum;
  a.tw = p->tw;
  a.split = p->split;
  a.fft = p->fft;
  char* base = (char*)ws->sp;
  a.acc = avg ? (double*)base : nullptr;
  a.used = avg ? (int*)(base + align256((int64_t)grid * bins * 8)) : nullptr;
  a.gwork = p->smem ? nullptr : base + acc_b;
  a.gstride = p->gstride;
  a.amp = amp_t;
  a.phase = phase_t;
  void* args[] = {&a};
  const bool f32 = p->host.dtype == PSG_F32;
  const void* k = avg ? (f32 ? (const void*)spectrum_kernel<float, true> : (const void*)spectrum_kernel<double, true>)
                      : (f32 ? (const void*)spectrum_kernel<float, false> : (const void*)spectrum_kernel<double, false>);
  if (nr > 0 || avg) CUDA_OK(cudaLaunchKernel(k, dim3(grid), dim3(256), args, p->smem, stream));
  if (avg) spectrum_finish<<<bins, 256, 0, stream>>>(a.acc, a.used, grid, bins, a.nfft, amp, (long long*)used);
  CUDA_OK(cudaGetLastError());
}

int psg_spectrum_average(const psg_spectrum_plan* plan, psg_workspace* ws, const void* block, int64_t rows, int32_t cols,
                         const int32_t* live, double dt_ms, int32_t first_col, int64_t row0, int64_t row1, double* amp,
                         int64_t* used, void* stream) {
  return guarded([&] {
    spectrum_launch(plan, ws, block, rows, cols, live, dt_ms, first_col, row0, row1, true, amp, used, nullptr, nullptr,
                    (cudaStream_t)stream);
  });
}
int psg_spectrum_amplitude(const psg_spectrum_plan* plan, psg_workspace* ws, const void* block, int64_t rows,
                           int32_t cols, const int32_t* live, double dt_ms, int32_t first_col, void* amp, void* phase,
                           void* stream) {
  return guarded([&] {
    spectrum_launch(plan, ws, block, rows, cols, live, dt_ms, first_col, 0, rows - 1, false, nullptr, nullptr, amp,
                    phase, (cudaStream_t)stream);
  });
}


// ------------------------------------------------------------- per-row scale
int psg_scale_rows(psg_workspace* ws, int32_t dtype, const void* src, void* dst, int64_t rows, int32_t cols,
                   const int32_t* live, const double* factors_host, void* stream) {
  return guarded([&] {
    if (!ws) throw InvalidArg("a workspace is required");
    if (dtype != PSG_F32 && dtype != PSG_F64) throw InvalidArg("dtype must be float32 or float64");
    if (rows < 0 || cols < 0) throw InvalidArg("rows and cols must be ≥ 0");
    if (rows > 0 && (!dst || !live || !factors_host)) throw InvalidArg("null argument");
    const int64_t esz = dtype == PSG_F32 ? 4 : 8;
    if (src && src != dst) {
      uintptr_t s0 = (uintptr_t)src, d0 = (uintptr_t)dst, bytes = (uintptr_t)(rows * cols * esz);
      if (s0 < d0 + bytes && d0 < s0 + bytes) throw InvalidArg("src and dst overlap without being the same block");
    }
    for (int64_t r = 0; r < rows; r++)
      if (std::isinf(factors_host[r]) || std::isinf(dtype == PSG_F32 ? (double)(float)factors_host[r] : factors_host[r]))
        throw InvalidArg("row " + std::to_string(r) + " has an infinite factor (" + std::to_string(factors_host[r]) + ")");
    if (rows == 0) return;
    ensure_device();
    sp_grow(ws, align256(rows * 8));
    cudaStream_t st = (cudaStream_t)stream;
    CUDA_OK(cudaMemcpyAsync(ws->sp, factors_host, (size_t)rows * 8, cudaMemcpyHostToDevice, st));
    const int grid = (int)std::min<int64_t>(rows, (int64_t)g_sm_count * 8);
    if (dtype == PSG_F32)
      scale_rows_kernel<float><<<grid, 256, 0, st>>>((const float*)(src ? src : dst), (float*)dst, rows, cols, live,
                                                     (const double*)ws->sp);
    else
      scale_rows_kernel<double><<<grid, 256, 0, st>>>((const double*)(src ? src : dst), (double*)dst, rows, cols, live,
                                                      (const double*)ws->sp);
    CUDA_OK(cudaGetLastError());
    // the factors' staging is reused by the next call: it must have landed
    CUDA_OK(cudaStreamSynchronize(st));
  });
}
// ------------------------------------------------------------- SEG-Y
int psg_segy_decode(const void* records, int64_t rows, int64_t record_bytes, int32_t header_bytes, int32_t samples,
                    int32_t format, int32_t little_endian, int32_t dtype, void* out, int32_t out_cols, void* stream) {
  return guarded([&] {
    const int sz = segy_sample_bytes(format);
    if (sz == 0) throw InvalidArg("SEG-Y data sample format " + std::to_string(format) + " is not supported");
    if (dtype != PSG_F32 && dtype != PSG_F64) throw InvalidArg("dtype must be float32 or float64");
    if (rows < 0 || header_bytes < 0 || samples < 0 || out_cols < 0) throw InvalidArg("negative size");
    if ((int64_t)header_bytes + (int64_t)samples * sz > record_bytes)
      throw InvalidArg("a record of " + std::to_string(record_bytes) + " bytes holds no " + std::to_string(samples) +
                       " samples of " + std::to_string(sz) + " bytes after a " + std::to_string(header_bytes) +
                       "-byte header");
    if (rows > 0 && (!records || (!out && out_cols > 0))) throw InvalidArg("null argument");
    if (rows == 0 || out_cols == 0) return;
    ensure_device();
    const int grid = (int)std::min<int64_t>(rows, (int64_t)g_sm_count * 8);
    cudaStream_t st = (cudaStream_t)stream;
    if (dtype == PSG_F32)
      segy_decode_kernel<float><<<grid, 256, 0, st>>>((const unsigned char*)records, rows, record_bytes, header_bytes,
                                                      samples, format, little_endian, (float*)out, out_cols);
    else
      segy_decode_kernel<double><<<grid, 256, 0, st>>>((const unsigned char*)records, rows, record_bytes, header_bytes,
                                                       samples, format, little_endian, (double*)out, out_cols);
    CUDA_OK(cudaGetLastError());
  });
}
int psg_segy_keys(const void* records, int64_t rows, int64_t record_bytes, int32_t little_endian, int32_t* status,
                  int32_t* num_samples, double* interval_us, double* offset, double* t0_ms, void* stream) {
  return guarded([&] {
    if (rows < 0) throw InvalidArg("negative size");
    if (record_bytes < 240) throw InvalidArg("a SEG-Y trace record holds a 240-byte header");
    if (rows > 0 && !records) throw InvalidArg("null argument");
    if (rows == 0) return;
    ensure_device();
    const int grid = (int)std::min<int64_t>((rows + 255) / 256, (int64_t)g_sm_count * 8);
    segy_keys_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>((const unsigned char*)records, rows, record_bytes,
                                                             little_endian, status, num_samples, interval_us, offset,
                                                             t0_ms);
    CUDA_OK(cudaGetLastError());
  });
}
int psg_stack_result(const psg_stack* st, void* dst, int32_t dtype, int32_t norm, void* stream) {
  return guarded([&] {
    if (!st || !dst) throw InvalidArg("null argument");
    long long total = (long long)st->rows * st->samples;
    if (!total) return;
    ensure_device();
    int g = (int)std::min<long long>((total + 255) / 256, (long long)g_sm_count * 16);
    cudaStream_t s = (cudaStream_t)stream;
    if (dtype == PSG_F32) stack_result_kernel<float><<<g, 256, 0, s>>>(st->num, st->cnt, total, norm, (float*)dst);
    else stack_result_kernel<double><<<g, 256, 0, s>>>(st->num, st->cnt, total, norm, (double*)dst);
    CUDA_OK(cudaGetLastError());
  });
}
int psg_stack_fold(const psg_stack* st, int32_t* dst, void* stream) {
  return guarded([&] {
    if (!st || !dst) throw InvalidArg("null argument");
    size_t n = (size_t)(st->rows * st->samples);
    if (n) CUDA_OK(cudaMemcpyAsync(dst, st->cnt, n * 4, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  });
}

}  // extern "C"

// traceStatsInto's finish: rms = sqrt(Σx²/n) for live rows, NaN for others.
// statsOf (gain/stats.nim:124-127) per row: a row that is not live
// (live[r] < 0) reads NaN for both; a live row with no live samples reads
// (0, 0); otherwise rms = sqrt(Σx²/n).
__global__ void trace_stats_finish(double* rms, double* mx, const int* live, long long rows, int cols) {
  long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= rows) return;
  if (live[r] < 0) {
    rms[r] = NAN;
    mx[r] = NAN;
    return;
  }
  int n = min(live[r], cols);
  if (n == 0) {
    rms[r] = 0;
    mx[r] = 0;
  } else {
    rms[r] = sqrt(rms[r] / (double)n);
  }
}

// ================================================================ serving
// A request loop for a viewer's zoom-window and panel requests (different
// trace counts, widths and plans). Requests are admitted by their device
// footprint into a fixed arena (no allocation per request), copied in on
// one stream, run together in one launch of the batched pipeline kernel (each
// trace with its own request's plan), and copied out on another stream, so
// that requests arriving while others are on the GPU join the next launch
// and the copies of one overlap the kernels of others. The results are those
// of the plain apply: the kernel computes each trace the same way alone or
// in a batch.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <thread>
#include <unordered_map>

namespace psg {
namespace {
double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Arena {
  int64_t size = 0;
  std::map<int64_t, int64_t> free_;  // offset → bytes
  void init(int64_t n) {
    size = n;
    free_.clear();
    free_[0] = n;
  }
  int64_t alloc(int64_t n) {
    n = (n + 255) / 256 * 256;
    for (auto it = free_.begin(); it != free_.end(); ++it)
      if (it->second >= n) {
        int64_t off = it->first, rest = it->second - n;
        free_.erase(it);
        if (rest) free_[off + n] = rest;
        return off;
      }
    return -1;
  }
  void release(int64_t off, int64_t n) {
    n = (n + 255) / 256 * 256;
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && off + n == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
};

// How the loop runs a request: rows of the batched generic kernel (float32
// single-part plans without a per-trace kernel of their own), rows of the
// batched trace kernel of its transform length (plans the plain apply runs
// on the trace kernel), or alone, part by part through the plain apply's
// launches (per-panel normalizations, float64, IIR filters, mutes, long
// traces). Each gives what the plain apply gives, bit for bit.
enum { K_GENERIC = 0, K_TRACE = 1, K_SOLO = 2 };

struct Req {
  uint64_t ticket = 0;
  const psg_plan* plan = nullptr;
  const void* src = nullptr;  // host memory (staged through the arena) or device memory
  void* dst = nullptr;
  const int32_t* live = nullptr;
  const double* start = nullptr;
  const double* key_off = nullptr;  // a muting plan's rows' offsets and t0Ms
  const double* key_t0 = nullptr;
  int32_t first_sample = 0;
  double dt_ms = 0;
  int64_t rows = 0;
  int32_t cols = 0;
  int esz = 4;
  bool device = false;  // the buffers are device memory: no copies in or out
  int kind = K_GENERIC;
  const TracePlanInfo* trace = nullptr;  // K_TRACE: the build whose batched kernel runs it
  int64_t off = -1, bytes = 0;
  // the device addresses the kernels read and write (the arena's or the caller's)
  char* d_data = nullptr;
  const char* d_src = nullptr;
  const int* d_live = nullptr;
  const double* d_start = nullptr;
  const double* d_off = nullptr;
  const double* d_t0 = nullptr;
  double t_submit = 0, t_done = 0;
  int status = PSG_OK;
  bool done = false;
  bool claimed = false;      // a thread is in psg_wait on it (one waiter per ticket)
  cudaEvent_t in = nullptr;  // its copy in finished
};

struct Batch {
  std::vector<Req*> reqs;
  cudaEvent_t kern = nullptr;  // its kernels finished
  cudaEvent_t done = nullptr;  // its copies out finished
  bool kern_done = false;
  int slot = 0;
};
}  // namespace
}  // namespace psg

struct psg_server {
  int device = 0;
  char* arena_d = nullptr;
  Arena arena;
  static const int kSlots = 4, kMaxJobs = 64;
  // copies in on one stream; each batch slot its own kernel and copy-out
  // streams, so a batch can start while another one's kernels run
  cudaStream_t s_in = nullptr, s_comp[kSlots] = {}, s_out[kSlots] = {};
  psg_workspace* ws[kSlots] = {};  // the plain apply's scratch for requests run alone
  Job* jobs_h = nullptr;  // pinned, kSlots × kMaxJobs
  long long* begin_h = nullptr;
  Job* jobs_d = nullptr;
  long long* begin_d = nullptr;
  int* status_d = nullptr;
  bool slot_busy[kSlots] = {};
  std::thread sched;
  std::mutex mu;
  std::condition_variable cv, cv_done;
  bool stop = false;
  std::deque<Req*> pending;
  std::vector<Req*> staged;
  std::vector<Batch*> inflight;
  std::vector<cudaEvent_t> events;  // a pool of reusable events
  std::unordered_map<uint64_t, Req*> by_ticket;
  uint64_t next_ticket = 1;
  // statistics
  int64_t completed = 0, samples = 0, launches = 0, batched_reqs = 0, refused = 0, kernels = 0, overlapped = 0;
  std::vector<double> lat;
  double t_first = 0, t_last = 0;
  std::string error;
};

namespace psg {
namespace {
// Arena bytes of a host request: its block, live lengths, window starts
// and (a muting plan) its rows' offsets and t0Ms; none for device buffers.
int64_t req_bytes(const Req& r) {
  if (r.device) return 0;
  return align256(r.rows * (int64_t)r.cols * r.esz) + align256(r.rows * 4) + align256(r.rows * 8) +
         (r.key_off ? 2 * align256(r.rows * 8) : 0);
}

cudaEvent_t get_event(psg_server* S) {
  if (!S->events.empty()) {
    cudaEvent_t e = S->events.back();
    S->events.pop_back();
    return e;
  }
  cudaEvent_t e;
  CUDA_OK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return e;
}
void put_event(psg_server* S, cudaEvent_t e) {
  if (e) S->events.push_back(e);
}

// Moves pending requests to staged: device requests at once; host requests
// when their bytes fit the arena (first come, first served), starting their
// copies in. The copies are issued with the lock released (a copy from
// pageable memory returns only when done), the requests in neither list
// meanwhile (cancel then finds them started).
void admit(psg_server* S, std::unique_lock<std::mutex>& lk) {
  std::vector<Req*> take;
  while (!S->pending.empty()) {
    Req* r = S->pending.front();
    if (r->device) {
      S->pending.pop_front();
      r->d_src = (const char*)r->src;
      r->d_data = (char*)r->dst;
      r->d_live = r->live;
      r->d_start = r->start;
      r->d_off = r->key_off;
      r->d_t0 = r->key_t0;
      S->staged.push_back(r);
      continue;
    }
    int64_t off = S->arena.alloc(r->bytes);
    if (off < 0) break;  // waits for memory to free up (FIFO)
    S->pending.pop_front();
    r->off = off;
    char* base = S->arena_d + off;
    const int64_t db = align256(r->rows * (int64_t)r->cols * r->esz), lb = align256(r->rows * 4),
                  sb = align256(r->rows * 8);
    r->d_src = nullptr;  // applied in place in the arena
    r->d_data = base;
    r->d_live = (const int*)(base + db);
    r->d_start = r->start ? (const double*)(base + db + lb) : nullptr;
    if (r->key_off) {
      r->d_off = (const double*)(base + db + lb + sb);
      r->d_t0 = (const double*)(base + db + lb + 2 * sb);
    }
    r->in = get_event(S);
    take.push_back(r);
  }
  if (take.empty()) return;
  lk.unlock();
  try {
    for (Req* r : take) {
      char* base = r->d_data;
      const int64_t db = align256(r->rows * (int64_t)r->cols * r->esz), lb = align256(r->rows * 4),
                    sb = align256(r->rows * 8);
      CUDA_OK(cudaMemcpyAsync(base, r->src, (size_t)(r->rows * (int64_t)r->cols * r->esz), cudaMemcpyHostToDevice,
                              S->s_in));
      CUDA_OK(cudaMemcpyAsync(base + db, r->live, r->rows * 4, cudaMemcpyHostToDevice, S->s_in));
      if (r->start) CUDA_OK(cudaMemcpyAsync(base + db + lb, r->start, r->rows * 8, cudaMemcpyHostToDevice, S->s_in));
      if (r->key_off) {
        CUDA_OK(cudaMemcpyAsync(base + db + lb + sb, r->key_off, r->rows * 8, cudaMemcpyHostToDevice, S->s_in));
        CUDA_OK(cudaMemcpyAsync(base + db + lb + 2 * sb, r->key_t0, r->rows * 8, cudaMemcpyHostToDevice, S->s_in));
      }
      CUDA_OK(cudaEventRecord(r->in, S->s_in));
    }
  } catch (...) {
    lk.lock();
    for (Req* r : take) S->staged.push_back(r);  // failed with the staged ones
    throw;
  }
  lk.lock();
  for (Req* r : take) S->staged.push_back(r);
}

// A staged request whose input is on the device.
bool ready(psg_server* S, Req* r) {
  if (!r->in) return true;
  if (cudaEventQuery(r->in) != cudaSuccess) return false;
  put_event(S, r->in);
  r->in = nullptr;
  return true;
}

Job job_of(const Req* r) {
  const psg_plan* p = r->plan;
  Job j{};
  j.src = r->d_src;
  j.dst = r->d_data;
  j.live = r->d_live;
  j.start_ms = r->d_start;
  j.steps = p->d_steps;
  j.rows = r->rows;
  j.cols = r->cols;
  j.first = p->host.parts[0].first;
  j.last = p->host.parts[0].second;
  j.dt_ms = r->dt_ms > 0 ? r->dt_ms : p->host.dt_ms;
  return j;
}

// A status from one of this library's entry points as an exception.
void throw_unless_ok(int st) {
  if (st == PSG_EINVAL) throw InvalidArg(t_err);
  if (st != PSG_OK) throw std::runtime_error(t_err);
}

void launch_batch_reqs(psg_server* S, Batch* b);

// One batch on a free slot: every staged request whose input is on the
// device (up to kMaxJobs, in arrival order). The generic rows go in one
// launch, each trace build's rows in one launch, the requests run alone
// after them part by part; then the host requests' copies out.
void launch_batch(psg_server* S, std::unique_lock<std::mutex>& lk) {
  int slot = -1;
  for (int i = 0; i < psg_server::kSlots; i++)
    if (!S->slot_busy[i]) {
      slot = i;
      break;
    }
  if (slot < 0 || S->staged.empty()) return;
  std::unique_ptr<Batch> b(new Batch());
  b->slot = slot;
  for (size_t i = 0; i < S->staged.size() && b->reqs.size() < (size_t)psg_server::kMaxJobs;) {
    Req* r = S->staged[i];
    if (ready(S, r)) {
      b->reqs.push_back(r);
      S->staged.erase(S->staged.begin() + i);
    } else {
      i++;
    }
  }
  if (b->reqs.empty()) return;
  try {
    launch_batch_reqs(S, b.get());
    // the copies out with the lock released (to pageable memory a copy
    // returns only when done); the slot stays taken meanwhile
    S->slot_busy[slot] = true;
    b->done = get_event(S);
    lk.unlock();
    try {
      cudaStream_t so = S->s_out[slot];
      for (Req* r : b->reqs)
        if (!r->device)
          CUDA_OK(cudaMemcpyAsync(r->dst, r->d_data, (size_t)(r->rows * (int64_t)r->cols * r->esz),
                                  cudaMemcpyDeviceToHost, so));
      CUDA_OK(cudaEventRecord(b->done, so));
    } catch (...) {
      lk.lock();
      S->slot_busy[slot] = false;
      throw;
    }
    lk.lock();
  } catch (const std::exception& e) {
    // the batch's requests fail; what was queued for them finishes first,
    // so that their arena memory is free to reuse
    S->error = e.what();
    cudaStreamSynchronize(S->s_comp[slot]);
    cudaStreamSynchronize(S->s_out[slot]);
    cudaGetLastError();
    const int code = dynamic_cast<const InvalidArg*>(&e) ? PSG_EINVAL : PSG_ECUDA;
    for (Req* r : b->reqs) {
      r->status = code;
      r->done = true;
      if (r->off >= 0) S->arena.release(r->off, r->bytes);
      r->off = -1;
    }
    put_event(S, b->kern);
    put_event(S, b->done);
    S->cv_done.notify_all();
    return;
  }
  S->launches++;
  S->batched_reqs += (int64_t)b->reqs.size();
  S->inflight.push_back(b.release());
}

void launch_batch_reqs(psg_server* S, Batch* b) {
  const int slot = b->slot;
  cudaStream_t sc = S->s_comp[slot], so = S->s_out[slot];
  // the launches over many requests' rows: the generic group first, then
  // one group per (trace build, recipe)
  struct Group {
    const TracePlanInfo* tp = nullptr;
    int rc = 0;
    std::vector<Req*> reqs;
  };
  std::vector<Group> groups(1);
  std::vector<Req*> solo;
  for (Req* r : b->reqs) {
    if (r->kind == K_SOLO) {
      solo.push_back(r);
      continue;
    }
    if (r->kind == K_GENERIC) {
      groups[0].reqs.push_back(r);
      continue;
    }
    const int rc = r->plan->trace_recipe[0];
    size_t g = 1;
    while (g < groups.size() && !(groups[g].tp == r->trace && groups[g].rc == rc)) g++;
    if (g == groups.size()) {
      groups.push_back(Group{});
      groups[g].tp = r->trace;
      groups[g].rc = rc;
    }
    groups[g].reqs.push_back(r);
  }
  Job* jh = S->jobs_h + slot * psg_server::kMaxJobs;
  long long* bh = S->begin_h + slot * psg_server::kMaxJobs;
  size_t nj = 0;
  std::vector<size_t> first(groups.size());
  for (size_t g = 0; g < groups.size(); g++) {
    first[g] = nj;
    long long total = 0;
    for (Req* r : groups[g].reqs) {
      jh[nj] = job_of(r);
      bh[nj] = total;
      total += r->rows;
      nj++;
    }
  }
  if (nj) {
    CUDA_OK(cudaMemcpyAsync(S->jobs_d + slot * psg_server::kMaxJobs, jh, nj * sizeof(Job), cudaMemcpyHostToDevice, sc));
    CUDA_OK(cudaMemcpyAsync(S->begin_d + slot * psg_server::kMaxJobs, bh, nj * sizeof(long long),
                            cudaMemcpyHostToDevice, sc));
  }
  for (size_t g = 0; g < groups.size(); g++) {
    const Group& G = groups[g];
    if (G.reqs.empty()) continue;
    PipeArgs a{};
    a.jobs = S->jobs_d + slot * psg_server::kMaxJobs + first[g];
    a.row_begin = S->begin_d + slot * psg_server::kMaxJobs + first[g];
    a.njobs = (int)G.reqs.size();
    a.status = S->status_d;
    long long total = 0;
    int xb = 0;
    size_t work = 0;
    for (Req* r : G.reqs) {
      total += r->rows;
      xb = std::max(xb, r->plan->x_bytes);
      work = std::max(work, r->plan->smem - (size_t)r->plan->work_off);
    }
    a.total_rows = total;
    if (total == 0) continue;
    if (G.tp) {
      // the trace build's batched kernel: one row buffer, its transform buffers
      const void* k = G.tp->batch[G.rc];
      const size_t sm = (size_t)xb + 2 * (size_t)G.tp->buf * 8;
      allow_smem(k);
      int per = 0;
      CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, G.tp->nt, sm));
      if (per <= 0) throw InvalidArg("a batch's traces do not fit the device's shared memory");
      a.x_bytes = xb;
      a.work_off = xb;
      a.tw_pass = G.reqs[0]->plan->trace_cands[0][0].tw;  // the build's table (every plan's holds the same)
      launch_pipe(k, (int)std::min<long long>(total, (long long)per * g_sm_count), G.tp->nt, sm, sc, a);
    } else {
      // one row buffer, or two when the prefetch costs no occupancy
      auto occ = [&](bool pf, size_t& sm) {
        sm = (size_t)((pf ? 2 : 1) * xb) + work;
        auto k = batch_kernel_for(pf);
        allow_smem(k);
        int per = 0;
        CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, kNT, sm));
        return per;
      };
      size_t sm1, sm2;
      int o1 = occ(false, sm1), o2 = occ(true, sm2);
      bool pf = o2 > 0 && o2 >= o1;
      a.x_bytes = xb;
      a.work_off = (pf ? 2 : 1) * xb;
      int per = pf ? o2 : o1;
      if (per <= 0) throw InvalidArg("a batch's traces do not fit the device's shared memory");
      launch_pipe(batch_kernel_for(pf), (int)std::min<long long>(total, (long long)per * g_sm_count), kNT,
                  pf ? sm2 : sm1, sc, a);
    }
    S->kernels++;
  }
  // requests run alone: the plain apply's part-by-part launches, with this
  // slot's workspace for per-panel statistics and long-trace work areas
  for (Req* r : solo) {
    const psg_plan* p = r->plan;
    throw_unless_ok(psg_workspace_reserve(S->ws[slot], p, r->rows, r->cols));
    psg_keys k{};
    k.offset = r->d_off;
    k.t0_ms = r->d_t0;
    k.first_sample = r->first_sample;
    const psg_keys* kp = p->needs_keys ? &k : nullptr;
    for (int part = 0; part < (int)p->host.parts.size(); part++) {
      const void* from = part == 0 ? r->d_src : nullptr;
      if (p->host.dtype == PSG_F32)
        launch_part<float>(p, S->ws[slot], part, from, r->d_data, r->rows, r->cols, r->d_live, r->d_start, sc, kp,
                           r->dt_ms);
      else
        launch_part<double>(p, S->ws[slot], part, from, r->d_data, r->rows, r->cols, r->d_live, r->d_start, sc, kp,
                            r->dt_ms);
      S->kernels++;
    }
  }
  CUDA_OK(cudaGetLastError());
  b->kern = get_event(S);
  CUDA_OK(cudaEventRecord(b->kern, sc));
  CUDA_OK(cudaStreamWaitEvent(so, b->kern, 0));
}

// Retires finished batches: their requests are done and their memory free.
bool retire(psg_server* S) {
  bool any = false;
  for (size_t i = 0; i < S->inflight.size();) {
    Batch* b = S->inflight[i];
    cudaError_t e = cudaEventQuery(b->done);
    if (e == cudaErrorNotReady) {
      i++;
      continue;
    }
    double t = now_s();
    for (Req* r : b->reqs) {
      r->status = e == cudaSuccess ? PSG_OK : PSG_ECUDA;
      r->t_done = t;
      r->done = true;
      if (r->off >= 0) S->arena.release(r->off, r->bytes);
      S->completed++;
      S->samples += r->rows * (int64_t)r->cols;
      S->lat.push_back(t - r->t_submit);
      S->t_last = t;
    }
    put_event(S, b->kern);
    put_event(S, b->done);
    S->slot_busy[b->slot] = false;
    delete b;
    S->inflight.erase(S->inflight.begin() + i);
    any = true;
  }
  return any;
}

// The loop: admits what fits, launches a batch when no batch's kernels are
// running, or, while some are, when the requests ready to run hold enough
// rows to fill the device on their own (a CTA per row on every SM, four
// deep): that batch then runs beside the others on its slot's streams.
// Requests arriving during a batch otherwise join the next one.
void sched_loop(psg_server* S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  const int64_t fill_rows = 4 * (int64_t)g_sm_count;
  while (true) {
    if (S->stop && S->pending.empty() && S->staged.empty() && S->inflight.empty()) break;
    try {
      admit(S, lk);
      int running = 0;
      for (Batch* b : S->inflight) {
        if (!b->kern_done) b->kern_done = cudaEventQuery(b->kern) == cudaSuccess;
        if (!b->kern_done) running++;
      }
      int64_t ready_rows = 0;
      for (Req* r : S->staged)
        if (ready(S, r)) ready_rows += std::max<int64_t>(r->rows, 1);
      if (ready_rows > 0 && (running == 0 || ready_rows >= fill_rows)) {
        if (running > 0) S->overlapped++;
        launch_batch(S, lk);
      }
      if (retire(S)) S->cv_done.notify_all();
    } catch (const std::exception& e) {
      S->error = e.what();
      for (Req* r : S->staged) {
        r->status = PSG_ECUDA;
        r->done = true;
      }
      S->staged.clear();
      S->cv_done.notify_all();
    }
    // idle: sleep until a submit; otherwise poll again within a few
    // microseconds (a finished batch is seen at once), spinning with the lock
    // released so that submitting and waiting threads get it meanwhile
    if (S->inflight.empty() && S->pending.empty() && S->staged.empty())
      S->cv.wait_for(lk, std::chrono::milliseconds(5));
    else {
      lk.unlock();
      const auto until = std::chrono::steady_clock::now() + std::chrono::microseconds(4);
      while (std::chrono::steady_clock::now() < until) std::this_thread::yield();
      lk.lock();
    }
  }
}
}  // namespace
}  // namespace psg

extern "C" {

int psg_server_create(int device, int64_t arena_bytes, psg_server** out) {
  return guarded([&] {
    if (!out) throw InvalidArg("null argument");
    if (arena_bytes < (1 << 20)) throw InvalidArg("the arena needs at least 1 MiB");
    CUDA_OK(cudaSetDevice(device));
    ensure_device();
    std::unique_ptr<psg_server> S(new psg_server());
    S->device = device;
    CUDA_OK(cudaMalloc(&S->arena_d, (size_t)arena_bytes));
    S->arena.init(arena_bytes);
    CUDA_OK(cudaStreamCreateWithFlags(&S->s_in, cudaStreamNonBlocking));
    for (int i = 0; i < psg_server::kSlots; i++) {
      CUDA_OK(cudaStreamCreateWithFlags(&S->s_comp[i], cudaStreamNonBlocking));
      CUDA_OK(cudaStreamCreateWithFlags(&S->s_out[i], cudaStreamNonBlocking));
      throw_unless_ok(psg_workspace_create(&S->ws[i]));
    }
    const int nj = psg_server::kSlots * psg_server::kMaxJobs;
    CUDA_OK(cudaMallocHost(&S->jobs_h, nj * sizeof(Job)));
    CUDA_OK(cudaMallocHost(&S->begin_h, nj * sizeof(long long)));
    CUDA_OK(cudaMalloc(&S->jobs_d, nj * sizeof(Job)));
    CUDA_OK(cudaMalloc(&S->begin_d, nj * sizeof(long long)));
    CUDA_OK(cudaMalloc(&S->status_d, 256));
    CUDA_OK(cudaMemset(S->status_d, 0, 256));
    psg_server* raw = S.release();
    raw->sched = std::thread(sched_loop, raw);
    *out = raw;
  });
}

void psg_server_destroy(psg_server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> g(S->mu);
    S->stop = true;
  }
  S->cv.notify_all();
  if (S->sched.joinable()) S->sched.join();
  for (auto& kv : S->by_ticket) delete kv.second;
  for (cudaEvent_t e : S->events) cudaEventDestroy(e);
  cudaFree(S->arena_d);
  cudaFree(S->jobs_d);
  cudaFree(S->begin_d);
  cudaFree(S->status_d);
  cudaFreeHost(S->jobs_h);
  cudaFreeHost(S->begin_h);
  cudaStreamDestroy(S->s_in);
  for (int i = 0; i < psg_server::kSlots; i++) {
    if (S->s_comp[i]) cudaStreamDestroy(S->s_comp[i]);
    if (S->s_out[i]) cudaStreamDestroy(S->s_out[i]);
    psg_workspace_destroy(S->ws[i]);
  }
  delete S;
}

}  // extern "C"

namespace psg {
namespace {
// Queues a request: host buffers (staged through the arena) or device
// buffers (the kernels read and write them in place), keys for a muting
// plan. Where the plain apply would take a request, so does the loop.
int submit(psg_server* S, const psg_plan* plan, const void* src, void* dst, int64_t rows, int32_t cols,
           const int32_t* live, const double* start_ms, const psg_keys* keys, double dt_ms, bool device,
           void* stream, uint64_t* ticket) {
  return guarded([&] {
    if (!S || !ticket) throw InvalidArg("null argument");
    check_apply(plan, nullptr, src, dst, rows, cols, live, dt_ms, false, keys);
    if (!src) throw InvalidArg("src is required");
    if (plan->needs_keys && (!keys->offset || !keys->t0_ms)) throw InvalidArg("the keys' offset and t0_ms are required");
    std::unique_ptr<Req> r(new Req());
    r->plan = plan;
    r->src = src;
    r->dst = dst;
    r->rows = rows;
    r->cols = cols;
    r->live = live;
    r->start = start_ms;
    r->dt_ms = dt_ms;
    r->esz = plan->host.dtype == PSG_F32 ? 4 : 8;
    r->device = device;
    if (plan->needs_keys) {
      r->key_off = keys->offset;
      r->key_t0 = keys->t0_ms;
      r->first_sample = keys->first_sample;
    }
    // how it runs: as the plain apply would, in a batch where it can
    bool single = plan->host.dtype == PSG_F32 && plan->host.parts.size() == 1 && !part_needs_panel(plan, 0) &&
                  !plan->wide && !plan->needs_keys;
    for (const StepHost& st : plan->host.steps)
      if (st.kind == ST_IIR) single = false;
    r->kind = K_SOLO;
    if (single) {
      const TracePlanInfo* tp = plan->trace.empty() ? nullptr : plan->trace[0];
      if (!tp) {
        r->kind = K_GENERIC;
      } else if (tp->batch[plan->trace_recipe[0]]) {
        r->kind = K_TRACE;
        r->trace = tp;
      }
    }
    r->bytes = req_bytes(*r);
    r->t_submit = now_s();
    std::lock_guard<std::mutex> g(S->mu);
    if (r->bytes > S->arena.size) {
      S->refused++;
      throw NoMemory("admission refused: the request needs " + std::to_string(r->bytes) +
                     " bytes of device memory, the loop holds " + std::to_string(S->arena.size));
    }
    if (device && stream) {
      // the caller's work on the buffers, queued on `stream`, comes first
      r->in = get_event(S);
      CUDA_OK(cudaEventRecord(r->in, (cudaStream_t)stream));
    }
    if (S->completed == 0 && S->by_ticket.empty()) S->t_first = r->t_submit;
    r->ticket = S->next_ticket++;
    *ticket = r->ticket;
    S->by_ticket[r->ticket] = r.get();
    S->pending.push_back(r.release());
    S->cv.notify_all();
  });
}
}  // namespace
}  // namespace psg

extern "C" {

int psg_submit(psg_server* S, const psg_plan* plan, const void* src_host, void* dst_host, int64_t rows, int32_t cols,
               const int32_t* live_host, const double* start_ms_host, double dt_ms, uint64_t* ticket) {
  return submit(S, plan, src_host, dst_host, rows, cols, live_host, start_ms_host, nullptr, dt_ms, false, nullptr,
                ticket);
}

int psg_submit_keyed(psg_server* S, const psg_plan* plan, const void* src_host, void* dst_host, int64_t rows,
                     int32_t cols, const int32_t* live_host, const double* start_ms_host, const psg_keys* keys_host,
                     double dt_ms, uint64_t* ticket) {
  return submit(S, plan, src_host, dst_host, rows, cols, live_host, start_ms_host, keys_host, dt_ms, false, nullptr,
                ticket);
}

int psg_submit_device(psg_server* S, const psg_plan* plan, const void* src, void* dst, int64_t rows, int32_t cols,
                      const int32_t* live, const double* start_ms, const psg_keys* keys, double dt_ms, void* stream,
                      uint64_t* ticket) {
  return submit(S, plan, src, dst, rows, cols, live, start_ms, keys, dt_ms, true, stream, ticket);
}

// A ticket has one waiter: the thread that waits claims the request under
// the lock, a second thread that waits on the same ticket meanwhile gets
// PSG_EINVAL, and only the claiming thread erases and frees it (after a
// timeout the claim is dropped and the ticket can be waited on again). A
// timeout that is not finite, or longer than about 30 years, waits until the
// request finishes; a negative one polls once.
int psg_wait(psg_server* S, uint64_t ticket, double timeout_ms) { return psg_wait_done(S, ticket, timeout_ms, nullptr); }

int psg_wait_done(psg_server* S, uint64_t ticket, double timeout_ms, double* done_s) {
  if (!S) {
    t_err = "null argument";
    return PSG_EINVAL;
  }
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->by_ticket.find(ticket);
  if (it == S->by_ticket.end()) {
    t_err = "unknown ticket " + std::to_string(ticket);
    return PSG_EINVAL;
  }
  Req* r = it->second;
  if (r->claimed) {
    t_err = "another thread is waiting on ticket " + std::to_string(ticket);
    return PSG_EINVAL;
  }
  r->claimed = true;
  const bool forever = !(timeout_ms <= 1e12);  // NaN, +Inf and huge values
  const double ms = forever ? 0.0 : std::max(timeout_ms, 0.0);
  auto deadline = std::chrono::steady_clock::now() + std::chrono::microseconds((int64_t)(ms * 1000));
  while (!r->done) {
    if (forever) {
      S->cv_done.wait(lk);
    } else if (S->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !r->done) {
      r->claimed = false;
      t_err = "the request did not finish within " + std::to_string(timeout_ms) + " ms";
      return PSG_ETIMEOUT;
    }
  }
  int st = r->status;
  if (done_s) *done_s = r->t_done;
  S->by_ticket.erase(ticket);
  delete r;
  if (st == PSG_ECANCELED) t_err = "the request was cancelled";
  else if (st != PSG_OK) t_err = S->error.empty() ? "a CUDA call of the request loop failed" : S->error;
  return st;
}

int psg_poll(psg_server* S, uint64_t ticket, int32_t* done) {
  if (!S || !done) {
    t_err = "null argument";
    return PSG_EINVAL;
  }
  std::lock_guard<std::mutex> g(S->mu);
  auto it = S->by_ticket.find(ticket);
  if (it == S->by_ticket.end()) {
    t_err = "unknown ticket " + std::to_string(ticket);
    return PSG_EINVAL;
  }
  *done = it->second->done ? 1 : 0;
  return PSG_OK;
}

int psg_cancel(psg_server* S, uint64_t ticket) {
  if (!S) {
    t_err = "null argument";
    return PSG_EINVAL;
  }
  std::lock_guard<std::mutex> g(S->mu);
  auto it = S->by_ticket.find(ticket);
  if (it == S->by_ticket.end()) {
    t_err = "unknown ticket " + std::to_string(ticket);
    return PSG_EINVAL;
  }
  Req* r = it->second;
  auto q = std::find(S->pending.begin(), S->pending.end(), r);
  if (q == S->pending.end()) {
    t_err = r->done ? "the request has finished" : "the request has started: wait for it";
    return PSG_EINVAL;
  }
  S->pending.erase(q);
  put_event(S, r->in);  // a device request's wait on its caller's stream
  r->in = nullptr;
  r->done = true;
  r->status = PSG_ECANCELED;
  S->cv_done.notify_all();
  return PSG_OK;
}

int psg_server_load(psg_server* S, int64_t* out2) {
  if (!S || !out2) {
    t_err = "null argument";
    return PSG_EINVAL;
  }
  std::lock_guard<std::mutex> g(S->mu);
  int64_t n = 0, samples = 0;
  auto add = [&](const Req* r) {
    n++;
    samples += r->rows * (int64_t)r->cols;
  };
  for (const Req* r : S->pending) add(r);
  for (const Req* r : S->staged) add(r);
  for (const Batch* b : S->inflight)
    for (const Req* r : b->reqs) add(r);
  out2[0] = n;
  out2[1] = samples;
  return PSG_OK;
}

int psg_server_counters(psg_server* S, int64_t* out4) {
  if (!S || !out4) {
    t_err = "null argument";
    return PSG_EINVAL;
  }
  std::lock_guard<std::mutex> g(S->mu);
  out4[0] = S->launches;
  out4[1] = S->kernels;
  out4[2] = S->overlapped;
  out4[3] = S->completed;
  return PSG_OK;
}

// {completed, samples, launches, mean requests per launch, p50 s, p99 s,
//  Msamples/s over the first submit to the last completion, refused}
int psg_server_stats(psg_server* S, double* out8, int reset) {
  if (!S || !out8) {
    t_err = "null argument";
    return PSG_EINVAL;
  }
  std::lock_guard<std::mutex> g(S->mu);
  std::vector<double> l = S->lat;
  std::sort(l.begin(), l.end());
  auto q = [&](double f) { return l.empty() ? 0.0 : l[std::min(l.size() - 1, (size_t)(f * (l.size() - 1) + 0.5))]; };
  out8[0] = (double)S->completed;
  out8[1] = (double)S->samples;
  out8[2] = (double)S->launches;
  out8[3] = S->launches ? (double)S->batched_reqs / (double)S->launches : 0.0;
  out8[4] = q(0.50);
  out8[5] = q(0.99);
  out8[6] = S->t_last > S->t_first ? (double)S->samples / (S->t_last - S->t_first) / 1e6 : 0.0;
  out8[7] = (double)S->refused;
  if (reset) {
    S->completed = S->samples = S->launches = S->batched_reqs = S->refused = 0;
    S->lat.clear();
    S->t_first = S->t_last = 0;
  }
  return PSG_OK;
}

}  // extern "C"
