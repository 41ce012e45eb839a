// psg_oracle.cpp — TEST INFRASTRUCTURE ONLY. The CPU oracle for processSEG's
// compiled-pipeline hot path: a plain C++ restatement of the reference's Nim
// algorithms (xrfez/processSEG v0.14.1), in float32 and float64, used by the
// tests as the checker and by bench.py's CPU-baseline leg. Nothing in the
// product library links, loads or calls this file.
//
// Parity status: the reference is Nim and no Nim toolchain exists here, so it
// cannot be compiled or run; its dependency parseSEG is not vendored either.
// This restatement is pinned by the reference's own known-answer tests and
// tolerances (tests/tfftplan.nim, tgain.nim, tfilterapply.nim,
// tfilterdesign.nim, tpipeline.nim, tcorrelate.nim), re-run against it in
// tests/test_oracle_pins.py. There are no golden vectors for this path in the
// reference (its noise comes from Nim's std/random, which is not portable).
//
// Each function cites the reference file:line it restates.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <complex>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../include/psg.h"

namespace orc {

static const double PI = 3.14159265358979323846;
static const double INF = std::numeric_limits<double>::infinity();
static const double NaN = std::numeric_limits<double>::quiet_NaN();

struct ValueError : std::runtime_error {
  explicit ValueError(const std::string& m) : std::runtime_error(m) {}
};

static std::string fmt(double v) {
  char b[64];
  snprintf(b, sizeof b, "%g", v);
  return b;
}

// ------------------------------------------------------------------ sums --
// core/sums.nim:12-23
template <class T> double sum64(const T* x, int64_t n) {
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int64_t m = n / 8 * 8;
  for (int64_t i = 0; i < m; i += 8)
    for (int j = 0; j < 8; j++) acc[j] += (double)x[i + j];
  double r = 0;
  for (int j = 0; j < 8; j++) r += acc[j];
  for (int64_t k = m; k < n; k++) r += (double)x[k];
  return r;
}
// core/sums.nim:25-40
template <class T> double sumIndexed64(const T* x, int64_t n) {
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0}, idx[8];
  for (int j = 0; j < 8; j++) idx[j] = j;
  int64_t m = n / 8 * 8;
  for (int64_t i = 0; i < m; i += 8)
    for (int j = 0; j < 8; j++) {
      acc[j] += idx[j] * (double)x[i + j];
      idx[j] += 8;
    }
  double r = 0;
  for (int j = 0; j < 8; j++) r += acc[j];
  for (int64_t k = m; k < n; k++) r += (double)k * (double)x[k];
  return r;
}
// gain/stats.nim:82-95
template <class T> double sumSq64(const T* x, int64_t n) {
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int64_t m = n / 8 * 8;
  for (int64_t i = 0; i < m; i += 8)
    for (int j = 0; j < 8; j++) {
      double v = (double)x[i + j];
      acc[j] += v * v;
    }
  double r = 0;
  for (int j = 0; j < 8; j++) r += acc[j];
  for (int64_t k = m; k < n; k++) r += (double)x[k] * (double)x[k];
  return r;
}
// gain/stats.nim:97-117: the integer maximum of the bits with the sign cleared
static double maxAbs(const float* x, int64_t n) {
  int32_t m = 0;
  for (int64_t i = 0; i < n; i++) {
    int32_t b;
    std::memcpy(&b, &x[i], 4);
    b &= 0x7FFFFFFF;
    m = b > m ? b : m;
  }
  float f;
  std::memcpy(&f, &m, 4);
  return (double)f;
}
static double maxAbs(const double* x, int64_t n) {
  int64_t m = 0;
  for (int64_t i = 0; i < n; i++) {
    int64_t b;
    std::memcpy(&b, &x[i], 8);
    b &= 0x7FFFFFFFFFFFFFFFLL;
    m = b > m ? b : m;
  }
  double f;
  std::memcpy(&f, &m, 8);
  return f;
}

static bool isFin(double x) { return std::isfinite(x); }
// gain/gain.nim:112-118
static bool finitePositive(double x) {
  int c = std::fpclassify(x);
  return (c == FP_NORMAL || c == FP_SUBNORMAL) && x > 0;
}
template <class T> bool fitsIn(double x) {
  return finitePositive(x) && finitePositive((double)(T)x);
}

// ------------------------------------------------------------------- FFT --
// fft/plan.nim:105-118
bool isFastLen(int64_t n) {
  if (n < 1) return false;
  int64_t k = n;
  for (int p : {2, 3, 5})
    while (k % p == 0) k /= p;
  return k == 1;
}
int64_t nextFastLen(int64_t n, bool even = true) {
  int64_t r = std::max<int64_t>(n, 1);
  while (!isFastLen(r) || (even && r % 2 == 1)) r++;
  return r;
}
// fft/plan.nim:120-132: 4s first, then a 2, 3s and 5s
static std::vector<int> factorize(int64_t n) {
  std::vector<int> r;
  int64_t k = n;
  while (k % 4 == 0) { r.push_back(4); k /= 4; }
  if (k % 2 == 0) { r.push_back(2); k /= 2; }
  for (int p : {3, 5})
    while (k % p == 0) { r.push_back(p); k /= p; }
  return r;
}

template <class T> struct FftPlan {
  int64_t n = 0, m = 0;
  std::vector<int> radices;
  std::vector<T> twRe, twIm, splitRe, splitIm;
  int64_t bins() const { return n / 2 + 1; }
};

// fft/plan.nim:136-160: twiddles computed in float64, stored as T
template <class T> FftPlan<T> initFftPlan(int64_t n) {
  if (!isFastLen(n))
    throw ValueError("an FFT length must be >= 1 with prime factors 2, 3 and 5 only, got " +
                     std::to_string(n));
  FftPlan<T> p;
  p.n = n;
  p.m = n % 2 == 0 ? n / 2 : n;
  p.radices = factorize(p.m);
  int64_t cur = p.m;
  for (int r : p.radices) {
    int64_t sub = cur / r;
    for (int64_t q = 0; q < sub; q++)
      for (int k = 1; k < r; k++) {
        double a = -2 * PI * (double)((q * k) % cur) / (double)cur;
        p.twRe.push_back((T)std::cos(a));
        p.twIm.push_back((T)std::sin(a));
      }
    cur = sub;
  }
  if (n % 2 == 0)
    for (int64_t k = 0; k <= p.m; k++) {
      double a = -2 * PI * (double)k / (double)n;
      p.splitRe.push_back((T)std::cos(a));
      p.splitIm.push_back((T)std::sin(a));
    }
  return p;
}

// fft/plan.nim:203-206
#define MULTW(yr, yi, wr, wi) \
  {                            \
    T t_ = yr * wr - yi * wi;  \
    yi = yr * wi + yi * wr;    \
    yr = t_;                   \
  }

// One Stockham DIF stage, fft/plan.nim:187-190 and the bfly/pass procs
// :225-417, with one lane: y[q + s·(r·p + k)] = (Σ_j x[q + s·(p + j·sub)]
// ω_r^{jk})·ω_cur^{pk}.
template <class T>
static void stage(int r, const T* xr, const T* xi, T* yr, T* yi, const T* tr, const T* ti,
                  int64_t sub, int64_t w) {
  for (int64_t p = 0; p < sub; p++) {
    int64_t a = p * w, b = (int64_t)r * p * w, o = sub * w, t = (int64_t)(r - 1) * p;
    for (int64_t i = 0; i < w; i++) {
      if (r == 2) {
        T ur = xr[a + i], ui = xi[a + i], vr = xr[a + o + i], vi = xi[a + o + i];
        yr[b + i] = ur + vr;
        yi[b + i] = ui + vi;
        T dr = ur - vr, di = ui - vi;
        MULTW(dr, di, tr[t], ti[t]);
        yr[b + w + i] = dr;
        yi[b + w + i] = di;
      } else if (r == 3) {
        const T c = (T)-0.5, s = (T)0.8660254037844386467637231707529362;
        T ar = xr[a + i], ai = xi[a + i];
        T t1r = xr[a + o + i] + xr[a + 2 * o + i], t1i = xi[a + o + i] + xi[a + 2 * o + i];
        T t2r = xr[a + o + i] - xr[a + 2 * o + i], t2i = xi[a + o + i] - xi[a + 2 * o + i];
        T m1r = ar + c * t1r, m1i = ai + c * t1i;
        T m2r = s * t2i, m2i = -s * t2r;
        yr[b + i] = ar + t1r;
        yi[b + i] = ai + t1i;
        T u1r = m1r + m2r, u1i = m1i + m2i, u2r = m1r - m2r, u2i = m1i - m2i;
        MULTW(u1r, u1i, tr[t], ti[t]);
        MULTW(u2r, u2i, tr[t + 1], ti[t + 1]);
        yr[b + w + i] = u1r;
        yi[b + w + i] = u1i;
        yr[b + 2 * w + i] = u2r;
        yi[b + 2 * w + i] = u2i;
      } else if (r == 4) {
        const T* x0r = xr + a; const T* x0i = xi + a;
        const T* x1r = xr + a + o; const T* x1i = xi + a + o;
        const T* x2r = xr + a + 2 * o; const T* x2i = xi + a + 2 * o;
        const T* x3r = xr + a + 3 * o; const T* x3i = xi + a + 3 * o;
        T t0r = x0r[i] + x2r[i], t0i = x0i[i] + x2i[i];
        T t1r = x0r[i] - x2r[i], t1i = x0i[i] - x2i[i];
        T t2r = x1r[i] + x3r[i], t2i = x1i[i] + x3i[i];
        T t3r = x1i[i] - x3i[i], t3i = x3r[i] - x1r[i];
        yr[b + i] = t0r + t2r;
        yi[b + i] = t0i + t2i;
        T u1r = t1r + t3r, u1i = t1i + t3i, u2r = t0r - t2r, u2i = t0i - t2i;
        T u3r = t1r - t3r, u3i = t1i - t3i;
        MULTW(u1r, u1i, tr[t], ti[t]);
        MULTW(u2r, u2i, tr[t + 1], ti[t + 1]);
        MULTW(u3r, u3i, tr[t + 2], ti[t + 2]);
        yr[b + w + i] = u1r; yi[b + w + i] = u1i;
        yr[b + 2 * w + i] = u2r; yi[b + 2 * w + i] = u2i;
        yr[b + 3 * w + i] = u3r; yi[b + 3 * w + i] = u3i;
      } else {  // 5
        const T c1 = (T)0.3090169943749474241022934171828191;
        const T c2 = (T)-0.8090169943749474241022934171828191;
        const T s1 = (T)0.9510565162951535721164393333793821;
        const T s2 = (T)0.5877852522924731291687059546390728;
        T ar = xr[a + i], ai = xi[a + i];
        T x1r = xr[a + o + i], x1i = xi[a + o + i], x2r = xr[a + 2 * o + i], x2i = xi[a + 2 * o + i];
        T x3r = xr[a + 3 * o + i], x3i = xi[a + 3 * o + i], x4r = xr[a + 4 * o + i], x4i = xi[a + 4 * o + i];
        T t1r = x1r + x4r, t1i = x1i + x4i, t2r = x2r + x3r, t2i = x2i + x3i;
        T t3r = x1r - x4r, t3i = x1i - x4i, t4r = x2r - x3r, t4i = x2i - x3i;
        T b1r = ar + c1 * t1r + c2 * t2r, b1i = ai + c1 * t1i + c2 * t2i;
        T b2r = ar + c2 * t1r + c1 * t2r, b2i = ai + c2 * t1i + c1 * t2i;
        T d1r = s1 * t3r + s2 * t4r, d1i = s1 * t3i + s2 * t4i;
        T d2r = s2 * t3r - s1 * t4r, d2i = s2 * t3i - s1 * t4i;
        yr[b + i] = ar + t1r + t2r;
        yi[b + i] = ai + t1i + t2i;
        T u1r = b1r + d1i, u1i = b1i - d1r, u4r = b1r - d1i, u4i = b1i + d1r;
        T u2r = b2r + d2i, u2i = b2i - d2r, u3r = b2r - d2i, u3i = b2i + d2r;
        MULTW(u1r, u1i, tr[t], ti[t]);
        MULTW(u2r, u2i, tr[t + 1], ti[t + 1]);
        MULTW(u3r, u3i, tr[t + 2], ti[t + 2]);
        MULTW(u4r, u4i, tr[t + 3], ti[t + 3]);
        yr[b + w + i] = u1r; yi[b + w + i] = u1i;
        yr[b + 2 * w + i] = u2r; yi[b + 2 * w + i] = u2i;
        yr[b + 3 * w + i] = u3r; yi[b + 3 * w + i] = u3i;
        yr[b + 4 * w + i] = u4r; yi[b + 4 * w + i] = u4i;
      }
    }
  }
}

// fft/plan.nim:421-450. Returns true when the result ended in (br, bi).
template <class T> bool complexForward(const FftPlan<T>& p, T* ar, T* ai, T* br, T* bi) {
  T *xr = ar, *xi = ai, *yr = br, *yi = bi;
  int64_t cur = p.m, s = 1, at = 0;
  for (int r : p.radices) {
    int64_t sub = cur / r;
    stage<T>(r, xr, xi, yr, yi, p.twRe.data() + at, p.twIm.data() + at, sub, s);
    at += sub * (r - 1);
    cur = sub;
    s *= r;
    std::swap(xr, yr);
    std::swap(xi, yi);
  }
  return xr == br;
}

// fft/plan.nim:501-542 (one lane)
template <class T> void fftForward(const FftPlan<T>& p, const T* x, T* re, T* im) {
  int64_t m = p.m;
  std::vector<T> ar(m), ai(m), br(m), bi(m);
  if (p.n % 2 == 1) {
    for (int64_t i = 0; i < m; i++) { ar[i] = x[i]; ai[i] = 0; }
  } else {
    for (int64_t k = 0; k < m; k++) { ar[k] = x[2 * k]; ai[k] = x[2 * k + 1]; }
  }
  bool inB = complexForward(p, ar.data(), ai.data(), br.data(), bi.data());
  const T* zr = inB ? br.data() : ar.data();
  const T* zi = inB ? bi.data() : ai.data();
  if (p.n % 2 == 1) {
    for (int64_t k = 0; k < p.bins(); k++) { re[k] = zr[k]; im[k] = zi[k]; }
    return;
  }
  T r0 = zr[0], i0 = zi[0];
  re[0] = r0 + i0; im[0] = 0;
  re[m] = r0 - i0; im[m] = 0;
  for (int64_t k = 1; k < m; k++) {
    // splitForward, fft/plan.nim:470-482
    T a_r = zr[k], a_i = zi[k], b_r = zr[m - k], b_i = zi[m - k];
    T wr = p.splitRe[k], wi = p.splitIm[k];
    T er = (T)0.5 * (a_r + b_r), ei = (T)0.5 * (a_i - b_i);
    T orr = (T)0.5 * (a_i + b_i), oi = (T)0.5 * (b_r - a_r);
    re[k] = er + wr * orr - wi * oi;
    im[k] = ei + wr * oi + wi * orr;
  }
}

// fft/plan.nim:544-595 (one lane)
template <class T> void fftInverse(const FftPlan<T>& p, const T* re, const T* im, T* x) {
  int64_t m = p.m;
  std::vector<T> ar(m), ai(m), br(m), bi(m);
  T scale = (T)1 / (T)p.n;
  if (p.n % 2 == 1) {
    ai[0] = re[0] * scale;
    ar[0] = 0;
    for (int64_t k = 1; k < p.bins(); k++) {
      T vr = re[k] * scale, vi = im[k] * scale;
      ai[k] = vr; ar[k] = vi;
      ai[m - k] = vr; ar[m - k] = -vi;
    }
  } else {
    T x0 = re[0], xm = re[m];
    ai[0] = (x0 + xm) * scale;
    ar[0] = (x0 - xm) * scale;
    for (int64_t k = 1; k < m; k++) {
      // splitInverse, fft/plan.nim:484-499
      T a_r = re[k], a_i = im[k], b_r = re[m - k], b_i = im[m - k];
      T wr = p.splitRe[k], wi = -p.splitIm[k];
      T er = a_r + b_r, ei = a_i - b_i, dr = a_r - b_r, di = a_i + b_i;
      T orr = dr * wr - di * wi, oi = dr * wi + di * wr;
      ai[k] = (er - oi) * scale;
      ar[k] = (ei + orr) * scale;
    }
  }
  bool inB = complexForward(p, ar.data(), ai.data(), br.data(), bi.data());
  const T* zr = inB ? bi.data() : ai.data();
  const T* zi = inB ? br.data() : ar.data();
  if (p.n % 2 == 1) {
    for (int64_t i = 0; i < m; i++) x[i] = zr[i];
  } else {
    for (int64_t k = 0; k < m; k++) { x[2 * k] = zr[k]; x[2 * k + 1] = zi[k]; }
  }
}

// ---------------------------------------------------------------- design --
// filter/design.nim:78-91, as the C-ABI's psg_filter_spec.
typedef psg_filter_spec Spec;
static bool hasLow(const Spec& s) { return s.f2 > 0; }
static bool hasHigh(const Spec& s) { return s.f3 < INF; }

// filter/design.nim:103-137
static void checkCorners(const Spec& c) {
  for (double f : {c.f1, c.f2, c.f3, c.f4})
    if (std::isnan(f)) throw ValueError("a corner is NaN");
  if (hasLow(c) && !(c.f1 >= 0 && c.f1 < c.f2))
    throw ValueError("a low cut needs 0 <= f1 < f2 (a sloped ramp)");
  if (!hasLow(c) && (c.f1 != 0 || c.f2 != 0)) throw ValueError("no low cut needs f1 = f2 = 0");
  if (hasHigh(c) && !(c.f3 < c.f4 && c.f4 < INF))
    throw ValueError("a high cut needs f3 < f4 < Inf (a sloped ramp)");
  if (!hasHigh(c) && c.f4 != INF) throw ValueError("no high cut needs f3 = f4 = Inf");
  if (hasLow(c) && hasHigh(c) && !(c.f2 <= c.f3)) throw ValueError("a band-pass needs f2 <= f3");
}
static void checkSlope(double s) {
  if (!(s > 0 && s < INF)) throw ValueError("a slope must be finite and > 0 dB/octave");
}
static void checkButter(double lowHz, double lowSlope, double highHz, double highSlope) {
  if (!(lowHz >= 0 && lowHz < INF)) throw ValueError("a low-cut corner must be finite and >= 0");
  if (!(highHz > 0)) throw ValueError("a high-cut corner must be > 0");
  if (lowHz > 0) checkSlope(lowSlope);
  if (highHz < INF) checkSlope(highSlope);
  if (!(lowHz < highHz)) throw ValueError("the low-cut corner must be below the high-cut one");
}
static void checkNotch(const psg_notch& n) {
  if (!(n.freq_hz > 0 && n.freq_hz < INF)) throw ValueError("a notch frequency must be finite and > 0");
  if (!(n.width_hz > 0 && n.width_hz < INF)) throw ValueError("a notch width must be finite and > 0");
}
// filter/design.nim:143-173
void validate(const Spec& spec, double dtMs) {
  if (!(dtMs > 0 && dtMs < INF)) throw ValueError("dtMs must be finite and > 0");
  double nyq = 500 / dtMs;
  if (spec.kind == PSG_RK_TRAPEZOID) {
    checkCorners(spec);
    if (hasHigh(spec) && spec.f4 > nyq) throw ValueError("f4 = " + fmt(spec.f4) + " Hz is above Nyquist");
    if (hasLow(spec) && spec.f2 >= nyq) throw ValueError("f2 is not below Nyquist");
  } else {
    checkButter(spec.low_hz, spec.low_slope, spec.high_hz, spec.high_slope);
    if (spec.high_hz < INF && spec.high_hz >= nyq) throw ValueError("the high-cut corner is not below Nyquist");
    if (spec.low_hz >= nyq) throw ValueError("the low-cut corner is not below Nyquist");
  }
  if (spec.n_notches < 0 || spec.n_notches > PSG_MAX_NOTCHES) throw ValueError("bad notch count");
  for (int i = 0; i < spec.n_notches; i++) {
    checkNotch(spec.notches[i]);
    if (spec.notches[i].freq_hz >= nyq) throw ValueError("a notch is not below Nyquist");
  }
}
// filter/design.nim:227-234
static double warp(double f, double dtMs) {
  double x = PI * f * dtMs / 1000;
  return x >= PI / 2 ? INF : std::tan(x);
}
static double ramp(double x) {
  if (x <= 0) return 0.0;
  if (x >= 1) return 1.0;
  double s = std::sin(PI / 2 * x);
  return s * s;
}
// filter/design.nim:236-255
double response(const Spec& spec, double f, double dtMs) {
  double r = 1.0;
  if (spec.kind == PSG_RK_TRAPEZOID) {
    if (hasLow(spec)) r *= ramp((f - spec.f1) / (spec.f2 - spec.f1));
    if (hasHigh(spec)) r *= 1 - ramp((f - spec.f3) / (spec.f4 - spec.f3));
  } else {
    double wf = warp(f, dtMs);
    if (spec.low_hz > 0)
      r *= (f <= 0 ? 0.0 : 1 / (1 + std::pow(warp(spec.low_hz, dtMs) / wf, spec.low_slope / 6)));
    if (spec.high_hz < INF)
      r *= (wf == INF ? 0.0 : 1 / (1 + std::pow(wf / warp(spec.high_hz, dtMs), spec.high_slope / 6)));
  }
  for (int i = 0; i < spec.n_notches; i++)
    r *= ramp(std::fabs(f - spec.notches[i].freq_hz) / (spec.notches[i].width_hz / 2));
  return r;
}
// filter/design.nim:257-265
template <class T> void responseInto(const Spec& spec, double dtMs, int64_t nfft, T* h) {
  int64_t bins = nfft / 2 + 1;
  double df = 1000 / ((double)nfft * dtMs);
  for (int64_t k = 0; k < bins; k++) h[k] = (T)response(spec, (double)k * df, dtMs);
  if (spec.zero_dc && bins > 0) h[0] = 0;
}
// filter/design.nim:267-282
double narrowestRampHz(const Spec& spec) {
  double r = INF;
  if (spec.kind == PSG_RK_TRAPEZOID) {
    if (hasLow(spec)) r = std::min(r, spec.f2 - spec.f1);
    if (hasHigh(spec)) r = std::min(r, spec.f4 - spec.f3);
  } else {
    if (spec.low_hz > 0) r = std::min(r, spec.low_hz * std::min(1.0, 24 / spec.low_slope) / 2);
    if (spec.high_hz < INF) r = std::min(r, spec.high_hz * std::min(1.0, 24 / spec.high_slope) / 2);
  }
  for (int i = 0; i < spec.n_notches; i++) r = std::min(r, spec.notches[i].width_hz / 2);
  return r;
}
// filter/design.nim:288-298
static int64_t energyLength(const std::vector<double>& h, double centre) {
  int64_t n = (int64_t)h.size();
  double total = centre * centre;
  for (int64_t j = 1; j < n; j++) total += h[j] * h[j];
  double e = centre * centre;
  int64_t r = 0;
  while (e < 0.999 * total && r < n / 2) {
    r++;
    e += h[r] * h[r] + (n - r != r ? h[n - r] * h[n - r] : 0.0);
  }
  return r;
}
static const int64_t maxImpulseGrid = 1 << 24;
// filter/design.nim:300-325
static int64_t featureLength(const Spec& spec, double dtMs) {
  double feature = narrowestRampHz(spec);
  if (feature == INF) return 0;
  double fs = 1000 / dtMs;
  double start = std::ceil(16 * fs / feature);
  int64_t n = start > (double)maxImpulseGrid ? maxImpulseGrid + 1
                                             : nextFastLen(std::max<int64_t>(64, (int64_t)start));
  while (true) {
    if (n > maxImpulseGrid)
      throw ValueError("the filter's impulse response is longer than " +
                       std::to_string(maxImpulseGrid / 8) + " samples");
    FftPlan<double> p = initFftPlan<double>(n);
    std::vector<double> re(p.bins()), im(p.bins(), 0.0), h(n);
    responseInto(spec, dtMs, n, re.data());
    fftInverse(p, re.data(), im.data(), h.data());
    int64_t L = std::max(energyLength(h, h[0]), energyLength(h, 1 - h[0]));
    if (L <= n / 8) return L;
    n = nextFastLen(2 * n);
  }
}
// filter/design.nim:327-351
static std::vector<Spec> features(const Spec& spec) {
  std::vector<Spec> r;
  Spec flat{};
  flat.kind = PSG_RK_TRAPEZOID;
  flat.f1 = 0; flat.f2 = 0; flat.f3 = INF; flat.f4 = INF;
  if (spec.kind == PSG_RK_TRAPEZOID) {
    if (hasLow(spec)) {
      Spec s = flat; s.f1 = spec.f1; s.f2 = spec.f2;
      r.push_back(s);
    }
    if (hasHigh(spec)) {
      Spec s = flat; s.f3 = spec.f3; s.f4 = spec.f4;
      r.push_back(s);
    }
  } else {
    if (spec.low_hz > 0) {
      Spec s{}; s.kind = PSG_RK_BUTTERWORTH;
      s.low_hz = spec.low_hz; s.low_slope = spec.low_slope; s.high_hz = INF; s.high_slope = spec.high_slope;
      r.push_back(s);
    }
    if (spec.high_hz < INF) {
      Spec s{}; s.kind = PSG_RK_BUTTERWORTH;
      s.low_hz = 0; s.low_slope = spec.low_slope; s.high_hz = spec.high_hz; s.high_slope = spec.high_slope;
      r.push_back(s);
    }
  }
  for (int i = 0; i < spec.n_notches; i++) {
    Spec s = flat;
    s.n_notches = 1;
    s.notches[0] = spec.notches[i];
    r.push_back(s);
  }
  return r;
}
// filter/design.nim:353-366
int64_t impulseLength(const Spec& spec, double dtMs) {
  validate(spec, dtMs);
  int64_t r = 0;
  for (const Spec& f : features(spec)) r = std::max(r, featureLength(f, dtMs));
  return r;
}

// ------------------------------------------------------------ filter/apply --
// filter/edges.nim:16-30
template <class T> void trendOf(int trend, const T* x, int64_t n, double& a, double& b) {
  if (trend == PSG_TR_NONE) { a = 0; b = 0; return; }
  if (trend == PSG_TR_MEAN) { a = sum64(x, n) / (double)n; b = 0; return; }
  double sx = sum64(x, n), nf = (double)n, mean = sx / nf;
  if (n == 1) { a = mean; b = 0; return; }
  double c = (nf - 1) / 2;
  double slope = (sumIndexed64(x, n) - c * sx) / (nf * (nf * nf - 1) / 12);
  a = mean - slope * c;
  b = slope;
}

template <class T> struct FilterPlan {
  Spec spec;
  FftPlan<T> fft;
  std::vector<T> gain, fall;
  int64_t pad = 0, margin = 0, samples = 0;
  bool reflect = false;
  double dtMs = 0, dcGain = 0;
  int trend = PSG_TR_LINEAR;
};

// filter/apply.nim:118-151
template <class T> FilterPlan<T> initFilterPlan(const Spec& spec, double dtMs, int64_t samples, int trend) {
  if (samples < 1) throw ValueError("a filter plan needs samples >= 1, got " + std::to_string(samples));
  validate(spec, dtMs);
  int64_t margin = impulseLength(spec, dtMs);
  double dcGain = response(spec, 0, dtMs);
  bool reflect = dcGain >= 0.5 || trend != PSG_TR_LINEAR;
  int64_t pad = reflect ? margin : std::min(margin, samples);
  int64_t n = samples + (reflect ? 4 : 2) * pad;
  double rmp = narrowestRampHz(spec);
  if (rmp < INF && pad == margin) n = std::max(n, (int64_t)std::ceil(2000 / (rmp * dtMs)));
  n = nextFastLen(n);
  FilterPlan<T> p;
  p.spec = spec;
  p.fft = initFftPlan<T>(n);
  p.gain.resize(p.fft.bins());
  responseInto(spec, dtMs, n, p.gain.data());
  p.fall.resize(pad);
  for (int64_t k = 1; k <= pad; k++) {
    double c = std::cos(PI / 2 * (double)k / (double)(pad + 1));
    p.fall[k - 1] = (T)(c * c);
  }
  p.pad = pad;
  p.margin = margin;
  p.samples = samples;
  p.dtMs = dtMs;
  p.dcGain = dcGain;
  p.trend = trend;
  p.reflect = reflect;
  return p;
}

// filter/apply.nim:194-216
template <class T> void packInto(const FilterPlan<T>& plan, const T* x, int64_t n, double a, double b, T* dst) {
  int64_t p = plan.pad;
  for (int64_t i = 0; i < n; i++) dst[p + i] = (T)((double)x[i] - (a + b * (double)i));
  if (plan.reflect) {
    T d0 = dst[p], dn = dst[p + n - 1];
    for (int64_t k = 1; k <= p; k++) {
      T r = dst[p + std::min(k, n - 1)];
      dst[p - k] = (d0 + d0 - r) * plan.fall[k - 1];
    }
    for (int64_t k = 1; k <= p; k++) {
      T r = dst[p + n - 1 - std::min(k, n - 1)];
      dst[p + n - 1 + k] = (dn + dn - r) * plan.fall[k - 1];
    }
  } else {
    for (int64_t k = 1; k <= p; k++) {
      dst[p - k] = 0;
      dst[p + n - 1 + k] = 0;
    }
  }
  for (int64_t j = 2 * p + n; j < plan.fft.n; j++) dst[j] = 0;
}
// filter/apply.nim:218-231
template <class T> void unpackFrom(const FilterPlan<T>& plan, const T* src, double a, double b, T* x, int64_t n) {
  int64_t p = plan.pad;
  double gb = b * plan.dcGain;
  double ga = plan.spec.zero_dc ? -gb * (double)(n - 1) / 2 : a * plan.dcGain;
  if (ga == 0 && gb == 0) {
    for (int64_t i = 0; i < n; i++) x[i] = src[p + i];
  } else {
    for (int64_t i = 0; i < n; i++) x[i] = (T)((double)src[p + i] + (ga + gb * (double)i));
  }
}
// filter/apply.nim:340-363 (one trace; the lanes forms compute the same
// expression per sample, filter/apply.nim:255-260)
template <class T> void applyFilter(const FilterPlan<T>& plan, T* x, int64_t n) {
  if (n == 0) return;
  int64_t nf = plan.fft.n, nb = plan.fft.bins();
  std::vector<T> buf(nf), re(nb), im(nb);
  double a, b;
  trendOf(plan.trend, x, n, a, b);
  packInto(plan, x, n, a, b, buf.data());
  fftForward(plan.fft, buf.data(), re.data(), im.data());
  for (int64_t k = 0; k < nb; k++) {  // gainRun, filter/apply.nim:234-247
    re[k] = re[k] * plan.gain[k];
    im[k] = im[k] * plan.gain[k];
  }
  fftInverse(plan.fft, re.data(), im.data(), buf.data());
  unpackFrom(plan, buf.data(), a, b, x, n);
}

// ----------------------------------------------------------------- basic --
// core/basic.nim:52-110
template <class T> void demean(T* x, int64_t n) {
  if (n == 0) return;
  T m = (T)(sum64(x, n) / (double)n);
  for (int64_t i = 0; i < n; i++) x[i] = x[i] - m;
}
template <class T> void detrend(T* x, int64_t n) {
  if (n == 0) return;
  double nf = (double)n, c = (nf - 1) / 2, sx = sum64(x, n), mean = sx / nf;
  double stt = nf * (nf * nf - 1) / 12;
  double slope = n > 1 ? (sumIndexed64(x, n) - c * sx) / stt : 0.0;
  T a = (T)(mean - slope * c), b = (T)slope;
  for (int32_t i = 0; i < (int32_t)n; i++) x[i] = x[i] - (a + b * (T)i);
}
template <class T> void scale(T* x, int64_t n, double factor) {
  T k = (T)factor;
  for (int64_t i = 0; i < n; i++) x[i] = x[i] * k;
}
template <class T> void clip(T* x, int64_t n, double lo, double hi) {
  T l = (T)lo, h = (T)hi;
  for (int64_t i = 0; i < n; i++) {
    T v = x[i];
    x[i] = v > h ? h : (v < l ? l : v);
  }
}
template <class T> void polarity(T* x, int64_t n) {
  for (int64_t i = 0; i < n; i++) x[i] = -x[i];
}

// ------------------------------------------------------------------ stats --
struct TraceStats { double rms = 0, maxAbs = 0; };
// gain/stats.nim:124-133
template <class T> TraceStats traceStats(const T* x, int64_t n) {
  TraceStats s;
  if (n == 0) return s;
  double sum = sumSq64(x, n), mx = maxAbs(x, n);
  s.rms = std::sqrt(sum / (double)n);
  s.maxAbs = mx;
  return s;
}
// gain/stats.nim:135-157
static void selectK(double* a, int64_t lo0, int64_t hi0, int64_t k) {
  int64_t lo = lo0, hi = hi0;
  while (hi > lo) {
    int64_t mid = (lo + hi) >> 1;
    if (a[mid] < a[lo]) std::swap(a[mid], a[lo]);
    if (a[hi] < a[lo]) std::swap(a[hi], a[lo]);
    if (a[hi] < a[mid]) std::swap(a[hi], a[mid]);
    double pivot = a[mid];
    int64_t i = lo, j = hi;
    while (i <= j) {
      while (a[i] < pivot) i++;
      while (a[j] > pivot) j--;
      if (i <= j) {
        std::swap(a[i], a[j]);
        i++;
        j--;
      }
    }
    if (k <= j) hi = j;
    else if (k >= i) lo = i;
    else return;
  }
}
// gain/stats.nim:159-182
template <class T> double percentileAbs(const T* x, int64_t n, double p) {
  if (n == 0) return 0;
  if (std::isnan(maxAbs(x, n))) return NaN;
  std::vector<double> a(n);
  for (int64_t i = 0; i < n; i++) a[i] = std::fabs((double)x[i]);
  double h = (double)(n - 1) * p / 100;
  int64_t k = std::min((int64_t)std::floor(h), n - 1);
  selectK(a.data(), 0, n - 1, k);
  double lower = a[k];
  if (k + 1 >= n) return lower;
  double upper = INF;
  for (int64_t i = k + 1; i < n; i++) upper = std::min(upper, a[i]);
  double f = h - (double)k;
  return f == 0 ? lower : lower + f * (upper - lower);
}

static const int histBins = 65536, histShift = 15, maxKey = 0xFEFF;
// gain/stats.nim:208-213
static int keyOf(float a) {
  uint32_t b;
  std::memcpy(&b, &a, 4);
  return std::min((int)(b >> histShift), maxKey);
}
static double binLow(int k) {
  uint32_t b = (uint32_t)k << histShift;
  float f;
  std::memcpy(&f, &b, 4);
  return (double)f;
}
// gain/stats.nim:237-251
static double orderStat(const std::vector<uint32_t>& h, int64_t j, double mx) {
  int64_t below = 0;
  for (int k = 0; k <= maxKey; k++) {
    int64_t c = h[k];
    if (below + c > j) {
      if (k == 0) return 0;
      double lo = binLow(k), hi = std::min(binLow(k + 1), mx);
      return std::min(std::max(lo + ((double)(j - below) + 0.5) / (double)c * (hi - lo), lo), mx);
    }
    below += c;
  }
  return mx;
}
struct PanelStats { double rms = 0, maxAbs = 0, clip = NaN; int64_t rows = 0, samples = 0; };
// gain/stats.nim:253-304 (the four interleaved ways fold to one histogram)
// signedLive: live[i] < 0 marks a row that is not live and live[i] == 0 a
// live row with no samples (isLive true, liveSamples 0), which the reference
// counts: sumSqMaxAbs of nothing is (0, 0) and usable (:267-276). Otherwise
// (the pipeline's flattening) live[i] == 0 is a row that is not processed.
template <class T>
PanelStats panelStats(const T* b, int64_t rows, int64_t cols, const int32_t* live, double clipP,
                      bool signedLive = false) {
  PanelStats r;
  double sum = 0, mx = 0;
  std::vector<char> use(rows, 0);
  for (int64_t i = 0; i < rows; i++) {
    if (signedLive ? live[i] < 0 : live[i] <= 0) continue;
    int64_t n = std::min<int64_t>(live[i], cols);
    double s = sumSq64(b + i * cols, n), m = maxAbs(b + i * cols, n);
    if (std::isnan(m) || std::isinf(m) || s == INF) continue;  // usable, :232-235
    use[i] = 1;
    sum += s;
    mx = std::max(mx, m);
    r.samples += n;
    r.rows++;
  }
  r.clip = NaN;
  if (r.samples == 0) return r;
  r.rms = std::sqrt(sum / (double)r.samples);
  r.maxAbs = mx;
  if (std::isnan(clipP)) return r;
  if (clipP == 100) { r.clip = mx; return r; }
  std::vector<uint32_t> h(histBins, 0);
  for (int64_t i = 0; i < rows; i++) {
    if (!use[i]) continue;
    const T* x = b + i * cols;
    for (int64_t j = 0; j < std::min<int64_t>(live[i], cols); j++) h[keyOf((float)std::fabs((double)x[j]))]++;
  }
  double rank = (double)(r.samples - 1) * clipP / 100;
  int64_t k = std::min((int64_t)std::floor(rank), r.samples - 1);
  double lower = orderStat(h, k, mx);
  double f = rank - (double)k;
  r.clip = (f == 0 || k + 1 >= r.samples) ? lower : lower + f * (orderStat(h, k + 1, mx) - lower);
  return r;
}

// traceStatsInto (gain/stats.nim:186-199) with statsOf (:124-127) and
// traceStats (:129-133): per row, NaN for a row that is not live
// (live[r] < 0), (0, 0) for a live row without samples, else the RMS and
// max |x| of its first live[r] samples (sumSq64's eight accumulators).
template <class T>
void traceStatsInto(const T* b, int64_t rows, int64_t cols, const int32_t* live, double* rms, double* mxo) {
  for (int64_t r = 0; r < rows; r++) {
    if (live[r] < 0) {
      rms[r] = NaN;
      mxo[r] = NaN;
      continue;
    }
    int64_t n = std::min<int64_t>(live[r], cols);
    if (n == 0) {
      rms[r] = 0;
      mxo[r] = 0;
      continue;
    }
    rms[r] = std::sqrt(sumSq64(b + r * cols, n) / (double)n);
    mxo[r] = maxAbs(b + r * cols, n);
  }
}

// ------------------------------------------------------------------- AGC --
struct AgcPlan {
  int mode = 0;
  int64_t half = 0, samples = 0;
  double dtMs = 0, target = 1, epsilon = 1e-9;
  std::vector<double> inv, rev;
};
// gain/gain.nim:272-302
AgcPlan initAgcPlan(double windowMs, double dtMs, int64_t samples, int mode, double target, double epsilon) {
  if (!finitePositive(dtMs)) throw ValueError("dtMs must be finite and positive, got " + fmt(dtMs));
  if (samples < 1 || samples > 2147483647LL)
    throw ValueError("an AGC plan needs samples in 1 .. int32.high, got " + std::to_string(samples));
  if (!finitePositive(windowMs))
    throw ValueError("an AGC window must be finite and positive, got " + fmt(windowMs) + " ms");
  double h = std::round(windowMs / (2 * dtMs));
  if (h < 1) throw ValueError("an AGC window of " + fmt(windowMs) + " ms is under 3 samples");
  if (h > (double)(1 << 26)) throw ValueError("an AGC window is too long");
  if (!finitePositive(target)) throw ValueError("an AGC target must be finite and positive");
  if (!finitePositive(epsilon)) throw ValueError("an AGC epsilon must be finite and positive");
  AgcPlan p;
  p.mode = mode;
  p.half = (int64_t)h;
  p.samples = samples;
  p.dtMs = dtMs;
  p.target = target;
  p.epsilon = epsilon;
  p.inv.assign(2 * p.half + 2, 0.0);
  for (size_t c = 1; c < p.inv.size(); c++) p.inv[c] = 1 / (double)c;
  p.rev.assign(2 * p.half + 1, 0.0);
  for (size_t m = 0; m < p.rev.size(); m++) p.rev[m] = 1 / (double)(2 * p.half + 1 - (int64_t)m);
  return p;
}
// gain/gain.nim:351-390: per block of w, s[i] the suffix sum to the block's
// end, p[e] the prefix sum from the block's start to e − 1 (0 at a start).
template <class T> static void blockSums(const T* x, int64_t n, int64_t w, int mode, double* s, double* p) {
  auto term = [mode](double v) { return mode == PSG_AGC_RMS ? v * v : std::fabs(v); };
  int64_t bs = 0;
  while (bs < n) {
    int64_t be = std::min(bs + w, n);
    double fwd = 0, bwd = 0;
    p[bs] = 0;
    for (int64_t k = 0; k < be - bs; k++) {
      fwd += term((double)x[bs + k]);
      p[bs + k + 1] = fwd;
      bwd += term((double)x[be - 1 - k]);
      s[be - 1 - k] = bwd;
    }
    bs = be;
  }
  if (n % w == 0) p[n] = 0;
}
// gain/gain.nim:392-461
template <class T> void agc(const AgcPlan& plan, T* x, int64_t n) {
  if (n == 0) return;
  double rms = traceStats(x, n).rms;
  if (rms == 0) return;
  int64_t h = plan.half, w = 2 * h + 1;
  std::vector<double> s(n + 1), p(n + 1);
  blockSums(x, n, w, plan.mode, s.data(), p.data());
  if (!fitsIn<T>(plan.target / rms / plan.epsilon)) return;
  bool rmsMode = plan.mode == PSG_AGC_RMS;
  double unit = rmsMode ? 1 / (rms * rms) : 1 / rms;
  T k = (T)(plan.target / rms), eps = (T)plan.epsilon;
  int64_t first = std::min(h, n), last = std::max(first, n - h);
  int64_t headCut = std::clamp(n - h, (int64_t)0, first);
  int64_t lastBlock = (n - 1) / w * w;
  int64_t tailCut = std::clamp(lastBlock + h, last, n);
  double pn = p[n];
  const double* inv = plan.inv.data();
  const double* rev = plan.rev.data();
  double unitW = unit / (double)w;
  double headWhole = headCut < first ? pn * unit * inv[n] : 0.0;
  auto step = [&](int64_t i, double meanOf) {
    T lv = rmsMode ? (T)std::sqrt((T)meanOf) : (T)meanOf;
    T gi = k / (lv + eps);
    x[i] = (T)(x[i] * (T)gi);
  };
  for (int64_t i = 0; i < headCut; i++) step(i, p[i + h + 1] * (unit * inv[i + h + 1]));
  for (int64_t i = headCut; i < first; i++) step(i, headWhole);
  for (int64_t i = first; i < last; i++) step(i, (s[i - h] + p[i + h + 1]) * unitW);
  for (int64_t i = last; i < tailCut; i++) step(i, (s[i - h] + pn) * (unit * rev[i + h + 1 - n]));
  for (int64_t i = tailCut; i < n; i++) step(i, s[i - h] * (unit * rev[i + h + 1 - n]));
}

// ------------------------------------------------------------- normalize --
struct NormPlan { int stat = 0, scope = 0; double target = 1, percentile = 99; int64_t samples = 0; };
// gain/gain.nim:153-167
NormPlan initNormalizePlan(int stat, int64_t samples, int scope, double target, double percentile) {
  if (samples < 1) throw ValueError("a normalize plan needs samples >= 1, got " + std::to_string(samples));
  if (!finitePositive(target)) throw ValueError("a normalize target must be finite and positive");
  if (!(percentile >= 0 && percentile <= 100)) throw ValueError("a percentile must be in 0 .. 100");
  NormPlan p;
  p.stat = stat; p.scope = scope; p.target = target; p.percentile = percentile; p.samples = samples;
  return p;
}
// gain/gain.nim:198-219
template <class T> void normalizeTrace(const NormPlan& plan, T* x, int64_t n) {
  double level;
  if (plan.stat == PSG_NORM_MAX) level = traceStats(x, n).maxAbs;
  else if (plan.stat == PSG_NORM_RMS) level = traceStats(x, n).rms;
  else level = percentileAbs(x, n, plan.percentile);
  if (finitePositive(level) && fitsIn<T>(plan.target / level)) scale(x, n, plan.target / level);
}
// gain/gain.nim:221-240
template <class T>
double panelFactor(const NormPlan& plan, const T* b, int64_t rows, int64_t cols, const int32_t* live) {
  double clipP = plan.stat == PSG_NORM_PERCENTILE ? plan.percentile : NaN;
  PanelStats s = panelStats(b, rows, cols, live, clipP);
  double level = plan.stat == PSG_NORM_MAX ? s.maxAbs : (plan.stat == PSG_NORM_RMS ? s.rms : s.clip);
  if (finitePositive(level) && fitsIn<T>(plan.target / level)) return plan.target / level;
  return NaN;
}

// ----------------------------------------------------------- gain curves --
typedef psg_gain_curve Curve;
// gain/curves.nim:132-152
double gainDbAt(const Curve& c, double tMs) {
  if (std::isnan(tMs)) return NaN;
  if (c.kind == PSG_GC_KNOTS && c.n_knots == 0) return NaN;
  if (c.kind == PSG_GC_KNOTS) {
    const psg_gain_knot* k = c.knots;
    int n = c.n_knots;
    if (tMs <= k[0].t_ms) return k[0].db;
    if (tMs >= k[n - 1].t_ms) return k[n - 1].db;
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (k[mid].t_ms <= tMs) lo = mid; else hi = mid;
    }
    double f = (tMs - k[lo].t_ms) / (k[hi].t_ms - k[lo].t_ms);
    return k[lo].db + f * (k[hi].db - k[lo].db);
  }
  if (c.kind == PSG_GC_POWER) return 20 * c.power * std::log10(std::max(tMs, c.min_ms) / c.ref_ms);
  return c.db_per_s * tMs / 1000;
}
// gain/curves.nim:154-160
double factorAt(const Curve& c, double tMs) {
  if (std::isnan(tMs)) return NaN;
  if (c.kind == PSG_GC_POWER) return std::pow(std::max(tMs, c.min_ms) / c.ref_ms, c.power);
  return std::pow(10.0, gainDbAt(c, tMs) / 20);
}
// gain/curves.nim:97-126 (builder checks)
static void checkCurve(const Curve& c) {
  if (c.kind == PSG_GC_KNOTS) {
    if (c.n_knots < 1 || c.n_knots > PSG_MAX_KNOTS) throw ValueError("a knot gain needs at least one knot");
    for (int i = 0; i < c.n_knots; i++) {
      if (!(isFin(c.knots[i].t_ms) && isFin(c.knots[i].db))) throw ValueError("a knot is not finite");
      if (i > 0 && !(c.knots[i].t_ms > c.knots[i - 1].t_ms)) throw ValueError("knot times must strictly increase");
    }
  } else if (c.kind == PSG_GC_POWER) {
    if (!isFin(c.power)) throw ValueError("a power must be finite");
    if (!(isFin(c.ref_ms) && c.ref_ms > 0)) throw ValueError("refMs must be finite and positive");
    if (!(isFin(c.min_ms) && c.min_ms > 0)) throw ValueError("minMs must be finite and positive");
  } else if (c.kind == PSG_GC_EXPONENTIAL) {
    if (!isFin(c.db_per_s)) throw ValueError("dbPerS must be finite");
  } else {
    throw ValueError("unknown gain curve kind");
  }
}
template <class T> struct CurvePlan {
  Curve curve;
  std::vector<T> table;
  double dtMs = 0, tMinMs = 0;
  int64_t samples = 0;
};
// gain/curves.nim:214-247
template <class T>
CurvePlan<T> initGainCurvePlan(const Curve& curve, double dtMs, int64_t samples, double tMinMs, double tMaxMs) {
  if (!(isFin(dtMs) && dtMs > 0)) throw ValueError("dtMs must be finite and positive");
  if (samples < 1) throw ValueError("a gain curve plan needs samples >= 1");
  checkCurve(curve);
  double hiMs = std::isnan(tMaxMs) ? tMinMs + (double)(samples - 1) * dtMs : tMaxMs;
  if (!(isFin(tMinMs) && isFin(hiMs))) throw ValueError("the table limits must be finite");
  if (hiMs < tMinMs) throw ValueError("tMaxMs is before tMinMs");
  double span = std::floor((hiMs - tMinMs) / dtMs + 1e-9);
  if (span >= (double)(1 << 26)) throw ValueError("a gain table is too long");
  int64_t len = (int64_t)span + 1;
  CurvePlan<T> p;
  p.curve = curve;
  p.dtMs = dtMs;
  p.tMinMs = tMinMs;
  p.samples = samples;
  p.table.resize(len);
  for (int64_t k = 0; k < len; k++) {
    double t = tMinMs + (double)k * dtMs;
    double g = factorAt(curve, t);
    p.table[k] = (T)g;
    if (std::isinf((double)p.table[k]) || std::isnan(g))
      throw ValueError("the gain at " + fmt(t) + " ms overflows");
  }
  return p;
}
struct TableSpan { int64_t s = 0, j0 = 0, j1 = 0; double f = 0; bool onGrid = false; };
// gain/curves.nim:316-329
template <class T> TableSpan spanOf(const CurvePlan<T>& plan, int64_t n, double startMs) {
  TableSpan r;
  double u = (startMs - plan.tMinMs) / plan.dtMs;
  if (!isFin(u) || std::fabs(u) > 1e15) { r.j0 = n; r.j1 = n; return r; }
  double rr = std::round(u);
  r.onGrid = std::fabs(u - rr) <= 1e-9 * std::max(1.0, std::fabs(u));
  r.s = (int64_t)(r.onGrid ? rr : std::floor(u));
  r.f = u - (double)r.s;
  int64_t last = (int64_t)plan.table.size() - (r.onGrid ? 1 : 2);
  r.j0 = std::clamp(-r.s, (int64_t)0, n);
  r.j1 = std::clamp(last - r.s + 1, r.j0, n);
  return r;
}
// gain/curves.nim:282-306, 331-337, and the workspace form :383-418
template <class T> void applyGainCurve(const CurvePlan<T>& plan, T* x, int64_t n, double startMs, int64_t cols) {
  if (n == 0 || std::isnan(startMs)) return;
  TableSpan sp = spanOf(plan, n, startMs);
  if (sp.j0 > 0 || sp.j1 < n) {
    std::vector<T> fac(cols);
    TableSpan full = spanOf(plan, cols, startMs);
    for (int64_t j = 0; j < full.j0; j++) fac[j] = (T)factorAt(plan.curve, startMs + (double)j * plan.dtMs);
    for (int64_t j = full.j1; j < cols; j++) fac[j] = (T)factorAt(plan.curve, startMs + (double)j * plan.dtMs);
    for (int64_t j = 0; j < sp.j0; j++) { T v = x[j]; x[j] = v == 0 ? v : v * fac[j]; }
    for (int64_t j = sp.j1; j < n; j++) { T v = x[j]; x[j] = v == 0 ? v : v * fac[j]; }
  }
  if (sp.j1 > sp.j0) {
    const T* tab = plan.table.data() + sp.s + sp.j0;
    T* xs = x + sp.j0;
    int64_t m = sp.j1 - sp.j0;
    if (sp.onGrid) {
      for (int64_t j = 0; j < m; j++) xs[j] = xs[j] * tab[j];
    } else {
      T f = (T)sp.f;
      for (int64_t j = 0; j < m; j++) {
        T a = tab[j];
        xs[j] = xs[j] * (a + f * (tab[j + 1] - a));
      }
    }
  }
}

// ---------------------------------------------------------- fft/spectrum --
template <class T> struct SpectrumPlan {
  FftPlan<T> fft;
  std::vector<T> taper;
  double taperSum = 0, dtMs = 0;
  bool demean = true;
};
// initSpectrumPlan, fft/spectrum.nim:79-107
template <class T> SpectrumPlan<T> initSpectrumPlan(double dtMs, int64_t windowLen, double taperFraction, int64_t nfft,
                                                   bool demean) {
  if (windowLen < 1) throw ValueError("a spectrum window needs >= 1 sample, got " + std::to_string(windowLen));
  if (!(dtMs > 0 && dtMs < INF)) throw ValueError("dtMs must be finite and > 0");
  if (!(taperFraction >= 0 && taperFraction <= 0.5)) throw ValueError("taperFraction must be in 0 .. 0.5");
  int64_t n = nfft;
  if (n == 0) {
    n = 1;
    while (n < windowLen) n <<= 1;
  }
  if (n < windowLen) throw ValueError("nfft is shorter than the window");
  SpectrumPlan<T> sp;
  sp.fft = initFftPlan<T>(n);
  sp.dtMs = dtMs;
  sp.demean = demean;
  sp.taper.resize(windowLen);
  int64_t ramp = (int64_t)std::round(taperFraction * (double)windowLen);
  for (int64_t i = 0; i < windowLen; i++) {
    int64_t d = std::min(i, windowLen - 1 - i);
    double w = 1.0;
    if (d < ramp) {
      double sv = std::sin(PI / 2 * (double)(d + 1) / (double)(ramp + 1));
      w = sv * sv;
    }
    sp.taper[i] = (T)w;
    sp.taperSum += (double)sp.taper[i];
  }
  return sp;
}
// windowInto, fft/spectrum.nim:261-281: returns Σw, NaN for a non-finite window
template <class T> double windowInto(const SpectrumPlan<T>& sp, const T* x, int64_t len, T* dst) {
  int64_t n = std::min<int64_t>(len, (int64_t)sp.taper.size());
  double sum = n > 0 ? sum64(x, n) : 0.0;
  bool finite = sum - sum == 0;
  T m = (sp.demean && n > 0 && finite) ? (T)(sum / (double)n) : (T)0;
  double sw = 0;
  if (n == (int64_t)sp.taper.size()) {
    for (int64_t j = 0; j < n; j++) dst[j] = (x[j] - m) * sp.taper[j];
    sw = sp.taperSum;
  } else {
    for (int64_t j = 0; j < n; j++) {
      T w = std::min(sp.taper[j], sp.taper[n - 1 - j]);
      dst[j] = (x[j] - m) * w;
      sw += (double)w;
    }
  }
  for (int64_t j = n; j < sp.fft.n; j++) dst[j] = (T)0;
  return finite ? sw : NaN;
}
template <class T> double sides(const SpectrumPlan<T>& sp, int64_t k) { return (k == 0 || 2 * k == sp.fft.n) ? 1.0 : 2.0; }
// amplitudeInto, fft/spectrum.nim:283-300
template <class T> void amplitudeInto(const SpectrumPlan<T>& sp, const T* x, int64_t len, T* amp, T* phase) {
  int64_t nb = sp.fft.bins();
  std::vector<T> xw(sp.fft.n), re(nb), im(nb);
  double sw = windowInto(sp, x, len, xw.data());
  fftForward(sp.fft, xw.data(), re.data(), im.data());
  for (int64_t k = 0; k < nb; k++) {
    amp[k] = (T)(std::hypot((double)re[k], (double)im[k]) * sides(sp, k) / sw);
    phase[k] = (T)std::atan2((double)im[k], (double)re[k]);
  }
}
// averageAmplitudeInto, fft/spectrum.nim:302-416 (rows in order, one at a time)
template <class T> int64_t averageAmplitude(const SpectrumPlan<T>& sp, const T* b, int64_t rows, int64_t cols,
                                            const int32_t* live, int64_t firstCol, int64_t r0, int64_t r1, double* amp) {
  int64_t nb = sp.fft.bins();
  std::vector<double> acc(nb, 0.0);
  std::vector<T> xw(sp.fft.n), re(nb), im(nb);
  int64_t used = 0;
  for (int64_t r = std::max<int64_t>(r0, 0); r <= std::min(r1, rows - 1); r++) {
    int64_t lv = std::min<int64_t>(std::max<int32_t>(live[r], 0), cols);
    if (lv <= firstCol) continue;
    int64_t last = std::min<int64_t>(lv, firstCol + (int64_t)sp.taper.size());
    double sw = windowInto(sp, b + r * cols + firstCol, last - firstCol, xw.data());
    if (!(sw > 0)) continue;
    fftForward(sp.fft, xw.data(), re.data(), im.data());
    double scale = 1 / (sw * sw);
    for (int64_t k = 0; k < nb; k++) {
      double rr = (double)re[k], ii = (double)im[k];
      acc[k] += (rr * rr + ii * ii) * scale;
    }
    used++;
  }
  for (int64_t k = 0; k < nb; k++) amp[k] = used > 0 ? std::sqrt(acc[k] / (double)used) * sides(sp, k) : 0.0;
  return used;
}

// ------------------------------------------------------------- filter/iir --
// A biquad, a0 = 1, with its 0 Hz gain (filter/iir.nim:82-111).
struct Sos {
  double b0, b1, b2, a1, a2, g;
};
static Sos mkSos(double b0, double b1, double b2, double a1, double a2) {
  return Sos{b0, b1, b2, a1, a2, (b0 + b1 + b2) / (1 + a1 + a2)};
}
// Complex division as Nim's std/complex `/` (Smith's method).
static void cdivNim(double xr, double xi, double yr, double yi, double& r_re, double& r_im) {
  double r, den;
  if (std::fabs(yr) < std::fabs(yi)) {
    r = yr / yi;
    den = yi + r * yr;
    r_re = (xr * r + xi) / den;
    r_im = (xi * r - xr) / den;
  } else {
    r = yi / yr;
    den = yr + r * yi;
    r_re = (xr + r * xi) / den;
    r_im = (xi - r * xr) / den;
  }
}
// butterSections, filter/iir.nim:113-148
static std::vector<Sos> butterSections(double fc, double dtMs, int order, bool high) {
  std::vector<Sos> res;
  double fs = 1000 / dtMs;
  double wc = 2 * fs * std::tan(PI * fc / fs);
  double k2 = 2 * fs;
  for (int k = 0; k < order / 2; k++) {
    double th = PI * (double)(2 * k + 1) / (double)(2 * order);
    double sr = -wc * std::sin(th), si = wc * std::cos(th);
    double zr, zi;
    cdivNim(k2 + sr, 0.0 + si, k2 - sr, 0.0 - si, zr, zi);
    double a1 = -2 * zr, a2 = zr * zr + zi * zi;
    if (high) {
      double g = (1 - a1 + a2) / 4;
      res.push_back(mkSos(g, -2 * g, g, a1, a2));
    } else {
      double g = (1 + a1 + a2) / 4;
      res.push_back(mkSos(g, 2 * g, g, a1, a2));
    }
  }
  if (order % 2 == 1) {
    double z = (k2 - wc) / (k2 + wc);
    double a1 = -z;
    if (high) {
      double g = (1 - a1) / 2;
      res.push_back(mkSos(g, -g, 0, a1, 0));
    } else {
      double g = (1 + a1) / 2;
      res.push_back(mkSos(g, g, 0, a1, 0));
    }
  }
  return res;
}
// causalLength, filter/iir.nim:150-182
static int64_t causalLength(const std::vector<Sos>& sections) {
  int64_t n = 1024;
  while (true) {
    std::vector<double> h(n, 0.0);
    h[0] = 1;
    for (const Sos& c : sections) {
      double s1 = 0, s2 = 0;
      for (int64_t j = 0; j < n; j++) {
        double x = h[j];
        double y = c.b0 * x + s1;
        s1 = c.b1 * x - c.a1 * y + s2;
        s2 = c.b2 * x - c.a2 * y;
        h[j] = y;
      }
    }
    double rest = 0, tail = 0;
    for (int64_t j = 1; j < n; j++) {
      rest += h[j] * h[j];
      if (j >= n - n / 4) tail += h[j] * h[j];
    }
    if (tail <= 1e-12 * std::max(rest, 1e-300) || n >= (int64_t(1) << 24)) {
      int64_t result = 0;
      for (double c0 : {h[0], 1 - h[0]}) {
        double total = c0 * c0 + rest, e = c0 * c0;
        int64_t L = 0;
        while (e < 0.9999 * total && L < n - 1) {
          L++;
          e += h[L] * h[L];
        }
        result = std::max(result, L);
      }
      return result;
    }
    n *= 2;
  }
}
static int iirPoles(double slope, double perPole, const char* side) {
  double n = slope / perPole;
  if (!(n >= 1 && n <= 32 && n == std::round(n)))
    throw ValueError(std::string("the ") + side + " slope of an IIR filter must be a multiple of " + fmt(perPole) +
                     " dB/octave, 1 .. 32 poles; got " + fmt(slope));
  return (int)n;
}
struct IirPlan {
  Spec spec;
  std::vector<Sos> sections;
  int phase = PSG_IP_ZERO, trend = PSG_TR_LINEAR;
  int64_t pad = 0, lead = 0, tail = 0, samples = 0;
  bool reflect = false;
  double dtMs = 0, dcGain = 1, dcSlope = 0;
};
// initIirPlan, filter/iir.nim:193-239
static IirPlan initIirPlan(const Spec& spec, double dtMs, int64_t samples, int phase, int trend) {
  if (samples < 1) throw ValueError("an IIR plan needs samples >= 1, got " + std::to_string(samples));
  validate(spec, dtMs);
  if (spec.kind != PSG_RK_BUTTERWORTH) throw ValueError("an IIR filter needs a Butterworth spec");
  if (spec.n_notches > 0 || spec.zero_dc) throw ValueError("an IIR filter takes no notches and no 0 Hz suppression");
  double perPole = phase == PSG_IP_ZERO ? 12.0 : 6.0;
  std::vector<Sos> lowSecs, highSecs;
  if (spec.low_hz > 0) lowSecs = butterSections(spec.low_hz, dtMs, iirPoles(spec.low_slope, perPole, "low-cut"), true);
  if (spec.high_hz < INF)
    highSecs = butterSections(spec.high_hz, dtMs, iirPoles(spec.high_slope, perPole, "high-cut"), false);
  IirPlan p;
  p.sections = lowSecs;
  p.sections.insert(p.sections.end(), highSecs.begin(), highSecs.end());
  p.spec = spec;
  p.phase = phase;
  p.pad = phase == PSG_IP_ZERO ? impulseLength(spec, dtMs) : std::max(causalLength(lowSecs), causalLength(highSecs));
  p.samples = samples;
  p.dtMs = dtMs;
  double g = 1.0, dg = 0.0;
  for (const Sos& c : p.sections) {
    double n1 = c.b0 + c.b1 + c.b2, d1 = 1 + c.a1 + c.a2;
    double gi = n1 / d1;
    double dgi = ((c.b1 + 2 * c.b2) * d1 - n1 * (c.a1 + 2 * c.a2)) / (d1 * d1);
    dg = dg * gi + g * dgi;
    g *= gi;
  }
  p.dcGain = phase == PSG_IP_ZERO ? g * g : g;
  p.dcSlope = phase == PSG_IP_ZERO ? 0.0 : dg;
  p.trend = trend;
  p.reflect = std::fabs(p.dcGain) >= 0.5 || trend != PSG_TR_LINEAR;
  p.lead = p.reflect ? p.pad : 0;
  p.tail = phase == PSG_IP_ZERO ? p.pad : 0;
  return p;
}
// sosKernel for one trace, filter/iir.nim:303-351: from rest or from the
// steady state of the first input, the state flushed to 0 below 1e-250
// every 256 steps.
static void sosSingle(double* buf, int64_t m, const Sos& c, bool steady, bool backward) {
  double s1 = 0, s2 = 0;
  if (steady && m > 0) {
    double u = buf[backward ? m - 1 : 0];
    double y = c.g * u;
    s2 = c.b2 * u - c.a2 * y;
    s1 = y - c.b0 * u;
  }
  int64_t done = 0;
  while (done < m) {
    int64_t run = std::min<int64_t>(256, m - done);
    for (int64_t k = 0; k < run; k++) {
      int64_t j = backward ? m - 1 - done - k : done + k;
      double x = buf[j];
      double y = c.b0 * x + s1;
      s1 = c.b1 * x - c.a1 * y + s2;
      s2 = c.b2 * x - c.a2 * y;
      buf[j] = y;
    }
    s1 = std::fabs(s1) < 1e-250 ? 0.0 : s1;
    s2 = std::fabs(s2) < 1e-250 ? 0.0 : s2;
    done += run;
  }
}
// applyFilter on one trace, filter/iir.nim:363-433 (packInto, runSingle, unpackFrom)
template <class T> void applyIir(const IirPlan& plan, T* x, int64_t n) {
  if (n <= 0) return;
  int64_t p = plan.lead, m = plan.lead + n + plan.tail;
  std::vector<double> buf(m, 0.0);
  double a, b;
  trendOf(plan.trend, x, n, a, b);
  for (int64_t i = 0; i < n; i++) buf[p + i] = (double)x[i] - (a + b * (double)i);
  if (plan.reflect) {
    double d0 = buf[p];
    for (int64_t k = 1; k <= p; k++) buf[p - k] = 2 * d0 - buf[p + std::min(k, n - 1)];
    double dn = buf[p + n - 1];
    for (int64_t k = 1; k <= plan.tail; k++) buf[p + n - 1 + k] = 2 * dn - buf[p + n - 1 - std::min(k, n - 1)];
  } else {
    for (int64_t k = 1; k <= plan.tail; k++) buf[p + n - 1 + k] = 0;
  }
  for (const Sos& c : plan.sections) sosSingle(buf.data(), m, c, plan.reflect, false);
  if (plan.phase == PSG_IP_ZERO)
    for (const Sos& c : plan.sections) sosSingle(buf.data(), m, c, plan.reflect, true);
  double ga = a * plan.dcGain - b * plan.dcSlope, gb = b * plan.dcGain;
  for (int64_t i = 0; i < n; i++) x[i] = (T)(buf[p + i] + (ga + gb * (double)i));
}

// ------------------------------------------------------------ core/mute --
// MuteCurve.muteTimeMs, core/mute.nim:103-123
double muteTimeMs(const psg_mute_curve& c, double msPerDist, double offset) {
  switch (c.kind) {
    case PSG_MK_TIME: return c.t_ms;
    case PSG_MK_LMO: return c.t0_ms + std::fabs(offset) * msPerDist + c.pad_ms;
    default: {
      double x = std::fabs(offset);
      if (std::isnan(x)) return NaN;
      int last = c.n_knots - 1;
      if (x <= c.offsets[0]) return c.times_ms[0];
      if (x >= c.offsets[last]) return c.times_ms[last];
      int lo = 0, hi = last;
      while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (c.offsets[mid] <= x) lo = mid; else hi = mid;
      }
      double u = (x - c.offsets[lo]) / (c.offsets[hi] - c.offsets[lo]);
      return c.times_ms[lo] + u * (c.times_ms[hi] - c.times_ms[lo]);
    }
  }
}
// core/mute.nim:127-137
int64_t firstAtOrAfter(double c, int64_t n) {
  if (!(c > 0)) return 0;
  if (c >= (double)n) return n;
  return (int64_t)std::ceil(c);
}
int64_t firstAfter(double c, int64_t n) {
  if (!(c >= 0)) return 0;
  if (c >= (double)n) return n;
  return (int64_t)std::floor(c) + 1;
}
// muteTop, core/mute.nim:139-159
template <class T> void muteTop(T* x, int64_t n, double startCol, double taperCols) {
  if (std::isnan(startCol)) return;
  if (!(taperCols < INF)) taperCols = 0.0;
  double rampStart = startCol - taperCols;
  int64_t zeroEnd = firstAtOrAfter(rampStart, n);
  for (int64_t j = 0; j < zeroEnd; j++) x[j] = T(0);
  if (taperCols > 0)
    for (int64_t j = zeroEnd; j < firstAtOrAfter(startCol, n); j++) {
      double w = std::sin(PI / 2 * ((double)j - rampStart) / taperCols);
      x[j] = T((double)x[j] * (w * w));
    }
}
// muteBottom, core/mute.nim:161-180
template <class T> void muteBottom(T* x, int64_t n, double endCol, double taperCols) {
  if (std::isnan(endCol)) return;
  if (!(taperCols < INF)) taperCols = 0.0;
  double rampEnd = endCol + taperCols;
  int64_t zeroStart = firstAfter(rampEnd, n);
  if (taperCols > 0)
    for (int64_t j = firstAfter(endCol, n); j < zeroStart; j++) {
      double w = std::sin(PI / 2 * (rampEnd - (double)j) / taperCols);
      x[j] = T((double)x[j] * (w * w));
    }
  for (int64_t j = zeroStart; j < n; j++) x[j] = T(0);
}
// The keys a mute reads per row (ChunkMeta.keys, core/types.nim:206-214).
struct RowKeys {
  const double* offset = nullptr;  // NULL: NaN
  const double* t0 = nullptr;      // NULL: NaN
  int64_t firstSample = 0;
  double dtMs = 0;
};

// -------------------------------------------------------------- pipeline --
enum StepKind { stDemean, stDetrend, stScale, stClip, stPolarity, stFilter, stAgc, stNormTrace, stNormPanel, stGainCurve,
                stMuteTop, stMuteBottom, stIir };
template <class T> struct Step {
  StepKind kind;
  IirPlan iir;
  psg_mute_curve mute{};
  double msPerDist = 0, taperMs = 0;
  double factor = 0, lo = 0, hi = 0;
  FilterPlan<T> filter;
  AgcPlan agc;
  NormPlan norm;
  CurvePlan<T> curve;
  int64_t margin() const {
    return kind == stFilter ? filter.margin : (kind == stAgc ? agc.half : (kind == stIir ? iir.pad : 0));
  }
};
static const char* opName(int k) {
  static const char* names[] = {"opDemean", "opDetrend", "opScale", "opGainDb", "opClip", "opPolarity",
                                "opMuteTop", "opMuteBottom", "opFilter", "opIir", "opAgc", "opNormalize",
                                "opGainCurve", "opCalibrate", "opUncalibrate"};
  return (k >= 0 && k < 15) ? names[k] : "opUnknown";
}
template <class T> struct Plan {
  std::vector<Step<T>> steps;
  std::vector<std::pair<int, int>> parts;  // [a, b) step ranges
  double dtMs = 0;
  int64_t samples = 0, recordSamples = 0, margin = 0;
};
// pipeline.nim:392-447
template <class T> Step<T> compileOp(const psg_op& op, double dtMs, int64_t samples, int64_t record) {
  Step<T> s;
  switch (op.kind) {
    case PSG_OP_DEMEAN: s.kind = stDemean; break;
    case PSG_OP_DETREND: s.kind = stDetrend; break;
    case PSG_OP_POLARITY: s.kind = stPolarity; break;
    case PSG_OP_SCALE:
      if (!isFin(op.factor)) throw ValueError("the factor must be finite, got " + fmt(op.factor));
      if (!isFin((double)(T)op.factor)) throw ValueError("a factor of " + fmt(op.factor) + " overflows");
      s.kind = stScale; s.factor = op.factor; break;
    case PSG_OP_GAIN_DB: {
      if (!isFin(op.factor)) throw ValueError("the gain must be finite, got " + fmt(op.factor) + " dB");
      double f = std::pow(10.0, op.factor / 20);
      if (!isFin(f) || !isFin((double)(T)f)) throw ValueError("a gain of " + fmt(op.factor) + " dB overflows");
      s.kind = stScale; s.factor = f; break;
    }
    case PSG_OP_CLIP:
      if (std::isnan(op.lo) || std::isnan(op.hi) || op.lo > op.hi)
        throw ValueError("clip limits must satisfy lo <= hi");
      s.kind = stClip; s.lo = op.lo; s.hi = op.hi; break;
    case PSG_OP_FILTER:
      s.kind = stFilter; s.filter = initFilterPlan<T>(op.filter, dtMs, samples, op.trend); break;
    case PSG_OP_AGC:
      s.kind = stAgc; s.agc = initAgcPlan(op.window_ms, dtMs, samples, op.agc_mode, op.target, op.epsilon); break;
    case PSG_OP_NORMALIZE:
      s.norm = initNormalizePlan(op.norm_stat, samples, op.norm_scope, op.norm_target, op.percentile);
      s.kind = op.norm_scope == PSG_PER_PANEL ? stNormPanel : stNormTrace; break;
    case PSG_OP_GAIN_CURVE:
      s.kind = stGainCurve; s.curve = initGainCurvePlan<T>(op.curve, dtMs, record, op.t_min_ms, op.t_max_ms); break;
    case PSG_OP_IIR:
      s.kind = stIir; s.iir = initIirPlan(op.filter, dtMs, samples, op.iir_phase, op.trend); break;
    case PSG_OP_MUTE_TOP:
    case PSG_OP_MUTE_BOTTOM: {
      // pipeline.nim:417-424 and the builders' checks, core/mute.nim:55-97
      const psg_mute_curve& c = op.mute;
      if (c.kind == PSG_MK_TIME) {
        if (!isFin(c.t_ms)) throw ValueError("a mute time must be finite, got " + fmt(c.t_ms));
      } else if (c.kind == PSG_MK_TABLE) {
        if (c.n_knots < 1 || c.n_knots > PSG_MAX_MUTE_KNOTS) throw ValueError("a mute table needs 1 .. 64 knots");
        for (int i = 0; i < c.n_knots; i++) {
          if (!isFin(c.offsets[i]) || c.offsets[i] < 0) throw ValueError("mute table offsets must be finite and >= 0");
          if (i > 0 && c.offsets[i] <= c.offsets[i - 1]) throw ValueError("mute table offsets must be strictly ascending");
          if (!isFin(c.times_ms[i])) throw ValueError("mute table times must be finite");
        }
      } else if (c.kind == PSG_MK_LMO) {
        if (!isFin(c.velocity) || c.velocity <= 0) throw ValueError("an LMO mute velocity must be finite and positive");
        if (!isFin(c.t0_ms) || !isFin(c.pad_ms)) throw ValueError("LMO mute times must be finite");
      } else {
        throw ValueError("unknown mute kind");
      }
      if (!isFin(op.taper_ms) || op.taper_ms < 0) throw ValueError("a mute taper must be finite and >= 0 ms, got " + fmt(op.taper_ms));
      s.kind = op.kind == PSG_OP_MUTE_TOP ? stMuteTop : stMuteBottom;
      s.mute = c;
      s.msPerDist = c.kind == PSG_MK_LMO ? 1000 / c.velocity : 0;
      s.taperMs = op.taper_ms;
      break;
    }
    default:
      throw ValueError("this op is not supported by the oracle");
  }
  return s;
}
// pipeline.nim:466-523
template <class T> Plan<T> compile(const psg_op* ops, int nops, double dtMs, int64_t samples, int64_t recordSamples) {
  if (!isFin(dtMs) || dtMs <= 0) throw ValueError("dtMs must be finite and positive, got " + fmt(dtMs));
  if (samples < 1) throw ValueError("a pipeline needs samples >= 1, got " + std::to_string(samples));
  if (recordSamples != 0 && recordSamples < samples) throw ValueError("recordSamples must be 0 or >= samples");
  Plan<T> p;
  int64_t record = std::max(samples, recordSamples);
  p.dtMs = dtMs; p.samples = samples; p.recordSamples = record;
  for (int i = 0; i < nops; i++) {
    try {
      p.steps.push_back(compileOp<T>(ops[i], dtMs, samples, record));
    } catch (const ValueError& e) {
      throw ValueError("op " + std::to_string(i) + " (" + opName(ops[i].kind) + "): " + e.what());
    }
  }
  int start = 0;
  for (int i = 0; i < (int)p.steps.size(); i++) {
    p.margin += p.steps[i].margin();
    if (p.steps[i].kind == stNormPanel && i > start) {
      p.parts.push_back({start, i});
      start = i;
    }
  }
  p.parts.push_back({start, (int)p.steps.size()});
  return p;
}
// pipeline.nim:671-688 on one row; `k` holds the row's keys (r: its index).
template <class T> void runStep(const Step<T>& s, T* x, int64_t n, double startMs, int64_t cols, const RowKeys& k,
                                int64_t r) {
  switch (s.kind) {
    case stIir: applyIir(s.iir, x, n); break;
    case stMuteTop:
    case stMuteBottom: {
      // muteCol, core/mute.nim:209-214, and the block forms :216-240
      double off = k.offset ? k.offset[r] : NaN, t0 = k.t0 ? k.t0[r] : NaN;
      double col = (muteTimeMs(s.mute, s.msPerDist, off) - t0) / k.dtMs - (double)k.firstSample;
      double taperCols = s.taperMs / k.dtMs;
      if (s.kind == stMuteTop) muteTop(x, n, col, taperCols);
      else muteBottom(x, n, col, taperCols);
      break;
    }
    case stDemean: demean(x, n); break;
    case stDetrend: detrend(x, n); break;
    case stPolarity: polarity(x, n); break;
    case stScale: scale(x, n, s.factor); break;
    case stClip: clip(x, n, s.lo, s.hi); break;
    case stFilter: applyFilter(s.filter, x, n); break;
    case stAgc: agc(s.agc, x, n); break;
    case stNormTrace: normalizeTrace(s.norm, x, n); break;
    case stNormPanel: break;
    case stGainCurve: applyGainCurve(s.curve, x, n, startMs, cols); break;
  }
}
// pipeline.nim:690-723 on rows [r0, r1): every step of the part per live row
// (rows are independent, so the reference's 256 KB tiles give the same values).
template <class T>
void runPart(const Plan<T>& plan, int part, const T* src, T* dst, int64_t r0, int64_t r1, int64_t cols,
             const int32_t* live, const double* startMs, double factor, const RowKeys& keys) {
  auto range = plan.parts[part];
  int first = (range.first < range.second && plan.steps[range.first].kind == stNormPanel) ? range.first + 1 : range.first;
  if (src && src != dst) std::memcpy(dst + r0 * cols, src + r0 * cols, (size_t)(r1 - r0) * cols * sizeof(T));
  for (int64_t r = r0; r < r1; r++) {
    int64_t n = live[r];
    if (n <= 0) continue;
    T* x = dst + r * cols;
    if (!std::isnan(factor)) scale(x, n, factor);
    for (int i = first; i < range.second; i++) runStep(plan.steps[i], x, n, startMs ? startMs[r] : NaN, cols, keys, r);
  }
}

// --------------------------------------------------------- process pool --
// core/pool.nim:123-308 restated: persistent threads woken per job; rows
// handed out in runs of about 256 KB (a multiple of 8 rows) by an atomic
// counter; a per-panel factor computed by worker 0 before its part.
class Pool {
 public:
  explicit Pool(int n) : n_(std::max(1, n)) {
    for (int i = 0; i < n_; i++) th_.emplace_back([this, i] { loop(i); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> g(mu_);
      quit_ = true;
      job_++;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  int size() const { return n_; }
  // Runs fn(worker) on every worker and waits.
  void run(const std::function<void(int)>& fn) {
    std::unique_lock<std::mutex> g(mu_);
    fn_ = &fn;
    pending_ = n_;
    job_++;
    cv_.notify_all();
    done_.wait(g, [this] { return pending_ == 0; });
    fn_ = nullptr;
  }

 private:
  void loop(int id) {
    uint64_t seen = 0;
    while (true) {
      const std::function<void(int)>* f;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return job_ != seen; });
        seen = job_;
        if (quit_) return;
        f = fn_;
      }
      (*f)(id);
      {
        std::lock_guard<std::mutex> g(mu_);
        if (--pending_ == 0) done_.notify_all();
      }
    }
  }
  int n_;
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  uint64_t job_ = 0;
  int pending_ = 0;
  bool quit_ = false;
  const std::function<void(int)>* fn_ = nullptr;
};

// pipeline.nim:725-734 with the pool's part/panel jobs, pool.nim:239-308.
template <class T>
void applyPool(Pool* pool, const Plan<T>& plan, const T* src, T* dst, int64_t rows, int64_t cols,
               const int32_t* live, const double* startMs, RowKeys keys = RowKeys()) {
  if (!(keys.dtMs > 0)) keys.dtMs = plan.dtMs;
  int64_t grain = std::max<int64_t>(8, (256 * 1024 / std::max<int64_t>(1, cols * (int64_t)sizeof(T))) / 8 * 8);
  for (int part = 0; part < (int)plan.parts.size(); part++) {
    bool from0 = part == 0 && src && src != dst;
    double factor = NaN;
    auto rg = plan.parts[part];
    if (rg.first < rg.second && plan.steps[rg.first].kind == stNormPanel)
      factor = panelFactor(plan.steps[rg.first].norm, from0 ? src : dst, rows, cols, live);
    const T* s = from0 ? src : nullptr;
    if (!pool) {
      runPart(plan, part, s, dst, 0, rows, cols, live, startMs, factor, keys);
      continue;
    }
    std::atomic<int64_t> next{0};
    std::function<void(int)> job = [&](int) {
      while (true) {
        int64_t a = next.fetch_add(grain);
        if (a >= rows) break;
        runPart(plan, part, s, dst, a, std::min(rows, a + grain), cols, live, startMs, factor, keys);
      }
    };
    pool->run(job);
  }
}

// ---------------------------------------------------------- correlation --
// vibroseis/kaiser.nim:4-14: the power series of I0, stopped once a term
// falls under 1e-17 of the running sum.
double besselI0(double x) {
  double term = 1.0, result = 1.0, q = x * x / 4;
  for (int k = 1; k <= 500; k++) {
    term *= q / (double)(k * k);
    result += term;
    if (term < result * 1e-17) break;
  }
  return result;
}
// vibroseis/taper.nim:69-74 (defaultParam), :125-145 (taperWeight)
double taperDefault(int shape) { return shape == 6 ? 6.0 : shape == 7 ? 0.4 : shape == 8 ? 2.0 : NaN; }
double taperWeight(int shape, double x, double param) {
  double p = std::isnan(param) ? taperDefault(shape) : param;
  x = std::clamp(x, 0.0, 1.0);
  switch (shape) {
    case 0: return x;
    case 1: return std::sin(PI / 2 * x);
    case 2: return 0.5 - 0.5 * std::cos(PI * x);
    case 3: return 0.54 - 0.46 * std::cos(PI * x);
    case 4: return 0.42 - 0.5 * std::cos(PI * x) + 0.08 * std::cos(2 * PI * x);
    case 5: return 0.35875 - 0.48829 * std::cos(PI * x) + 0.14128 * std::cos(2 * PI * x) - 0.01168 * std::cos(3 * PI * x);
    case 6: { double u = 1 - x; return besselI0(p * std::sqrt(std::max(0.0, 1 - u * u))) / besselI0(p); }
    case 7: { double u = (1 - x) / p; return std::exp(-0.5 * u * u); }
    case 8: return std::pow(x, p);
    default: throw ValueError("unknown taper shape");
  }
}
// vibroseis/sweep.nim:292-301 (linear law), :331-342 (sweepInto),
// taper.nim:160-179 (applyTaper)
template <class T>
std::vector<T> linearSweep(double f1, double f2, double lengthMs, double dtMs, double tStart, double tEnd, int shape,
                           double param, double phaseDeg, double amplitude) {
  double steps = lengthMs / dtMs;
  double r = std::round(steps);
  int64_t n = std::fabs(steps - r) <= 1e-6 ? (int64_t)r : (int64_t)std::floor(steps);
  std::vector<T> x(n);
  double dt = dtMs / 1000, Tl = lengthMs / 1000, rate = (f2 - f1) / Tl;
  double p0 = phaseDeg * (PI / 180.0);
  for (int64_t j = 0; j < n; j++) {
    double t = (double)j * dt;
    double ph = 2 * PI * (f1 * t + 0.5 * rate * t * t);
    x[j] = (T)(amplitude * std::sin(p0 + ph));
  }
  double sweepMs = (double)n * dtMs;
  double s = std::isnan(tStart) ? 0.0 : tStart, e = std::isnan(tEnd) ? 0.0 : tEnd;
  if (s > 0)
    for (int64_t j = 0; j < n && (double)j * dtMs < s; j++)
      x[j] = (T)((double)x[j] * taperWeight(shape, (double)j * dtMs / s, param));
  if (e > 0)
    for (int64_t j = n - 1; j >= 0 && sweepMs - (double)j * dtMs < e; j--)
      x[j] = (T)((double)x[j] * taperWeight(shape, (sweepMs - (double)j * dtMs) / e, param));
  return x;
}

// vibroseis/sweep.nim:234-329 and :375-420: the non-linear laws' frequency,
// the phase integral (closed form for linear and table, Gauss–Legendre with
// 4 points per interval otherwise) and the harmonics, without validation
// (the tests feed valid specs). Law codes: 0 linear, 1 dB/octave, 2 dB/Hz,
// 3 exponential, 4 table.
struct OSweep {
  int law;
  double f1, f2, lengthMs, dtMs, boostDb;
  std::vector<double> tt, tf;  // table times (ms) and frequencies
};
double oExpm1(double x) {  // sweep.nim:236-241
  double u = std::exp(x);
  if (u == 1) return x;
  if (u - 1 == -1) return -1.0;
  return (u - 1) * x / std::log(u);
}
double oLn1p(double x) {  // sweep.nim:243-246
  double u = 1 + x;
  if (u == 1) return x;
  return std::log(u) * x / (u - 1);
}
double oFrequencyAt(const OSweep& s, double tMs) {  // sweep.nim:248-284
  double T = s.lengthMs;
  double x = std::clamp(tMs, 0.0, T) / T;
  double f1 = s.f1, f2 = s.f2;
  if (x <= 0) return f1;
  if (x >= 1) return f2;
  auto within = [&](double f) { return std::clamp(f, std::min(f1, f2), std::max(f1, f2)); };
  if (s.law == 0) return within(f1 + (f2 - f1) * x);
  if (s.law == 3) return within(f1 * std::pow(f2 / f1, x));
  if (s.law == 1) {
    double octaveDb = 20 * std::log10(2.0) / 2;
    double m = s.boostDb / octaveDb + 1;
    if (std::fabs(m) < 1e-12) return within(f1 * std::pow(f2 / f1, x));
    return within(f1 * std::pow(1 + x * oExpm1(m * std::log(f2 / f1)), 1 / m));
  }
  if (s.law == 2) {
    double k = s.boostDb * std::log(10.0) / 10;
    double e = oExpm1(k * (f2 - f1));
    if (std::fabs(k * (f2 - f1)) < 1e-12) return within(f1 + (f2 - f1) * x);
    return within(f1 + oLn1p(x * e) / k);
  }
  double t = std::clamp(tMs, 0.0, T);
  size_t i = 1;
  while (i < s.tt.size() - 1 && s.tt[i] < t) i++;
  return s.tf[i - 1] + (s.tf[i] - s.tf[i - 1]) * (t - s.tt[i - 1]) / (s.tt[i] - s.tt[i - 1]);
}
std::vector<double> oPhases(const OSweep& s, int64_t n) {  // sweep.nim:292-329
  std::vector<double> ph(n);
  double dt = s.dtMs / 1000, T = s.lengthMs / 1000;
  if (s.law == 0) {
    double rate = (s.f2 - s.f1) / T;
    for (int64_t j = 0; j < n; j++) {
      double t = (double)j * dt;
      ph[j] = 2 * PI * (s.f1 * t + 0.5 * rate * t * t);
    }
  } else if (s.law == 4) {
    double acc = 0;
    size_t i = 1;
    for (int64_t j = 0; j < n; j++) {
      double tMs = (double)j * s.dtMs;
      while (i < s.tt.size() - 1 && s.tt[i] <= tMs) {
        acc += 0.5 * (s.tf[i - 1] + s.tf[i]) * (s.tt[i] - s.tt[i - 1]) / 1000;
        i++;
      }
      double sec = (std::min(tMs, s.tt[i]) - s.tt[i - 1]) / 1000;
      double slope = (s.tf[i] - s.tf[i - 1]) / ((s.tt[i] - s.tt[i - 1]) / 1000);
      ph[j] = 2 * PI * (acc + s.tf[i - 1] * sec + 0.5 * slope * sec * sec);
    }
  } else {
    static const double nodes[4] = {-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526};
    static const double weights[4] = {0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538};
    double acc = 0;
    if (n > 0) ph[0] = 0;
    for (int64_t j = 1; j < n; j++) {
      double a = (double)(j - 1) * s.dtMs, h = 0.5 * s.dtMs, sum = 0;
      for (int q = 0; q < 4; q++) sum += weights[q] * oFrequencyAt(s, a + h + h * nodes[q]);
      acc += sum * h / 1000;
      ph[j] = 2 * PI * acc;
    }
  }
  return ph;
}
// sweepHarmonicsInto (sweep.nim:375-420) into n samples of T; harmonics as
// (order, amp, phaseDeg) triples; nh 0: the plain sweep.
template <class T>
std::vector<T> oSweepSamples(const OSweep& s, const double* harm, int nh, double phaseDeg, double amplitude,
                             double ts, double te, int shape, double param, int64_t n) {
  double steps = s.lengthMs / s.dtMs, r = std::round(steps);
  int64_t nSweep = std::fabs(steps - r) <= 1e-6 ? (int64_t)r : (int64_t)std::floor(steps);
  int64_t m = std::min(n, nSweep);
  std::vector<double> ph = oPhases(s, m);
  double p0 = phaseDeg * (PI / 180.0), nyq = 500.0 / s.dtMs;
  std::vector<T> x(n, T(0));
  for (int64_t j = 0; j < m; j++) {
    double p = p0 + ph[j], v = 0;
    if (nh == 0) {
      v = std::sin(p);
    } else {
      double f = oFrequencyAt(s, (double)j * s.dtMs);
      for (int k = 0; k < nh; k++) {
        double order = harm[3 * k], amp = harm[3 * k + 1], pd = harm[3 * k + 2];
        if (order == 1 || order * f < nyq) v += amp * std::sin(order * p + pd * (PI / 180.0));
      }
    }
    x[j] = (T)(amplitude * v);
  }
  double sa = std::isnan(ts) ? 0.0 : ts, ea = std::isnan(te) ? 0.0 : te;
  int64_t len = std::min(n, nSweep);
  double sweepMs = n >= nSweep ? (double)nSweep * s.dtMs : s.lengthMs;
  if (sa > 0)
    for (int64_t j = 0; j < len && (double)j * s.dtMs < sa; j++)
      x[j] = (T)((double)x[j] * taperWeight(shape, (double)j * s.dtMs / sa, param));
  if (ea > 0)
    for (int64_t j = len - 1; j >= 0 && sweepMs - (double)j * s.dtMs < ea; j--)
      x[j] = (T)((double)x[j] * taperWeight(shape, (sweepMs - (double)j * s.dtMs) / ea, param));
  return x;
}

template <class T> struct CorrPlan {
  FftPlan<T> fft;
  std::vector<T> mulRe, mulIm;
  int64_t shift = 0, recordSamples = 0, outSamples = 0, pilotSamples = 0;
  double dtMs = 0, scale = 1;
};
// vibroseis/correlate.nim:82-160
template <class T>
CorrPlan<T> initCorrelationPlan(const double* pilot, int64_t plen, double pilotDt, double pilotT0, double dtMs,
                                int64_t recordSamples, int64_t outSamples, int mode, double epsPercent, bool normalize) {
  if (plen < 2) throw ValueError("a pilot needs at least two samples");
  double energy = 0;
  for (int64_t i = 0; i < plen; i++) {
    if (!isFin(pilot[i])) throw ValueError("pilot sample is not finite");
    energy += pilot[i] * pilot[i];
  }
  if (energy == 0) throw ValueError("the pilot is all zeros");
  if (!(dtMs > 0 && dtMs < INF)) throw ValueError("dtMs must be finite and positive");
  if (!(std::fabs(pilotDt - dtMs) <= 1e-9 * dtMs)) throw ValueError("the pilot is sampled at another interval");
  if (recordSamples < 1) throw ValueError("recordSamples must be >= 1");
  int64_t outN = outSamples == 0 ? recordSamples - plen : outSamples;
  if (outN < 1) throw ValueError("the pilot is not shorter than the record");
  if (outSamples < 0 || outN > recordSamples) throw ValueError("outSamples must be in 0 .. recordSamples");
  if (mode == PSG_CM_DECONVOLVE && !(epsPercent > 0 && epsPercent < INF)) throw ValueError("epsPercent");
  double s = pilotT0 / dtMs;
  if (std::fabs(s) >= (double)(recordSamples + plen)) throw ValueError("no lag reaches the output");
  int64_t whole = (int64_t)std::round(s);
  double frac = s - (double)whole;
  int64_t n = nextFastLen(recordSamples + plen + 64 + std::llabs(whole));
  CorrPlan<T> p;
  p.fft = initFftPlan<T>(n);
  int64_t bins = p.fft.bins();
  FftPlan<double> pf = initFftPlan<double>(n);
  std::vector<double> x(n, 0.0), pr(bins), pi(bins);
  for (int64_t j = 0; j < plen; j++) x[j] = pilot[j];
  fftForward(pf, x.data(), pr.data(), pi.data());
  double peakPow = 0;
  for (int64_t k = 0; k < bins; k++) peakPow = std::max(peakPow, pr[k] * pr[k] + pi[k] * pi[k]);
  double eps = mode == PSG_CM_DECONVOLVE ? epsPercent / 100 * peakPow : 0.0;
  std::vector<double> w(bins);
  double peak = 0;
  for (int64_t k = 0; k < bins; k++) {
    double p2 = pr[k] * pr[k] + pi[k] * pi[k];
    w[k] = mode == PSG_CM_DECONVOLVE ? 1 / (p2 + eps) : 1.0;
    double g = p2 * w[k];
    peak += (k == 0 || (n % 2 == 0 && k == bins - 1)) ? g : 2 * g;
  }
  peak /= (double)n;
  double scale = normalize ? 1 / peak : 1.0;
  p.mulRe.resize(bins);
  p.mulIm.resize(bins);
  for (int64_t k = 0; k < bins; k++) {
    double ws = w[k] * scale;
    double ar = pr[k] * ws, ai = -pi[k] * ws;
    double th = 2 * PI * (double)k * frac / (double)n;
    double cr = std::cos(th), ci = std::sin(th);
    p.mulRe[k] = (T)(ar * cr - ai * ci);
    p.mulIm[k] = (T)(ai * cr + ar * ci);
  }
  if (n % 2 == 0) p.mulIm[bins - 1] = 0;
  p.shift = whole;
  p.recordSamples = recordSamples;
  p.outSamples = outN;
  p.pilotSamples = plen;
  p.dtMs = dtMs;
  p.scale = scale;
  return p;
}
// vibroseis/correlate.nim:271-274, 292-326 (one record)
template <class T> void correlateOne(const CorrPlan<T>& plan, const T* x, int64_t live, T* y, int64_t cols) {
  int64_t n = plan.fft.n, bins = plan.fft.bins();
  std::vector<T> buf(n, (T)0), re(bins), im(bins);
  for (int64_t j = 0; j < live; j++) buf[j] = x[j];
  fftForward(plan.fft, buf.data(), re.data(), im.data());
  for (int64_t k = 0; k < bins; k++) {
    T a = re[k], b = im[k], mr = plan.mulRe[k], mi = plan.mulIm[k];
    re[k] = a * mr - b * mi;
    im[k] = a * mi + b * mr;
  }
  fftInverse(plan.fft, re.data(), im.data(), buf.data());
  int64_t wrapped = std::clamp(1 - plan.pilotSamples - plan.shift, (int64_t)0, cols);
  int64_t direct = std::clamp(-plan.shift, wrapped, cols);
  int64_t last = std::clamp(plan.recordSamples - plan.shift, direct, cols);
  int64_t wrap = plan.shift + n;
  for (int64_t m = 0; m < wrapped; m++) y[m] = 0;
  for (int64_t m = wrapped; m < direct; m++) y[m] = buf[m + wrap];
  for (int64_t m = direct; m < last; m++) y[m] = buf[m + plan.shift];
  for (int64_t m = last; m < cols; m++) y[m] = 0;
}

}  // namespace orc

// ==================================================================== C ABI
using namespace orc;

static thread_local std::string g_err;
template <class F> static int guard(F&& f) {
  try {
    f();
    g_err.clear();
    return PSG_OK;
  } catch (const ValueError& e) {
    g_err = e.what();
    return PSG_EINVAL;
  } catch (const std::exception& e) {
    g_err = e.what();
    return PSG_EINVAL;
  }
}

struct OrcPlan {
  int dtype;
  void* p;  // Plan<float>* or Plan<double>*
};

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }
int orc_is_fast_len(int64_t n) { return isFastLen(n) ? 1 : 0; }
int64_t orc_next_fast_len(int64_t n, int even) { return nextFastLen(n, even != 0); }

int orc_fft_forward(int dtype, int64_t n, const void* x, void* re, void* im) {
  return guard([&] {
    if (dtype == PSG_F32) {
      auto p = initFftPlan<float>(n);
      fftForward(p, (const float*)x, (float*)re, (float*)im);
    } else {
      auto p = initFftPlan<double>(n);
      fftForward(p, (const double*)x, (double*)re, (double*)im);
    }
  });
}
int orc_fft_inverse(int dtype, int64_t n, const void* re, const void* im, void* x) {
  return guard([&] {
    if (dtype == PSG_F32) {
      auto p = initFftPlan<float>(n);
      fftInverse(p, (const float*)re, (const float*)im, (float*)x);
    } else {
      auto p = initFftPlan<double>(n);
      fftInverse(p, (const double*)re, (const double*)im, (double*)x);
    }
  });
}
int orc_response(const psg_filter_spec* spec, double f, double dtMs, double* out) {
  return guard([&] { *out = response(*spec, f, dtMs); });
}
int orc_impulse_length(const psg_filter_spec* spec, double dtMs, int64_t* out) {
  return guard([&] { *out = impulseLength(*spec, dtMs); });
}
// FilterPlan facts: margin, pad, nfft, reflect, dcGain, and the gain table
// (nfft/2 + 1 doubles when gain_out is not NULL).
int orc_filter_plan_info(const psg_filter_spec* spec, int dtype, double dtMs, int64_t samples, int trend,
                         int64_t* margin, int64_t* pad, int64_t* nfft, int* reflect, double* dcGain,
                         double* gain_out) {
  return guard([&] {
    auto p = initFilterPlan<double>(*spec, dtMs, samples, trend);
    *margin = p.margin; *pad = p.pad; *nfft = p.fft.n; *reflect = p.reflect; *dcGain = p.dcGain;
    if (gain_out) {
      if (dtype == PSG_F32) {
        auto q = initFilterPlan<float>(*spec, dtMs, samples, trend);
        for (size_t k = 0; k < q.gain.size(); k++) gain_out[k] = q.gain[k];
      } else {
        for (size_t k = 0; k < p.gain.size(); k++) gain_out[k] = p.gain[k];
      }
    }
  });
}
int orc_required_margin(const psg_op* ops, int nops, double dtMs, int64_t* out) {
  return guard([&] {
    if (!isFin(dtMs) || dtMs <= 0) throw ValueError("dtMs must be finite and positive, got " + fmt(dtMs));
    int64_t m = 0;
    for (int i = 0; i < nops; i++) {
      try {
        if (ops[i].kind == PSG_OP_FILTER) {
          validate(ops[i].filter, dtMs);
          m += impulseLength(ops[i].filter, dtMs);
        } else if (ops[i].kind == PSG_OP_AGC) {
          m += initAgcPlan(ops[i].window_ms, dtMs, 1, ops[i].agc_mode, ops[i].target, ops[i].epsilon).half;
        } else if (ops[i].kind == PSG_OP_IIR) {
          m += initIirPlan(ops[i].filter, dtMs, 1, ops[i].iir_phase, ops[i].trend).pad;
        }
      } catch (const ValueError& e) {
        throw ValueError("op " + std::to_string(i) + " (" + opName(ops[i].kind) + "): " + e.what());
      }
    }
    *out = m;
  });
}
// SpectrumPlan's nfft and Σw; averageAmplitudeInto over rows r0 .. r1
// (returns the rows averaged in *used); amplitudeInto per row (windows up to
// each row's live end; rows × bins of amp and phase).
int orc_spectrum(int dtype, double dtMs, int64_t windowLen, double taperFraction, int64_t nfft, int demean,
                 const void* b, int64_t rows, int64_t cols, const int32_t* live, int64_t firstCol, int64_t r0,
                 int64_t r1, double* avg, int64_t* used, void* amp, void* phase, int64_t* nfftOut, double* taperSum) {
  return guard([&] {
    auto run = [&](auto tag) {
      typedef decltype(tag) T;
      SpectrumPlan<T> sp = initSpectrumPlan<T>(dtMs, windowLen, taperFraction, nfft, demean != 0);
      if (nfftOut) *nfftOut = sp.fft.n;
      if (taperSum) *taperSum = sp.taperSum;
      if (avg) *used = averageAmplitude(sp, (const T*)b, rows, cols, live, firstCol, r0, r1, avg);
      if (amp) {
        int64_t nb = sp.fft.bins();
        for (int64_t r = 0; r < rows; r++) {
          int64_t lv = std::min<int64_t>(std::max<int32_t>(live[r], 0), cols);
          int64_t n = std::max<int64_t>(0, std::min<int64_t>(lv, firstCol + windowLen) - firstCol);
          amplitudeInto(sp, (const T*)b + r * cols + firstCol, n, (T*)amp + r * nb, (T*)phase + r * nb);
        }
      }
    };
    if (dtype == PSG_F32) run(float());
    else run(double());
  });
}
// IirPlan's order, requiredMargin, dcGain and magnitudeAt (filter/iir.nim:
// 241-278) at the frequencies f[0 .. nf).
int orc_iir_info(const psg_filter_spec* spec, double dtMs, int64_t samples, int phase, int trend, int* order,
                 int64_t* pad, double* dcGain, const double* f, int64_t nf, double* mag) {
  return guard([&] {
    IirPlan p = initIirPlan(*spec, dtMs, samples, phase, trend);
    int o = 0;
    for (const Sos& c : p.sections) o += c.a2 == 0 ? 1 : 2;
    *order = o;
    *pad = p.pad;
    *dcGain = p.dcGain;
    for (int64_t i = 0; i < nf; i++) {
      double w = 2 * PI * f[i] * dtMs / 1000;
      double zr = std::cos(w), zi = -std::sin(w);
      double z2r = zr * zr - zi * zi, z2i = zr * zi + zi * zr;
      double hr = 1, hi = 0;
      for (const Sos& c : p.sections) {
        double nr = c.b0 + c.b1 * zr + c.b2 * z2r, ni = c.b1 * zi + c.b2 * z2i;
        double dr = 1.0 + c.a1 * zr + c.a2 * z2r, di = c.a1 * zi + c.a2 * z2i;
        double qr, qi;
        cdivNim(nr, ni, dr, di, qr, qi);
        double tr = hr * qr - hi * qi, ti = hr * qi + hi * qr;
        hr = tr;
        hi = ti;
      }
      double a = std::hypot(hr, hi);
      mag[i] = phase == PSG_IP_ZERO ? a * a : a;
    }
  });
}
// applyFilter of an IIR plan on one trace of n samples, in place (float64).
int orc_iir_apply(const psg_filter_spec* spec, double dtMs, int64_t samples, int phase, int trend, double* x,
                  int64_t n) {
  return guard([&] {
    IirPlan p = initIirPlan(*spec, dtMs, samples, phase, trend);
    if (n > samples) throw ValueError("a trace longer than the plan's samples");
    applyIir(p, x, n);
  });
}
int orc_plan_compile(const psg_op* ops, int nops, int dtype, double dtMs, int64_t samples, int64_t record,
                     void** out) {
  return guard([&] {
    OrcPlan* op = new OrcPlan{dtype, nullptr};
    try {
      if (dtype == PSG_F32) op->p = new Plan<float>(compile<float>(ops, nops, dtMs, samples, record));
      else op->p = new Plan<double>(compile<double>(ops, nops, dtMs, samples, record));
    } catch (...) {
      delete op;
      throw;
    }
    *out = op;
  });
}
void orc_plan_destroy(void* h) {
  OrcPlan* op = (OrcPlan*)h;
  if (!op) return;
  if (op->dtype == PSG_F32) delete (Plan<float>*)op->p;
  else delete (Plan<double>*)op->p;
  delete op;
}
int64_t orc_plan_margin(void* h) {
  OrcPlan* op = (OrcPlan*)h;
  return op->dtype == PSG_F32 ? ((Plan<float>*)op->p)->margin : ((Plan<double>*)op->p)->margin;
}
int orc_plan_part_count(void* h) {
  OrcPlan* op = (OrcPlan*)h;
  return (int)(op->dtype == PSG_F32 ? ((Plan<float>*)op->p)->parts.size() : ((Plan<double>*)op->p)->parts.size());
}
int64_t orc_plan_step_nfft(void* h, int step) {
  OrcPlan* op = (OrcPlan*)h;
  if (op->dtype == PSG_F32) {
    auto& s = ((Plan<float>*)op->p)->steps[step];
    return s.kind == stFilter ? s.filter.fft.n : 0;
  }
  auto& s = ((Plan<double>*)op->p)->steps[step];
  return s.kind == stFilter ? s.filter.fft.n : 0;
}
// isLive / liveSamples / sampleTimeMs flattened, core/types.nim:212-240
// (mode 1: the correlation rule, vibroseis/correlate.nim:442-443).
int orc_rows_flatten(const int32_t* status, const int32_t* numSamples, const double* t0, int64_t rows, int32_t first,
                     double dtMs, const int64_t* failed, int64_t nfailed, int32_t cols, int32_t mode, int32_t* live,
                     double* startMs) {
  return guard([&] {
    std::vector<char> isFailed(rows, 0);
    for (int64_t i = 0; i < nfailed; i++)
      if (failed[i] >= 0 && failed[i] < rows) isFailed[failed[i]] = 1;
    for (int64_t r = 0; r < rows; r++) {
      // mode 3: the rule of mode 0, with the rows it leaves out marked -1
      bool use = mode == 0 || mode == 3 ? ((status[r] == PSG_TS_LIVE || status[r] == PSG_TS_UNKNOWN) && !isFailed[r])
                                        : (status[r] != PSG_TS_DEAD && !isFailed[r]);
      int64_t n = std::clamp<int64_t>((int64_t)numSamples[r] - first, 0, cols);
      live[r] = use ? (int32_t)n : (mode == 3 ? -1 : 0);
      if (startMs) startMs[r] = (t0 ? t0[r] : NaN) + (double)(first) * dtMs;
    }
  });
}
// apply(plan, src, dst, meta), pipeline.nim:725-772; threads > 1 runs through
// the ProcessPool clone. src NULL: in place.
int orc_plan_apply(void* h, const void* src, void* dst, int64_t rows, int64_t cols, const int32_t* live,
                   const double* startMs, int threads) {
  return guard([&] {
    OrcPlan* op = (OrcPlan*)h;
    std::unique_ptr<Pool> pool(threads > 1 ? new Pool(threads) : nullptr);
    if (op->dtype == PSG_F32)
      applyPool(pool.get(), *(Plan<float>*)op->p, (const float*)src, (float*)dst, rows, cols, live, startMs);
    else
      applyPool(pool.get(), *(Plan<double>*)op->p, (const double*)src, (double*)dst, rows, cols, live, startMs);
  });
}
// The same with the rows' keys, which a plan with mutes reads: offset and
// t0Ms per row (NULL: NaN), the block's first sample and the rows' interval.
int orc_plan_apply_keyed(void* h, const void* src, void* dst, int64_t rows, int64_t cols, const int32_t* live,
                         const double* startMs, const double* offset, const double* t0, int64_t firstSample,
                         double dtMs, int threads) {
  return guard([&] {
    OrcPlan* op = (OrcPlan*)h;
    std::unique_ptr<Pool> pool(threads > 1 ? new Pool(threads) : nullptr);
    RowKeys k;
    k.offset = offset;
    k.t0 = t0;
    k.firstSample = firstSample;
    k.dtMs = dtMs;
    if (op->dtype == PSG_F32)
      applyPool(pool.get(), *(Plan<float>*)op->p, (const float*)src, (float*)dst, rows, cols, live, startMs, k);
    else
      applyPool(pool.get(), *(Plan<double>*)op->p, (const double*)src, (double*)dst, rows, cols, live, startMs, k);
  });
}
// The CPU baseline: `iters` applies of the plan through one pool of
// `threads` workers (created once, as a viewer's pool is), each sample timed;
// returns the median and minimum seconds (bench/benchutil.nim:96-126 method,
// warm-up included in `warm`).
// The reference harness's timing (bench/benchutil.nim:96-126): `warm` runs,
// then `samples` samples, each running batches of 1, 2, 4 … applies until at
// least min_sample_ms have passed, timed as elapsed / applies; the median and
// the minimum of the samples, and the applies run in all.
int orc_bench_apply(void* h, const void* src, void* dst, int64_t rows, int64_t cols, const int32_t* live,
                    const double* startMs, int threads, int warm, int samples, double min_sample_ms,
                    double* median_s, double* min_s, int64_t* applies) {
  return guard([&] {
    OrcPlan* op = (OrcPlan*)h;
    Pool pool(threads);
    auto once = [&] {
      if (op->dtype == PSG_F32)
        applyPool(&pool, *(Plan<float>*)op->p, (const float*)src, (float*)dst, rows, cols, live, startMs);
      else
        applyPool(&pool, *(Plan<double>*)op->p, (const double*)src, (double*)dst, rows, cols, live, startMs);
    };
    for (int i = 0; i < warm; i++) once();
    std::vector<double> t;
    int64_t total = 0;
    for (int k = 0; k < samples; k++) {
      int64_t n = 0, batch = 1;
      auto t0 = std::chrono::steady_clock::now();
      double el = 0;
      while (true) {
        for (int64_t b = 0; b < batch; b++) once();
        n += batch;
        batch *= 2;
        el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el * 1e3 >= min_sample_ms) break;
      }
      t.push_back(el / (double)n);
      total += n;
    }
    std::sort(t.begin(), t.end());
    *median_s = t.empty() ? 0 : t[t.size() / 2];
    *min_s = t.empty() ? 0 : t[0];
    if (applies) *applies = total;
  });
}
// Single-op kernels on one row, for unit checks.
int orc_agc_row(int dtype, double windowMs, double dtMs, int mode, double target, double eps, void* x, int64_t n) {
  return guard([&] {
    AgcPlan p = initAgcPlan(windowMs, dtMs, std::max<int64_t>(n, 1), mode, target, eps);
    if (dtype == PSG_F32) agc(p, (float*)x, n); else agc(p, (double*)x, n);
  });
}
int orc_panel_stats(int dtype, const void* b, int64_t rows, int64_t cols, const int32_t* live, double clipP,
                    int signedLive, double* out5) {
  return guard([&] {
    PanelStats s = dtype == PSG_F32 ? panelStats((const float*)b, rows, cols, live, clipP, signedLive != 0)
                                    : panelStats((const double*)b, rows, cols, live, clipP, signedLive != 0);
    out5[0] = s.rms; out5[1] = s.maxAbs; out5[2] = s.clip; out5[3] = (double)s.rows; out5[4] = (double)s.samples;
  });
}
int orc_trace_stats(int dtype, const void* b, int64_t rows, int64_t cols, const int32_t* live, double* rms,
                    double* mx) {
  return guard([&] {
    if (dtype == PSG_F32) traceStatsInto((const float*)b, rows, cols, live, rms, mx);
    else traceStatsInto((const double*)b, rows, cols, live, rms, mx);
  });
}
int orc_percentile_abs(int dtype, const void* x, int64_t n, double p, double* out) {
  return guard([&] {
    *out = dtype == PSG_F32 ? percentileAbs((const float*)x, n, p) : percentileAbs((const double*)x, n, p);
  });
}
// table: n_table (t_ms, f_hz) pairs; harm: nh (order, amp, phaseDeg) triples
int orc_sweep_samples(int law, double f1, double f2, double lengthMs, double dtMs, double boostDb,
                      const double* table, int n_table, const double* harm, int nh, double phaseDeg, double amp,
                      double ts, double te, int shape, double param, int dtype, void* out, int64_t n) {
  return guard([&] {
    OSweep s{law, f1, f2, lengthMs, dtMs, boostDb, {}, {}};
    for (int i = 0; i < n_table; i++) {
      s.tt.push_back(table[2 * i]);
      s.tf.push_back(table[2 * i + 1]);
    }
    if (dtype == PSG_F32) {
      auto v = oSweepSamples<float>(s, harm, nh, phaseDeg, amp, ts, te, shape, param, n);
      std::memcpy(out, v.data(), v.size() * 4);
    } else {
      auto v = oSweepSamples<double>(s, harm, nh, phaseDeg, amp, ts, te, shape, param, n);
      std::memcpy(out, v.data(), v.size() * 8);
    }
  });
}
int orc_sweep_frequency_at(int law, double f1, double f2, double lengthMs, double dtMs, double boostDb,
                           const double* table, int n_table, double tMs, double* out) {
  return guard([&] {
    OSweep s{law, f1, f2, lengthMs, dtMs, boostDb, {}, {}};
    for (int i = 0; i < n_table; i++) {
      s.tt.push_back(table[2 * i]);
      s.tf.push_back(table[2 * i + 1]);
    }
    *out = oFrequencyAt(s, tMs);
  });
}
int orc_taper_weight(int shape, double x, double param, double* out) {
  return guard([&] { *out = taperWeight(shape, x, param); });
}
int orc_linear_sweep(double f1, double f2, double lengthMs, double dtMs, double ts, double te, int shape,
                     double param, double phaseDeg, double amp, int dtype, void* out, int64_t* n_out) {
  return guard([&] {
    if (dtype == PSG_F32) {
      auto v = linearSweep<float>(f1, f2, lengthMs, dtMs, ts, te, shape, param, phaseDeg, amp);
      if (out) std::memcpy(out, v.data(), v.size() * 4);
      *n_out = (int64_t)v.size();
    } else {
      auto v = linearSweep<double>(f1, f2, lengthMs, dtMs, ts, te, shape, param, phaseDeg, amp);
      if (out) std::memcpy(out, v.data(), v.size() * 8);
      *n_out = (int64_t)v.size();
    }
  });
}
// correlateInto (block form) with rows `live` (mode 1 flattening; 0: zeros).
int orc_correlate(const double* pilot, int64_t plen, double pilotDt, double pilotT0, int dtype, double dtMs,
                  int64_t recordSamples, int64_t outSamples, int mode, double epsPercent, int normalize,
                  const void* src, void* dst, int64_t rows, int64_t cols, const int32_t* live, int64_t* nfft_out,
                  double* scale_out) {
  return guard([&] {
    if (dtype == PSG_F32) {
      auto p = initCorrelationPlan<float>(pilot, plen, pilotDt, pilotT0, dtMs, recordSamples, outSamples, mode,
                                          epsPercent, normalize != 0);
      if (nfft_out) *nfft_out = p.fft.n;
      if (scale_out) *scale_out = p.scale;
      for (int64_t r = 0; r < rows && src; r++)
        correlateOne(p, (const float*)src + r * cols, live[r], (float*)dst + r * p.outSamples, p.outSamples);
    } else {
      auto p = initCorrelationPlan<double>(pilot, plen, pilotDt, pilotT0, dtMs, recordSamples, outSamples, mode,
                                           epsPercent, normalize != 0);
      if (nfft_out) *nfft_out = p.fft.n;
      if (scale_out) *scale_out = p.scale;
      for (int64_t r = 0; r < rows && src; r++)
        correlateOne(p, (const double*)src + r * cols, live[r], (double*)dst + r * p.outSamples, p.outSamples);
    }
  });
}
// RecordStack rsVertical, vibroseis/vstack.nim:186-202, 357-380, 439-471:
// adds rows with live[r] > 0 into num/count (float64 / int32 arrays of
// out_rows × samples) at row_map[r] (NULL: r), skipping non-finite rows.
int orc_stack_add(int dtype, const void* b, int64_t rows, int64_t cols, const int32_t* live, const int32_t* rowMap,
                  double* num, int32_t* cnt, int64_t samples) {
  return guard([&] {
    for (int64_t r = 0; r < rows; r++) {
      int64_t o = rowMap ? rowMap[r] : r;
      if (o < 0 || live[r] <= 0) continue;
      int64_t n = live[r];
      double s = 0;
      for (int64_t j = 0; j < n; j++) {
        double v = dtype == PSG_F32 ? (double)((const float*)b)[r * cols + j] : ((const double*)b)[r * cols + j];
        s += v - v;
      }
      if (s != 0 || std::isnan(s)) continue;
      for (int64_t j = 0; j < n; j++) {
        double v = dtype == PSG_F32 ? (double)((const float*)b)[r * cols + j] : ((const double*)b)[r * cols + j];
        num[o * samples + j] += v;
        cnt[o * samples + j] += 1;
      }
    }
  });
}

}  // extern "C"
