// psg_plan.cpp — host side of libpsgcuda.so: validating ops and compiling a
// pipeline into the tables the device kernels read (filter responses, FFT
// twiddles, pad tapers, gain tables, correlation multipliers), all generated
// in float64. The arithmetic on samples runs on the GPU (psg_cuda.cu).
//
// Reference: src/processSEG/pipeline.nim (compile), filter/design.nim
// (responses, impulse length), filter/apply.nim:118-151 (filter plan),
// gain/gain.nim:272-302 (AGC plan), gain/curves.nim:214-247 (gain tables),
// vibroseis/correlate.nim:82-160, sweep.nim, taper.nim (correlation plan).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstring>
#include <limits>

#include "psg_internal.h"

namespace psg {

namespace {
const double kPi = 3.14159265358979323846;
const double kInf = std::numeric_limits<double>::infinity();
const double kNaN = std::numeric_limits<double>::quiet_NaN();
typedef std::complex<double> cd;

std::string num(double v) {
  char b[48];
  snprintf(b, sizeof b, "%g", v);
  return b;
}
bool fin(double x) { return std::isfinite(x); }
bool fin_pos(double x) {
  int c = std::fpclassify(x);
  return (c == FP_NORMAL || c == FP_SUBNORMAL) && x > 0;
}
template <class T> bool fits(double x) { return fin_pos(x) && fin_pos((double)(T)x); }
bool fits_dtype(int dtype, double x) { return dtype == PSG_F32 ? fits<float>(x) : fits<double>(x); }
double as_dtype(int dtype, double x) { return dtype == PSG_F32 ? (double)(float)x : x; }

// A mixed-radix decimation-in-time FFT in float64 on the host, for the
// plan-time transforms (impulse lengths, pilot spectra). `w` holds
// exp(sign·2πi·j/N) for the top length N; a sub-transform reads it at a stride.
void dit(const cd* in, int64_t istride, cd* out, int64_t n, const std::vector<cd>& w, int64_t wstride,
         std::vector<cd>& tmp) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  int r = n % 4 == 0 ? 4 : (n % 2 == 0 ? 2 : (n % 3 == 0 ? 3 : 5));
  int64_t m = n / r;
  for (int q = 0; q < r; q++) dit(in + q * istride, istride * r, out + q * m, m, w, wstride * r, tmp);
  const int64_t N = (int64_t)w.size();
  cd t[5];
  for (int64_t k = 0; k < m; k++) {
    for (int q = 0; q < r; q++) t[q] = out[q * m + k] * w[(q * k * wstride) % N];
    for (int s = 0; s < r; s++) {
      cd acc = 0;
      for (int q = 0; q < r; q++) acc += t[q] * w[((int64_t)q * s * m * wstride) % N];
      tmp[k + m * s] = acc;
    }
  }
  std::copy(tmp.begin(), tmp.begin() + n, out);
}
// Forward (sign −1) or unscaled inverse (sign +1) complex FFT of a 2·3·5-smooth length.
std::vector<cd> cfft(const std::vector<cd>& x, int sign) {
  int64_t n = (int64_t)x.size();
  std::vector<cd> w(n), out(n), tmp(n);
  for (int64_t j = 0; j < n; j++) {
    double a = sign * 2 * kPi * (double)j / (double)n;
    w[j] = cd(std::cos(a), std::sin(a));
  }
  dit(x.data(), 1, out.data(), n, w, 1, tmp);
  return out;
}
}  // namespace

bool same_interval(double dt, double plan_dt) { return std::fabs(dt - plan_dt) <= 1e-9 * plan_dt; }

// ----------------------------------------------------------------- lengths
// fft/plan.nim:105-118
bool fast_len(int64_t n) {
  if (n < 1) return false;
  for (int p : {2, 3, 5})
    while (n % p == 0) n /= p;
  return n == 1;
}
int64_t next_fast(int64_t n, bool even) {
  int64_t r = n < 1 ? 1 : n;
  while (!fast_len(r) || (even && (r & 1))) r++;
  return r;
}

// -------------------------------------------------------------- FFT tables
// The device runs Stockham passes of radix 2, 3, 4, 5, 6, 8, 9, 10, 12, 15 or
// 16 (the composite ones as small DFTs in registers). The factorization of m
// minimizes a cost model of a pass on a CTA of `threads`: ceil(butterflies /
// threads) rounds of R elements each, at the small DFT's arithmetic per
// element plus the pass's shared-memory traffic and twiddle multiply.
// The twiddle of output k of butterfly p in a pass of `cur` points is
// exp(−2πi·p·k/cur) (fft/plan.nim:146-155), read from one table of
// exp(−2πi·e/m).
namespace {
double radix_cost(int r) {
  switch (r) {
    case 2: return 2.0;
    case 3: return 5.3;
    case 4: return 4.0;
    case 5: return 6.8;
    case 6: return 6.2;
    case 8: return 6.0;
    case 9: return 8.0;
    case 10: return 7.4;
    case 12: return 7.3;
    case 15: return 8.6;
    case 16: return 7.0;
  }
  return 1e9;
}
std::vector<int> plan_radices(int64_t m, int threads, int max_radix) {
  static const int kRadix[] = {16, 15, 12, 10, 9, 8, 6, 5, 4, 3, 2};
  // best[d] for every divisor d of m: the cheapest passes whose product is d
  std::vector<int64_t> divs;
  for (int64_t d = 1; d * d <= m; d++)
    if (m % d == 0) {
      divs.push_back(d);
      if (d * d != m) divs.push_back(m / d);
    }
  std::sort(divs.begin(), divs.end());
  std::vector<double> best(divs.size(), 1e300);
  std::vector<int> choice(divs.size(), 0);
  auto index = [&](int64_t d) { return (int)(std::lower_bound(divs.begin(), divs.end(), d) - divs.begin()); };
  best[0] = 0;  // d = 1
  for (size_t i = 1; i < divs.size(); i++) {
    int64_t d = divs[i];
    for (int r : kRadix) {
      if (r > max_radix || d % r != 0) continue;
      double bf = (double)(m / r);
      double rounds = std::ceil(bf / threads);
      double pass = rounds * r * (radix_cost(r) + 2.0 + 5.0 * (r - 1) / r + 10.0 / r);
      double c = best[index(d / r)] + pass;
      if (c < best[i] - 1e-9) {
        best[i] = c;
        choice[i] = r;
      }
    }
  }
  std::vector<int> out;
  int64_t d = m;
  while (d > 1) {
    int r = choice[index(d)];
    if (r == 0) throw InvalidArg("no FFT factorization of " + std::to_string(m));
    out.push_back(r);
    d /= r;
  }
  // larger radices first: their passes have the fewest butterflies
  std::sort(out.begin(), out.end(), std::greater<int>());
  return out;
}
}  // namespace

FftTables fft_tables(int64_t n, int max_radix) {
  if (!fast_len(n) || n % 2 != 0) throw InvalidArg("the device FFT needs an even 2·3·5-smooth length, got " + std::to_string(n));
  FftTables t;
  t.n = n;
  t.m = n / 2;
  t.radices = plan_radices(t.m, 256, max_radix);
  // One table for every pass: the twiddle of output k of butterfly p in the
  // pass after radices of product s (cur = m / s points) is
  // ω_cur^{p·k} = ω_m^{p·k·s}, and p·k·s < m.
  for (int64_t e = 0; e < t.m; e++) {
    double a = -2 * kPi * (double)e / (double)t.m;
    t.tw_re.push_back(std::cos(a));
    t.tw_im.push_back(std::sin(a));
  }
  for (int64_t j = 0; j <= t.m; j++) {
    double a = -2 * kPi * (double)j / (double)n;
    t.split_re.push_back(std::cos(a));
    t.split_im.push_back(std::sin(a));
  }
  return t;
}

// ------------------------------------------------------------------ design
namespace {
bool low_cut(const psg_filter_spec& s) { return s.f2 > 0; }
bool high_cut(const psg_filter_spec& s) { return s.f3 < kInf; }
void need(bool ok, const std::string& m) {
  if (!ok) throw InvalidArg(m);
}
// filter/design.nim:103-137
void check_spec_shape(const psg_filter_spec& s) {
  if (s.kind == PSG_RK_TRAPEZOID) {
    need(!(std::isnan(s.f1) || std::isnan(s.f2) || std::isnan(s.f3) || std::isnan(s.f4)), "a corner is NaN");
    if (low_cut(s)) need(s.f1 >= 0 && s.f1 < s.f2, "a low cut needs 0 ≤ f1 < f2 (a sloped ramp), got f1 = " + num(s.f1) + ", f2 = " + num(s.f2));
    else need(s.f1 == 0 && s.f2 == 0, "no low cut needs f1 = f2 = 0");
    if (high_cut(s)) need(s.f3 < s.f4 && s.f4 < kInf, "a high cut needs f3 < f4 < Inf (a sloped ramp), got f3 = " + num(s.f3) + ", f4 = " + num(s.f4));
    else need(s.f4 == kInf, "no high cut needs f3 = f4 = Inf");
    if (low_cut(s) && high_cut(s)) need(s.f2 <= s.f3, "a band-pass needs f2 ≤ f3");
  } else if (s.kind == PSG_RK_BUTTERWORTH) {
    need(s.low_hz >= 0 && s.low_hz < kInf, "a low-cut corner must be finite and ≥ 0 (0: none), got " + num(s.low_hz));
    need(s.high_hz > 0, "a high-cut corner must be > 0 (Inf: none), got " + num(s.high_hz));
    if (s.low_hz > 0) need(s.low_slope > 0 && s.low_slope < kInf, "a slope must be finite and > 0 dB/octave, got " + num(s.low_slope));
    if (s.high_hz < kInf) need(s.high_slope > 0 && s.high_slope < kInf, "a slope must be finite and > 0 dB/octave, got " + num(s.high_slope));
    need(s.low_hz < s.high_hz, "the low-cut corner must be below the high-cut one");
  } else {
    throw InvalidArg("unknown response kind " + std::to_string(s.kind));
  }
  need(s.n_notches >= 0 && s.n_notches <= PSG_MAX_NOTCHES, "at most 8 notches");
  for (int i = 0; i < s.n_notches; i++) {
    need(s.notches[i].freq_hz > 0 && s.notches[i].freq_hz < kInf, "a notch frequency must be finite and > 0, got " + num(s.notches[i].freq_hz));
    need(s.notches[i].width_hz > 0 && s.notches[i].width_hz < kInf, "a notch width must be finite and > 0, got " + num(s.notches[i].width_hz));
  }
}
double tan_warp(double f, double dt_ms) {
  double x = kPi * f * dt_ms / 1000;
  return x >= kPi / 2 ? kInf : std::tan(x);
}
double sin2_ramp(double x) {
  if (x <= 0) return 0.0;
  if (x >= 1) return 1.0;
  double s = std::sin(kPi / 2 * x);
  return s * s;
}
double narrowest(const psg_filter_spec& s) {
  double r = kInf;
  if (s.kind == PSG_RK_TRAPEZOID) {
    if (low_cut(s)) r = std::min(r, s.f2 - s.f1);
    if (high_cut(s)) r = std::min(r, s.f4 - s.f3);
  } else {
    if (s.low_hz > 0) r = std::min(r, s.low_hz * std::min(1.0, 24 / s.low_slope) / 2);
    if (s.high_hz < kInf) r = std::min(r, s.high_hz * std::min(1.0, 24 / s.high_slope) / 2);
  }
  for (int i = 0; i < s.n_notches; i++) r = std::min(r, s.notches[i].width_hz / 2);
  return r;
}
// The bin gains of an FFT of `nfft` points (filter/design.nim:257-265).
std::vector<double> bin_gains(const psg_filter_spec& s, double dt_ms, int64_t nfft) {
  int64_t bins = nfft / 2 + 1;
  std::vector<double> h(bins);
  double df = 1000 / ((double)nfft * dt_ms);
  for (int64_t k = 0; k < bins; k++) h[k] = spec_response(s, (double)k * df, dt_ms);
  if (s.zero_dc && bins > 0) h[0] = 0;
  return h;
}
// The half length holding 99.9 % of the energy of a symmetric impulse whose
// centre sample is `c` (filter/design.nim:288-298).
int64_t half_energy(const std::vector<double>& h, double c) {
  int64_t n = (int64_t)h.size();
  double total = c * c;
  for (int64_t j = 1; j < n; j++) total += h[j] * h[j];
  double e = c * c;
  int64_t L = 0;
  while (e < 0.999 * total && L < n / 2) {
    ++L;
    e += h[L] * h[L] + (n - L != L ? h[n - L] * h[n - L] : 0.0);
  }
  return L;
}
// One feature's impulse length, the longer of H and 1 − H, on a grid grown
// until the impulse fits in an eighth of it (filter/design.nim:300-325).
int64_t feature_len(const psg_filter_spec& s, double dt_ms) {
  const int64_t max_grid = 1 << 24;
  double feat = narrowest(s);
  if (feat == kInf) return 0;
  double start = std::ceil(16 * (1000 / dt_ms) / feat);
  int64_t n = start > (double)max_grid ? max_grid + 1 : next_fast(std::max<int64_t>(64, (int64_t)start));
  while (true) {
    if (n > max_grid)
      throw InvalidArg("the filter's impulse response is longer than " + std::to_string(max_grid / 8) +
                       " samples at " + num(dt_ms) + " ms (narrowest ramp " + num(feat) + " Hz)");
    std::vector<double> g = bin_gains(s, dt_ms, n);
    std::vector<cd> full(n);
    for (int64_t k = 0; k < (int64_t)g.size(); k++) {
      full[k] = g[k];
      if (k > 0 && k < n - k) full[n - k] = g[k];
    }
    std::vector<cd> t = cfft(full, +1);
    std::vector<double> h(n);
    for (int64_t j = 0; j < n; j++) h[j] = t[j].real() / (double)n;
    int64_t L = std::max(half_energy(h, h[0]), half_energy(h, 1 - h[0]));
    if (L <= n / 8) return L;
    n = next_fast(2 * n);
  }
}
}  // namespace

// filter/design.nim:143-173
void validate_spec(const psg_filter_spec& s, double dt_ms) {
  need(dt_ms > 0 && dt_ms < kInf, "dtMs must be finite and > 0, got " + num(dt_ms));
  check_spec_shape(s);
  double nyq = 500 / dt_ms;
  if (s.kind == PSG_RK_TRAPEZOID) {
    if (high_cut(s)) need(!(s.f4 > nyq), "f4 = " + num(s.f4) + " Hz is above Nyquist (" + num(nyq) + " Hz at " + num(dt_ms) + " ms)");
    if (low_cut(s)) need(!(s.f2 >= nyq), "f2 = " + num(s.f2) + " Hz is not below Nyquist (" + num(nyq) + " Hz)");
  } else {
    if (s.high_hz < kInf) need(!(s.high_hz >= nyq), "the high-cut corner " + num(s.high_hz) + " Hz is not below Nyquist (" + num(nyq) + " Hz)");
    need(!(s.low_hz >= nyq), "the low-cut corner " + num(s.low_hz) + " Hz is not below Nyquist (" + num(nyq) + " Hz)");
  }
  for (int i = 0; i < s.n_notches; i++)
    need(!(s.notches[i].freq_hz >= nyq), "a notch at " + num(s.notches[i].freq_hz) + " Hz is not below Nyquist (" + num(nyq) + " Hz)");
}

// filter/design.nim:236-255
double spec_response(const psg_filter_spec& s, double f, double dt_ms) {
  double g = 1.0;
  if (s.kind == PSG_RK_TRAPEZOID) {
    if (low_cut(s)) g *= sin2_ramp((f - s.f1) / (s.f2 - s.f1));
    if (high_cut(s)) g *= 1 - sin2_ramp((f - s.f3) / (s.f4 - s.f3));
  } else {
    double wf = tan_warp(f, dt_ms);
    if (s.low_hz > 0) g *= f <= 0 ? 0.0 : 1 / (1 + std::pow(tan_warp(s.low_hz, dt_ms) / wf, s.low_slope / 6));
    if (s.high_hz < kInf) g *= wf == kInf ? 0.0 : 1 / (1 + std::pow(wf / tan_warp(s.high_hz, dt_ms), s.high_slope / 6));
  }
  for (int i = 0; i < s.n_notches; i++) g *= sin2_ramp(std::fabs(f - s.notches[i].freq_hz) / (s.notches[i].width_hz / 2));
  return g;
}

// filter/design.nim:327-366: each edge and notch measured on its own.
int64_t spec_impulse_length(const psg_filter_spec& s, double dt_ms) {
  validate_spec(s, dt_ms);
  psg_filter_spec flat{};
  flat.kind = PSG_RK_TRAPEZOID;
  flat.f3 = flat.f4 = kInf;
  std::vector<psg_filter_spec> parts;
  if (s.kind == PSG_RK_TRAPEZOID) {
    if (low_cut(s)) { psg_filter_spec a = flat; a.f1 = s.f1; a.f2 = s.f2; parts.push_back(a); }
    if (high_cut(s)) { psg_filter_spec a = flat; a.f3 = s.f3; a.f4 = s.f4; parts.push_back(a); }
  } else {
    psg_filter_spec b{};
    b.kind = PSG_RK_BUTTERWORTH;
    b.low_slope = s.low_slope;
    b.high_slope = s.high_slope;
    if (s.low_hz > 0) { psg_filter_spec a = b; a.low_hz = s.low_hz; a.high_hz = kInf; parts.push_back(a); }
    if (s.high_hz < kInf) { psg_filter_spec a = b; a.low_hz = 0; a.high_hz = s.high_hz; parts.push_back(a); }
  }
  for (int i = 0; i < s.n_notches; i++) {
    psg_filter_spec a = flat;
    a.n_notches = 1;
    a.notches[0] = s.notches[i];
    parts.push_back(a);
  }
  int64_t L = 0;
  for (auto& p : parts) L = std::max(L, feature_len(p, dt_ms));
  return L;
}

// filter/apply.nim:118-151
FilterHost filter_plan(const psg_filter_spec& s, double dt_ms, int64_t samples, int trend, int max_radix) {
  need(samples >= 1, "a filter plan needs samples ≥ 1, got " + std::to_string(samples));
  need(trend >= PSG_TR_NONE && trend <= PSG_TR_LINEAR, "unknown trend removal " + std::to_string(trend));
  validate_spec(s, dt_ms);
  FilterHost f;
  f.spec = s;
  f.trend = trend;
  f.margin = spec_impulse_length(s, dt_ms);
  f.dc_gain = spec_response(s, 0, dt_ms);
  f.reflect = f.dc_gain >= 0.5 || trend != PSG_TR_LINEAR;
  f.pad = f.reflect ? f.margin : std::min(f.margin, samples);
  int64_t n = samples + (f.reflect ? 4 : 2) * f.pad;
  double rmp = narrowest(s);
  if (rmp < kInf && f.pad == f.margin) n = std::max(n, (int64_t)std::ceil(2000 / (rmp * dt_ms)));
  f.nfft = next_fast(n);
  f.gain = bin_gains(s, dt_ms, f.nfft);
  f.fall.resize(f.pad);
  for (int64_t k = 1; k <= f.pad; k++) {
    double c = std::cos(kPi / 2 * (double)k / (double)(f.pad + 1));
    f.fall[k - 1] = c * c;
  }
  f.fft = fft_tables(f.nfft, max_radix);
  return f;
}

// ------------------------------------------------------------- gain curves
// gain/curves.nim:132-160
double gain_factor_at(const psg_gain_curve& c, double t) {
  if (std::isnan(t)) return kNaN;
  if (c.kind == PSG_GC_POWER) return std::pow(std::max(t, c.min_ms) / c.ref_ms, c.power);
  double db;
  if (c.kind == PSG_GC_KNOTS) {
    if (c.n_knots == 0) return kNaN;
    const psg_gain_knot* k = c.knots;
    int n = c.n_knots;
    if (t <= k[0].t_ms) db = k[0].db;
    else if (t >= k[n - 1].t_ms) db = k[n - 1].db;
    else {
      int lo = 0, hi = n - 1;
      while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        (k[mid].t_ms <= t ? lo : hi) = mid;
      }
      double f = (t - k[lo].t_ms) / (k[hi].t_ms - k[lo].t_ms);
      db = k[lo].db + f * (k[hi].db - k[lo].db);
    }
  } else {
    db = c.db_per_s * t / 1000;
  }
  return std::pow(10.0, db / 20);
}
namespace {
void check_curve(const psg_gain_curve& c) {
  if (c.kind == PSG_GC_KNOTS) {
    need(c.n_knots >= 1, "the curve has no knots: build it with knotGain, powerGain or exponentialGain");
    need(c.n_knots <= PSG_MAX_KNOTS, "at most 64 knots");
    for (int i = 0; i < c.n_knots; i++) {
      need(fin(c.knots[i].t_ms) && fin(c.knots[i].db), "knot " + std::to_string(i) + " is not finite");
      if (i > 0) need(c.knots[i].t_ms > c.knots[i - 1].t_ms, "knot times must strictly increase");
    }
  } else if (c.kind == PSG_GC_POWER) {
    need(fin(c.power), "a power must be finite, got " + num(c.power));
    need(fin(c.ref_ms) && c.ref_ms > 0, "refMs must be finite and positive, got " + num(c.ref_ms));
    need(fin(c.min_ms) && c.min_ms > 0, "minMs must be finite and positive, got " + num(c.min_ms));
  } else if (c.kind == PSG_GC_EXPONENTIAL) {
    need(fin(c.db_per_s), "dbPerS must be finite, got " + num(c.db_per_s));
  } else {
    throw InvalidArg("unknown gain curve kind " + std::to_string(c.kind));
  }
}

const char* op_name(int k) {
  static const char* names[] = {"opDemean", "opDetrend", "opScale", "opGainDb", "opClip",
                                "opPolarity", "opMuteTop", "opMuteBottom", "opFilter", "opIir",
                                "opAgc", "opNormalize", "opGainCurve", "opCalibrate", "opUncalibrate"};
  return (k >= 0 && k < 15) ? names[k] : "op?";
}

// gain/gain.nim:272-296
int64_t agc_half(double window_ms, double dt_ms, int64_t samples, double target, double epsilon) {
  need(fin_pos(dt_ms), "dtMs must be finite and positive, got " + num(dt_ms));
  need(samples >= 1 && samples <= 2147483647LL, "an AGC plan needs samples in 1 .. int32.high, got " + std::to_string(samples));
  need(fin_pos(window_ms), "an AGC window must be finite and positive, got " + num(window_ms) + " ms");
  double h = std::round(window_ms / (2 * dt_ms));
  need(h >= 1, "an AGC window of " + num(window_ms) + " ms is under 3 samples at " + num(dt_ms) + " ms");
  need(h <= (double)(1 << 26), "an AGC window of " + num(window_ms) + " ms is too long");
  need(fin_pos(target), "an AGC target must be finite and positive, got " + num(target));
  need(fin_pos(epsilon), "an AGC epsilon must be finite and positive, got " + num(epsilon));
  return (int64_t)h;
}

// timeMute / tableMute / lmoMute (core/mute.nim:55-97): what the builders
// check, for curves that come through the C ABI.
void check_mute(const psg_mute_curve& c) {
  switch (c.kind) {
    case PSG_MK_TIME:
      need(fin(c.t_ms), "a mute time must be finite, got " + num(c.t_ms));
      break;
    case PSG_MK_TABLE:
      need(c.n_knots >= 1, "a mute table needs at least one knot");
      need(c.n_knots <= PSG_MAX_MUTE_KNOTS, "a mute table takes at most " + std::to_string(PSG_MAX_MUTE_KNOTS) + " knots");
      for (int i = 0; i < c.n_knots; i++) {
        need(fin(c.offsets[i]) && c.offsets[i] >= 0, "mute table offsets must be finite and ≥ 0, got " + num(c.offsets[i]));
        need(i == 0 || c.offsets[i] > c.offsets[i - 1], "mute table offsets must be strictly ascending: " +
                                                           num(c.offsets[i > 0 ? i - 1 : 0]) + " is followed by " + num(c.offsets[i]));
        need(fin(c.times_ms[i]), "mute table times must be finite, got " + num(c.times_ms[i]));
      }
      break;
    case PSG_MK_LMO:
      need(fin(c.velocity) && c.velocity > 0, "an LMO mute velocity must be finite and positive, got " + num(c.velocity));
      need(fin(c.t0_ms) && fin(c.pad_ms), "LMO mute times must be finite, got t0Ms " + num(c.t0_ms) + ", padMs " + num(c.pad_ms));
      break;
    default:
      throw InvalidArg("unknown mute kind " + std::to_string(c.kind));
  }
}

// pipeline.nim:392-447
StepHost compile_op(const psg_op& op, int dtype, double dt_ms, int64_t samples, int64_t record, int max_radix) {
  StepHost s;
  switch (op.kind) {
    case PSG_OP_DEMEAN: s.kind = ST_DEMEAN; break;
    case PSG_OP_DETREND: s.kind = ST_DETREND; break;
    case PSG_OP_POLARITY: s.kind = ST_POLARITY; break;
    case PSG_OP_SCALE:
      need(fin(op.factor), "the factor must be finite, got " + num(op.factor));
      need(fin(as_dtype(dtype, op.factor)), "a factor of " + num(op.factor) + " overflows " + (dtype ? "float64" : "float32"));
      s.kind = ST_SCALE;
      s.factor = op.factor;
      break;
    case PSG_OP_GAIN_DB: {
      need(fin(op.factor), "the gain must be finite, got " + num(op.factor) + " dB");
      double f = std::pow(10.0, op.factor / 20);
      need(fin(f) && fin(as_dtype(dtype, f)), "a gain of " + num(op.factor) + " dB overflows " + (dtype ? "float64" : "float32"));
      s.kind = ST_SCALE;
      s.factor = f;
      break;
    }
    case PSG_OP_CLIP:
      need(!(std::isnan(op.lo) || std::isnan(op.hi) || op.lo > op.hi),
           "clip limits must satisfy lo ≤ hi, got " + num(op.lo) + " .. " + num(op.hi));
      s.kind = ST_CLIP;
      s.lo = op.lo;
      s.hi = op.hi;
      break;
    case PSG_OP_FILTER:
      s.kind = ST_FILTER;
      s.filter = filter_plan(op.filter, dt_ms, samples, op.trend, max_radix);
      break;
    case PSG_OP_AGC:
      need(op.agc_mode == PSG_AGC_RMS || op.agc_mode == PSG_AGC_MEAN_ABS, "unknown AGC mode");
      s.kind = ST_AGC;
      s.half = agc_half(op.window_ms, dt_ms, samples, op.target, op.epsilon);
      s.agc_mode = op.agc_mode;
      s.target = op.target;
      s.epsilon = op.epsilon;
      break;
    case PSG_OP_NORMALIZE:
      // gain/gain.nim:153-167
      need(samples >= 1, "a normalize plan needs samples ≥ 1");
      need(fin_pos(op.norm_target), "a normalize target must be finite and positive, got " + num(op.norm_target));
      need(op.percentile >= 0 && op.percentile <= 100, "a percentile must be in 0 .. 100, got " + num(op.percentile));
      need(op.norm_stat >= 0 && op.norm_stat <= 2, "unknown normalization statistic");
      need(op.norm_scope == PSG_PER_TRACE || op.norm_scope == PSG_PER_PANEL, "unknown normalization scope");
      s.kind = op.norm_scope == PSG_PER_PANEL ? ST_NORM_PANEL : ST_NORM_TRACE;
      s.stat = op.norm_stat;
      s.scope = op.norm_scope;
      s.norm_target = op.norm_target;
      s.percentile = op.percentile;
      break;
    case PSG_OP_GAIN_CURVE: {
      // gain/curves.nim:214-247, tabulated over the record (pipeline.nim:441-443)
      check_curve(op.curve);
      double hi = std::isnan(op.t_max_ms) ? op.t_min_ms + (double)(record - 1) * dt_ms : op.t_max_ms;
      need(fin(op.t_min_ms) && fin(hi), "the table limits must be finite, got " + num(op.t_min_ms) + " .. " + num(hi));
      need(!(hi < op.t_min_ms), "tMaxMs " + num(hi) + " is before tMinMs " + num(op.t_min_ms));
      double span = std::floor((hi - op.t_min_ms) / dt_ms + 1e-9);
      need(span < (double)(1 << 26), "a gain table of " + num(span) + " samples is too long");
      s.kind = ST_GAIN_CURVE;
      s.curve = op.curve;
      s.t_min_ms = op.t_min_ms;
      s.table.resize((size_t)span + 1);
      for (size_t k = 0; k < s.table.size(); k++) {
        double t = op.t_min_ms + (double)k * dt_ms;
        double g = gain_factor_at(op.curve, t);
        need(!(std::isinf(as_dtype(dtype, g)) || std::isnan(g)), "the gain at " + num(t) + " ms (" + num(g) + ") overflows");
        s.table[k] = g;
      }
      break;
    }
    case PSG_OP_MUTE_TOP:
    case PSG_OP_MUTE_BOTTOM:
      check_mute(op.mute);
      need(fin(op.taper_ms) && op.taper_ms >= 0, "a mute taper must be finite and ≥ 0 ms, got " + num(op.taper_ms));
      s.kind = op.kind == PSG_OP_MUTE_TOP ? ST_MUTE_TOP : ST_MUTE_BOTTOM;
      s.mute = op.mute;
      s.ms_per_dist = op.mute.kind == PSG_MK_LMO ? 1000 / op.mute.velocity : 0;
      s.taper_ms = op.taper_ms;
      break;
    case PSG_OP_IIR:
      s.kind = ST_IIR;
      s.iir = iir_plan(op.filter, dt_ms, samples, op.iir_phase, op.trend);
      break;
    case PSG_OP_CALIBRATE:
    case PSG_OP_UNCALIBRATE:
      throw InvalidArg("calibration resolves its factors from the SEG-D keys and file scales of a reader, "
                       "which this library does not have: apply resolved per-row factors with scaleRows");
    default:
      throw InvalidArg("unknown op kind " + std::to_string(op.kind));
  }
  return s;
}

std::atomic<uint64_t> g_generation{0};
}  // namespace

// pipeline.nim:466-523
PlanHost compile_plan(const psg_op* ops, int n_ops, int dtype, double dt_ms, int64_t samples,
                      int64_t record_samples, int max_radix) {
  need(dtype == PSG_F32 || dtype == PSG_F64, "dtype must be float32 or float64");
  need(fin(dt_ms) && dt_ms > 0, "dtMs must be finite and positive, got " + num(dt_ms));
  need(samples >= 1, "a pipeline needs samples ≥ 1, got " + std::to_string(samples));
  need(samples <= (1 << 20), "a pipeline takes at most 2²⁰ samples per trace on the device");
  need(record_samples == 0 || record_samples >= samples,
       "recordSamples (" + std::to_string(record_samples) + ") must be 0 or ≥ samples (" + std::to_string(samples) +
           "): it is the length of the traces a window of `samples` is cut from");
  need(n_ops >= 0 && (n_ops == 0 || ops != nullptr), "no ops");
  PlanHost p;
  p.dtype = dtype;
  p.dt_ms = dt_ms;
  p.samples = samples;
  p.record_samples = std::max(samples, record_samples);
  for (int i = 0; i < n_ops; i++) {
    try {
      p.steps.push_back(compile_op(ops[i], dtype, dt_ms, samples, p.record_samples, max_radix));
    } catch (const InvalidArg& e) {
      throw InvalidArg(std::string("op ") + std::to_string(i) + " (" + op_name(ops[i].kind) + "): " + e.what());
    }
  }
  int start = 0;
  for (int i = 0; i < (int)p.steps.size(); i++) {
    p.margin += p.steps[i].margin();
    if (p.steps[i].kind == ST_NORM_PANEL && i > start) {
      p.parts.push_back({start, i});
      start = i;
    }
  }
  p.parts.push_back({start, (int)p.steps.size()});
  p.generation = g_generation.fetch_add(1) + 1;
  return p;
}

// pipeline.nim:525-548
int64_t required_margin(const psg_op* ops, int n_ops, double dt_ms) {
  need(fin(dt_ms) && dt_ms > 0, "dtMs must be finite and positive, got " + num(dt_ms));
  int64_t m = 0;
  for (int i = 0; i < n_ops; i++) {
    try {
      if (ops[i].kind == PSG_OP_FILTER) m += spec_impulse_length(ops[i].filter, dt_ms);
      else if (ops[i].kind == PSG_OP_AGC) m += agc_half(ops[i].window_ms, dt_ms, 1, ops[i].target, ops[i].epsilon);
      else if (ops[i].kind == PSG_OP_IIR) m += iir_plan(ops[i].filter, dt_ms, 1, ops[i].iir_phase, ops[i].trend).pad;
    } catch (const InvalidArg& e) {
      throw InvalidArg(std::string("op ") + std::to_string(i) + " (" + op_name(ops[i].kind) + "): " + e.what());
    }
  }
  return m;
}

// ------------------------------------------------------------- IIR filters
namespace {
// Complex a/b by Smith's method (scaled by the larger part of b).
void cdiv(double ar, double ai, double br, double bi, double& qr, double& qi) {
  if (std::fabs(br) < std::fabs(bi)) {
    double r = br / bi, den = bi + r * br;
    qr = (ar * r + ai) / den;
    qi = (ai * r - ar) / den;
  } else {
    double r = bi / br, den = br + r * bi;
    qr = (ar + r * ai) / den;
    qi = (ai - r * ar) / den;
  }
}
Biquad biquad(double b0, double b1, double b2, double a1, double a2) {
  return Biquad{b0, b1, b2, a1, a2, (b0 + b1 + b2) / (1 + a1 + a2)};
}
// butterSections (filter/iir.nim:113-148): a digital Butterworth low-pass or
// high-pass of `order` poles, −3 dB at fc, by the bilinear transform
// prewarped at fc. The analog prototype's poles are wc·(−sin θ ± i cos θ),
// θ = π(2k + 1)/(2N); each conjugate pair maps to z = (2fs + s)/(2fs − s).
std::vector<Biquad> butter_sections(double fc, double dt_ms, int order, bool high) {
  std::vector<Biquad> out;
  double fs = 1000 / dt_ms;
  double wc = 2 * fs * std::tan(kPi * fc / fs);
  double k2 = 2 * fs;
  for (int k = 0; k < order / 2; k++) {
    double th = kPi * (double)(2 * k + 1) / (double)(2 * order);
    double sr = -wc * std::sin(th), si = wc * std::cos(th);
    double zr, zi;
    cdiv(k2 + sr, si, k2 - sr, -si, zr, zi);
    double a1 = -2 * zr, a2 = zr * zr + zi * zi;
    if (high) {
      double g = (1 - a1 + a2) / 4;  // gain 1 at Nyquist
      out.push_back(biquad(g, -2 * g, g, a1, a2));
    } else {
      double g = (1 + a1 + a2) / 4;  // gain 1 at 0 Hz
      out.push_back(biquad(g, 2 * g, g, a1, a2));
    }
  }
  if (order % 2 == 1) {
    double z = (k2 - wc) / (k2 + wc), a1 = -z;
    if (high) {
      double g = (1 - a1) / 2;
      out.push_back(biquad(g, -g, 0, a1, 0));
    } else {
      double g = (1 + a1) / 2;
      out.push_back(biquad(g, g, 0, a1, 0));
    }
  }
  return out;
}
// causalLength (filter/iir.nim:150-182): the samples after a spike holding
// 99.99 % of the energy of the cascade's causal impulse response h (or of
// δ − h, whichever is longer), h run from rest until its last quarter holds
// under 1e-12 of the energy.
int64_t causal_length(const std::vector<Biquad>& secs) {
  const double frac = 0.9999;
  for (int64_t n = 1024;; n *= 2) {
    std::vector<double> h(n, 0.0);
    h[0] = 1;
    for (const Biquad& c : secs) {
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
    if (tail <= 1e-12 * std::max(rest, 1e-300) || n >= (1 << 24)) {
      int64_t best = 0;
      for (double c0 : {h[0], 1 - h[0]}) {
        double total = c0 * c0 + rest, e = c0 * c0;
        int64_t L = 0;
        while (e < frac * total && L < n - 1) {
          L++;
          e += h[L] * h[L];
        }
        best = std::max(best, L);
      }
      return best;
    }
  }
}
int poles(double slope, double per_pole, const char* side) {
  double n = slope / per_pole;
  need(n >= 1 && n <= 32 && n == std::round(n),
       std::string("the ") + side + " slope of an IIR filter must be a multiple of " + num(per_pole) +
           " dB/octave (" + std::to_string((int)per_pole) + " per pole), 1 .. 32 poles; got " + num(slope));
  return (int)n;
}
}  // namespace

// initIirPlan (filter/iir.nim:193-239)
IirHost iir_plan(const psg_filter_spec& s, double dt_ms, int64_t samples, int phase, int trend) {
  need(samples >= 1, "an IIR plan needs samples ≥ 1, got " + std::to_string(samples));
  need(phase == PSG_IP_ZERO || phase == PSG_IP_MINIMUM, "unknown IIR phase " + std::to_string(phase));
  need(trend >= PSG_TR_NONE && trend <= PSG_TR_LINEAR, "unknown trend removal " + std::to_string(trend));
  validate_spec(s, dt_ms);
  need(s.kind == PSG_RK_BUTTERWORTH,
       "an IIR filter needs a Butterworth spec (butterLowCut, butterHighCut, butterBandPass)");
  need(s.n_notches == 0 && !s.zero_dc, "an IIR filter takes no notches and no 0 Hz suppression");
  IirHost p;
  p.spec = s;
  p.phase = phase;
  p.trend = trend;
  double per_pole = phase == PSG_IP_ZERO ? 12.0 : 6.0;
  std::vector<Biquad> low, high;
  if (s.low_hz > 0) low = butter_sections(s.low_hz, dt_ms, poles(s.low_slope, per_pole, "low-cut"), true);
  if (s.high_hz < kInf) high = butter_sections(s.high_hz, dt_ms, poles(s.high_slope, per_pole, "high-cut"), false);
  p.sections = low;
  p.sections.insert(p.sections.end(), high.begin(), high.end());
  p.pad = phase == PSG_IP_ZERO ? spec_impulse_length(s, dt_ms) : std::max(causal_length(low), causal_length(high));
  // G(1) and G'(1) of the cascade from each section's N(q)/D(q), q = 1/z
  double g = 1, dg = 0;
  for (const Biquad& c : p.sections) {
    double n1 = c.b0 + c.b1 + c.b2, d1 = 1 + c.a1 + c.a2;
    double gi = n1 / d1;
    double dgi = ((c.b1 + 2 * c.b2) * d1 - n1 * (c.a1 + 2 * c.a2)) / (d1 * d1);
    dg = dg * gi + g * dgi;
    g *= gi;
  }
  p.dc_gain = phase == PSG_IP_ZERO ? g * g : g;
  p.dc_slope = phase == PSG_IP_ZERO ? 0.0 : dg;
  p.reflect = std::fabs(p.dc_gain) >= 0.5 || trend != PSG_TR_LINEAR;
  p.lead = p.reflect ? p.pad : 0;
  p.tail = phase == PSG_IP_ZERO ? p.pad : 0;
  return p;
}
// magnitudeAt (filter/iir.nim:268-278): |H| (minimum phase) or |H|² (zero
// phase) at f Hz from the sections.
double iir_magnitude(const IirHost& p, double f, double dt_ms) {
  double w = 2 * kPi * f * dt_ms / 1000;
  double zr = std::cos(w), zi = -std::sin(w);       // z^-1
  double z2r = zr * zr - zi * zi, z2i = 2 * zr * zi;  // z^-2
  double hr = 1, hi = 0;
  for (const Biquad& c : p.sections) {
    double nr = c.b0 + c.b1 * zr + c.b2 * z2r, ni = c.b1 * zi + c.b2 * z2i;
    double dr = 1 + c.a1 * zr + c.a2 * z2r, di = c.a1 * zi + c.a2 * z2i;
    double qr, qi;
    cdiv(nr, ni, dr, di, qr, qi);
    double tr = hr * qr - hi * qi;
    hi = hr * qi + hi * qr;
    hr = tr;
  }
  double a = std::hypot(hr, hi);
  return p.phase == PSG_IP_ZERO ? a * a : a;
}
int iir_order(const IirHost& p) {
  int o = 0;
  for (const Biquad& c : p.sections) o += c.a2 == 0 ? 1 : 2;
  return o;
}

// ---------------------------------------------------------------- spectra
// initSpectrumPlan (fft/spectrum.nim:79-107)
SpectrumHost spectrum_plan(int dtype, double dt_ms, int64_t window, double taper_fraction, int64_t nfft,
                           bool demean, int max_radix) {
  need(dtype == PSG_F32 || dtype == PSG_F64, "dtype must be float32 or float64");
  need(window >= 1, "a spectrum window needs ≥ 1 sample, got " + std::to_string(window));
  need(dt_ms > 0 && dt_ms < kInf, "dtMs must be finite and > 0, got " + num(dt_ms));
  need(taper_fraction >= 0 && taper_fraction <= 0.5, "taperFraction must be in 0 .. 0.5, got " + num(taper_fraction));
  int64_t n = nfft;
  if (n == 0) {
    n = 1;
    while (n < window) n *= 2;  // nextPowerOfTwo
  }
  need(n >= window, "nfft " + std::to_string(n) + " is shorter than the window (" + std::to_string(window) + ")");
  need(fast_len(n), "an FFT length must be 2·3·5-smooth, got " + std::to_string(n));
  need(n <= (1 << 22), "a spectrum FFT of " + std::to_string(n) + " points is too long for the device");
  SpectrumHost p;
  p.dtype = dtype;
  p.dt_ms = dt_ms;
  p.window = window;
  p.nfft = n;
  p.bins = n / 2 + 1;
  p.demean = demean;
  p.odd = (n & 1) != 0;
  p.fft = fft_tables(p.odd ? 2 * n : n, max_radix);
  const int64_t ramp = (int64_t)std::round(taper_fraction * (double)window);
  p.taper.resize(window);
  for (int64_t i = 0; i < window; i++) {
    const int64_t d = std::min(i, window - 1 - i);  // from the nearer end
    double w = 1.0;
    if (d < ramp) {
      double s = std::sin(kPi / 2 * (double)(d + 1) / (double)(ramp + 1));
      w = s * s;
    }
    p.taper[i] = as_dtype(dtype, w);
    p.taper_sum += p.taper[i];
  }
  return p;
}

// --------------------------------------------------------------- vibroseis
namespace {
// vibroseis/kaiser.nim:4-14: I0 by its power series Σ (x²/4)^k / (k!)²,
// stopped once a term is below 1e-17 of the sum (about 70 terms at 50).
double bessel_i0(double x) {
  double term = 1, sum = 1, q = x * x / 4;
  for (int k = 1; k <= 500; k++) {
    term *= q / (double)(k * k);
    sum += term;
    if (term < sum * 1e-17) break;
  }
  return sum;
}
}  // namespace

// vibroseis/taper.nim:69-74: β = 6 (Kaiser), σ = 0.4 (Gaussian), p = 2
// (power); NaN for the shapes without a parameter.
double taper_default_param(int shape) {
  switch (shape) {
    case 6: return 6.0;
    case 7: return 0.4;
    case 8: return 2.0;
    default: return std::nan("");
  }
}

// vibroseis/taper.nim:79-97 (validate): the lengths ≥ 0 and finite or NaN,
// and the shape's parameter (NaN: its default) in range.
void check_taper(double start_ms, double end_ms, int shape, double param) {
  need(shape >= 0 && shape <= 8, "taper shape " + std::to_string(shape) + " is not one of 0 .. 8");
  for (double v : {start_ms, end_ms})
    need(std::isnan(v) || (v >= 0 && v < kInf), "a taper length must be ≥ 0 and finite (or NaN for none), got " + num(v));
  const double p = std::isnan(param) ? taper_default_param(shape) : param;
  if (shape == 6) need(p >= 0 && p <= 50, "a Kaiser taper needs 0 ≤ β ≤ 50, got " + num(p));
  if (shape == 7) need(p > 0 && p < kInf, "a Gaussian taper needs σ > 0, got " + num(p));
  if (shape == 8) need(p > 0 && p < kInf, "a power taper needs an exponent > 0, got " + num(p));
}

// vibroseis/taper.nim:125-145: w(x) on x clamped to [0, 1].
double taper_weight(int shape, double x, double param) {
  const double p = std::isnan(param) ? taper_default_param(shape) : param;
  x = std::min(1.0, std::max(0.0, x));
  switch (shape) {
    case 0: return x;
    case 1: return std::sin(kPi / 2 * x);
    case 2: return 0.5 - 0.5 * std::cos(kPi * x);
    case 3: return 0.54 - 0.46 * std::cos(kPi * x);
    case 4: return 0.42 - 0.5 * std::cos(kPi * x) + 0.08 * std::cos(2 * kPi * x);
    case 5: return 0.35875 - 0.48829 * std::cos(kPi * x) + 0.14128 * std::cos(2 * kPi * x) - 0.01168 * std::cos(3 * kPi * x);
    case 6: { double u = 1 - x; return bessel_i0(p * std::sqrt(std::max(0.0, 1 - u * u))) / bessel_i0(p); }
    case 7: { double u = (1 - x) / p; return std::exp(-0.5 * u * u); }
    case 8: return std::pow(x, p);
    default: throw InvalidArg("taper shape " + std::to_string(shape) + " is not one of 0 .. 8");
  }
}

// vibroseis/taper.nim:147-179 (checkFits, applyTaper) on values of dtype
// held as doubles: each product rounds to dtype, as T(float64(x)·w).
void apply_taper(int dtype, double* x, int64_t n, double dt_ms, double start_ms, double end_ms, int shape,
                 double param) {
  need(dt_ms > 0 && dt_ms < kInf, "dtMs must be finite and positive, got " + num(dt_ms));
  const double sweep_ms = (double)std::max<int64_t>(n, 0) * dt_ms;
  check_taper(start_ms, end_ms, shape, param);
  const double s = std::isnan(start_ms) ? 0.0 : start_ms, e = std::isnan(end_ms) ? 0.0 : end_ms;
  need(!(s + e > sweep_ms * (1 + 1e-9)), "the sweep tapers overlap: " + num(s) + " + " + num(e) +
                                             " ms is longer than the " + num(sweep_ms) + " ms sweep");
  if (s > 0)
    for (int64_t j = 0; j < n && (double)j * dt_ms < s; j++)
      x[j] = as_dtype(dtype, x[j] * taper_weight(shape, (double)j * dt_ms / s, param));
  if (e > 0)
    for (int64_t j = n - 1; j >= 0 && sweep_ms - (double)j * dt_ms < e; j--)
      x[j] = as_dtype(dtype, x[j] * taper_weight(shape, (sweep_ms - (double)j * dt_ms) / e, param));
}

// ------------------------------------------------------------------ sweeps
namespace {
// 20·log10(2)/2: dB per octave of dt/df ∝ f (sweep.nim:234).
const double kOctaveDb = 20 * std::log10(2.0) / 2;
const double kMaxDbPerOctaveTotal = 300, kMaxDbPerHzTotal = 150;

// exp(x) − 1 and ln(1 + x) by Kahan's correction, as sweep.nim:236-246
// writes them (not libm's expm1 / log1p: the phases must match its bits).
double kahan_expm1(double x) {
  double u = std::exp(x);
  if (u == 1) return x;
  if (u - 1 == -1) return -1.0;
  return (u - 1) * x / std::log(u);
}
double kahan_ln1p(double x) {
  double u = 1 + x;
  return u == 1 ? x : std::log(u) * x / (u - 1);
}

void check_freq(double f, double limit, double nyq, const std::string& what) {
  need(f > 0 && f < kInf, what + " must be > 0 Hz, got " + num(f));
  need(!(f > nyq), what + " = " + num(f) + " Hz is above Nyquist (" + num(nyq) + " Hz): it would alias");
  need(!(f > limit * (1 + 1e-12)), what + " = " + num(f) + " Hz is above the anti-alias limit " + num(limit) +
                                       " Hz (maxNyquistFraction · Nyquist); raise maxNyquistFraction to allow it");
}

// The 4-point Gauss–Legendre rule on [−1, 1]: nodes ±√(3/7 ∓ (2/7)√(6/5)),
// weights (18 ± √30)/36, as the decimal values sweep.nim:286-290 holds.
const double kGlNodes[4] = {-0.8611363115940526, -0.3399810435848563, 0.3399810435848563, 0.8611363115940526};
const double kGlWeights[4] = {0.3478548451374538, 0.6521451548625461, 0.6521451548625461, 0.3478548451374538};

// sweep.nim:292-329 (phasesInto): 2π·∫₀ᵗ f in radians, without φ₀.
void sweep_phases(const SweepHost& s, double* phase, int64_t n) {
  const double dt = s.dt_ms / 1000, T = s.length_ms / 1000;
  if (s.law == PSG_SL_LINEAR) {
    const double rate = (s.f2 - s.f1) / T;
    for (int64_t j = 0; j < n; j++) {
      double t = (double)j * dt;
      phase[j] = 2 * kPi * (s.f1 * t + 0.5 * rate * t * t);
    }
  } else if (s.law == PSG_SL_TABLE) {
    // piecewise linear f: the phase is piecewise quadratic, exact per piece
    const auto& tab = s.table;
    double acc = 0;
    size_t i = 1;
    for (int64_t j = 0; j < n; j++) {
      const double tms = (double)j * s.dt_ms;
      while (i < tab.size() - 1 && tab[i].t_ms <= tms) {
        acc += 0.5 * (tab[i - 1].f_hz + tab[i].f_hz) * (tab[i].t_ms - tab[i - 1].t_ms) / 1000;
        i++;
      }
      const psg_sweep_point a = tab[i - 1], b = tab[i];
      const double sec = (std::min(tms, b.t_ms) - a.t_ms) / 1000;
      const double slope = (b.f_hz - a.f_hz) / ((b.t_ms - a.t_ms) / 1000);
      phase[j] = 2 * kPi * (acc + a.f_hz * sec + 0.5 * slope * sec * sec);
    }
  } else {
    double acc = 0;
    if (n > 0) phase[0] = 0;
    for (int64_t j = 1; j < n; j++) {
      const double a = (double)(j - 1) * s.dt_ms, h = 0.5 * s.dt_ms;
      double sum = 0;
      for (int q = 0; q < 4; q++) sum += kGlWeights[q] * sweep_frequency_at(s, a + h + h * kGlNodes[q]);
      acc += sum * h / 1000;
      phase[j] = 2 * kPi * acc;
    }
  }
}
}  // namespace

// sweep.nim:112-119 (sweepLen) with core/types.nim:147-160 (samplesInLength:
// a quotient within 1e-6 of a whole number is that number, else floor).
int64_t sweep_len(const SweepHost& s) {
  if (!(s.dt_ms > 0 && s.dt_ms < kInf)) return 0;
  if (!(s.length_ms > 0 && s.length_ms < kInf)) return 0;
  const double steps = s.length_ms / s.dt_ms;
  if (!(steps >= 1 && steps <= 2147483647.0)) return 0;
  const double r = std::round(steps);
  return std::fabs(steps - r) <= 1e-6 ? (int64_t)r : (int64_t)std::floor(steps);
}

// sweep.nim:132-183 (validate, with checkFreq :123-130 and the taper's
// checkFits, taper.nim:147-158).
void sweep_validate(const SweepHost& s) {
  need(s.dt_ms > 0 && s.dt_ms < kInf, "dtMs must be finite and positive, got " + num(s.dt_ms));
  need(s.length_ms >= s.dt_ms && s.length_ms < kInf, "lengthMs must be at least one sample interval, got " + num(s.length_ms));
  const double steps = s.length_ms / s.dt_ms;
  need(!(steps > 2147483647.0), "a sweep of " + num(s.length_ms) + " ms at " + num(s.dt_ms) + " ms is over 2³¹ samples");
  need(!(std::fabs(steps - std::round(steps)) > 1e-6),
       "lengthMs = " + num(s.length_ms) + " must be a whole number of samples of " + num(s.dt_ms) + " ms");
  need(s.max_nyq > 0 && s.max_nyq <= 1, "maxNyquistFraction must be in (0, 1], got " + num(s.max_nyq));
  need(fin(s.amplitude), "the amplitude must be finite, got " + num(s.amplitude));
  need(fin(s.phase_deg), "startPhaseDeg must be finite, got " + num(s.phase_deg));
  const double nyq = 500 / s.dt_ms, limit = s.max_nyq * nyq;
  check_freq(s.f1, limit, nyq, "f1Hz");
  check_freq(s.f2, limit, nyq, "f2Hz");
  switch (s.law) {
    case PSG_SL_DB_PER_OCTAVE:
    case PSG_SL_DB_PER_HZ: {
      need(fin(s.boost_db), "boostDb must be finite, got " + num(s.boost_db));
      const bool hz = s.law == PSG_SL_DB_PER_HZ;
      const double total = hz ? std::fabs(s.boost_db * (s.f2 - s.f1)) : std::fabs(s.boost_db * std::log2(s.f2 / s.f1));
      const double lim = hz ? kMaxDbPerHzTotal : kMaxDbPerOctaveTotal;
      need(!(total > lim), "a boost of " + num(s.boost_db) + (hz ? " dB/Hz" : " dB/octave") + " from " + num(s.f1) +
                               " to " + num(s.f2) + " Hz adds up to " + num(std::round(10 * total) / 10) +
                               " dB, over the limit of " + num(lim));
      break;
    }
    case PSG_SL_TABLE: {
      const auto& t = s.table;
      need(t.size() >= 2, "a table sweep needs at least two points");
      need(t[0].t_ms == 0, "a sweep table must start at 0 ms, got " + num(t[0].t_ms));
      need(!(std::fabs(t.back().t_ms - s.length_ms) > 1e-9 * s.length_ms),
           "a sweep table must end at lengthMs = " + num(s.length_ms) + ", got " + num(t.back().t_ms));
      for (size_t i = 0; i < t.size(); i++) {
        check_freq(t[i].f_hz, limit, nyq, "the table frequency at " + num(t[i].t_ms) + " ms");
        need(i == 0 || t[i].t_ms > t[i - 1].t_ms,
             "sweep table times must increase: " + num(i ? t[i - 1].t_ms : 0) + " then " + num(t[i].t_ms));
      }
      need(s.f1 == t[0].f_hz && s.f2 == t.back().f_hz, "a table sweep's f1Hz and f2Hz must be its first and last frequencies");
      break;
    }
    case PSG_SL_LINEAR:
    case PSG_SL_EXPONENTIAL: break;
    default: throw InvalidArg("sweep law " + std::to_string(s.law) + " is not one of 0 .. 4");
  }
  check_taper(s.taper_start, s.taper_end, s.taper_shape, s.taper_param);
  const double ts = std::isnan(s.taper_start) ? 0.0 : s.taper_start, te = std::isnan(s.taper_end) ? 0.0 : s.taper_end;
  need(!(ts + te > s.length_ms * (1 + 1e-9)), "the sweep tapers overlap: " + num(ts) + " + " + num(te) +
                                                  " ms is longer than the " + num(s.length_ms) + " ms sweep");
}

// sweep.nim:248-284 (frequencyAt): f1 at 0 and f2 at lengthMs exactly, the
// laws clamped between the two; the spec is assumed valid.
double sweep_frequency_at(const SweepHost& s, double t_ms) {
  const double T = s.length_ms, f1 = s.f1, f2 = s.f2;
  const double x = std::min(std::max(t_ms, 0.0), T) / T;
  if (x <= 0) return f1;
  if (x >= 1) return f2;
  const double lo = std::min(f1, f2), hi = std::max(f1, f2);
  auto within = [&](double f) { return std::min(std::max(f, lo), hi); };
  switch (s.law) {
    case PSG_SL_LINEAR: return within(f1 + (f2 - f1) * x);
    case PSG_SL_EXPONENTIAL: return within(f1 * std::pow(f2 / f1, x));
    case PSG_SL_DB_PER_OCTAVE: {
      // f^m linear in time, written in f2/f1 so that no power of a frequency overflows
      const double m = s.boost_db / kOctaveDb + 1;
      if (std::fabs(m) < 1e-12) return within(f1 * std::pow(f2 / f1, x));
      return within(f1 * std::pow(1 + x * kahan_expm1(m * std::log(f2 / f1)), 1 / m));
    }
    case PSG_SL_DB_PER_HZ: {
      const double k = s.boost_db * std::log(10.0) / 10;  // dt/df ∝ exp(k·f)
      const double e = kahan_expm1(k * (f2 - f1));
      if (std::fabs(k * (f2 - f1)) < 1e-12) return within(f1 + (f2 - f1) * x);
      return within(f1 + kahan_ln1p(x * e) / k);
    }
    default: {
      const double t = std::min(std::max(t_ms, 0.0), T);
      const auto& tab = s.table;
      size_t i = 1;
      while (i < tab.size() - 1 && tab[i].t_ms < t) i++;
      const psg_sweep_point a = tab[i - 1], b = tab[i];
      return a.f_hz + (b.f_hz - a.f_hz) * (t - a.t_ms) / (b.t_ms - a.t_ms);
    }
  }
}

// sweep.nim:436-463 (phaseAt): φ₀ + 2π·∫₀ᵗ f for the laws with a closed
// form; NaN for the boosted ones.
double sweep_phase_at(const SweepHost& s, double t_ms) {
  const double t = std::min(std::max(t_ms, 0.0), s.length_ms) / 1000, T = s.length_ms / 1000;
  const double p0 = s.phase_deg * (kPi / 180);
  switch (s.law) {
    case PSG_SL_LINEAR: return p0 + 2 * kPi * (s.f1 * t + 0.5 * (s.f2 - s.f1) / T * t * t);
    case PSG_SL_EXPONENTIAL: {
      const double r = std::log(s.f2 / s.f1);
      if (std::fabs(r) < 1e-12) return p0 + 2 * kPi * s.f1 * t;
      return p0 + 2 * kPi * s.f1 * T / r * kahan_expm1(r * t / T);
    }
    case PSG_SL_TABLE: {
      double acc = 0;
      const double tm = t * 1000;
      const auto& tab = s.table;
      for (size_t i = 1; i < tab.size(); i++) {
        const psg_sweep_point a = tab[i - 1], b = tab[i];
        if (tm <= b.t_ms) {
          const double sec = (tm - a.t_ms) / 1000;
          const double slope = (b.f_hz - a.f_hz) / ((b.t_ms - a.t_ms) / 1000);
          return p0 + 2 * kPi * (acc + a.f_hz * sec + 0.5 * slope * sec * sec);
        }
        acc += 0.5 * (a.f_hz + b.f_hz) * (b.t_ms - a.t_ms) / 1000;
      }
      return p0 + 2 * kPi * acc;
    }
    default: return kNaN;
  }
}

// sweep.nim:465-473 (segySweepType): 1 linear, 3 exponential (or a dB/octave
// law of −3.0103 dB), 4 other.
int sweep_segy_type(const SweepHost& s) {
  switch (s.law) {
    case PSG_SL_LINEAR: return 1;
    case PSG_SL_EXPONENTIAL: return 3;
    case PSG_SL_DB_PER_OCTAVE: return std::fabs(s.boost_db + kOctaveDb) < 1e-9 ? 3 : 4;
    default: return 4;
  }
}

// sweep.nim:331-342 (sweepInto) and :351-420 (checkHarmonic, taperPrefix,
// sweepHarmonicsInto): n samples of dtype held as doubles, each rounded to
// dtype before the ramps; samples past the sweep are 0.
std::vector<double> sweep_samples(const SweepHost& s, const std::vector<psg_sweep_harmonic>& harmonics, int64_t n,
                                  int dtype) {
  sweep_validate(s);
  need(n >= 1, "a sweep buffer needs at least one sample, got " + std::to_string(n));
  for (const auto& h : harmonics) {
    need(h.order > 0 && h.order < kInf, "a harmonic order must be finite and > 0, got " + num(h.order));
    need(fin(h.amp), "a harmonic amplitude must be finite, got " + num(h.amp));
    need(fin(h.phase_deg), "a harmonic phase must be finite, got " + num(h.phase_deg));
  }
  const int64_t n_sweep = sweep_len(s), m = std::min(n, n_sweep);
  std::vector<double> phase((size_t)m), x((size_t)n, 0.0);
  sweep_phases(s, phase.data(), m);
  const double p0 = s.phase_deg * (kPi / 180), nyq = 500.0 / s.dt_ms;
  for (int64_t j = 0; j < m; j++) {
    const double p = p0 + phase[j];
    double v = 0;
    if (harmonics.empty()) {
      v = std::sin(p);
    } else {
      const double f = sweep_frequency_at(s, (double)j * s.dt_ms);
      for (const auto& h : harmonics)
        if (h.order == 1 || h.order * f < nyq) v += h.amp * std::sin(h.order * p + h.phase_deg * (kPi / 180));
    }
    x[j] = as_dtype(dtype, s.amplitude * v);
  }
  if (n >= n_sweep) {
    apply_taper(dtype, x.data(), n_sweep, s.dt_ms, s.taper_start, s.taper_end, s.taper_shape, s.taper_param);
  } else {
    // the ramps of the whole sweep on its first n samples (taperPrefix)
    const double ts = std::isnan(s.taper_start) ? 0.0 : s.taper_start, te = std::isnan(s.taper_end) ? 0.0 : s.taper_end;
    if (ts > 0)
      for (int64_t j = 0; j < n && (double)j * s.dt_ms < ts; j++)
        x[j] = as_dtype(dtype, x[j] * taper_weight(s.taper_shape, (double)j * s.dt_ms / ts, s.taper_param));
    if (te > 0)
      for (int64_t j = n - 1; j >= 0 && s.length_ms - (double)j * s.dt_ms < te; j--)
        x[j] = as_dtype(dtype, x[j] * taper_weight(s.taper_shape, (s.length_ms - (double)j * s.dt_ms) / te, s.taper_param));
  }
  return x;
}

// vibroseis/correlate.nim:82-160
CorrHost corr_plan(const double* pilot, int64_t plen, double pilot_dt, double pilot_t0, double dt_ms,
                   int64_t record, int64_t out, int mode, double eps_percent, bool normalize, int max_radix) {
  need(plen >= 2, "a pilot needs at least two samples, got " + std::to_string(plen));
  need(pilot_dt > 0 && pilot_dt < kInf, "a pilot's dtMs must be finite and positive");
  need(fin(pilot_t0), "a pilot's t0Ms must be finite, got " + num(pilot_t0));
  double energy = 0;
  for (int64_t i = 0; i < plen; i++) {
    need(fin(pilot[i]), "pilot sample " + std::to_string(i) + " is not finite");
    energy += pilot[i] * pilot[i];
  }
  need(energy != 0, "the pilot is all zeros");
  need(dt_ms > 0 && dt_ms < kInf, "dtMs must be finite and positive, got " + num(dt_ms));
  need(same_interval(pilot_dt, dt_ms), "the pilot is sampled at " + num(pilot_dt) + " ms, the records at " + num(dt_ms) + " ms: resample the pilot first (resamplePilot)");
  need(record >= 1, "recordSamples must be ≥ 1, got " + std::to_string(record));
  int64_t out_n = out == 0 ? record - plen : out;
  need(out_n >= 1, "the pilot (" + std::to_string(plen) + " samples) is not shorter than the record (" + std::to_string(record) + "): no listen time; pass outSamples");
  need(out >= 0 && out_n <= record, "outSamples must be in 0 .. recordSamples, got " + std::to_string(out));
  need(mode == PSG_CM_CORRELATE || mode == PSG_CM_DECONVOLVE, "unknown correlation mode");
  if (mode == PSG_CM_DECONVOLVE) need(eps_percent > 0 && eps_percent < kInf, "epsPercent must be finite and positive, got " + num(eps_percent));
  double s = pilot_t0 / dt_ms;
  need(std::fabs(s) < (double)(record + plen), "the pilot starts " + num(pilot_t0) + " ms from the time break: no lag reaches the output");
  CorrHost c;
  int64_t whole = (int64_t)std::round(s);
  double frac = s - (double)whole;
  c.n = next_fast(record + plen + 64 + std::llabs(whole));
  int64_t bins = c.n / 2 + 1;
  std::vector<cd> x(c.n, cd(0, 0));
  for (int64_t j = 0; j < plen; j++) x[j] = pilot[j];
  std::vector<cd> P = cfft(x, -1);
  double peak_pow = 0;
  for (int64_t k = 0; k < bins; k++) peak_pow = std::max(peak_pow, std::norm(P[k]));
  double eps = mode == PSG_CM_DECONVOLVE ? eps_percent / 100 * peak_pow : 0.0;
  std::vector<double> w(bins);
  double peak = 0;
  for (int64_t k = 0; k < bins; k++) {
    double p2 = std::norm(P[k]);
    w[k] = mode == PSG_CM_DECONVOLVE ? 1 / (p2 + eps) : 1.0;
    double g = p2 * w[k];
    peak += (k == 0 || (c.n % 2 == 0 && k == bins - 1)) ? g : 2 * g;
  }
  peak /= (double)c.n;
  c.scale = normalize ? 1 / peak : 1.0;
  c.mul_re.resize(bins);
  c.mul_im.resize(bins);
  for (int64_t k = 0; k < bins; k++) {
    double th = 2 * kPi * (double)k * frac / (double)c.n;
    cd m = std::conj(P[k]) * (w[k] * c.scale) * cd(std::cos(th), std::sin(th));
    c.mul_re[k] = m.real();
    c.mul_im[k] = m.imag();
  }
  c.mul_im[bins - 1] = 0;  // the inverse takes Nyquist as real
  c.shift = whole;
  c.record = record;
  c.out = out_n;
  c.pilot_len = plen;
  c.dt_ms = dt_ms;
  c.mode = mode;
  c.fft = fft_tables(c.n, max_radix);
  return c;
}

}  // namespace psg
