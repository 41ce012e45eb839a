// A host-side exercise of the plan compiler (processseg_b200/csrc/psg_plan.cpp)
// and the CPU oracle (oracle/psg_oracle.cpp), built by
// tests/test_sanitizers.py with AddressSanitizer and UndefinedBehaviorSanitizer:
// every op kind, both dtypes, valid and invalid parameters, ragged rows,
// spectra, IIR filters, correlation. Exits 0 when every call behaved; a
// sanitizer report ends the process with an error.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "../processseg_b200/csrc/psg_internal.h"

extern "C" {
int orc_plan_compile(const psg_op* ops, int nops, int dtype, double dtMs, int64_t samples, int64_t record, void** out);
void orc_plan_destroy(void* h);
int orc_plan_apply_keyed(void* h, const void* src, void* dst, int64_t rows, int64_t cols, const int32_t* live,
                         const double* startMs, const double* offset, const double* t0, int64_t firstSample,
                         double dtMs, int threads);
int orc_spectrum(int dtype, double dtMs, int64_t windowLen, double taperFraction, int64_t nfft, int demean,
                 const void* b, int64_t rows, int64_t cols, const int32_t* live, int64_t firstCol, int64_t r0,
                 int64_t r1, double* avg, int64_t* used, void* amp, void* phase, int64_t* nfftOut, double* taperSum);
int orc_iir_apply(const psg_filter_spec* spec, double dtMs, int64_t samples, int phase, int trend, double* x,
                  int64_t n);
int orc_correlate(const double* pilot, int64_t plen, double pilotDt, double pilotT0, int dtype, double dtMs,
                  int64_t recordSamples, int64_t outSamples, int mode, double epsPercent, int normalize,
                  const void* src, void* dst, int64_t rows, int64_t cols, const int32_t* live, int64_t* nfft_out,
                  double* scale_out);
}

namespace psg {
void set_error(const std::string&) {}
}

static int failures = 0;
#define CHECK(c)                                                  \
  do {                                                            \
    if (!(c)) {                                                   \
      std::fprintf(stderr, "check failed line %d: %s\n", __LINE__, #c); \
      failures++;                                                 \
    }                                                             \
  } while (0)

static psg_filter_spec trapezoid(double f1, double f2, double f3, double f4) {
  psg_filter_spec s{};
  s.kind = PSG_RK_TRAPEZOID;
  s.f1 = f1, s.f2 = f2, s.f3 = f3, s.f4 = f4;
  s.low_hz = 0, s.high_hz = INFINITY;
  return s;
}
static psg_filter_spec butter(double lo, double hi, double slope) {
  psg_filter_spec s{};
  s.kind = PSG_RK_BUTTERWORTH;
  s.f1 = 0, s.f2 = 0, s.f3 = INFINITY, s.f4 = INFINITY;
  s.low_hz = lo, s.low_slope = slope, s.high_hz = hi, s.high_slope = slope;
  return s;
}
static psg_op op(int kind) {
  psg_op o{};
  o.kind = kind;
  o.trend = PSG_TR_LINEAR;
  o.t_max_ms = NAN;
  o.target = 1;
  o.epsilon = 1e-9;
  o.norm_target = 1;
  o.percentile = 99;
  return o;
}

static std::vector<std::vector<psg_op>> flows() {
  std::vector<std::vector<psg_op>> f;
  psg_op demean = op(PSG_OP_DEMEAN), bp = op(PSG_OP_FILTER), agc = op(PSG_OP_AGC), nrm = op(PSG_OP_NORMALIZE);
  bp.filter = trapezoid(4, 8, 60, 80);
  agc.window_ms = 300;
  nrm.norm_stat = PSG_NORM_PERCENTILE;
  f.push_back({demean, bp, agc});
  f.push_back({demean, bp, agc, nrm});
  psg_op panel = nrm;
  panel.norm_scope = PSG_PER_PANEL;
  f.push_back({bp, panel, agc});
  psg_op iir = op(PSG_OP_IIR);
  iir.filter = butter(4, 60, 24);
  psg_op iirm = iir;
  iirm.iir_phase = PSG_IP_MINIMUM;
  iirm.trend = PSG_TR_MEAN;
  f.push_back({iir, agc});
  f.push_back({demean, iirm});
  psg_op top = op(PSG_OP_MUTE_TOP), bottom = op(PSG_OP_MUTE_BOTTOM);
  top.mute.kind = PSG_MK_LMO;
  top.mute.velocity = 2000;
  top.taper_ms = 30;
  bottom.mute.kind = PSG_MK_TABLE;
  bottom.mute.n_knots = 3;
  double offs[3] = {0, 1000, 3000}, times[3] = {2500, 3200, 5000};
  std::memcpy(bottom.mute.offsets, offs, sizeof(offs));
  std::memcpy(bottom.mute.times_ms, times, sizeof(times));
  bottom.taper_ms = 60;
  f.push_back({top, bp, bottom});
  psg_op gc = op(PSG_OP_GAIN_CURVE);
  gc.curve.kind = PSG_GC_POWER;
  gc.curve.power = 2;
  gc.curve.ref_ms = 1000;
  gc.curve.min_ms = 10;
  psg_op clip = op(PSG_OP_CLIP);
  clip.lo = -2, clip.hi = 2;
  f.push_back({op(PSG_OP_DETREND), bp, gc, clip, op(PSG_OP_POLARITY)});
  return f;
}

int main() {
  std::mt19937_64 rng(5);
  std::normal_distribution<double> nd(0, 1);
  // the host plan compiler, valid and invalid
  for (auto& fl : flows()) {
    for (int dtype : {PSG_F32, PSG_F64})
      for (int64_t n : {(int64_t)1, (int64_t)2, (int64_t)7, (int64_t)500, (int64_t)2001}) {
        try {
          psg::PlanHost p = psg::compile_plan(fl.data(), (int)fl.size(), dtype, 2.0, n, 0, dtype ? 8 : 12);
          CHECK(!p.parts.empty());
        } catch (const psg::InvalidArg&) {
        }
      }
    try {
      (void)psg::required_margin(fl.data(), (int)fl.size(), 2.0);
    } catch (const psg::InvalidArg&) {
    }
  }
  for (double dt : {0.0, -1.0, (double)NAN, 2.0})
    for (int64_t n : {(int64_t)0, (int64_t)-3, (int64_t)10}) {
      auto fl = flows()[0];
      try {
        psg::compile_plan(fl.data(), (int)fl.size(), PSG_F32, dt, n, 0, 12);
        CHECK(dt == 2.0 && n == 10);
      } catch (const psg::InvalidArg&) {
      }
    }
  for (double slope : {12.0, 18.0, 24.0, 48.0, 400.0})
    for (int ph : {PSG_IP_ZERO, PSG_IP_MINIMUM}) {
      try {
        psg::IirHost h = psg::iir_plan(butter(3, 80, slope), 2.0, 1000, ph, PSG_TR_LINEAR);
        CHECK(psg::iir_order(h) > 0);
        CHECK(std::isfinite(psg::iir_magnitude(h, 30, 2.0)));
      } catch (const psg::InvalidArg&) {
      }
    }
  for (int64_t w : {(int64_t)1, (int64_t)2, (int64_t)3, (int64_t)257, (int64_t)501, (int64_t)4000})
    for (int64_t nfft : {(int64_t)0, (int64_t)375, (int64_t)4096}) {
      try {
        psg::SpectrumHost s = psg::spectrum_plan(PSG_F32, 2.0, w, 0.1, nfft, true, 12);
        CHECK(s.bins == s.nfft / 2 + 1);
      } catch (const psg::InvalidArg&) {
      }
    }
  // the oracle on ragged rows with keys
  const int64_t rows = 9, cols = 700;
  std::vector<double> x64(rows * cols);
  for (auto& v : x64) v = nd(rng);
  std::vector<float> x32(x64.begin(), x64.end());
  std::vector<int32_t> live = {700, 0, 1, 2, 350, 699, 700, 17, 500};
  std::vector<double> start(rows, 0.0), offset(rows), t0(rows, 0.0);
  for (int64_t r = 0; r < rows; r++) offset[r] = 100.0 * (double)r;
  offset[3] = NAN;
  for (auto& fl : flows())
    for (int dtype : {PSG_F32, PSG_F64}) {
      void* h = nullptr;
      if (orc_plan_compile(fl.data(), (int)fl.size(), dtype, 2.0, cols, 0, &h) != 0) continue;
      std::vector<double> d64(rows * cols);
      std::vector<float> d32(rows * cols);
      const void* src = dtype ? (const void*)x64.data() : (const void*)x32.data();
      void* dst = dtype ? (void*)d64.data() : (void*)d32.data();
      CHECK(orc_plan_apply_keyed(h, src, dst, rows, cols, live.data(), start.data(), offset.data(), t0.data(), 3, 2.0,
                                 2) == 0);
      orc_plan_destroy(h);
    }
  for (int dtype : {PSG_F32, PSG_F64}) {
    std::vector<double> avg(2049);
    int64_t used = 0, nf = 0;
    double sw = 0;
    const void* src = dtype ? (const void*)x64.data() : (const void*)x32.data();
    CHECK(orc_spectrum(dtype, 2.0, 300, 0.2, 0, 1, src, rows, cols, live.data(), 5, 0, rows - 1, avg.data(), &used,
                       nullptr, nullptr, &nf, &sw) == 0);
    std::vector<double> amp(rows * (nf / 2 + 1)), ph(rows * (nf / 2 + 1));
    std::vector<float> amp32(amp.size()), ph32(ph.size());
    CHECK(orc_spectrum(dtype, 2.0, 300, 0.2, 0, 1, src, rows, cols, live.data(), 5, 0, -1, nullptr, nullptr,
                       dtype ? (void*)amp.data() : (void*)amp32.data(), dtype ? (void*)ph.data() : (void*)ph32.data(),
                       nullptr, nullptr) == 0);
  }
  psg_filter_spec bs = butter(2, 90, 24);
  std::vector<double> tr(x64.begin(), x64.begin() + 700);
  CHECK(orc_iir_apply(&bs, 2.0, 700, PSG_IP_ZERO, PSG_TR_LINEAR, tr.data(), 700) == 0);
  std::vector<double> pilot(300);
  for (int j = 0; j < 300; j++) pilot[j] = std::sin(0.05 * j * (1 + j * 0.01));
  std::vector<float> cout_(rows * 400);
  int64_t nf = 0;
  double sc = 0;
  CHECK(orc_correlate(pilot.data(), 300, 2.0, 0.0, PSG_F32, 2.0, cols, 400, PSG_CM_CORRELATE, 1.0, 1, x32.data(),
                      cout_.data(), rows, cols, live.data(), &nf, &sc) == 0);
  std::printf("sanitized harness: %d failures\n", failures);
  return failures == 0 ? 0 : 1;
}
