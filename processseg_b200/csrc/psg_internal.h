// psg_internal.h — shared by the host plan compiler (psg_plan.cpp) and the
// device side (psg_cuda.cu) of libpsgcuda.so. Not part of the public ABI.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/psg.h"

namespace psg {

// A ValueError of the reference: an invalid op, plan, shape or interval.
struct InvalidArg : std::runtime_error {
  explicit InvalidArg(const std::string& m) : std::runtime_error(m) {}
};
// An AssertionDefect of the reference: a workspace not reserved for the plan.
struct WorkspaceError : std::runtime_error {
  explicit WorkspaceError(const std::string& m) : std::runtime_error(m) {}
};
// Admission refused: the work needs more device memory than it may hold.
struct NoMemory : std::runtime_error {
  explicit NoMemory(const std::string& m) : std::runtime_error(m) {}
};
struct CudaError : std::runtime_error {
  explicit CudaError(const std::string& m) : std::runtime_error(m) {}
};

void set_error(const std::string& m);

// ------------------------------------------------------------------- lengths
bool fast_len(int64_t n);
int64_t next_fast(int64_t n, bool even = true);

// ------------------------------------------------------------------ FFT plan
// The complex FFT of length m that a real FFT of length n = 2m runs: the
// Stockham passes (radix per pass, first pass first) and their twiddles,
// generated in float64. The device reads the twiddles as T.
struct FftTables {
  int64_t n = 0, m = 0;
  std::vector<int> radices;
  std::vector<double> tw_re, tw_im;       // exp(−2πi·e/m), e < m
  std::vector<double> split_re, split_im; // exp(−2πik/n), k = 0 .. m
};
FftTables fft_tables(int64_t n, int max_radix = 16);

// --------------------------------------------------------------- filter plan
struct FilterHost {
  psg_filter_spec spec{};
  int trend = PSG_TR_LINEAR;
  int64_t margin = 0, pad = 0, nfft = 0;
  bool reflect = false;
  double dc_gain = 0;
  std::vector<double> gain;  // nfft/2 + 1 bins
  std::vector<double> fall;  // pad values
  FftTables fft;
};
void validate_spec(const psg_filter_spec& s, double dt_ms);
double spec_response(const psg_filter_spec& s, double f_hz, double dt_ms);
int64_t spec_impulse_length(const psg_filter_spec& s, double dt_ms);
FilterHost filter_plan(const psg_filter_spec& s, double dt_ms, int64_t samples, int trend, int max_radix = 16);

// ------------------------------------------------------------- IIR filters
// A second-order section in transposed direct form II (a0 = 1) and its gain
// at 0 Hz, g = (b0 + b1 + b2)/(1 + a1 + a2).
struct Biquad {
  double b0, b1, b2, a1, a2, g;
};
struct IirHost {
  psg_filter_spec spec{};
  std::vector<Biquad> sections;  // low-cut (high-pass) sections, then high-cut
  int phase = PSG_IP_ZERO, trend = PSG_TR_LINEAR;
  int64_t pad = 0, lead = 0, tail = 0;  // requiredMargin; padded samples before and after
  bool reflect = false;  // odd-reflection pads and steady-state starts (else zeros, from rest)
  double dc_gain = 1, dc_slope = 0;
};
IirHost iir_plan(const psg_filter_spec& s, double dt_ms, int64_t samples, int phase, int trend);
double iir_magnitude(const IirHost& p, double f_hz, double dt_ms);
int iir_order(const IirHost& p);

// ---------------------------------------------------------------- the plan
enum StepKind {
  ST_DEMEAN = 0, ST_DETREND, ST_SCALE, ST_CLIP, ST_POLARITY, ST_FILTER, ST_AGC,
  ST_NORM_TRACE, ST_NORM_PANEL, ST_GAIN_CURVE, ST_MUTE_TOP, ST_MUTE_BOTTOM, ST_IIR
};

struct StepHost {
  int kind = 0;
  double factor = 0, lo = 0, hi = 0;
  FilterHost filter;
  // AGC
  int64_t half = 0;
  int agc_mode = 0;
  double target = 1, epsilon = 1e-9;
  // normalize
  int stat = 0, scope = 0;
  double norm_target = 1, percentile = 99;
  // gain curve
  psg_gain_curve curve{};
  std::vector<double> table;
  double t_min_ms = 0;
  // mutes (core/mute.nim): the curve, 1000/velocity of an LMO mute, the taper
  psg_mute_curve mute{};
  double ms_per_dist = 0, taper_ms = 0;
  // IIR filter
  IirHost iir;
  int64_t margin() const {
    return kind == ST_FILTER ? filter.margin : (kind == ST_AGC ? half : (kind == ST_IIR ? iir.pad : 0));
  }
};

struct PlanHost {
  int dtype = PSG_F32;
  double dt_ms = 0;
  int64_t samples = 0, record_samples = 0, margin = 0;
  uint64_t generation = 0;
  std::vector<StepHost> steps;
  std::vector<std::pair<int, int>> parts;  // [a, b)
};

PlanHost compile_plan(const psg_op* ops, int n_ops, int dtype, double dt_ms, int64_t samples,
                      int64_t record_samples, int max_radix = 12);
int64_t required_margin(const psg_op* ops, int n_ops, double dt_ms);
double gain_factor_at(const psg_gain_curve& c, double t_ms);
bool same_interval(double dt, double plan_dt);

// --------------------------------------------------------------- spectra
// SpectrumPlan (fft/spectrum.nim:79-107): a window of `window` samples,
// tapered and zero-padded to nfft. The device FFT is complex: of nfft/2
// points over sample pairs for an even nfft (then the real-FFT split), of
// nfft points over the samples for an odd one.
struct SpectrumHost {
  int dtype = PSG_F32;
  double dt_ms = 0;
  int64_t window = 0, nfft = 0, bins = 0;
  bool demean = true, odd = false;
  std::vector<double> taper;  // the weights, rounded to T
  double taper_sum = 0;       // Σ of the T weights, in float64
  FftTables fft;
};
SpectrumHost spectrum_plan(int dtype, double dt_ms, int64_t window, double taper_fraction, int64_t nfft,
                           bool demean, int max_radix);

// ----------------------------------------------------------- correlation
struct CorrHost {
  int64_t n = 0, shift = 0, record = 0, out = 0, pilot_len = 0;
  double dt_ms = 0, scale = 1;
  int mode = 0;
  std::vector<double> mul_re, mul_im;
  FftTables fft;
};
CorrHost corr_plan(const double* pilot, int64_t plen, double pilot_dt, double pilot_t0, double dt_ms,
                   int64_t record, int64_t out, int mode, double eps_percent, bool normalize, int max_radix = 16);
// vibroseis/sweep.nim: a SweepSpec with its taper inline.
struct SweepHost {
  int law = PSG_SL_LINEAR;
  double f1 = 0, f2 = 0, length_ms = 0, dt_ms = 0, boost_db = 0;
  std::vector<psg_sweep_point> table;
  double phase_deg = 0, amplitude = 1;
  double taper_start = 0, taper_end = 0, taper_param = 0;
  int taper_shape = 0;
  double max_nyq = 0.8;
};
int64_t sweep_len(const SweepHost& s);
void sweep_validate(const SweepHost& s);
double sweep_frequency_at(const SweepHost& s, double t_ms);
double sweep_phase_at(const SweepHost& s, double t_ms);
int sweep_segy_type(const SweepHost& s);
std::vector<double> sweep_samples(const SweepHost& s, const std::vector<psg_sweep_harmonic>& harmonics, int64_t n,
                                  int dtype);
double taper_default_param(int shape);
void check_taper(double start_ms, double end_ms, int shape, double param);
double taper_weight(int shape, double x, double param);
void apply_taper(int dtype, double* x, int64_t n, double dt_ms, double start_ms, double end_ms, int shape,
                 double param);

}  // namespace psg
