/*
 * psg.h — C ABI of libpsgcuda.so, the B200 (sm_100a) implementation of
 * processSEG's compiled-pipeline hot path.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, returns a
 * `psg_status` and never throws or aborts. After a non-zero status,
 * `psg_last_error` gives the message of the calling thread's last failure.
 * PSG_EINVAL mirrors the reference's ValueError and is returned before any
 * sample changes; PSG_EWORKSPACE mirrors its AssertionDefect for a workspace
 * that was not reserved for the plan. Data never fails: NaN and Inf stay in
 * their own row, as in the reference.
 *
 * Reference interfaces (paths within xrfez/processSEG v0.14.1) that each
 * declaration replaces are cited beside it.
 */
#ifndef PSG_H
#define PSG_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
typedef enum psg_status {
  PSG_OK = 0,
  PSG_EINVAL = 1,     /* ValueError: bad op, plan, shape, interval, width    */
  PSG_EWORKSPACE = 2, /* AssertionDefect: workspace not reserved for the plan */
  PSG_ENOMEM = 3,     /* device memory or admission refused                  */
  PSG_ETIMEOUT = 4,   /* a bounded wait ran out                              */
  PSG_ECUDA = 5,      /* a CUDA call failed (message has the CUDA error)     */
  PSG_ENODEV = 6,     /* no usable sm_100 device                             */
  PSG_ECANCELED = 7   /* a served request was cancelled before it started    */
} psg_status;

/* ------------------------------------------------------------- enumerations
 * The numbering follows the reference's enums so that ops built in any host
 * language keep their meaning.                                             */
typedef enum psg_dtype { PSG_F32 = 0, PSG_F64 = 1 } psg_dtype;

/* OpKind, src/processSEG/pipeline.nim:92-108 */
typedef enum psg_op_kind {
  PSG_OP_DEMEAN = 0, PSG_OP_DETREND = 1, PSG_OP_SCALE = 2, PSG_OP_GAIN_DB = 3,
  PSG_OP_CLIP = 4, PSG_OP_POLARITY = 5, PSG_OP_MUTE_TOP = 6,
  PSG_OP_MUTE_BOTTOM = 7, PSG_OP_FILTER = 8, PSG_OP_IIR = 9, PSG_OP_AGC = 10,
  PSG_OP_NORMALIZE = 11, PSG_OP_GAIN_CURVE = 12, PSG_OP_CALIBRATE = 13,
  PSG_OP_UNCALIBRATE = 14
} psg_op_kind;

/* TrendRemoval, src/processSEG/filter/edges.nim:9-14 */
typedef enum psg_trend { PSG_TR_NONE = 0, PSG_TR_MEAN = 1, PSG_TR_LINEAR = 2 } psg_trend;
/* ResponseKind, src/processSEG/filter/design.nim:69-72 */
typedef enum psg_response_kind { PSG_RK_TRAPEZOID = 0, PSG_RK_BUTTERWORTH = 1 } psg_response_kind;
/* AgcMode, src/processSEG/gain/gain.nim:92-95 */
typedef enum psg_agc_mode { PSG_AGC_RMS = 0, PSG_AGC_MEAN_ABS = 1 } psg_agc_mode;
/* NormStat / NormScope, src/processSEG/gain/gain.nim:72-81 */
typedef enum psg_norm_stat { PSG_NORM_MAX = 0, PSG_NORM_RMS = 1, PSG_NORM_PERCENTILE = 2 } psg_norm_stat;
typedef enum psg_norm_scope { PSG_PER_TRACE = 0, PSG_PER_PANEL = 1 } psg_norm_scope;
/* GainCurveKind, src/processSEG/gain/curves.nim:65-69 */
typedef enum psg_curve_kind { PSG_GC_KNOTS = 0, PSG_GC_POWER = 1, PSG_GC_EXPONENTIAL = 2 } psg_curve_kind;
/* Trace status as ChunkMeta.isLive reads it, src/processSEG/core/types.nim:221-224 */
typedef enum psg_trace_status {
  PSG_TS_UNKNOWN = 0, PSG_TS_LIVE = 1, PSG_TS_DEAD = 2, PSG_TS_AUX = 3
} psg_trace_status;
/* CorrelationMode, src/processSEG/vibroseis/correlate.nim:61-64 */
typedef enum psg_corr_mode { PSG_CM_CORRELATE = 0, PSG_CM_DECONVOLVE = 1 } psg_corr_mode;
/* FoldNorm of stackInto, src/processSEG/vibroseis/vstack.nim:439 */
typedef enum psg_fold_norm { PSG_FN_NONE = 0, PSG_FN_FOLD = 1, PSG_FN_SQRT_FOLD = 2 } psg_fold_norm;

#define PSG_MAX_NOTCHES 8
#define PSG_MAX_KNOTS 64

/* ------------------------------------------------------------ op descriptors
 * FilterSpec, src/processSEG/filter/design.nim:78-91 (notches inline).      */
typedef struct psg_notch { double freq_hz, width_hz; } psg_notch;
typedef struct psg_filter_spec {
  int32_t kind;       /* psg_response_kind */
  int32_t zero_dc;    /* withZeroDc */
  int32_t n_notches;
  int32_t _pad;
  double f1, f2, f3, f4;                          /* trapezoid corners, Hz */
  double low_hz, low_slope, high_hz, high_slope;  /* Butterworth */
  psg_notch notches[PSG_MAX_NOTCHES];
} psg_filter_spec;

/* GainCurve, src/processSEG/gain/curves.nim:71-80 (knots inline). */
typedef struct psg_gain_knot { double t_ms, db; } psg_gain_knot;
typedef struct psg_gain_curve {
  int32_t kind;       /* psg_curve_kind */
  int32_t n_knots;
  double power, ref_ms, min_ms, db_per_s;
  psg_gain_knot knots[PSG_MAX_KNOTS];
} psg_gain_curve;

/* MuteCurve, src/processSEG/core/mute.nim:37-49 (table knots inline). A
 * time mute: t_ms on every trace. A table: |offset| knots (finite, ≥ 0,
 * strictly ascending) and their times, linear between and flat beyond. An
 * LMO mute: t0_ms + |offset|·1000/velocity + pad_ms. */
typedef enum psg_mute_kind { PSG_MK_TIME = 0, PSG_MK_TABLE = 1, PSG_MK_LMO = 2 } psg_mute_kind;
#define PSG_MAX_MUTE_KNOTS 64
typedef struct psg_mute_curve {
  int32_t kind;       /* psg_mute_kind */
  int32_t n_knots;
  double t_ms;                          /* time */
  double velocity, t0_ms, pad_ms;       /* LMO */
  double offsets[PSG_MAX_MUTE_KNOTS];   /* table */
  double times_ms[PSG_MAX_MUTE_KNOTS];
} psg_mute_curve;

/* IirPhase, src/processSEG/filter/iir.nim:76-80 */
typedef enum psg_iir_phase { PSG_IP_ZERO = 0, PSG_IP_MINIMUM = 1 } psg_iir_phase;

/* Op, src/processSEG/pipeline.nim:117-174, as one plain struct: the fields a
 * kind does not use are ignored. */
typedef struct psg_op {
  int32_t kind;        /* psg_op_kind */
  int32_t trend;       /* filter and IIR filter: psg_trend */
  double factor;       /* scale: factor; gain dB: dB */
  double lo, hi;       /* clip */
  psg_filter_spec filter;
  double window_ms, target, epsilon;  /* agc */
  int32_t agc_mode;    /* psg_agc_mode */
  int32_t norm_stat;   /* psg_norm_stat */
  int32_t norm_scope;  /* psg_norm_scope */
  int32_t iir_phase;   /* IIR filter: psg_iir_phase */
  double norm_target, percentile;     /* normalize */
  psg_gain_curve curve;
  double t_min_ms, t_max_ms;          /* gain curve table span (NaN: record end) */
  psg_mute_curve mute;                /* top and bottom mutes */
  double taper_ms;                    /* mute taper on the muted side */
} psg_op;

/* The trace keys a mute reads (ChunkMeta.keys, src/processSEG/core/types.nim:
 * 206-214, with the window origin): per row its offset and t0Ms (arrays of
 * `rows` doubles; NaN: unknown, and a mute that needs it leaves the row
 * alone; a NULL array reads as all NaN) and the block's first sample of the
 * trace (ChunkMeta.firstSample). */
typedef struct psg_keys {
  const double* offset;
  const double* t0_ms;
  int32_t first_sample;
  int32_t _pad;
} psg_keys;

/* ------------------------------------------------------------------ handles */
typedef struct psg_plan psg_plan;           /* PipelinePlan[T]                 */
typedef struct psg_workspace psg_workspace; /* Workspace (a device arena)      */
typedef struct psg_corr_plan psg_corr_plan; /* CorrelationPlan[T]              */
typedef struct psg_stack psg_stack;         /* RecordStack[T], rsVertical      */

/* The calling thread's last error message (empty after success). */
const char* psg_last_error(void);
/* Selects and checks the device (sm_100 required). */
int psg_init(int device);
/* Library version string. */
const char* psg_version(void);

/* --------------------------------------------------------- lengths / margins */
/* isFastLen / nextFastLen, src/processSEG/fft/plan.nim:105-118 */
int psg_is_fast_len(int64_t n);
int64_t psg_next_fast_len(int64_t n, int even);
/* impulseLength, src/processSEG/filter/design.nim:353-366 */
int psg_impulse_length(const psg_filter_spec* spec, double dt_ms, int32_t* out);
/* response, src/processSEG/filter/design.nim:236-255 */
int psg_response(const psg_filter_spec* spec, double f_hz, double dt_ms, double* out);
/* initIirPlan, src/processSEG/filter/iir.nim:193-239, on the host: the
 * cascade's order (poles of one pass), requiredMargin and gain at 0 Hz
 * (G(1), or G(1)² for zero phase) of a Butterworth spec (any pointer may be
 * NULL). PSG_EINVAL for what initIirPlan rejects. */
int psg_iir_design(const psg_filter_spec* spec, double dt_ms, int32_t samples, int32_t phase,
                   int32_t trend, int32_t* order, int32_t* margin, double* dc_gain);
/* IirPlan.magnitudeAt, src/processSEG/filter/iir.nim:268-278: |H| (minimum
 * phase) or |H|² (zero phase) at n frequencies (host arrays). */
int psg_iir_magnitude(const psg_filter_spec* spec, double dt_ms, int32_t phase,
                      const double* f_hz, int32_t n, double* out);
/* Pipeline.requiredMargin, src/processSEG/pipeline.nim:525-548 */
int psg_required_margin(const psg_op* ops, int32_t n_ops, double dt_ms, int32_t* out);
/* decodeWindow, src/processSEG/pipeline.nim:550-560: out[0..1] = first, last */
void psg_decode_window(int64_t shown_first, int64_t shown_last, int64_t margin,
                       int64_t trace_len, int64_t* out);

/* --------------------------------------------------------------- plans */
/* compile, src/processSEG/pipeline.nim:466-523. Uploads the plan's tables to
 * the current device once. A trace is processed in one CTA's shared memory;
 * when its FFT or AGC work areas do not fit beside it there, they go to
 * per-CTA slices of global memory held by the workspace (the plan's
 * psg_plan_workspace_bytes counts them). A trace itself longer than shared
 * memory holds (about 56,000 float32 or 28,000 float64 samples) is
 * PSG_EINVAL. PSG_WIDE=1 in the environment lays out any plan that way. */
int psg_plan_compile(const psg_op* ops, int32_t n_ops, int32_t dtype, double dt_ms,
                     int32_t samples, int32_t record_samples, psg_plan** out);
void psg_plan_destroy(psg_plan* plan);
/* requiredMargin / generation / samples / recordSamples / partCount,
 * src/processSEG/pipeline.nim:562-647 */
int32_t psg_plan_margin(const psg_plan* plan);
uint64_t psg_plan_generation(const psg_plan* plan);
int32_t psg_plan_samples(const psg_plan* plan);
int32_t psg_plan_record_samples(const psg_plan* plan);
int32_t psg_plan_part_count(const psg_plan* plan);
/* partNeedsPanel, src/processSEG/pipeline.nim:649-654: 1 when part `part`
 * starts with a per-panel normalization, else 0 (also for no such part). */
int32_t psg_plan_part_needs_panel(const psg_plan* plan, int32_t part);
/* 1 when the plan mutes: it is applied with its rows' keys (the _keyed
 * entry points; the others refuse it with PSG_EINVAL). */
int32_t psg_plan_needs_keys(const psg_plan* plan);
/* ------------------------------------------------------------ launch tuning
 * A float32 part of exactly demean, filter (zero pads), AGC (and a per-trace
 * normalization) whose transform length has compile-time builds runs on the
 * trace kernel. Its launch shapes: each build (the reference's FFT stages
 * grouped into passes one way, a register budget, a CTA width), with or
 * without the next row's copy in flight, on a persistent grid or one CTA
 * per row. Every shape gives the same bits. The first apply of such a part
 * at a row count of a new class (the count's bit length) times every shape
 * on the call's own input into a scratch block, each timed launch after a
 * write of twice the L2's size has flushed that input from it (waiting for
 * the stream once), and keeps the fastest for that class; PSG_TUNE=0 in the environment at
 * compile keeps the first shape, and so does an apply under stream capture
 * before the class is tuned. No counterpart in the reference, whose FFT plan
 * has one factorization per length (fft/plan.nim:120-160). */
/* The number of launch shapes of part `part` (0 when the part runs on
 * pipeline_kernel or does not exist). */
int32_t psg_plan_trace_shapes(const psg_plan* plan, int32_t part);
/* Pins part `part` to launch shape `shape` for every row count (-1 unpins:
 * the tuner's choices apply again). PSG_EINVAL for a part without shapes or
 * a shape out of range. */
int psg_plan_pin_trace(psg_plan* plan, int32_t part, int32_t shape);
/* The launch shapes and the tuner's record as JSON, written into buf (cap
 * bytes with the terminating NUL, truncated to fit); *needed (when not
 * NULL) gets the full length + 1. {"parts": [{"part", "pinned", "shapes":
 * [{"m", "threads", "min_blocks", "passes", "prefetch", "grid",
 * "ctas_per_sm", "smem"}]}], "tuned": [{"part", "class", "rows", "us",
 * "choice"}]}. */
int psg_plan_tuning(const psg_plan* plan, char* buf, int64_t cap, int64_t* needed);
int32_t psg_plan_len(const psg_plan* plan);
/* For step i of the plan: its FFT length (0 for steps without one) and the
 * pad laid out each side (FilterPlan.nfft / pad, filter/apply.nim:161-164). */
int32_t psg_plan_step_nfft(const psg_plan* plan, int32_t step);
int32_t psg_plan_step_margin(const psg_plan* plan, int32_t step);
/* Scratch bytes of device memory the plan needs for `rows` rows
 * (WorkspaceSize, src/processSEG/pipeline.nim:599-602), with the global
 * work areas of a plan with long traces. */
int64_t psg_plan_workspace_bytes(const psg_plan* plan, int64_t rows, int32_t cols);

/* --------------------------------------------------------------- workspace */
/* initWorkspace / reserve, src/processSEG/core/workspace.nim:50-96: a
 * grow-only device arena, plus pinned host staging for the host-pointer
 * entry points. One per thread (or stream) of callers. */
int psg_workspace_create(psg_workspace** out);
void psg_workspace_destroy(psg_workspace* ws);
/* Grows ws for `plan` applied to up to `rows` rows (and the staging of a
 * host-memory apply `cols` wide); with plan NULL, for the statistics of up to
 * `rows` rows (psg_panel_stats; panelStatsWorkspace, gain/stats.nim:57-58). */
int psg_workspace_reserve(psg_workspace* ws, const psg_plan* plan, int64_t rows,
                          int32_t cols);
int64_t psg_workspace_bytes(const psg_workspace* ws);

/* --------------------------------------------------------------- rows
 * ChunkMeta flattened (isLive, liveSamples, sampleTimeMs,
 * src/processSEG/core/types.nim:212-240) into two per-row arrays on the host:
 * live[r] = the samples to process (0: the row is not processed) and
 * start_ms[r] = the time of column 0 (NaN when unknown). mode 0 is the
 * processing rule (live or unknown status, not failed); mode 1 the
 * correlation rule (not dead, not failed: auxiliary rows are correlated,
 * src/processSEG/vibroseis/correlate.nim:442-443); mode 2 every row that is
 * not failed (scaleRows, core/calibrate.nim:575-581); mode 3 the processing
 * rule of mode 0 with the rows it does not take marked −1, so that a live row
 * with no live samples (0) stays apart from a row that is not live
 * (traceStatsInto, src/processSEG/gain/stats.nim:186-199). `t0_ms` may be
 * NULL (NaN). */
int psg_rows_flatten(const int32_t* status, const int32_t* num_samples,
                     const double* t0_ms, int64_t rows, int32_t first_sample,
                     double dt_ms, const int64_t* failed, int64_t n_failed,
                     int32_t cols, int32_t mode, int32_t* live_out,
                     double* start_ms_out);

/* checkApply, src/processSEG/pipeline.nim:619-641: the checks psg_apply
 * makes before touching a sample, without any device work: a compiled plan,
 * src (NULL: in place) and dst of rows × cols not overlapping unless they
 * are the same block, dt_ms the plan's interval (relative 1e-9), cols at
 * most the plan's samples. PSG_EINVAL with the reference's message. */
int psg_check_apply(const psg_plan* plan, const void* src, const void* dst, int64_t rows,
                    int32_t cols, double dt_ms);
/* --------------------------------------------------------------- apply
 * apply(plan, src, dst, meta, ws), src/processSEG/pipeline.nim:736-772.
 * Device pointers; `src` NULL (or equal to `dst`) runs in place. `live` and
 * `start_ms` are device arrays of `rows` values (psg_rows_flatten). `dt_ms`
 * is the rows' interval (ChunkMeta.dtMs), checked against the plan with
 * sameInterval. Rows that are not live, and samples past a row's live
 * length, are copied unchanged from src. Asynchronous on `stream`
 * (a cudaStream_t; NULL: the legacy default stream). */
int psg_apply(const psg_plan* plan, psg_workspace* ws, const void* src, void* dst,
              int64_t rows, int32_t cols, const int32_t* live, const double* start_ms,
              double dt_ms, void* stream);
/* psg_apply with the rows' trace keys (device arrays), which a plan with
 * mutes needs: the mute column of row r is (t − t0_ms[r])/dt_ms −
 * first_sample, t the curve's time at offset[r] (core/mute.nim:209-214). */
int psg_apply_keyed(const psg_plan* plan, psg_workspace* ws, const void* src, void* dst,
                    int64_t rows, int32_t cols, const int32_t* live, const double* start_ms,
                    const psg_keys* keys, double dt_ms, void* stream);
/* The same from and to host memory (pinned memory overlaps best): the
 * host→device copy of src, live and start_ms, the apply, and the
 * device→host copy of dst, all on `stream`; returns after dst is written. */
int psg_apply_host(const psg_plan* plan, psg_workspace* ws, const void* src_host,
                   void* dst_host, int64_t rows, int32_t cols, const int32_t* live_host,
                   const double* start_ms_host, double dt_ms, void* stream);
/* psg_apply_host with the rows' trace keys (host arrays). */
int psg_apply_host_keyed(const psg_plan* plan, psg_workspace* ws, const void* src_host,
                         void* dst_host, int64_t rows, int32_t cols, const int32_t* live_host,
                         const double* start_ms_host, const psg_keys* keys_host, double dt_ms,
                         void* stream);
/* psg_apply_host_keyed without waiting: returns once the copies and kernels
 * are queued on the workspace's streams (after the work already queued on
 * `stream`); psg_workspace_sync returns when they are done. Consecutive
 * calls on one workspace overlap (one panel's copies out with the next
 * one's copies in): the host arrays of a call (src, dst, live, start_ms,
 * keys) must stay valid and unchanged until psg_workspace_sync, and pinned
 * memory is what overlaps. */
int psg_apply_host_async(const psg_plan* plan, psg_workspace* ws, const void* src_host,
                         void* dst_host, int64_t rows, int32_t cols, const int32_t* live_host,
                         const double* start_ms_host, const psg_keys* keys_host, double dt_ms,
                         void* stream);
int psg_workspace_sync(psg_workspace* ws);

/* Parts API, src/processSEG/pipeline.nim:643-723: the per-panel factor of a
 * part (NaN: the block is left alone) over the whole block, on the device;
 * `factor_out` is a device double. */
int psg_panel_factor(const psg_plan* plan, psg_workspace* ws, int32_t part,
                     const void* block, int64_t rows, int32_t cols, const int32_t* live,
                     double* factor_out, void* stream);
/* runPart, src/processSEG/pipeline.nim:690-723: the steps of part `part` on
 * the rows of dst (copied from `src` first when it is not NULL: the first
 * part of a src → dst apply only). For a part that starts with a per-panel
 * normalization, `factor` is a device double (from psg_panel_factor or
 * psg_panel_factor_from) that scales the live rows first; NaN or NULL
 * leaves them alone. Checks as psg_apply (checkApply). */
int psg_run_part(const psg_plan* plan, psg_workspace* ws, int32_t part, const void* src,
                 void* dst, int64_t rows, int32_t cols, const int32_t* live,
                 const double* start_ms, double dt_ms, const double* factor, void* stream);
/* psg_run_part with the rows' trace keys (device arrays). */
int psg_run_part_keyed(const psg_plan* plan, psg_workspace* ws, int32_t part, const void* src,
                       void* dst, int64_t rows, int32_t cols, const int32_t* live,
                       const double* start_ms, const psg_keys* keys, double dt_ms,
                       const double* factor, void* stream);

/* A panel split by traces over several devices (or calls): the per-panel
 * factor of panelFactor (src/processSEG/gain/gain.nim:221-240, over
 * panelStats, gain/stats.nim:253-304) from statistics that merge.
 * psg_panel_partials writes, for this shard's rows, PSG_PANEL_PARTIAL_DOUBLES
 * device doubles: [0] Σx², [1] samples, [2] rows (over the usable rows: live,
 * finite, Σx² not overflowing), [3] maxAbs, then 65536 histogram counts of
 * the float32 bits of |x| >> 15 (exact integers; zeros unless the part's
 * statistic is a percentile). Shards merge by summing every entry except
 * [3], which takes the maximum (two all-reduces over the ranks).
 * psg_panel_factor_from turns merged partials into the factor (a device
 * double). One shard's partials give the same factor, bit for bit, as
 * psg_panel_factor over that shard. */
#define PSG_PANEL_PARTIAL_HEAD 4
#define PSG_PANEL_PARTIAL_DOUBLES (PSG_PANEL_PARTIAL_HEAD + 65536)
int psg_panel_partials(const psg_plan* plan, psg_workspace* ws, int32_t part,
                       const void* block, int64_t rows, int32_t cols, const int32_t* live,
                       double* partial, void* stream);
int psg_panel_factor_from(const psg_plan* plan, psg_workspace* ws, int32_t part,
                          const double* partial, double* factor_out, void* stream);

/* appliedResponseInto, src/processSEG/pipeline.nim:840-880 (responseModuli,
 * pipeline.nim:774-838): the response of the flow `ops` as applied. A unit
 * impulse at sample samples / 2 of one live row (t0 = 0) runs through the
 * compiled plan on the device, with every filter's trend removal set to
 * PSG_TR_NONE (the caller's ops are not changed); gain[i] (host) receives
 * |sum_j x[j] exp(-2 pi i hz[i] j dt)| of that output, in float64 on the
 * device. hz and gain are host arrays of n_hz doubles. Compiles a plan and
 * allocates the impulse row on every call; ws is grown to the plan when it
 * does not already hold it. PSG_EINVAL when the flow does not compile.
 * Synchronous, on a stream of its own (after the workspace's queued host
 * applies). */
int psg_applied_response(const psg_op* ops, int32_t n_ops, int32_t dtype, double dt_ms,
                         int32_t samples, const double* hz, int32_t n_hz, double* gain,
                         psg_workspace* ws);

/* ------------------------------------------------------------ graph replay
 * One psg_apply_keyed call (device pointers) captured into a CUDA graph for
 * replay (the "CUDA-graph replay" of the batched path; no counterpart in the
 * reference, whose apply is a CPU call): psg_graph_launch then runs the same
 * apply on `stream` with one host call instead of the checks and per-part
 * launches. The checks run once, at capture (PSG_EINVAL / PSG_EWORKSPACE as
 * psg_apply). The graph keeps the call's pointers: the plan, the workspace
 * (not grown while the graph lives), src, dst and the row arrays must stay
 * valid, and their contents are read at each launch. */
typedef struct psg_graph psg_graph;
int psg_graph_capture(const psg_plan* plan, psg_workspace* ws, const void* src, void* dst,
                      int64_t rows, int32_t cols, const int32_t* live, const double* start_ms,
                      const psg_keys* keys, double dt_ms, psg_graph** out);
int psg_graph_launch(psg_graph* graph, void* stream);
void psg_graph_destroy(psg_graph* graph);

/* ----------------------------------------------------------- statistics */
/* traceStatsInto, src/processSEG/gain/stats.nim:186-199: rms and maxAbs per
 * row into device arrays of `rows` doubles. `live` is psg_rows_flatten's
 * mode 3 (on the device): a row with live[r] < 0 is not live and reads NaN
 * for both; a live row reads the statistics of its first min(live[r], cols)
 * samples, (0, 0) when it has none (statsOf, stats.nim:124-127). PSG_EINVAL
 * for a dtype other than PSG_F32 or PSG_F64. */
int psg_trace_stats(const void* block, int32_t dtype, int64_t rows, int32_t cols,
                    const int32_t* live, double* rms_out, double* max_abs_out,
                    void* stream);
/* panelStats, src/processSEG/gain/stats.nim:253-304. out (device) receives
 * {rms, maxAbs, clip, rows, samples} as doubles. clip_percentile NaN skips
 * the histogram. `live` is psg_rows_flatten's mode 3 (on the device): rows
 * with live[r] < 0 are not live and left out; a live row with no live
 * samples (0) counts among `rows` and adds no samples, as in the reference.
 * PSG_EINVAL for a dtype other than PSG_F32 or PSG_F64. */
int psg_panel_stats(psg_workspace* ws, const void* block, int32_t dtype, int64_t rows,
                    int32_t cols, const int32_t* live, double clip_percentile,
                    double* out, void* stream);

/* panelStats without allocating: the same computation and output as
 * psg_panel_stats, for callers that cannot call cudaMalloc, such as a
 * viewer's frame loop that reads display-gain statistics every frame from
 * inside a fixed device-memory budget, or code that must not allocate on a
 * stream it shares with other work. No counterpart in the reference (its
 * panelStats takes a Workspace the caller grew beforehand).
 * Its scratch is a fixed array inside the library, about 1.25 MiB, that every
 * GPU which loads the library holds until the process exits; it takes at
 * most PSG_STATIC_MAX_ROWS rows (PSG_EINVAL beyond). The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress): make
 * that first call before any stream capture. Every call shares the one
 * array and it keeps the last call's contents, so calls that overlap on the
 * GPU (on different streams, or from different host threads) race: order
 * them on one stream. The cached address does not survive a device reset
 * (cudaDeviceReset): do not call this again on a device after resetting it. */
#define PSG_STATIC_MAX_ROWS 65536
int psg_panel_stats_static(const void* block, int32_t dtype, int64_t rows, int32_t cols,
                           const int32_t* live, double clip_percentile, double* out,
                           void* stream);

/* ------------------------------------------------------------- spectra */
/* SpectrumPlan, src/processSEG/fft/spectrum.nim:79-107: windows of
 * window_len samples at dt_ms, demeaned (demean != 0) and tapered over
 * taper_fraction of each end (a sin² ramp), zero-padded to nfft (0: the
 * next power of two of the window). PSG_EINVAL for what initSpectrumPlan
 * rejects. */
typedef struct psg_spectrum_plan psg_spectrum_plan;
int psg_spectrum_plan_create(int32_t dtype, double dt_ms, int32_t window_len, double taper_fraction,
                             int32_t nfft, int32_t demean, psg_spectrum_plan** out);
void psg_spectrum_plan_destroy(psg_spectrum_plan* plan);
/* nfft, bins (nfft/2 + 1), the window length and Σ of its taper weights. */
int psg_spectrum_plan_info(const psg_spectrum_plan* plan, int32_t* nfft, int32_t* bins,
                           int32_t* window_len, double* taper_sum);
/* averageAmplitudeInto, fft/spectrum.nim:267-416: the power-averaged
 * amplitude spectrum of the window first_col ..< first_col + window_len of
 * the live rows row0 .. row1 (clipped to the block) of a device block:
 * sqrt(mean over the rows of |X[k]|²/Σw²)·(2, or 1 at 0 Hz and Nyquist).
 * Rows with no live sample past first_col, or a NaN or infinite sample in
 * the window, are left out. amp: device, bins doubles (zeros when no row
 * counts); used (device int64, may be NULL): the rows averaged. The
 * workspace's spectrum scratch grows on the first call that needs it.
 * Asynchronous on `stream`. */
int psg_spectrum_average(const psg_spectrum_plan* plan, psg_workspace* ws, const void* block,
                         int64_t rows, int32_t cols, const int32_t* live, double dt_ms,
                         int32_t first_col, int64_t row0, int64_t row1, double* amp,
                         int64_t* used, void* stream);
/* amplitudeInto, fft/spectrum.nim:283-300, for every row of a device
 * block: its window (up to its live end) to the scaled amplitude
 * |X[k]|·sides/Σw and the phase atan2(Im, Re) from the window's first
 * sample, into device arrays of rows × bins values of the plan's dtype (a
 * row without samples in the window gets NaN amplitudes). */
int psg_spectrum_amplitude(const psg_spectrum_plan* plan, psg_workspace* ws, const void* block,
                           int64_t rows, int32_t cols, const int32_t* live, double dt_ms,
                           int32_t first_col, void* amp, void* phase, void* stream);

/* ------------------------------------------------------- per-row scale */
/* scaleRows / scaleRowsInto, src/processSEG/core/calibrate.nim:562-612 (the
 * scaling `calibrate` does with its resolved per-row factors): row r of src
 * times T(factors_host[r]) over its first live[r] samples into dst (src NULL
 * or dst: in place), the rest of dst copied from src. live from
 * psg_rows_flatten mode 2 (every row but the failed ones, to its live
 * length). A NaN factor fills the row's live samples with NaN; an infinite
 * one (also in float32) is PSG_EINVAL before any sample changes. Device
 * blocks; returns when the factors' staging in the workspace is free. */
int psg_scale_rows(psg_workspace* ws, int32_t dtype, const void* src, void* dst, int64_t rows,
                   int32_t cols, const int32_t* live, const double* factors_host, void* stream);

/* --------------------------------------------------------------- SEG-Y */
/* The decode a reader does before the path (parseSEG's trace reading, which
 * the reference does not vendor), on the device: `rows` raw trace records
 * of record_bytes each (device memory), a header of header_bytes (240 for
 * SEG-Y) and then `samples` samples of data sample format `format` (SEG-Y
 * rev 2 codes 1 IBM float, 2 int32, 3 int16, 5 IEEE float32, 6 IEEE
 * float64, 7 int24, 8 int8, 10 uint32, 11 uint16, 15 uint24, 16 uint8),
 * big-endian unless little_endian, into a device block of out_cols columns
 * of dtype (zeros past `samples`). Each value converts exactly to float64
 * first, then rounds to dtype. Asynchronous on `stream`. */
int psg_segy_decode(const void* records, int64_t rows, int64_t record_bytes, int32_t header_bytes,
                    int32_t samples, int32_t format, int32_t little_endian, int32_t dtype,
                    void* out, int32_t out_cols, void* stream);
/* The trace-header keys of the same records (SEG-Y rev 2 trace header):
 * status from the trace identification code (bytes 29-30: 1 live, 2 dead,
 * 0 unknown, others auxiliary), offset (37-40), t0 = the delay recording
 * time in ms (109-110), the number of samples (115-116) and the sample
 * interval in µs (117-118). Device arrays of `rows` values; any may be
 * NULL. */
int psg_segy_keys(const void* records, int64_t rows, int64_t record_bytes, int32_t little_endian,
                  int32_t* status, int32_t* num_samples, double* interval_us, double* offset,
                  double* t0_ms, void* stream);

/* ----------------------------------------------------------- vibroseis */
/* Sweep taper shapes (TaperShape, src/processSEG/vibroseis/taper.nim:46-58):
 * 0 linear, 1 cosine, 2 cos², 3 Hamming, 4 Blackman, 5 Blackman–Harris,
 * 6 Kaiser (param β, default 6), 7 Gaussian (σ in ramp lengths, default 0.4),
 * 8 power (exponent p, default 2). A NaN param takes the shape's default. */
enum psg_taper_shape {
  PSG_TP_LINEAR = 0, PSG_TP_COSINE = 1, PSG_TP_COS2 = 2, PSG_TP_HAMMING = 3,
  PSG_TP_BLACKMAN = 4, PSG_TP_BLACKMAN_HARRIS = 5, PSG_TP_KAISER = 6,
  PSG_TP_GAUSSIAN = 7, PSG_TP_POWER = 8
};
/* taperWeight, src/processSEG/vibroseis/taper.nim:125-145: the ramp w(x) of
 * `shape` at x clamped to [0, 1]. The parameter is not validated, as in the
 * reference; an unknown shape is PSG_EINVAL. */
int psg_taper_weight(int32_t shape, double x, double param, double* out);
/* applyTaper, src/processSEG/vibroseis/taper.nim:160-179 (with validate and
 * checkFits, :79-158): ramps of start_ms and end_ms (0 or NaN: none) applied
 * in place to n host samples of dtype whose sample j is at j·dt_ms; each
 * product rounds to dtype. PSG_EINVAL, with nothing written, for a dt_ms
 * that is not finite and positive, a bad length or parameter, or ramps
 * longer than n·dt_ms together. */
int psg_apply_taper(int32_t dtype, void* x, int64_t n, double dt_ms, double start_ms,
                    double end_ms, int32_t shape, double param);
/* Sweep laws (SweepLaw, src/processSEG/vibroseis/sweep.nim:68-74): the
 * instantaneous frequency from f1 at 0 to f2 at length_ms, linear in time,
 * with the amplitude spectrum boosted by boost_db per octave or per Hz,
 * exponential in time, or piecewise linear through a table. */
enum psg_sweep_law {
  PSG_SL_LINEAR = 0, PSG_SL_DB_PER_OCTAVE = 1, PSG_SL_DB_PER_HZ = 2,
  PSG_SL_EXPONENTIAL = 3, PSG_SL_TABLE = 4
};
/* SweepPoint, sweep.nim:76-79. */
typedef struct psg_sweep_point {
  double t_ms;
  double f_hz;
} psg_sweep_point;
/* SweepSpec, sweep.nim:81-94 (the taper's fields inline). A table sweep's
 * f1_hz / f2_hz / length_ms are its first and last points' (tableSweep,
 * sweep.nim:221-232); the table is borrowed for the call. */
typedef struct psg_sweep {
  int32_t law;                  /* psg_sweep_law */
  int32_t taper_shape;          /* psg_taper_shape */
  double f1_hz, f2_hz, length_ms, dt_ms;
  double boost_db;              /* dB per octave or per Hz */
  const psg_sweep_point* table; /* PSG_SL_TABLE only */
  int64_t n_table;
  double start_phase_deg, amplitude;
  double taper_start_ms, taper_end_ms, taper_param;
  double max_nyquist_fraction;  /* 0.8 in the reference's builders */
} psg_sweep;
/* SweepHarmonic, sweep.nim:96-103: amp · sin(order·φ + phase_deg in rad). */
typedef struct psg_sweep_harmonic {
  double order, amp, phase_deg;
} psg_sweep_harmonic;

/* validate, sweep.nim:132-183 (with the taper's checkFits): PSG_EINVAL and
 * the reference's message for an invalid spec. */
int psg_sweep_validate(const psg_sweep* spec);
/* sweepLen, sweep.nim:112-119: lengthMs / dtMs in whole samples; 0 for a
 * length or interval that validate refuses. */
int psg_sweep_len(const psg_sweep* spec, int64_t* n);
/* frequencyAt, sweep.nim:248-284 (t_ms clamped to 0 .. length_ms); phaseAt,
 * sweep.nim:436-463 (NaN for the two boosted laws, which have no closed
 * form). The spec is validated first. */
int psg_sweep_frequency_at(const psg_sweep* spec, double t_ms, double* out);
int psg_sweep_phase_at(const psg_sweep* spec, double t_ms, double* out);
/* sweepInto / sweepHarmonicsInto, sweep.nim:292-434: n host samples of dtype
 * (n_harmonics 0 and n = sweepLen: the sweep alone; a longer buffer is the
 * sweep followed by zeros, a shorter one its first n samples). The phase is
 * in float64: closed form for the linear and table laws, 4-point
 * Gauss–Legendre per sample interval for the others; each sample rounds to
 * dtype before the ramps. SEG-Y sweep type (segySweepType, :465-473) in
 * *segy_type when it is not NULL. */
int psg_sweep_samples(const psg_sweep* spec, const psg_sweep_harmonic* harmonics,
                      int32_t n_harmonics, int32_t dtype, void* out, int64_t n,
                      int32_t* segy_type);
/* linearSweep + sweepSamples (a psg_sweep of PSG_SL_LINEAR through
 * psg_sweep_samples). `out` is host memory of *n_out values of dtype (NULL:
 * just report the length). */
int psg_linear_sweep(double f1_hz, double f2_hz, double length_ms, double dt_ms,
                     double taper_start_ms, double taper_end_ms, int32_t taper_shape,
                     double taper_param, double start_phase_deg, double amplitude,
                     double max_nyquist_fraction, int32_t dtype, void* out,
                     int64_t* n_out);
/* initCorrelationPlan, src/processSEG/vibroseis/correlate.nim:82-160: the
 * pilot (host samples of pilot_dtype) spectrum in float64, the multiplier
 * stored as dtype on the device. */
int psg_corr_plan_create(const void* pilot, int32_t pilot_dtype, int64_t pilot_len,
                         double pilot_dt_ms, double pilot_t0_ms, int32_t dtype,
                         double dt_ms, int32_t record_samples, int32_t out_samples,
                         int32_t mode, double eps_percent, int32_t normalize,
                         psg_corr_plan** out);
void psg_corr_plan_destroy(psg_corr_plan* plan);
int32_t psg_corr_plan_nfft(const psg_corr_plan* plan);
int32_t psg_corr_plan_out_samples(const psg_corr_plan* plan);
double psg_corr_plan_scale(const psg_corr_plan* plan);
/* correlateInto (block form), src/processSEG/vibroseis/correlate.nim:421-464:
 * device src [rows, cols ≤ recordSamples], dst [rows, outSamples]; `live`
 * from psg_rows_flatten mode 1 (0: a zero row). */
int psg_correlate(const psg_corr_plan* plan, const void* src, void* dst, int64_t rows,
                  int32_t cols, const int32_t* live, double dt_ms, void* stream);

/* RecordStack rsVertical, src/processSEG/vibroseis/vstack.nim:118-471:
 * float64 sums and int32 counts on the device. */
int psg_stack_create(int64_t rows, int32_t samples, double dt_ms, psg_stack** out);
void psg_stack_destroy(psg_stack* st);
int psg_stack_clear(psg_stack* st, void* stream);
/* addRecord: rows of `block` (device, dtype) with live[r] > 0 into output
 * row row_map[r] (device int32; NULL: r; < 0: skipped); a row with a
 * non-finite sample is skipped. */
int psg_stack_add(psg_stack* st, const void* block, int32_t dtype, int64_t rows,
                  int32_t cols, const int32_t* live, const int32_t* row_map,
                  void* stream);
/* correlateInto fused with addRecord: each correlated row is also added to
 * the stack in one launch. `live` selects the rows to correlate (mode 1);
 * `stack_live` (device, NULL: outSamples for every row) the samples of each
 * correlated row to add (0: not added; addRecord adds live rows only, mode
 * 0 with cols = outSamples); row_map as psg_stack_add. `dst` may be NULL
 * when only the stack is wanted. */
int psg_correlate_stack(const psg_corr_plan* plan, psg_stack* st, const void* src,
                        void* dst, int64_t rows, int32_t cols, const int32_t* live,
                        const int32_t* stack_live, const int32_t* row_map, double dt_ms,
                        void* stream);
/* stackInto, src/processSEG/vibroseis/vstack.nim:439-471: dst device
 * [rows, samples] of dtype. */
int psg_stack_result(const psg_stack* st, void* dst, int32_t dtype, int32_t norm,
                     void* stream);
/* foldInto: counts, device int32 [rows, samples]. */
int psg_stack_fold(const psg_stack* st, int32_t* dst, void* stream);

/* ------------------------------------------------------------- serving
 * A request loop for a viewer (the reference's viewer loop,
 * tests/utils/viewersim.nim:155-200, calls pool.apply per stale entry; here
 * requests from any thread are batched on the GPU as they arrive). Requests
 * are admitted by device footprint into a fixed arena of `arena_bytes`,
 * copied in, run in batches, and copied out, so the copies of one request
 * overlap the kernels of others. In a batch, the float32 single-part
 * requests run together: one launch of the batched pipeline kernel for the
 * plans without a trace kernel (each trace with its own request's plan and
 * width), one launch of each transform length's batched trace kernel for
 * the others; requests of any other plan (a per-panel normalization, whose
 * factor comes from the request's own rows; float64; IIR filters; mutes;
 * traces too long for shared memory) run after them with the plain apply's
 * launches. A batch starts when none is running, or beside running ones
 * when the requests ready for it hold at least four rows per SM (up to four
 * batches at once, each on its own streams). Results equal psg_apply_host's
 * (psg_apply's for device buffers) bit for bit. */
typedef struct psg_server psg_server;
int psg_server_create(int device, int64_t arena_bytes, psg_server** out);
void psg_server_destroy(psg_server* server);
/* Queues a request (host buffers; pinned memory overlaps best). Returns
 * PSG_ENOMEM when the request alone needs more than the arena holds. The plan
 * and the buffers must stay valid until psg_wait returns. */
int psg_submit(psg_server* server, const psg_plan* plan, const void* src_host, void* dst_host,
               int64_t rows, int32_t cols, const int32_t* live_host,
               const double* start_ms_host, double dt_ms, uint64_t* ticket);
/* psg_submit for a plan that mutes: its rows' keys (host arrays, copied in
 * with the block; psg_submit refuses such a plan with PSG_EINVAL). */
int psg_submit_keyed(psg_server* server, const psg_plan* plan, const void* src_host,
                     void* dst_host, int64_t rows, int32_t cols, const int32_t* live_host,
                     const double* start_ms_host, const psg_keys* keys_host, double dt_ms,
                     uint64_t* ticket);
/* A request whose buffers are already on the server's device (src, dst,
 * live, start_ms and the keys' arrays: device memory): no copies, the
 * kernels read src and write dst directly; no arena bytes. The request runs
 * after the work queued on `stream` (the caller's, or NULL when the buffers
 * are final already) at the time of the call. `keys` only for a plan that
 * mutes (else NULL). */
int psg_submit_device(psg_server* server, const psg_plan* plan, const void* src, void* dst,
                      int64_t rows, int32_t cols, const int32_t* live, const double* start_ms,
                      const psg_keys* keys, double dt_ms, void* stream, uint64_t* ticket);
/* Waits for a request (PSG_ETIMEOUT after timeout_ms; a timeout that is not
 * finite or above 1e12 ms waits until the request finishes) and releases its
 * ticket; PSG_ECANCELED for a request cancelled before it started. A ticket
 * has one waiter: a second thread that waits on it while the first does
 * gets PSG_EINVAL. */
int psg_wait(psg_server* server, uint64_t ticket, double timeout_ms);
/* psg_wait that also gives the time the request finished (the loop saw its
 * copies out done), in seconds of the host's monotonic clock
 * (CLOCK_MONOTONIC: Python's time.perf_counter), so that a caller can
 * measure latency from when the request was due. */
int psg_wait_done(psg_server* server, uint64_t ticket, double timeout_ms, double* done_s);
/* *done = 1 when the request has finished (or was cancelled), without
 * waiting or releasing its ticket. */
int psg_poll(psg_server* server, uint64_t ticket, int32_t* done);
/* Cancels a request that has not started (not yet admitted to the arena):
 * PSG_OK, and psg_wait then returns PSG_ECANCELED; its buffers are not
 * touched. PSG_EINVAL for an unknown ticket or a request already started
 * (it runs to completion: wait for it). */
int psg_cancel(psg_server* server, uint64_t ticket);
/* out[8]: completed, samples, launches, requests per launch, p50 and p99
 * latency (s, submit to completion), Msamples/s, refused; reset != 0 clears. */
int psg_server_stats(psg_server* server, double* out, int reset);
/* The loop's counters since it was created: {batches, kernel launches
 * (batched launches and the part launches of requests run alone), batches
 * started beside running ones, requests completed}. */
int psg_server_counters(psg_server* server, int64_t* out4);
/* The loop's outstanding work now: {requests, samples} queued, staged or in
 * a running batch (what a front end placing requests over several devices'
 * loops reads to pick the least loaded). */
int psg_server_load(psg_server* server, int64_t* out2);

#ifdef __cplusplus
}
#endif
#endif /* PSG_H */
