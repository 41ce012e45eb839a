"""ctypes view of ``include/psg.h`` and the loader of ``libpsgcuda.so``.

The structs mirror the C header field for field; the enums keep the
reference's numbering (``OpKind``, ``TrendRemoval``, ``AgcMode`` ... in
src/processSEG/pipeline.nim:92-108, filter/edges.nim:9-14,
gain/gain.nim:72-95, gain/curves.nim:65-69).

The library is built in-tree by ``processseg_b200/csrc/build.py`` (or
``__graft_entry__.build()``). There is no fallback: importing the compute
entry points without the library raises ``ImportError``.
"""
from __future__ import annotations

import ctypes as C
import os

MAX_NOTCHES = 8
MAX_KNOTS = 64
MAX_MUTE_KNOTS = 64

# psg_status
OK, EINVAL, EWORKSPACE, ENOMEM, ETIMEOUT, ECUDA, ENODEV, ECANCELED = range(8)
# psg_dtype
F32, F64 = 0, 1
# psg_op_kind (OpKind)
(OP_DEMEAN, OP_DETREND, OP_SCALE, OP_GAIN_DB, OP_CLIP, OP_POLARITY, OP_MUTE_TOP,
 OP_MUTE_BOTTOM, OP_FILTER, OP_IIR, OP_AGC, OP_NORMALIZE, OP_GAIN_CURVE,
 OP_CALIBRATE, OP_UNCALIBRATE) = range(15)
OP_NAMES = ["opDemean", "opDetrend", "opScale", "opGainDb", "opClip", "opPolarity",
            "opMuteTop", "opMuteBottom", "opFilter", "opIir", "opAgc", "opNormalize",
            "opGainCurve", "opCalibrate", "opUncalibrate"]
# psg_trend
TR_NONE, TR_MEAN, TR_LINEAR = 0, 1, 2
# psg_response_kind
RK_TRAPEZOID, RK_BUTTERWORTH = 0, 1
# psg_agc_mode
AGC_RMS, AGC_MEAN_ABS = 0, 1
# psg_norm_stat / psg_norm_scope
NORM_MAX, NORM_RMS, NORM_PERCENTILE = 0, 1, 2
PER_TRACE, PER_PANEL = 0, 1
# psg_panel_partials: [Σx², samples, rows, maxAbs] + 65536 histogram counts
PANEL_PARTIAL_HEAD = 4
PANEL_PARTIAL_DOUBLES = PANEL_PARTIAL_HEAD + 65536
# psg_curve_kind
GC_KNOTS, GC_POWER, GC_EXPONENTIAL = 0, 1, 2
# psg_trace_status
TS_UNKNOWN, TS_LIVE, TS_DEAD, TS_AUX = 0, 1, 2, 3
# psg_mute_kind (MuteKind) / psg_iir_phase (IirPhase)
MK_TIME, MK_TABLE, MK_LMO = 0, 1, 2
IP_ZERO, IP_MINIMUM = 0, 1
# psg_corr_mode / psg_fold_norm
CM_CORRELATE, CM_DECONVOLVE = 0, 1
FN_NONE, FN_FOLD, FN_SQRT_FOLD = 0, 1, 2


class Notch(C.Structure):
    _fields_ = [("freq_hz", C.c_double), ("width_hz", C.c_double)]


class FilterSpecC(C.Structure):
    _fields_ = [("kind", C.c_int32), ("zero_dc", C.c_int32), ("n_notches", C.c_int32),
                ("_pad", C.c_int32),
                ("f1", C.c_double), ("f2", C.c_double), ("f3", C.c_double), ("f4", C.c_double),
                ("low_hz", C.c_double), ("low_slope", C.c_double),
                ("high_hz", C.c_double), ("high_slope", C.c_double),
                ("notches", Notch * MAX_NOTCHES)]


class GainKnotC(C.Structure):
    _fields_ = [("t_ms", C.c_double), ("db", C.c_double)]


class GainCurveC(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n_knots", C.c_int32),
                ("power", C.c_double), ("ref_ms", C.c_double), ("min_ms", C.c_double),
                ("db_per_s", C.c_double), ("knots", GainKnotC * MAX_KNOTS)]


SL_LINEAR, SL_DB_PER_OCTAVE, SL_DB_PER_HZ, SL_EXPONENTIAL, SL_TABLE = range(5)


class MuteCurveC(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n_knots", C.c_int32), ("t_ms", C.c_double),
                ("velocity", C.c_double), ("t0_ms", C.c_double), ("pad_ms", C.c_double),
                ("offsets", C.c_double * MAX_MUTE_KNOTS), ("times_ms", C.c_double * MAX_MUTE_KNOTS)]


class KeysC(C.Structure):
    _fields_ = [("offset", C.c_void_p), ("t0_ms", C.c_void_p), ("first_sample", C.c_int32),
                ("_pad", C.c_int32)]


class SweepPointC(C.Structure):
    _fields_ = [("t_ms", C.c_double), ("f_hz", C.c_double)]


class SweepC(C.Structure):
    _fields_ = [("law", C.c_int32), ("taper_shape", C.c_int32), ("f1_hz", C.c_double),
                ("f2_hz", C.c_double), ("length_ms", C.c_double), ("dt_ms", C.c_double),
                ("boost_db", C.c_double), ("table", C.c_void_p), ("n_table", C.c_int64),
                ("start_phase_deg", C.c_double), ("amplitude", C.c_double),
                ("taper_start_ms", C.c_double), ("taper_end_ms", C.c_double),
                ("taper_param", C.c_double), ("max_nyquist_fraction", C.c_double)]


class SweepHarmonicC(C.Structure):
    _fields_ = [("order", C.c_double), ("amp", C.c_double), ("phase_deg", C.c_double)]


class OpC(C.Structure):
    _fields_ = [("kind", C.c_int32), ("trend", C.c_int32), ("factor", C.c_double),
                ("lo", C.c_double), ("hi", C.c_double), ("filter", FilterSpecC),
                ("window_ms", C.c_double), ("target", C.c_double), ("epsilon", C.c_double),
                ("agc_mode", C.c_int32), ("norm_stat", C.c_int32), ("norm_scope", C.c_int32),
                ("iir_phase", C.c_int32), ("norm_target", C.c_double), ("percentile", C.c_double),
                ("curve", GainCurveC), ("t_min_ms", C.c_double), ("t_max_ms", C.c_double),
                ("mute", MuteCurveC), ("taper_ms", C.c_double)]


def ops_array(ops) -> C.Array:
    """A C array of ``psg_op`` from ``Op`` objects (their ``to_c``)."""
    arr = (OpC * max(1, len(ops)))()
    for i, op in enumerate(ops):
        arr[i] = op.to_c()
    return arr


_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpsgcuda.so")
_lib = None

P = C.c_void_p
I32, I64, DBL = C.c_int32, C.c_int64, C.c_double


def _declare(lib):
    sig = {
        "psg_last_error": (C.c_char_p, []),
        "psg_version": (C.c_char_p, []),
        "psg_init": (C.c_int, [C.c_int]),
        "psg_is_fast_len": (C.c_int, [I64]),
        "psg_next_fast_len": (I64, [I64, C.c_int]),
        "psg_impulse_length": (C.c_int, [C.POINTER(FilterSpecC), DBL, C.POINTER(I32)]),
        "psg_response": (C.c_int, [C.POINTER(FilterSpecC), DBL, DBL, C.POINTER(DBL)]),
        "psg_required_margin": (C.c_int, [C.POINTER(OpC), I32, DBL, C.POINTER(I32)]),
        "psg_iir_design": (C.c_int, [C.POINTER(FilterSpecC), DBL, I32, I32, I32, C.POINTER(I32), C.POINTER(I32),
                                     C.POINTER(DBL)]),
        "psg_iir_magnitude": (C.c_int, [C.POINTER(FilterSpecC), DBL, I32, P, I32, P]),
        "psg_decode_window": (None, [I64, I64, I64, I64, C.POINTER(I64)]),
        "psg_plan_compile": (C.c_int, [C.POINTER(OpC), I32, I32, DBL, I32, I32, C.POINTER(P)]),
        "psg_plan_destroy": (None, [P]),
        "psg_plan_margin": (I32, [P]),
        "psg_plan_generation": (C.c_uint64, [P]),
        "psg_plan_samples": (I32, [P]),
        "psg_plan_record_samples": (I32, [P]),
        "psg_plan_part_count": (I32, [P]),
        "psg_plan_part_needs_panel": (I32, [P, I32]),
        "psg_plan_len": (I32, [P]),
        "psg_plan_step_nfft": (I32, [P, I32]),
        "psg_plan_step_margin": (I32, [P, I32]),
        "psg_plan_workspace_bytes": (I64, [P, I64, I32]),
        "psg_workspace_create": (C.c_int, [C.POINTER(P)]),
        "psg_workspace_destroy": (None, [P]),
        "psg_workspace_reserve": (C.c_int, [P, P, I64, I32]),
        "psg_workspace_bytes": (I64, [P]),
        "psg_rows_flatten": (C.c_int, [P, P, P, I64, I32, DBL, P, I64, I32, I32, P, P]),
        "psg_apply": (C.c_int, [P, P, P, P, I64, I32, P, P, DBL, P]),
        "psg_apply_host": (C.c_int, [P, P, P, P, I64, I32, P, P, DBL, P]),
        "psg_apply_keyed": (C.c_int, [P, P, P, P, I64, I32, P, P, C.POINTER(KeysC), DBL, P]),
        "psg_apply_host_keyed": (C.c_int, [P, P, P, P, I64, I32, P, P, C.POINTER(KeysC), DBL, P]),
        "psg_apply_host_async": (C.c_int, [P, P, P, P, I64, I32, P, P, C.POINTER(KeysC), DBL, P]),
        "psg_workspace_sync": (C.c_int, [P]),
        "psg_graph_capture": (C.c_int, [P, P, P, P, I64, I32, P, P, C.POINTER(KeysC), DBL, C.POINTER(P)]),
        "psg_graph_launch": (C.c_int, [P, P]),
        "psg_graph_destroy": (None, [P]),
        "psg_plan_needs_keys": (I32, [P]),
        "psg_plan_trace_shapes": (I32, [P, I32]),
        "psg_plan_pin_trace": (C.c_int, [P, I32, I32]),
        "psg_plan_tuning": (C.c_int, [P, P, I64, C.POINTER(I64)]),
        "psg_applied_response": (C.c_int, [C.POINTER(OpC), I32, I32, DBL, I32, P, I32, P, P]),
        "psg_spectrum_plan_create": (C.c_int, [I32, DBL, I32, DBL, I32, I32, C.POINTER(P)]),
        "psg_spectrum_plan_destroy": (None, [P]),
        "psg_spectrum_plan_info": (C.c_int, [P, C.POINTER(I32), C.POINTER(I32), C.POINTER(I32), C.POINTER(DBL)]),
        "psg_spectrum_average": (C.c_int, [P, P, P, I64, I32, P, DBL, I32, I64, I64, P, P, P]),
        "psg_spectrum_amplitude": (C.c_int, [P, P, P, I64, I32, P, DBL, I32, P, P, P]),
        "psg_segy_decode": (C.c_int, [P, I64, I64, I32, I32, I32, I32, I32, P, I32, P]),
        "psg_poll": (C.c_int, [P, C.c_uint64, C.POINTER(I32)]),
        "psg_cancel": (C.c_int, [P, C.c_uint64]),
        "psg_scale_rows": (C.c_int, [P, I32, P, P, I64, I32, P, P, P]),
        "psg_segy_keys": (C.c_int, [P, I64, I64, I32, P, P, P, P, P, P]),
        "psg_panel_factor": (C.c_int, [P, P, I32, P, I64, I32, P, P, P]),
        "psg_run_part": (C.c_int, [P, P, I32, P, P, I64, I32, P, P, DBL, P, P]),
        "psg_run_part_keyed": (C.c_int, [P, P, I32, P, P, I64, I32, P, P, C.POINTER(KeysC), DBL, P, P]),
        "psg_panel_partials": (C.c_int, [P, P, I32, P, I64, I32, P, P, P]),
        "psg_panel_factor_from": (C.c_int, [P, P, I32, P, P, P]),
        "psg_trace_stats": (C.c_int, [P, I32, I64, I32, P, P, P, P]),
        "psg_panel_stats": (C.c_int, [P, P, I32, I64, I32, P, DBL, P, P]),
        "psg_panel_stats_static": (C.c_int, [P, I32, I64, I32, P, DBL, P, P]),
        "psg_linear_sweep": (C.c_int, [DBL, DBL, DBL, DBL, DBL, DBL, I32, DBL, DBL, DBL, DBL, I32, P,
                                       C.POINTER(I64)]),
        "psg_taper_weight": (C.c_int, [I32, DBL, DBL, C.POINTER(DBL)]),
        "psg_check_apply": (C.c_int, [P, P, P, I64, I32, DBL]),
        "psg_sweep_validate": (C.c_int, [C.POINTER(SweepC)]),
        "psg_sweep_len": (C.c_int, [C.POINTER(SweepC), C.POINTER(I64)]),
        "psg_sweep_frequency_at": (C.c_int, [C.POINTER(SweepC), DBL, C.POINTER(DBL)]),
        "psg_sweep_phase_at": (C.c_int, [C.POINTER(SweepC), DBL, C.POINTER(DBL)]),
        "psg_sweep_samples": (C.c_int, [C.POINTER(SweepC), C.POINTER(SweepHarmonicC), I32, I32, P, I64,
                                        C.POINTER(I32)]),
        "psg_apply_taper": (C.c_int, [I32, P, I64, DBL, DBL, DBL, I32, DBL]),
        "psg_corr_plan_create": (C.c_int, [P, I32, I64, DBL, DBL, I32, DBL, I32, I32, I32, DBL, I32,
                                           C.POINTER(P)]),
        "psg_corr_plan_destroy": (None, [P]),
        "psg_corr_plan_nfft": (I32, [P]),
        "psg_corr_plan_out_samples": (I32, [P]),
        "psg_corr_plan_scale": (DBL, [P]),
        "psg_correlate": (C.c_int, [P, P, P, I64, I32, P, DBL, P]),
        "psg_stack_create": (C.c_int, [I64, I32, DBL, C.POINTER(P)]),
        "psg_stack_destroy": (None, [P]),
        "psg_stack_clear": (C.c_int, [P, P]),
        "psg_stack_add": (C.c_int, [P, P, I32, I64, I32, P, P, P]),
        "psg_correlate_stack": (C.c_int, [P, P, P, P, I64, I32, P, P, P, DBL, P]),
        "psg_stack_result": (C.c_int, [P, P, I32, I32, P]),
        "psg_stack_fold": (C.c_int, [P, P, P]),
        "psg_server_create": (C.c_int, [C.c_int, I64, C.POINTER(P)]),
        "psg_server_destroy": (None, [P]),
        "psg_submit": (C.c_int, [P, P, P, P, I64, I32, P, P, DBL, C.POINTER(C.c_uint64)]),
        "psg_server_counters": (C.c_int, [P, P]),
        "psg_server_load": (C.c_int, [P, P]),
        "psg_wait_done": (C.c_int, [P, C.c_uint64, DBL, C.POINTER(DBL)]),
        "psg_submit_keyed": (C.c_int, [P, P, P, P, I64, I32, P, P, C.POINTER(KeysC), DBL, C.POINTER(C.c_uint64)]),
        "psg_submit_device": (C.c_int, [P, P, P, P, I64, I32, P, P, C.POINTER(KeysC), DBL, P, C.POINTER(C.c_uint64)]),
        "psg_wait": (C.c_int, [P, C.c_uint64, DBL]),
        "psg_server_stats": (C.c_int, [P, C.POINTER(DBL), C.c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return sig


EXPORTED = None


def lib():
    """The loaded ``libpsgcuda.so``; raises ``ImportError`` when it is missing."""
    global _lib, EXPORTED
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; "
                "g.build()'` (there is no CPU fallback)")
        _lib = C.CDLL(LIB_PATH)
        EXPORTED = _declare(_lib)
    return _lib


class PsgError(RuntimeError):
    """A CUDA or device failure reported by the library."""


def check(status: int):
    """Maps a ``psg_status`` to the reference's exceptions: ``ValueError`` for
    PSG_EINVAL (raised before any sample changes) and ``AssertionError`` for
    PSG_EWORKSPACE (the reference's AssertionDefect)."""
    if status == OK:
        return
    msg = lib().psg_last_error().decode("utf-8", "replace")
    if status == EINVAL:
        raise ValueError(msg)
    if status == EWORKSPACE:
        raise AssertionError(msg)
    if status == ENOMEM:
        raise MemoryError(msg)
    if status == ETIMEOUT:
        raise TimeoutError(msg)
    raise PsgError(f"status {status}: {msg}")
