"""processseg_b200: processSEG's compiled-pipeline hot path on NVIDIA B200
(sm_100a), behind the reference's API (initPipeline / compile / apply,
Workspace, ChunkMeta, requiredMargin, decodeWindow, correlation and vertical
stacking). The compute runs in ``libpsgcuda.so`` (hand-written CUDA kernels
behind a C ABI, ``include/psg.h``); this package is its host-side mirror of
the reference's Nim interface.
"""
from . import _abi
from ._abi import (AGC_MEAN_ABS, AGC_RMS, CM_CORRELATE, CM_DECONVOLVE, F32, F64, FN_FOLD,
                   FN_NONE, FN_SQRT_FOLD, NORM_MAX, NORM_PERCENTILE, NORM_RMS, PER_PANEL,
                   PER_TRACE, TR_LINEAR, TR_MEAN, TR_NONE, TS_AUX, TS_DEAD, TS_LIVE, TS_UNKNOWN)
from .design import (Corners, FilterSpec, GainCurve, GainKnot, bandPass, butterBandPass,
                     butterHighCut, butterLowCut, exponentialGain, highCut, knotGain, lowCut,
                     powerGain)
from .ops import (Op, Pipeline, agcOp, bandPassOp, clipOp, decodeWindow, demeanOp, detrendOp,
                  filterOp, gainCurveOp, gainDbOp, iirOp, initPipeline, muteBottomOp, muteTopOp,
                  normalizeOp, polarityOp, scaleOp)
from .mute import MuteCurve, lmoMute, tableMute, timeMute
from .iir import IirPlan, initIirPlan
from .pool import ProcessPool, newProcessPool
from . import segy
from .calibrate import scaleRows, scaleRowsInto
from .spectrum import (SpectrumPlan, amplitudePhaseInto, circularMeanDeg, dbAbsolute, dbPeak, initSpectrumPlan,
                       removeDelayInto, toDbInto, unwrapPhaseInto)

# Reference enum names (pipeline.nim / gain.nim / edges.nim)
trNone, trMean, trLinear = TR_NONE, TR_MEAN, TR_LINEAR
agcRms, agcMeanAbs = AGC_RMS, AGC_MEAN_ABS
normMax, normRms, normPercentile = NORM_MAX, NORM_RMS, NORM_PERCENTILE
perTrace, perPanel = PER_TRACE, PER_PANEL
tsUnknown, tsLive, tsDead, tsAux = TS_UNKNOWN, TS_LIVE, TS_DEAD, TS_AUX
cmCorrelate, cmDeconvolve = CM_CORRELATE, CM_DECONVOLVE
fnNone, fnFold, fnSqrtFold = FN_NONE, FN_FOLD, FN_SQRT_FOLD
float32, float64 = F32, F64
mkTime, mkTable, mkLmo = _abi.MK_TIME, _abi.MK_TABLE, _abi.MK_LMO
ipZero, ipMinimum = _abi.IP_ZERO, _abi.IP_MINIMUM
from .meta import ChunkMeta, initChunkMeta, liveMeta
from .plan import PipelinePlan, Workspace, compile, initWorkspace
from .vibroseis import (CorrelationPlan, Pilot, RecordStack, SweepHarmonic, SweepPoint, SweepSpec, SweepTaper,
                        applyTaper, dbPerHzSweep, dbPerOctaveSweep, defaultTaperParam, exponentialSweep,
                        generatePilot, initCorrelationPlan, initPilot, initRecordStack, initSweepTaper, pilotFromRow,
                        sweepFromHeaders, sweepOverrides,
                        linearSweep, noTaper, segyTaperType, slDbPerHz, slDbPerOctave, slExponential, slLinear,
                        slTable, sweepHarmonics, tableSweep, taperWeight, tpBlackman, tpBlackmanHarris, tpCos2,
                        tpCosine, tpGaussian, tpHamming, tpKaiser, tpLinear, tpPower)
from .server import Server, ServerPool, leastLoaded
from .stats import PanelStats, TraceStats, panelStats, traceStatsInto
