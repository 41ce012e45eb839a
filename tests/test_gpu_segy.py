"""SEG-Y decode on the device (psg_segy_decode / psg_segy_keys) against the
oracle bit for bit: every sample format, both byte orders, float32 and
float64 blocks, columns past the samples; then decoded int16 and IBM
records through a pipeline plan against the oracle's apply of the same
decoded samples."""
import numpy as np
import pytest

import processseg_b200 as P
from processseg_b200 import _abi as A
from processseg_b200 import segy, synth
from oracle import oracle as O

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu, pytest.mark.usefixtures("built")]


@pytest.mark.parametrize("slack", [0, 6])
@pytest.mark.parametrize("little", [False, True])
@pytest.mark.parametrize("fmt", [1, 2, 3, 5, 6, 7, 8, 10, 11, 15, 16])
def test_decode_matches_oracle_bit_for_bit(fmt, little, slack):
    """Records packed back to back (the word-wide reads of 2- and 4-byte
    samples) and with 6 bytes of slack after each (the byte-wise reads)."""
    sz = segy.SAMPLE_BYTES[fmt]
    rng = np.random.default_rng(fmt * 2 + little)
    rec = rng.integers(0, 256, (37, 240 + 501 * sz + slack), dtype=np.uint8)
    for T, npdt in ((P.float32, np.float32), (P.float64, np.float64)):
        got = segy.decodeTraces(rec, 501, fmt, T, little, outCols=520).cpu().numpy()
        want = O.segy_decode(rec, 501, fmt, npdt, little, out_cols=520)
        assert got.dtype == want.dtype
        same = (got == want) | (np.isnan(got) & np.isnan(want))
        assert same.all(), (fmt, little, T)


def test_keys_match_oracle():
    rng = np.random.default_rng(11)
    rec = rng.integers(0, 256, (300, 240 + 64), dtype=np.uint8)
    rec[:, 28:30] = rng.integers(0, 4, (300, 1)).astype(np.uint8) * np.array([0, 1], np.uint8)
    for little in (False, True):
        k = segy.traceKeys(rec, little)
        status, ns, us, off, t0 = O.segy_keys(rec, little)
        assert np.array_equal(k["status"], status) and np.array_equal(k["numSamples"], ns)
        assert np.array_equal(k["intervalUs"], us) and np.array_equal(k["offset"], off)
        assert np.array_equal(k["t0Ms"], t0)


def records_of(data, live, fmt, offsets):
    """Big-endian SEG-Y records of float samples: IBM (1) or int16 (3)."""
    rows, n = data.shape
    sz = segy.SAMPLE_BYTES[fmt]
    rec = np.zeros((rows, 240 + n * sz), np.uint8)
    for r in range(rows):
        h = rec[r]
        h[28:30] = list((1).to_bytes(2, "big"))
        h[36:40] = list(int(offsets[r]).to_bytes(4, "big", signed=True))
        h[114:116] = list(int(live[r]).to_bytes(2, "big"))
        h[116:118] = list((2000).to_bytes(2, "big"))
    if fmt == 3:
        q = np.clip(np.round(data * 1000), -32768, 32767).astype(">i2")
        rec[:, 240:] = q.view(np.uint8).reshape(rows, -1)
    else:
        x = data.astype(np.float64)
        s = (x < 0).astype(np.uint64)
        a = np.abs(x)
        e = np.where(a > 0, np.floor(np.log2(np.where(a > 0, a, 1)) / 4) + 65, 0).astype(np.int64)
        f = np.where(a > 0, np.round(np.ldexp(a, 24 - 4 * (e - 64))), 0).astype(np.uint64)
        over = f >= (1 << 24)
        f = np.where(over, f >> np.uint64(4), f)
        e = np.where(over, e + 1, e)
        w = (s << np.uint64(31)) | (e.astype(np.uint64) << np.uint64(24)) | f
        rec[:, 240:] = w.astype(">u4").view(np.uint8).reshape(rows, -1)
    return rec


@pytest.mark.parametrize("fmt", [1, 3])
def test_decode_then_apply(fmt):
    g = synth.c1()
    live = g.numSamples
    rec = records_of(g.data, live, fmt, g.offsets)
    keys = segy.traceKeys(rec)
    meta = segy.chunkMetaOf(keys)
    assert meta.dtMs == 2.0
    x = segy.decodeTraces(rec, 2001, fmt, P.float32)
    want_in = O.segy_decode(rec, 2001, fmt, np.float32)
    assert np.array_equal(x.cpu().numpy(), want_in)
    flow = [P.demeanOp(), P.bandPassOp(P.Corners(4, 8, 60, 80)), P.agcOp(500)]
    plan = P.initPipeline(flow).compile(P.float32, 2.0, 2001)
    ws = P.initWorkspace()
    ws.reserve(plan, rows=x.shape[0], cols=2001)
    plan.apply(x, meta, ws)
    torch.cuda.synchronize()
    want = O.OraclePlan(flow, A.F32, 2.0, 2001).apply(want_in, *meta.flat(2001))
    got = x.cpu().numpy()
    for r in range(got.shape[0]):
        rms = float(np.sqrt(np.mean(want[r].astype(np.float64) ** 2)))
        assert np.max(np.abs(got[r] - want[r])) <= 1e-5 * rms
