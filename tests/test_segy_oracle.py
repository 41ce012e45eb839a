"""The SEG-Y decode's oracle on the CPU (test infrastructure), pinned by
published IBM hexadecimal floating-point values and by an independent exact
evaluation of the format's definition (−1)^s · (f / 2^24) · 16^(e − 64) in
rational arithmetic; the integer and IEEE formats by Python's struct module;
the trace-header keys by hand-built headers."""
import struct
from fractions import Fraction

import numpy as np
import pytest

from processseg_b200 import _abi as A
from oracle import oracle as O

IBM_KNOWN = [(0xC276A000, -118.625), (0x42640000, 100.0), (0x41100000, 1.0), (0x00000000, 0.0),
             (0x40800000, 0.5), (0xC1100000, -1.0), (0x42100000, 16.0), (0x3F800000, 0.5 / 16)]


def record(words, sz=4, little=False, header=None):
    rec = np.zeros((1, 240 + sz * len(words)), np.uint8)
    if header is not None:
        rec[0, :240] = header
    for i, w in enumerate(words):
        rec[0, 240 + sz * i:240 + sz * (i + 1)] = list(int(w).to_bytes(sz, "little" if little else "big"))
    return rec


def ibm_exact(w):
    s, e, f = w >> 31, (w >> 24) & 0x7F, w & 0xFFFFFF
    v = Fraction(f, 1 << 24) * Fraction(16) ** (e - 64)
    return float(-v if s else v)


def test_ibm_known_values():
    got = O.segy_decode(record([w for w, _ in IBM_KNOWN]), len(IBM_KNOWN), 1, np.float64)[0]
    assert got.tolist() == [v for _, v in IBM_KNOWN]


def test_ibm_matches_its_definition_exactly():
    rng = np.random.default_rng(7)
    words = rng.integers(0, 1 << 32, 2000, dtype=np.uint64).tolist() + [0x7FFFFFFF, 0xFFFFFFFF, 0x00000001, 0x80000000]
    got64 = O.segy_decode(record(words), len(words), 1, np.float64)[0]
    got32 = O.segy_decode(record(words), len(words), 1, np.float32)[0]
    for w, g64, g32 in zip(words, got64, got32):
        want = ibm_exact(int(w))
        assert g64 == want
        with np.errstate(over="ignore"):
            assert g32 == np.float32(want) or (np.isnan(g32) and np.isnan(want))


@pytest.mark.parametrize("little", [False, True])
def test_integer_and_ieee_formats(little):
    rng = np.random.default_rng(3)
    for fmt, sz, pack in ((2, 4, "i"), (3, 2, "h"), (5, 4, "f"), (6, 8, "d"), (8, 1, "b"), (10, 4, "I"),
                          (11, 2, "H"), (16, 1, "B")):
        raw = rng.integers(0, 256, (5, 240 + 7 * sz), dtype=np.uint8)
        got = O.segy_decode(raw, 7, fmt, np.float64, little)
        for r in range(5):
            for j in range(7):
                b = bytes(raw[r, 240 + sz * j:240 + sz * (j + 1)])
                want = struct.unpack(("<" if little else ">") + pack, b)[0]
                assert got[r, j] == want or (np.isnan(got[r, j]) and np.isnan(want))
    # 24-bit integers
    raw = record([0x000001, 0xFFFFFF, 0x800000, 0x7FFFFF], 3, little)
    assert O.segy_decode(raw, 4, 7, np.float64, little)[0].tolist() == [1, -1, -8388608, 8388607]
    assert O.segy_decode(raw, 4, 15, np.float64, little)[0].tolist() == [1, 16777215, 8388608, 8388607]


def test_trace_header_keys():
    h = np.zeros(240, np.uint8)
    h[28:30] = list((1).to_bytes(2, "big"))
    h[36:40] = list((-1250).to_bytes(4, "big", signed=True))
    h[108:110] = list((-40).to_bytes(2, "big", signed=True))
    h[114:116] = list((3001).to_bytes(2, "big"))
    h[116:118] = list((2000).to_bytes(2, "big"))
    rec = np.vstack([record([0], header=h)] * 3)
    rec[1, 28:30] = [0, 2]
    rec[2, 28:30] = [0, 7]
    status, ns, us, off, t0 = O.segy_keys(rec)
    assert status.tolist() == [A.TS_LIVE, A.TS_DEAD, A.TS_AUX]
    assert ns.tolist() == [3001] * 3 and us.tolist() == [2000.0] * 3
    assert off.tolist() == [-1250.0] * 3 and t0.tolist() == [-40.0] * 3
