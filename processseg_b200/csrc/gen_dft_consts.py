"""Writes psg_dft_consts.h: cos and −sin of 2π·e/R (the forward twiddles
ω_R^e = exp(−2πi·e/R)) for the composite in-register DFT sizes the device
FFT uses. Angles are reduced to the first quadrant first, so quarter turns
are exact. Run from this directory: python gen_dft_consts.py"""
import math
from fractions import Fraction

SIZES = [6, 9, 10, 12, 15, 16]


def cos_sin(e, R):
    x = Fraction(e, R) % 1              # turns
    k = math.floor(x * 4)                # quadrant
    r = x - Fraction(k, 4)               # [0, 1/4) turns
    if r == 0:
        c0, s0 = 1.0, 0.0
    elif r == Fraction(1, 8):
        c0 = s0 = math.sqrt(0.5)
    else:
        a = 2 * math.pi * float(r)
        c0, s0 = math.cos(a), math.sin(a)
    return [(c0, s0), (-s0, c0), (-c0, -s0), (s0, -c0)][k]


lines = ["// Generated by gen_dft_consts.py: the forward twiddles exp(-2*pi*i*e/R) of the",
         "// composite in-register DFTs, in float64 (cast to the sample type at use).",
         "#pragma once", "", "namespace psgd {", "template <int R> struct DftW;"]
for R in SIZES:
    cs = [cos_sin(e, R) for e in range(R)]
    def chain(vals):
        expr = repr(vals[-1] + 0.0)
        for e in range(len(vals) - 2, -1, -1):
            expr = f"e == {e} ? {vals[e] + 0.0!r} : {expr}"
        return expr
    lines.append(f"template <> struct DftW<{R}> {{")
    lines.append(f"  static __host__ __device__ constexpr double c(int e) {{ return {chain([v[0] for v in cs])}; }}")
    lines.append(f"  static __host__ __device__ constexpr double s(int e) {{ return {chain([-v[1] for v in cs])}; }}")
    lines.append("};")
lines += ["}  // namespace psgd", ""]
open("psg_dft_consts.h", "w").write("\n".join(lines))
