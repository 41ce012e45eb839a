// psg_trace.cuh — the float32 trace kernel of libpsgcuda.so: the plan parts
// demean → zero-phase FFT filter → AGC (→ per-trace normalization) with zero
// pads, with the transform's length known at compile time, and the float32
// correlation kernel of the same make.
//
// What differs from pipeline_kernel's recipe path (same inputs; outputs
// within the parity bar of both, closer to the reference's float32 bits):
//  * The filter's transforms (RPlan) run the reference's own stages (4s, a 2,
//    3s, 5s) with its butterflies, twiddles and roundings (no fused
//    multiply-add), two consecutive stages fused per shared-memory pass; the
//    split · gain · unsplit between the transforms runs once per bin pair in
//    the reference's order. Radices, strides and butterfly counts are
//    constants; each build groups the stages its own way (the host's tuner
//    picks among builds and launch shapes, which give the same bits).
//  * The demean, trend and AGC-level sums are float64, in an order that does
//    not depend on the build (kNT lanes, then the warps in order).
//  * One row buffer: the row is read only by the forward transform's first
//    pass, so the next row's bulk copy goes in right after the forward
//    transform (or the row shares the first transform buffer); the inverse
//    transform's last pass unpacks the filtered row into the buffer it does
//    not read, and the AGC writes its output into the other one.
//  * The AGC's window sums come from registers: a warp takes consecutive
//    window groups, each group's outputs needing the suffix sums of one
//    block and the prefix sums of the next (w = 2h + 1 = the block length,
//    so the window [i − h, i + h] spans exactly those two), scanned in
//    registers as pipeline_kernel scans them into shared memory, with the
//    same sums, divisors and gain arithmetic (gain/gain.nim:351-461).
//  * BATCH: the rows of many served requests' jobs in one launch.
#pragma once

#include "psg_kernel.cuh"
#include "psg_trace.h"

namespace psg {
namespace tk {

// ------------------------------------------------------- compile-time plan
// A complex FFT of M points in NP Stockham passes of radices Rs..., run by a
// CTA of NT threads (one trace per CTA), MINB CTAs per SM asked of the
// register allocator.
template <int M_, int NT_, int MINB_, int... Rs> struct FPlan {
  static constexpr int M = M_, NT = NT_, MINB = MINB_, NP = (int)sizeof...(Rs);
  static constexpr int R[NP] = {Rs...};
  static constexpr int radix(int i) { return R[i]; }
  // the product of the radices before pass i
  static constexpr int stride(int i) {
    int s = 1;
    for (int j = 0; j < i; j++) s *= R[j];
    return s;
  }
  // twiddles of one butterfly: R − 1 values, padded to an even count
  static constexpr int tws(int r) { return (r - 1 + 1) & ~1; }
  // where pass i's twiddles start in the plan's table (complex values)
  static constexpr int tw_off(int i) {
    int o = 0;
    for (int j = 0; j < i; j++) o += M / (stride(j) * R[j]) * tws(R[j]);
    return o;
  }
  static constexpr int tw_len() { return tw_off(NP - 1); }
  static_assert(stride(NP) == M, "the radices multiply to M");
};

__device__ __forceinline__ float2* smem_c() { return reinterpret_cast<float2*>(psg_dyn_smem); }

// A row of floats in the block's dynamic shared memory, held as an offset
// from the shared symbol (in floats): accesses through it compile to 32-bit
// shared loads and stores, where a pointer chosen at run time between the
// row buffers would be a generic 64-bit one.
struct SRow {
  int o;
  __device__ __forceinline__ float& operator[](int i) const { return reinterpret_cast<float*>(psg_dyn_smem)[o + i]; }
};

// A pass's inputs from the buffer at complex offset o.
struct BufLd {
  int o;
  __device__ __forceinline__ float2 operator()(int c, int) const { return smem_c()[o + c]; }
};
// A pass's outputs into the buffer at complex offset o.
struct BufSt {
  int o;
  __device__ __forceinline__ void operator()(int c, float2 v) const { smem_c()[o + c] = v; }
};

// Pass I of plan P (fft/plan.nim:187-190, decimation in frequency): butterfly
// b = p·S + q takes inputs b + j·B (B = M/R butterflies, j < R) and writes
// outputs q + S·(R·p + k) = b + S·(R − 1)·p + S·k, each output k ≥ 1 times
// the twiddle ω_M^{p·k·S} (table entry tw_off(I) + p·tws(R) + k − 1). The
// last pass (S·R = M) has p = 0 and no twiddles. ld(c, j) gives input c,
// st(c, v) takes output c.
template <class P, int I, class LD, class ST>
__device__ __forceinline__ void pass(const float2* __restrict__ tw, const LD& ld, const ST& st) {
  constexpr int R = P::radix(I), S = P::stride(I), M = P::M, NT = P::NT;
  constexpr int B = M / R;
  constexpr bool LAST = I == P::NP - 1;
  constexpr int U = (B + NT - 1) / NT;
  constexpr int TW = P::tws(R);
#pragma unroll
  for (int u = 0; u < U; u++) {
    const int b = (int)threadIdx.x + u * NT;
    if (B % NT != 0 && b >= B) continue;
    float2 v[R];
#pragma unroll
    for (int j = 0; j < R; j++) v[j] = ld(b + j * B, j);
    Dft<float2, float, R>::run(v);
    int base = b;
    if constexpr (!LAST) {
      const int p = b / S;
      const float4* t = reinterpret_cast<const float4*>(tw + P::tw_off(I) + p * TW);
#pragma unroll
      for (int k = 1; k < R; k += 2) {
        const float4 w = __ldg(t + (k - 1) / 2);
        v[k] = cmul(v[k], make_float2(w.x, w.y));
        if (k + 1 < R) v[k + 1] = cmul(v[k + 1], make_float2(w.z, w.w));
      }
      base = b + (S * (R - 1)) * p;
    }
#pragma unroll
    for (int k = 0; k < R; k++) st(base + S * k, v[k]);
  }
}

// Passes I .. NP − 1, pass I reading the buffer at x and writing the one at
// y (alternating after it); the last pass's outputs go to `last`. Every pass
// but the last ends with a barrier.
template <class P, int I> struct Passes {
  template <class ST> static __device__ __forceinline__ void run(int x, int y, const float2* tw, const ST& last) {
    if constexpr (I == P::NP - 1) {
      pass<P, I>(tw, BufLd{x}, last);
    } else {
      pass<P, I>(tw, BufLd{x}, BufSt{y});
      __syncthreads();
      Passes<P, I + 1>::run(y, x, tw, last);
    }
  }
};

// A forward complex FFT whose first pass takes its inputs from ld (the
// pack or the bridge) and writes the buffer at `b`; `a` is the other buffer.
// The last pass's outputs go to `last` (no barrier after it).
template <class P, class LD, class ST>
__device__ __forceinline__ void fft(int a, int b, const float2* tw, const LD& ld, const ST& last) {
  if constexpr (P::NP == 1) {
    pass<P, 0>(tw, ld, last);
  } else {
    pass<P, 0>(tw, ld, BufSt{b});
    __syncthreads();
    Passes<P, 1>::run(b, a, tw, last);
  }
}
// The buffer the last pass of fft(a, b, …) reads (pass NP − 2 wrote it) and
// the other one, which it may write.
template <class P> __device__ __forceinline__ int last_in(int a, int b) { return P::NP % 2 == 0 ? b : a; }
template <class P> __device__ __forceinline__ int last_out(int a, int b) { return P::NP % 2 == 0 ? a : b; }

// ------------------------------------------- the reference's rounding
// The filter's transforms as the reference rounds them in float32: its
// stages (radix 4 first, then a 2, then 3s and 5s, fft/plan.nim:120-132),
// its butterflies (fft/plan.nim:225-417) with every product and sum rounded
// on its own (no fused multiply-add) in the reference's order, and its
// per-stage twiddles ω_cur^{(p·k) mod cur} (fft/plan.nim:136-160). Two
// consecutive stages run as one pass in registers: a thread holding the R1·R2
// inputs of R2 butterflies of the first stage holds the inputs of R1
// butterflies of the second, so the arithmetic, and every rounding, is the
// two stages' while the data crosses shared memory once.
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
// Sums and differences on a complex value's two parts at once (sm_100's
// paired float32 instructions, written in PTX with the rounding stated), each
// part rounded as the scalar form is. ppm gives (a.x + b.x, a.y − b.y) and pmp
// (a.x − b.x, a.y + b.y) as fma.rn.f32x2(b, (±1, ∓1), a), whose products are
// exact, so the one rounding is the sum's or difference's, zero signs
// included. Products stay scalar (pm): a paired multiply feeding a paired add
// came out fused into one rounding on sm_100a even with .rn stated (a third
// of radix-5 butterflies differed), scalar products into paired sums do not.
__device__ __forceinline__ unsigned long long pk2(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ float2 upk2(unsigned long long r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
__device__ __forceinline__ float2 pa(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk2(a)), "l"(pk2(b)));
  return upk2(d);
}
__device__ __forceinline__ float2 ps(float2 a, float2 b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk2(a)), "l"(pk2(b)));
  return upk2(d);
}
__device__ __forceinline__ float2 pm(float c, float2 b) { return make_float2(fm(c, b.x), fm(c, b.y)); }
template <int SX> __device__ __forceinline__ float2 pmix(float2 a, float2 b) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(pk2(b)), "l"(pk2(make_float2((float)SX, (float)-SX))), "l"(pk2(a)));
  return upk2(d);
}
__device__ __forceinline__ float2 ppm(float2 a, float2 b) { return pmix<1>(a, b); }
__device__ __forceinline__ float2 pmp(float2 a, float2 b) { return pmix<-1>(a, b); }

// MULTW (fft/plan.nim:203-206): re = yr·wr − yi·wi, im = yr·wi + yi·wr
// (four scalar products, then the difference and the sum as one pair).
__device__ __forceinline__ float2 mul_tw(float2 y, float2 w) {
  return pmp(make_float2(fm(y.x, w.x), fm(y.x, w.y)), make_float2(fm(y.y, w.y), fm(y.y, w.x)));
}

// The reference's butterfly of radix R on v[0 .. R) (outputs in place, k-th
// output at v[k], before its twiddle); every operation the reference applies
// to both parts alike runs on the pair.
template <int R> struct RefDft;
template <> struct RefDft<2> {
  static __device__ __forceinline__ void run(float2* v) {
    const float2 u = v[0], w = v[1];
    v[0] = pa(u, w);
    v[1] = ps(u, w);
  }
};
template <> struct RefDft<3> {
  static __device__ __forceinline__ void run(float2* v) {
    const float c = -0.5f, s = (float)0.8660254037844386467637231707529362;
    const float2 a = v[0];
    const float2 t1 = pa(v[1], v[2]), t2 = ps(v[1], v[2]);
    const float2 m1 = pa(a, pm(c, t1));
    const float2 m2 = make_float2(fm(s, t2.y), fm(-s, t2.x));
    v[0] = pa(a, t1);
    v[1] = pa(m1, m2);
    v[2] = ps(m1, m2);
  }
};
template <> struct RefDft<4> {
  static __device__ __forceinline__ void run(float2* v) {
    const float2 x0 = v[0], x1 = v[1], x2 = v[2], x3 = v[3];
    const float2 t0 = pa(x0, x2), t1 = ps(x0, x2), t2 = pa(x1, x3);
    const float2 t3 = make_float2(fs(x1.y, x3.y), fs(x3.x, x1.x));
    v[0] = pa(t0, t2);
    v[1] = pa(t1, t3);
    v[2] = ps(t0, t2);
    v[3] = ps(t1, t3);
  }
};
template <> struct RefDft<5> {
  static __device__ __forceinline__ void run(float2* v) {
    const float c1 = (float)0.3090169943749474241022934171828191, c2 = (float)-0.8090169943749474241022934171828191;
    const float s1 = (float)0.9510565162951535721164393333793821, s2 = (float)0.5877852522924731291687059546390728;
    const float2 a = v[0];
    const float2 t1 = pa(v[1], v[4]), t2 = pa(v[2], v[3]);
    const float2 t3 = ps(v[1], v[4]), t4 = ps(v[2], v[3]);
    const float2 b1 = pa(pa(a, pm(c1, t1)), pm(c2, t2));
    const float2 b2 = pa(pa(a, pm(c2, t1)), pm(c1, t2));
    const float2 d1 = pa(pm(s1, t3), pm(s2, t4));
    const float2 d2 = ps(pm(s2, t3), pm(s1, t4));
    // (b.x + d.y, b.y − d.x) and (b.x − d.y, b.y + d.x)
    const float2 e1 = make_float2(d1.y, d1.x), e2 = make_float2(d2.y, d2.x);
    v[0] = pa(pa(a, t1), t2);
    v[1] = ppm(b1, e1);
    v[4] = pmp(b1, e1);
    v[2] = ppm(b2, e2);
    v[3] = pmp(b2, e2);
  }
};

// One pass: stage R1 alone (R2 = 0) or stages R1 then R2.
template <int R1, int R2 = 0> struct Grp {
  static constexpr int r1 = R1, r2 = R2, R = R2 ? R1 * R2 : R1;
};

// A transform of M points in passes Gs... (each one or two of the
// reference's stages), run by a CTA of NT threads, MINB CTAs per SM asked of
// the register allocator. Pass i of radix R (the product of its stages)
// moves data as a Stockham pass of that radix: butterfly b = p·S + q takes
// inputs b + j·M/R and writes outputs q + S·(R·p + k).
template <int M_, int NT_, int MINB_, class... Gs> struct RPlan {
  static constexpr int M = M_, NT = NT_, MINB = MINB_, NP = (int)sizeof...(Gs);
  static constexpr int G1[NP] = {Gs::r1...};
  static constexpr int G2[NP] = {Gs::r2...};
  static constexpr int radix(int i) { return G2[i] ? G1[i] * G2[i] : G1[i]; }
  static constexpr int stride(int i) {
    int s = 1;
    for (int j = 0; j < i; j++) s *= radix(j);
    return s;
  }
  // a butterfly's twiddles: R − 1 of them (R2·(R1 − 1) of the first stage
  // then R2 − 1 of the second), padded to an even count
  static constexpr int tws(int r) { return (r - 1 + 1) & ~1; }
  static constexpr int tw_off(int i) {
    int o = 0;
    for (int j = 0; j < i; j++) o += M / (stride(j) * radix(j)) * tws(radix(j));
    return o;
  }
  static_assert(stride(NP) == M, "the stages multiply to M");
  // The first pass writes outputs R·b + k (stride 1): for an even R, lanes
  // of a warp store 8-byte values R·8 bytes apart, into a quarter or less of
  // the banks. Its buffer is then laid out with one spare element after
  // every R (output c at c + c/R), which spreads those stores over all banks;
  // the second pass reads it so (input c = b + j·B at b + b/R + j·(B + B/R),
  // B a multiple of R).
  static constexpr int PAD = (NP > 1 && radix(0) % 2 == 0) ? radix(0) : 0;
  // complex elements of one transform buffer
  static constexpr int BUF = M + (PAD ? M / (PAD ? PAD : 1) : 0);
};

// Pass I of RPlan P. The first stage's butterflies are p + jB·(M/(S·R))
// (jB < R2) of a stage over cur = M/S points: its input jA is the pass's
// input jB + R2·jA, its output kA (times ω_cur^{((p + jB·M/(S·R))·kA) mod
// cur}) the second stage's input jB of its butterfly kA; that one's output kB
// (times ω_{cur/R1}^{(p·kB) mod (cur/R1)}) is the pass's output R1·kB + kA.
// The last stage of a transform has p = 0 and unit twiddles (the reference
// multiplies by (1, −0), which leaves every value as it is): they are
// skipped.
// OUTPAD (the first pass, stride 1): its outputs go to the padded layout
// (output c = R·p + k at c + p); INPAD (the second pass): ld is a BufLd of a
// buffer in that layout.
template <class P, int I, int OUTPAD = 0, int INPAD = 0, class LD, class ST>
__device__ __forceinline__ void ref_pass(const float2* __restrict__ tw, const LD& ld, const ST& st) {
  constexpr int R = P::radix(I), R1 = P::G1[I], R2 = P::G2[I], S = P::stride(I), M = P::M, NT = P::NT;
  constexpr int B = M / R;
  constexpr bool LAST = I == P::NP - 1;
  constexpr int U = (B + NT - 1) / NT;
  constexpr int TW = P::tws(R);
  static_assert(OUTPAD == 0 || (S == 1 && OUTPAD == R), "the padded layout is the first pass's");
  static_assert(INPAD == 0 || B % INPAD == 0, "the second pass's inputs stay B + B/R apart");
#pragma unroll
  for (int u = 0; u < U; u++) {
    const int b = (int)threadIdx.x + u * NT;
    if (B % NT != 0 && b >= B) continue;
    float2 v[R];
    if constexpr (INPAD != 0) {
      const float2* x = smem_c() + ld.o + b + b / INPAD;
#pragma unroll
      for (int j = 0; j < R; j++) v[j] = x[j * (B + B / INPAD)];
    } else {
#pragma unroll
      for (int j = 0; j < R; j++) v[j] = ld(b + j * B, j);
    }
    const int p = LAST ? 0 : b / S;
    const float2* t = tw + P::tw_off(I) + p * TW;
    float2 out[R];
    if constexpr (R2 == 0) {
      RefDft<R1>::run(v);
#pragma unroll
      for (int k = 0; k < R; k++) out[k] = (k == 0 || LAST) ? v[k] : mul_tw(v[k], __ldg(t + k - 1));
    } else {
      float2 mid[R2][R1];
#pragma unroll
      for (int jB = 0; jB < R2; jB++) {
        float2 a[R1];
#pragma unroll
        for (int jA = 0; jA < R1; jA++) a[jA] = v[jB + R2 * jA];
        RefDft<R1>::run(a);
#pragma unroll
        for (int kA = 0; kA < R1; kA++) mid[jB][kA] = kA == 0 ? a[0] : mul_tw(a[kA], __ldg(t + jB * (R1 - 1) + kA - 1));
      }
#pragma unroll
      for (int kA = 0; kA < R1; kA++) {
        float2 c[R2];
#pragma unroll
        for (int jB = 0; jB < R2; jB++) c[jB] = mid[jB][kA];
        RefDft<R2>::run(c);
#pragma unroll
        for (int kB = 0; kB < R2; kB++)
          out[R1 * kB + kA] = (kB == 0 || LAST) ? c[kB] : mul_tw(c[kB], __ldg(t + R2 * (R1 - 1) + kB - 1));
      }
    }
    const int base = b + (S * (R - 1)) * p + (OUTPAD ? p : 0);
#pragma unroll
    for (int k = 0; k < R; k++) st(base + S * k, out[k]);
  }
}

template <class P, int I> struct RefPasses {
  template <class ST> static __device__ __forceinline__ void run(int x, int y, const float2* tw, const ST& last) {
    constexpr int IN = I == 1 ? P::PAD : 0;
    if constexpr (I == P::NP - 1) {
      ref_pass<P, I, 0, IN>(tw, BufLd{x}, last);
    } else {
      ref_pass<P, I, 0, IN>(tw, BufLd{x}, BufSt{y});
      __syncthreads();
      RefPasses<P, I + 1>::run(y, x, tw, last);
    }
  }
};
// The transform of plan P, as fft().
template <class P, class LD, class ST>
__device__ __forceinline__ void ref_fft(int a, int b, const float2* tw, const LD& ld, const ST& last) {
  if constexpr (P::NP == 1) {
    ref_pass<P, 0>(tw, ld, last);
  } else {
    ref_pass<P, 0, P::PAD>(tw, ld, BufSt{b});
    __syncthreads();
    RefPasses<P, 1>::run(b, a, tw, last);
  }
}

// The reference's real-FFT steps between the transforms, in float32:
// splitForward (fft/plan.nim:470-482) of the forward transform's output z,
// the bin gains (gainRun, filter/apply.nim:234-247), and splitInverse with
// the 1/n scale and the swap into the inverse transform's input
// (fft/plan.nim:484-499, 544-567). Input c of the inverse needs the bins c
// and m − c, both split from z[c] and z[m − c]. `sp[c]` holds the split
// twiddles (re, im) of bins c and m − c, `g[c]` the gains of bins c and
// m − c (of bins 0 and m for c = 0).
struct RefBridgeLd {
  int zo, m;
  const float4* __restrict__ sp;
  const float2* __restrict__ g;
  float scale;
  __device__ __forceinline__ float2 operator()(int c, int j) const {
    const float2* z = smem_c() + zo;
    if (j == 0 && c == 0) {
      const float2 z0 = z[0];
      const float2 gg = __ldg(g);
      const float x0 = fm(fa(z0.x, z0.y), gg.x), xm = fm(fs(z0.x, z0.y), gg.y);
      return make_float2(fm(fs(x0, xm), scale), fm(fa(x0, xm), scale));
    }
    const float2 A = z[c], Bv = z[m - c];
    const float4 w = __ldg(sp + c);
    const float2 gg = __ldg(g + c);
    // the split of bins c (A, B) and m − c (B, A): their even and odd parts
    // share |terms| (x − y = −(y − x) exactly)
    const float er = fm(0.5f, fa(A.x, Bv.x)), ei = fm(0.5f, fs(A.y, Bv.y));
    const float orr = fm(0.5f, fa(A.y, Bv.y)), oi = fm(0.5f, fs(Bv.x, A.x));
    float Xr = fs(fa(er, fm(w.x, orr)), fm(w.y, oi));
    float Xi = fa(fa(ei, fm(w.x, oi)), fm(w.y, orr));
    float Yr = fs(fa(er, fm(w.z, orr)), fm(w.w, -oi));
    float Yi = fa(fa(-ei, fm(w.z, -oi)), fm(w.w, orr));
    Xr = fm(Xr, gg.x);
    Xi = fm(Xi, gg.x);
    Yr = fm(Yr, gg.y);
    Yi = fm(Yi, gg.y);
    // splitInverse of bin c with a = X[c], b = X[m − c], ω = (wr, −wi)
    const float e_r = fa(Xr, Yr), e_i = fs(Xi, Yi), dr = fs(Xr, Yr), di = fa(Xi, Yi);
    const float wr = w.x, wi = -w.y;
    const float o_r = fs(fm(dr, wr), fm(di, wi)), o_i = fa(fm(dr, wi), fm(di, wr));
    return make_float2(fm(fa(e_i, o_r), scale), fm(fs(e_r, o_i), scale));
  }
};

// The same steps for a pair of inputs at once, in place: bins c and m − c
// come from z[c] and z[m − c] and give the inverse transform's inputs c and
// m − c, so one thread splits, scales and unsplits both (every rounding as
// RefBridgeLd's: the pair's even and odd parts are shared, up to exact sign
// changes and commuted sums). The thread taking c = 0 also takes c = m/2
// when m is even (both their own partners).
template <int M, int NT>
__device__ __forceinline__ void ref_bridge_pairs(int zo, const float4* __restrict__ sp, const float2* __restrict__ g,
                                                 float scale) {
  float2* z = smem_c() + zo;
  constexpr int PAIRS = (M - 1) / 2;  // c = 1 .. PAIRS with m − c > c
  for (int t = threadIdx.x; t <= PAIRS; t += NT) {
    if (t == 0) {
      const float2 z0 = z[0];
      const float2 gg = __ldg(g);
      const float x0 = fm(fa(z0.x, z0.y), gg.x), xm = fm(fs(z0.x, z0.y), gg.y);
      z[0] = make_float2(fm(fs(x0, xm), scale), fm(fa(x0, xm), scale));
      if constexpr (M % 2 == 0) {
        // c = m/2 pairs with itself: bin m/2 from A = B = z[m/2]
        constexpr int c = M / 2;
        const float2 A = z[c];
        const float4 w = __ldg(sp + c);
        const float gc = __ldg(g + c).x;
        const float er = fm(0.5f, fa(A.x, A.x)), ei = fm(0.5f, fs(A.y, A.y));
        const float orr = fm(0.5f, fa(A.y, A.y)), oi = fm(0.5f, fs(A.x, A.x));
        const float Xr = fm(fs(fa(er, fm(w.x, orr)), fm(w.y, oi)), gc);
        const float Xi = fm(fa(fa(ei, fm(w.x, oi)), fm(w.y, orr)), gc);
        const float e_r = fa(Xr, Xr), e_i = fs(Xi, Xi), dr = fs(Xr, Xr), di = fa(Xi, Xi);
        const float wr = w.x, wi = -w.y;
        const float o_r = fs(fm(dr, wr), fm(di, wi)), o_i = fa(fm(dr, wi), fm(di, wr));
        z[c] = make_float2(fm(fa(e_i, o_r), scale), fm(fs(e_r, o_i), scale));
      }
      continue;
    }
    const int c = t, d = M - t;
    const float2 A = z[c], Bv = z[d];
    const float4 w = __ldg(sp + c);  // split twiddles of bins c (x, y) and m − c (z, w)
    const float2 gg = __ldg(g + c);  // gains of bins c and m − c
    const float er = fm(0.5f, fa(A.x, Bv.x)), ei = fm(0.5f, fs(A.y, Bv.y));
    const float orr = fm(0.5f, fa(A.y, Bv.y)), oi = fm(0.5f, fs(Bv.x, A.x));
    const float Xr = fm(fs(fa(er, fm(w.x, orr)), fm(w.y, oi)), gg.x);
    const float Xi = fm(fa(fa(ei, fm(w.x, oi)), fm(w.y, orr)), gg.x);
    const float Yr = fm(fs(fa(er, fm(w.z, orr)), fm(w.w, -oi)), gg.y);
    const float Yi = fm(fa(fa(-ei, fm(w.z, -oi)), fm(w.w, orr)), gg.y);
    // splitInverse of bin c (a = X, b = Y) and of bin m − c (a = Y, b = X)
    const float e_r = fa(Xr, Yr), e_i = fs(Xi, Yi), dr = fs(Xr, Yr), di = fa(Xi, Yi);
    {
      const float wr = w.x, wi = -w.y;
      const float o_r = fs(fm(dr, wr), fm(di, wi)), o_i = fa(fm(dr, wi), fm(di, wr));
      z[c] = make_float2(fm(fa(e_i, o_r), scale), fm(fs(e_r, o_i), scale));
    }
    {
      const float wr = w.z, wi = -w.w;
      const float o_r = fs(fm(-dr, wr), fm(di, wi)), o_i = fa(fm(-dr, wi), fm(di, wr));
      z[d] = make_float2(fm(fa(-e_i, o_r), scale), fm(fs(e_r, o_i), scale));
    }
  }
}

// ----------------------------------------------------------- pack, unpack
// packInto with zero pads (filter/apply.nim:194-216) as the first pass reads
// it: complex input c holds real samples 2c and 2c + 1 of the padded trace,
// sample j = i + p being x[i] − pre − (a + b·i) in float64 rounded once to
// float32 for 0 ≤ i < n, 0 in the pads.
struct PackLd {
  SRow X;
  int n, p;
  float pre;
  double a, b;
  // the demeaned sample x − pre (float32, as the demean step leaves it),
  // less the trend, each operation rounded as the reference's
  __device__ __forceinline__ float at(int i) const {
    const double t = __dadd_rn(a, __dmul_rn(b, (double)i));
    return __double2float_rn(__dsub_rn((double)fs(X[i], pre), t));
  }
  __device__ __forceinline__ float2 operator()(int c, int) const {
    const int i0 = 2 * c - p;
    float r0 = 0.f, r1 = 0.f;
    if ((unsigned)i0 < (unsigned)n) r0 = at(i0);
    if ((unsigned)(i0 + 1) < (unsigned)n) r1 = at(i0 + 1);
    return make_float2(r0, r1);
  }
};

// The real-FFT bridge (split · bin gain · unsplit · 1/n · swap) of
// BridgeLoad, reading the forward transform's output at zo.
struct BridgeLd {
  int zo, m;
  const Quad<float>* __restrict__ ab;
  __device__ __forceinline__ float2 operator()(int c, int j) const {
    const float2* z = smem_c() + zo;
    if (j == 0 && c == 0) {
      const float2 z0 = z[0];
      const float4 q = __ldg(reinterpret_cast<const float4*>(ab));
      const float x0 = (z0.x + z0.y) * q.x, xm = (z0.x - z0.y) * q.y;
      return make_float2(x0 - xm, x0 + xm);
    }
    const float2 u = z[c], v = z[m - c];
    const float4 q = __ldg(reinterpret_cast<const float4*>(ab) + c);
    // A·conj(u) + B·v
    return make_float2(q.x * u.x + q.y * u.y + q.z * v.x - q.w * v.y, q.y * u.x - q.x * u.y + q.z * v.y + q.w * v.x);
  }
};

// unpackFrom (filter/apply.nim:218-231) as the inverse transform's last pass
// writes: output c is the swapped pair of real samples 2c (its imaginary
// part) and 2c + 1 (its real part); sample j = i + p of the padded trace
// goes to x[i] for 0 ≤ i < n, plus the trend ga + gb·i in float64 when the
// filter passes it.
template <bool ADD> struct UnpackSt {
  SRow X;
  int n, p;
  double ga, gb;
  __device__ __forceinline__ void put(int i, float v) const {
    if ((unsigned)i < (unsigned)n) {
      if (ADD) v = __double2float_rn(__dadd_rn((double)v, __dadd_rn(ga, __dmul_rn(gb, (double)i))));
      X[i] = v;
    }
  }
  __device__ __forceinline__ void operator()(int c, float2 v) const {
    const int i0 = 2 * c - p;
    put(i0, v.y);
    put(i0 + 1, v.x);
  }
};

// ------------------------------------------------------------- reductions
// The CTA's static shared memory for the trace kernel: per-warp partial
// sums, the scalars one warp computes for the rest, the radix selection's
// histogram (normalization), and the row buffers' copy bookkeeping.
template <int NT> struct TkShared {
  static constexpr int W = NT / 32;
  double part[2][2][W];      // two sets (alternating reductions) of two sums per warp
  unsigned long long umax[2][W];
  float sc[8];               // scalars for the whole CTA
  double dsc[4];
  int isc[4];
};

// Each warp's sums of (x, y) in float64 into part[set]; lane 0 of warp 0
// later folds them (fold2). The caller puts a barrier between the two.
template <int NT> __device__ __forceinline__ void warp_sums2(double x, double y, TkShared<NT>& S, int set) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    x += __shfl_xor_sync(0xffffffffu, x, o);
    y += __shfl_xor_sync(0xffffffffu, y, o);
  }
  if ((threadIdx.x & 31) == 0) {
    S.part[set][0][threadIdx.x >> 5] = x;
    S.part[set][1][threadIdx.x >> 5] = y;
  }
}
// In lane 0 of warp 0 (after the barrier): the warps' sums in warp order.
template <int NT> __device__ __forceinline__ void fold2(const TkShared<NT>& S, int set, double& x, double& y) {
  x = 0;
  y = 0;
#pragma unroll
  for (int w = 0; w < NT / 32; w++) {
    x += S.part[set][0][w];
    y += S.part[set][1][w];
  }
}

// ----------------------------------------------------------------- the AGC
// The AGC of one trace (gain/gain.nim:351-461) from X[0, n) into Y[0, n),
// with r = 1/rms (the terms' scale), k = target/rms and eps as float32.
// Window groups: group g (g = 0 .. nb, nb blocks of w = 2h + 1 samples)
// holds the outputs i = (g − 1)·w + h + d, d < w; their window sum is the
// suffix sum from d of block g − 1 plus the exclusive prefix sum to d of
// block g (an absent block adds nothing; past the end of a short last
// block the prefix is that block's total, P[n]). Lane l holds d in
// [l·E, l·E + E). Each warp takes consecutive groups, carrying a block's
// terms from one group (its prefix side) to the next (its suffix side).
// The sums, divisors (w; i + h + 1 at the head; n at the whole-trace head;
// n − (i − h) at the tail) and gain are pipeline_kernel's.
template <int NT, int E, bool NEED_MX>
__device__ __forceinline__ unsigned long long agc_groups(const SRow X, const SRow Y, int n,
                                                         int h, bool rms_mode, float r, float k, float eps) {
  constexpr int W = NT / 32;
  const int w = 2 * h + 1;
  const int nb = (n + w - 1) / w;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int j0 = lane * E;
  const int G = nb + 1;
  const int per = (G + W - 1) / W;
  const int g0 = warp * per, g1 = min(G, g0 + per);
  const float invW = __frcp_rn((float)w);
  unsigned long long mx = 0;
  auto load = [&](float (&t)[E], int blk) {
    const int base = blk * w;
    const int L = (blk < 0 || blk >= nb) ? 0 : min(w, n - base);
#pragma unroll
    for (int e = 0; e < E; e++) {
      float v = 0.f;
      if (j0 + e < L) {
        const float s = X[base + j0 + e] * r;
        v = rms_mode ? s * s : fabsf(s);
      }
      t[e] = v;
    }
    return L;
  };
  if (g0 >= g1) return mx;
  float tc[E];
  load(tc, g0 - 1);
  for (int g = g0; g < g1; g++) {
    float tn[E];
    const int L1 = load(tn, g);  // block g: the prefix side
    // prefix sums of block g: the value at position j + 1 (j < L1) is
    // below + inc[j − l·E], as pipeline_kernel writes P
    float inc[E];
    float run = 0.f;
#pragma unroll
    for (int e = 0; e < E; e++) {
      run += tn[e];
      inc[e] = run;
    }
    const float below = warp_excl_prefix(run);
    const float prev_last = __shfl_up_sync(0xffffffffu, below + inc[E - 1], 1);  // P at j0 (lane l − 1's last)
    float pn = 0.f;  // P[n]: the short last block's total
    if (L1 > 0 && L1 < w) {
      const int jl = L1 - 1, ll = jl / E, el = jl - ll * E;
      float mine = 0.f;
#pragma unroll
      for (int e = 0; e < E; e++)
        if (e == el) mine = below + inc[e];
      pn = __shfl_sync(0xffffffffu, mine, ll);
    }
    // suffix sums of block g − 1: S at j = above + incs[j − l·E]
    float incs[E];
    run = 0.f;
#pragma unroll
    for (int e = E - 1; e >= 0; e--) {
      run += tc[e];
      incs[e] = run;
    }
    const float above = warp_excl_suffix(run);
    const int ibase = (g - 1) * w + h;  // the output at d = 0
    const bool interior = g >= 1 && (g + 1) * w - 2 < n;  // every output of the group has a whole window
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int d = j0 + e;
      const int i = ibase + d;
      if (d < w && i >= 0 && i < n) {
        float pv;
        if (d == 0) pv = 0.f;
        else if (d - 1 >= L1) pv = pn;
        else pv = e == 0 ? prev_last : below + inc[e - 1];
        const float sum = g >= 1 ? (above + incs[e]) + pv : pv;
        float inv;
        if (interior) {
          inv = invW;
        } else {
          const int cnt = min(i + h, n - 1) - max(i - h, 0) + 1;
          inv = cnt == w ? invW : __frcp_rn((float)cnt);
        }
        const float y = X[i] * agc_gain(sum * inv, k, eps, rms_mode);
        Y[i] = y;
        if (NEED_MX) {
          const unsigned long long bb = abs_bits(y);
          mx = bb > mx ? bb : mx;
        }
      }
    }
#pragma unroll
    for (int e = 0; e < E; e++) tc[e] = tn[e];
  }
  return mx;
}

// ------------------------------------------------------------------ kernel
// Stores a row from shared memory: 16-byte vectors where the destination
// allows, Y's elements [0, len) (Y placed so that Y + head is 16-byte
// aligned when `to` + head is).
template <int NT> __device__ __forceinline__ void store_row(const SRow Y, float* __restrict__ to, int len) {
  const int head = min((int)((4 - (((uintptr_t)to >> 2) & 3)) & 3), len);
  const int nv = (len - head) >> 2;
  for (int i = threadIdx.x; i < head; i += NT) to[i] = Y[i];
  float4* gv = reinterpret_cast<float4*>(to + head);
  if (((Y.o + head) & 3) == 0) {
    const float4* yv = reinterpret_cast<const float4*>(psg_dyn_smem) + ((Y.o + head) >> 2);
    for (int v = threadIdx.x; v < nv; v += NT) __stcs(gv + v, yv[v]);
  } else {
    for (int v = threadIdx.x; v < nv; v += NT) {
      const int i = head + 4 * v;
      __stcs(gv + v, make_float4(Y[i], Y[i + 1], Y[i + 2], Y[i + 3]));
    }
  }
  for (int i = head + 4 * nv + threadIdx.x; i < len; i += NT) to[i] = Y[i];
}

// The trace kernel: P the filter's transform, RECIPE the step chain
// (RC_DFA: demean, filter, AGC; RC_DFAN: then a per-trace normalization),
// PF the next row's bulk copy issued as soon as the row buffer is free (after
// the forward transform, or after a row that is only copied) so that it
// lands under the rest of the row's work, E the AGC's samples per lane (its
// window w ≤ 32·E), BATCH the rows of many requests' jobs in one launch
// (the request loop: a.jobs, a.row_begin, a.total_rows). Row handling (bulk
// copy, ragged ends, src → dst copy of dead rows and of samples past the
// live length) is pipeline_kernel's.
// Shared memory: the row buffer X, then the two transform buffers; the
// filtered trace F and the AGC's output Y take the transform buffers' place
// once the inverse transform no longer needs them.
template <class P, int RECIPE, bool PF, int E, bool BATCH = false>
__global__ void __launch_bounds__(P::NT, P::MINB) trace_kernel(PipeArgs a) {
  constexpr int NT = P::NT;
  static_assert(RECIPE != RC_DFAN || NT == kNT, "the normalization step runs at the pipeline kernels' CTA width");
  __shared__ TkShared<NT> S;
  __shared__ SharedMem smem;  // the radix selection of the normalization
  Shared SN{&smem, 0};
  __shared__ __align__(8) uint64_t bar;
  __shared__ RowSlot slot;
  __shared__ int s_ok;
  const long long total = BATCH ? a.total_rows : a.job.rows;
  constexpr int esz = 4;
  // thread 0: the bulk copy of row t into the row buffer
  auto issue = [&](long long t) {
    const RowCtx<float> c = row_ctx<float, BATCH>(a, t);
    const int len = c.copy ? c.cols : c.n;
    const uintptr_t ga = (uintptr_t)c.from, ge = ga + (uintptr_t)len * esz;
    const int off = (int)(ga & 15);
    uintptr_t lo = ga & ~(uintptr_t)15, hi = (ge + 15) & ~(uintptr_t)15;
    if (lo < (uintptr_t)c.blk_lo) lo += 16;
    if (hi > (uintptr_t)c.blk_hi) hi -= 16;
    if (len > 0 && hi > lo) {
      const int head = lo > ga ? (int)((lo - ga) / esz) : 0;
      const int tail = hi < ge ? (int)((hi - ga) / esz) : len;
      const uint32_t body = (uint32_t)(hi - lo);
      slot = RowSlot{head, tail, (int)body, len, off};
      mbar_arrive_expect_tx(&bar, body);
      bulk_load(psg_dyn_smem + off + ((long long)lo - (long long)ga), reinterpret_cast<const void*>(lo), body, &bar);
    } else {
      slot = RowSlot{len, len, 0, len, off};
      mbar_arrive(&bar);
    }
  };
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_init_fence();
    if (PF && blockIdx.x < total) issue(blockIdx.x);
  }
  __syncthreads();
  // the two transform buffers (complex offsets), after the row buffer
  const int ao = a.work_off / 8, bo = ao + P::BUF;
  uint32_t phase = 0;
  for (long long t = blockIdx.x; t < total; t += gridDim.x) {
    const long long tn = t + gridDim.x;
    if (!PF && threadIdx.x == 0) {
      fence_proxy_async();
      issue(t);
    }
    if (threadIdx.x < 32) {
      const bool ok = mbar_wait(&bar, phase, 1ll << 26);
      if (threadIdx.x == 0) s_ok = ok ? 1 : 0;
    }
    __syncthreads();
    if (!s_ok) {
      if (threadIdx.x == 0) {
        atomicExch(a.status, 1);
        mbar_wait(&bar, phase, 1ll << 26);
      }
      return;
    }
    mbar_try_wait(&bar, phase);
    phase ^= 1;
    const RowCtx<float> c = row_ctx<float, BATCH>(a, t);
    const RowSlot sl = slot;
    const SRow X{sl.off >> 2};
    for (int i = threadIdx.x; i < sl.head; i += NT) X[i] = c.from[i];
    for (int i = sl.tail + threadIdx.x; i < sl.len; i += NT) X[i] = c.from[i];
    if (sl.head > 0 || sl.tail < sl.len) __syncthreads();
    const int n = c.n;
    const int len = c.copy ? c.cols : n;
    bool issued = false;  // the same in every thread
    if (n > 0) {
      const DevStep* d = c.steps + c.first;
      const DevStep& fd = d[1];
      // (1) the demean (core/basic.nim:52-58): the mean of the live samples
      // from a float64 sum, rounded to float32; x' = x − mean in float32.
      // Every float64 sum of the kernel runs in the same order whatever the
      // build: kNT lanes each summing samples kNT apart, then the warps'
      // trees in warp order (a wider CTA's other warps add zeros), so the
      // builds of one transform length give the same bits.
      {
        double s1 = 0;
        if (threadIdx.x < kNT)
          for (int i = threadIdx.x; i < n; i += kNT) s1 += (double)X[i];
        warp_sums2<NT>(s1, 0.0, S, 0);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double s1, u;
        fold2<NT>(S, 0, s1, u);
        S.sc[0] = (float)(s1 / (double)n);
      }
      __syncthreads();
      const float mean = S.sc[0];
      // (2) the filter's trend of x' (filter/edges.nim:16-30): Σx' and
      // Σi·x' in float64
      {
        double s1 = 0, si = 0, ti = (double)threadIdx.x;
        if (threadIdx.x < kNT)
          for (int i = threadIdx.x; i < n; i += kNT, ti += (double)kNT) {
            const double v = (double)fs(X[i], mean);
            s1 += v;
            si += ti * v;
          }
        warp_sums2<NT>(s1, si, S, 1);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double s1, si;
        fold2<NT>(S, 1, s1, si);
        double ta, tb;
        trend_from(fd.trend, Stats{s1, si, 0, 0}, n, ta, tb);
        S.dsc[0] = ta;
        S.dsc[1] = tb;
      }
      __syncthreads();
      const double ta = S.dsc[0], tb = S.dsc[1];
      const float2* tw = reinterpret_cast<const float2*>(a.tw_pass);  // the build's per-pass twiddles
      const int pad = fd.pad;
      // the samples past the live length go out now, from the row buffer
      // that the next row's copy takes over after the forward transform
      for (int i = n + threadIdx.x; i < len; i += NT) c.to[i] = X[i];
      // (3) the forward transform of the packed trace
      ref_fft<P>(ao, bo, tw, PackLd{X, n, pad, mean, ta, tb}, BufSt{last_out<P>(ao, bo)});
      __syncthreads();
      if (PF && tn < total) {
        if (threadIdx.x == 0) {
          fence_proxy_async();
          issue(tn);
        }
        issued = true;
      }
      const int zo = last_out<P>(ao, bo);
      // (4) split, gains, unsplit and the inverse transform, its last pass
      // unpacking the filtered trace F into the buffer that pass does not
      // read; the AGC's output Y (aligned like the destination row) then
      // takes the buffer it read
      const double gb = tb * fd.dc_gain;
      const double ga = fd.zero_dc ? -gb * (double)(n - 1) / 2 : ta * fd.dc_gain;
      const int za = zo == ao ? bo : ao;  // the inverse's first pass writes the other buffer
      constexpr bool EVEN = P::NP % 2 == 0;
      const SRow F{2 * (EVEN ? zo : za)};
      const int yal = (int)(((uintptr_t)c.to >> 2) & 3);
      const SRow Y{2 * (EVEN ? za : zo) + (n + yal <= 2 * P::BUF ? yal : 0)};
      ref_bridge_pairs<P::M, NT>(zo, reinterpret_cast<const float4*>(fd.ref_split),
                                 reinterpret_cast<const float2*>(fd.ref_gain), fd.ref_scale);
      __syncthreads();
      const BufLd br{zo};
      if (ga == 0 && gb == 0) {
        ref_fft<P>(zo, za, tw, br, UnpackSt<false>{F, n, pad, 0, 0});
      } else {
        ref_fft<P>(zo, za, tw, br, UnpackSt<true>{F, n, pad, ga, gb});
      }
      __syncthreads();
      // (5) the AGC's level from Σx² of the filtered trace in float64 (each
      // square exact there)
      {
        double acc = 0;
        if (threadIdx.x < kNT)
          for (int i = threadIdx.x; i < n; i += kNT) {
            const double v = (double)F[i];
            acc = fma(v, v, acc);
          }
        warp_sums2<NT>(acc, 0.0, S, 0);
      }
      __syncthreads();
      const DevStep& ag = d[2];
      if (threadIdx.x == 0) {
        double s2d, unused;
        fold2<NT>(S, 0, s2d, unused);
        const double rms = sqrt(s2d / (double)n);
        const bool run = !(rms == 0 || !fits_d<float>(ag.target / rms / ag.epsilon));
        S.isc[1] = run ? 1 : 0;
        S.sc[1] = (float)(1 / rms);
        S.sc[2] = (float)(ag.target / rms);
        S.sc[3] = (float)ag.epsilon;
      }
      __syncthreads();
      const bool agc_run = S.isc[1] != 0;
      unsigned long long mx = 0;
      if (agc_run) {
        mx = agc_groups<NT, E, RECIPE == RC_DFAN>(F, Y, n, ag.half, ag.agc_mode == PSG_AGC_RMS, S.sc[1], S.sc[2],
                                                  S.sc[3]);
      } else if (RECIPE == RC_DFAN) {
        for (int i = threadIdx.x; i < n; i += NT) {
          const unsigned long long bb = abs_bits(F[i]);
          mx = bb > mx ? bb : mx;
        }
      }
      const SRow Z = agc_run ? Y : F;  // the row's processed samples
      if constexpr (RECIPE == RC_DFAN) {
        // (6) per-trace normalization of the AGC's output (its max |x| for
        // the NaN rule of the percentile, gain/gain.nim:198-219)
        float* z = reinterpret_cast<float*>(psg_dyn_smem) + Z.o;
        Stats st{0, 0, 0, 0};
        st.mx = bits_value(block_max_u64(mx, SN.m->redu[SN.flip]), 0.f);
        SN.flip ^= 1;
        const DevStep& nd = d[3];
        if (nd.stat == PSG_NORM_RMS) {
          // Σx² of the normalization's input: a float64 pass (not fused; the
          // benchmarked chains normalize by a percentile)
          double acc = 0;
          for (int i = threadIdx.x; i < n; i += NT) acc += (double)z[i] * (double)z[i];
          st.s2 = block_sum(acc, SN.m->red[SN.flip][0]);
          SN.flip ^= 1;
          __syncthreads();
        }
        __syncthreads();
        step_norm_trace<float, 0>(nd, st, z, n, SN);
      }
      // (7) the processed samples out, 16-byte stores where the
      // destination allows
      __syncthreads();
      store_row<NT>(Z, c.to, n);
    } else if (c.copy) {
      // a dead row (or one with no live samples): copied as it is
      store_row<NT>(X, c.to, len);
    }
    __syncthreads();
    if (PF && !issued && tn < total && threadIdx.x == 0) {
      fence_proxy_async();
      issue(tn);
    }
  }
}

// ------------------------------------------------------------ correlation
// A record's complex input c: samples 2c and 2c + 1 from global memory (the
// forward transform's first pass reads them there), 0 past its n samples.
struct RecLd {
  const float* __restrict__ x;
  int n;
  bool al8;  // x is 8-byte aligned: a pair of samples in one load
  __device__ __forceinline__ float2 operator()(int c, int) const {
    const int k = 2 * c;
    if (al8 && k + 1 < n) return __ldg(reinterpret_cast<const float2*>(x) + c);
    return make_float2(k < n ? __ldg(x + k) : 0.f, k + 1 < n ? __ldg(x + k + 1) : 0.f);
  }
};

// correlateInto (vibroseis/correlate.nim:205-300, 421-464) with the
// transform of plan P, one record per CTA pass: the forward transform of the
// zero-padded record, the bridge × conj(pilot spectrum) × phase map read by
// the inverse transform's first pass, then corr_rows's lag scatter
// (lagSpans: column c reads lag c + shift, wrapped by nfft for negative
// lags) and the vertical-stack add (vstack.nim:186-202, rows with a
// non-finite value skipped).
template <class P>
__global__ void __launch_bounds__(P::NT, P::MINB) corr_trace_kernel(CorrArgs a) {
  constexpr int NT = P::NT, M = P::M;
  __shared__ SharedMem S;
  const float* src = reinterpret_cast<const float*>(a.src);
  float* dst = reinterpret_cast<float*>(a.dst);
  const float2* tw = reinterpret_cast<const float2*>(a.tw_pass);
  const Quad<float>* ab = reinterpret_cast<const Quad<float>*>(a.bridge);
  const int wrapped = min(max(1 - a.pilot_len - a.shift, 0), a.out);
  const int direct = min(max(-a.shift, wrapped), a.out);
  const int last = min(max(a.record - a.shift, direct), a.out);
  constexpr int zo = P::NP % 2 == 0 ? 0 : M;       // the forward transform's output
  constexpr int za = zo == 0 ? M : 0;
  constexpr int yo = P::NP % 2 == 0 ? zo : za;     // the inverse transform's output
  for (long long r = blockIdx.x; r < a.rows; r += gridDim.x) {
    const int n = min(max(a.live[r], 0), a.cols);
    const float2* y = nullptr;
    if (n > 0) {
      const float* rx = src + r * (long long)a.cols;
      fft<P>(0, M, tw, RecLd{rx, n, ((uintptr_t)rx & 7) == 0}, BufSt{zo});
      __syncthreads();
      fft<P>(zo, za, tw, BridgeLd{zo, M, ab}, BufSt{yo});
      __syncthreads();
      y = smem_c() + yo;
    }
    auto value = [&](int c) -> float {
      if (!y || c < wrapped || c >= last) return 0.f;
      const int idx = c < direct ? c + a.shift + a.nfft : c + a.shift;
      const float2 v = y[idx >> 1];
      return (idx & 1) ? v.x : v.y;
    };
    const int o = a.stack_on ? (a.row_map ? a.row_map[r] : (int)r) : -1;
    const int sn = !a.stack_on ? 0
                   : a.stack_live ? min(max(a.stack_live[r], 0), a.stack_samples) : min(a.out, a.stack_samples);
    const bool take = a.stack_on && o >= 0 && o < a.stack_rows && sn > 0;
    constexpr int KV = 8;  // output samples a thread keeps in registers
    if (max(a.out, sn) <= KV * NT) {
      // one pass over the lags: the output row, the finite check and the
      // values the stack adds, kept in registers
      float vals[KV];
      double bad = 0;
      float* d = dst ? dst + r * (long long)a.out : nullptr;
#pragma unroll
      for (int k = 0; k < KV; k++) {
        const int c = threadIdx.x + k * NT;
        const float v = value(c);
        vals[k] = v;
        if (d && c < a.out) d[c] = v;
        if (take && c < sn) bad += (double)v - (double)v;  // allFinite: x − x is 0 for finite x
      }
      if (take) {
        bad = block_sum(bad, S.red[0][0]);
        if (bad == 0) {
          double* nm = a.num + (long long)o * a.stack_samples;
          int* ct = a.cnt + (long long)o * a.stack_samples;
#pragma unroll
          for (int k = 0; k < KV; k++) {
            const int c = threadIdx.x + k * NT;
            if (c < sn) {
              atomicAdd(nm + c, (double)vals[k]);
              atomicAdd(ct + c, 1);
            }
          }
        }
      }
      __syncthreads();
      continue;
    }
    if (dst) {
      float* d = dst + r * (long long)a.out;
      for (int c = threadIdx.x; c < a.out; c += NT) d[c] = value(c);
    }
    if (a.stack_on) {
      if (take) {
        double bad = 0;
        for (int c = threadIdx.x; c < sn; c += NT) {
          const double v = (double)value(c);
          bad += v - v;  // allFinite: x − x is 0 for finite x
        }
        bad = block_sum(bad, S.red[0][0]);
        if (bad == 0) {
          double* nm = a.num + (long long)o * a.stack_samples;
          int* ct = a.cnt + (long long)o * a.stack_samples;
          for (int c = threadIdx.x; c < sn; c += NT) {
            atomicAdd(nm + c, (double)value(c));
            atomicAdd(ct + c, 1);
          }
        }
      }
    }
    __syncthreads();
  }
}

// The host's description of a trace-kernel build (psg_trace.h): plan P with
// AGC lane width E, its kernels by recipe and prefetch (the normalization
// recipe only at the pipeline kernels' CTA width).
template <class P, int E> TracePlanInfo info() {
  TracePlanInfo t{};
  t.m = P::M;
  t.nt = P::NT;
  t.np = P::NP;
  for (int i = 0; i < P::NP; i++) {
    t.radix[i] = P::radix(i);
    t.g1[i] = P::G1[i];
    t.g2[i] = P::G2[i];
  }
  t.agc_e = E;
  t.min_blocks = P::MINB;
  t.buf = P::BUF;
  t.kernel[0][0] = (const void*)trace_kernel<P, RC_DFA, false, E>;
  t.kernel[0][1] = (const void*)trace_kernel<P, RC_DFA, true, E>;
  if constexpr (P::NT == kNT) {
    t.kernel[1][0] = (const void*)trace_kernel<P, RC_DFAN, false, E>;
    t.kernel[1][1] = (const void*)trace_kernel<P, RC_DFAN, true, E>;
  }
  return t;
}

// The same with the request loop's batched kernels (the prefetch form).
template <class P, int E> TracePlanInfo info_served() {
  TracePlanInfo t = info<P, E>();
  t.batch[0] = (const void*)trace_kernel<P, RC_DFA, true, E, true>;
  if constexpr (P::NT == kNT) t.batch[1] = (const void*)trace_kernel<P, RC_DFAN, true, E, true>;
  return t;
}

// The same for a correlation build (kernel[0][0]).
template <class P> TracePlanInfo corr_info() {
  TracePlanInfo t{};
  t.m = P::M;
  t.nt = P::NT;
  t.np = P::NP;
  for (int i = 0; i < P::NP; i++) {
    t.radix[i] = P::radix(i);
    t.g1[i] = P::radix(i);
  }
  t.min_blocks = P::MINB;
  t.buf = P::M;
  t.kernel[0][0] = (const void*)corr_trace_kernel<P>;
  return t;
}

}  // namespace tk

}  // namespace psg
