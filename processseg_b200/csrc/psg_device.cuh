// psg_device.cuh — device building blocks of libpsgcuda.so: complex helpers,
// block reductions and the shared-memory mixed-radix FFT.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "psg_dft_consts.h"

namespace psgd {

template <class T> struct C2;
template <> struct C2<float> { typedef float2 type; };
template <> struct C2<double> { typedef double2 type; };

template <class V> __device__ __forceinline__ V cadd(V a, V b) { return {a.x + b.x, a.y + b.y}; }
template <class V> __device__ __forceinline__ V csub(V a, V b) { return {a.x - b.x, a.y - b.y}; }
// (a·w) as the reference's mulTw: re = ar·wr − ai·wi, im = ar·wi + ai·wr
template <class V> __device__ __forceinline__ V cmul(V a, V w) {
  return {a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x};
}
// −i·a
template <class V> __device__ __forceinline__ V cmul_negi(V a) { return {a.y, -a.x}; }

// ------------------------------------------------------------ reductions
// Sums over the block; every thread gets the result. `red` holds ≥ 32 values.
template <class T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <class T> __device__ T block_sum(T v, T* red) {
  v = warp_sum(v);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  T r = l < nw ? red[l] : (T)0;
  r = warp_sum(r);
  return r;
}
__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
    v = u > v ? u : v;
  }
  return v;
}
__device__ inline unsigned long long block_max_u64(unsigned long long v, unsigned long long* red) {
  v = warp_max_u64(v);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  unsigned long long r = l < nw ? red[l] : 0ull;
  return warp_max_u64(r);
}

// Bits of |x| as an unsigned integer: for non-negative floats the integer
// order is the float order, and every NaN sorts above +Inf
// (gain/stats.nim:97-117).
__device__ __forceinline__ unsigned long long abs_bits(float v) {
  return (unsigned long long)(__float_as_uint(v) & 0x7FFFFFFFu);
}
__device__ __forceinline__ unsigned long long abs_bits(double v) {
  return (unsigned long long)__double_as_longlong(v) & 0x7FFFFFFFFFFFFFFFull;
}
__device__ __forceinline__ double bits_value(unsigned long long b, float) {
  return (double)__uint_as_float((unsigned)b);
}
__device__ __forceinline__ double bits_value(unsigned long long b, double) {
  return __longlong_as_double((long long)b);
}

// ------------------------------------------------------------ small DFTs
// Forward DFTs of 2, 3, 4, 5 and 8 points in registers (ω = exp(−2πi/R)).
// The 2..5-point forms are the butterflies of src/processSEG/fft/plan.nim:225-366.
template <class V, class T> __device__ __forceinline__ void dft2(V* v) {
  V a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}
template <class V, class T> __device__ __forceinline__ void dft3(V* v) {
  const T c = (T)-0.5, s = (T)0.8660254037844386467637231707529362;
  V a = v[0];
  V t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
  V m1 = {a.x + c * t1.x, a.y + c * t1.y};
  V m2 = {s * t2.y, -s * t2.x};
  v[0] = cadd(a, t1);
  v[1] = cadd(m1, m2);
  v[2] = csub(m1, m2);
}
template <class V, class T> __device__ __forceinline__ void dft4(V* v) {
  V t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
  V t2 = cadd(v[1], v[3]);
  V t3 = {v[1].y - v[3].y, v[3].x - v[1].x};  // (x1 − x3)·(−i)
  v[0] = cadd(t0, t2);
  v[1] = cadd(t1, t3);
  v[2] = csub(t0, t2);
  v[3] = csub(t1, t3);
}
template <class V, class T> __device__ __forceinline__ void dft5(V* v) {
  const T c1 = (T)0.3090169943749474241022934171828191, c2 = (T)-0.8090169943749474241022934171828191;
  const T s1 = (T)0.9510565162951535721164393333793821, s2 = (T)0.5877852522924731291687059546390728;
  V a = v[0];
  V t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]), t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
  V b1 = {a.x + c1 * t1.x + c2 * t2.x, a.y + c1 * t1.y + c2 * t2.y};
  V b2 = {a.x + c2 * t1.x + c1 * t2.x, a.y + c2 * t1.y + c1 * t2.y};
  V d1 = {s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y};
  V d2 = {s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y};
  v[0] = {a.x + t1.x + t2.x, a.y + t1.y + t2.y};
  v[1] = {b1.x + d1.y, b1.y - d1.x};
  v[4] = {b1.x - d1.y, b1.y + d1.x};
  v[2] = {b2.x + d2.y, b2.y - d2.x};
  v[3] = {b2.x - d2.y, b2.y + d2.x};
}
// 8 points as two 4-point DFTs and a radix-2 combine with ω8^k.
template <class V, class T> __device__ __forceinline__ void dft8(V* v) {
  const T h = (T)0.7071067811865475244008443621048490;
  V e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
  dft4<V, T>(e);
  dft4<V, T>(o);
  V o1 = {(o[1].x + o[1].y) * h, (o[1].y - o[1].x) * h};   // ·(√½ − i√½)
  V o2 = cmul_negi(o[2]);                                      // ·(−i)
  V o3 = {(o[3].y - o[3].x) * h, -(o[3].x + o[3].y) * h};   // ·(−√½ − i√½)
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], o1);
  v[5] = csub(e[1], o1);
  v[2] = cadd(e[2], o2);
  v[6] = csub(e[2], o2);
  v[3] = cadd(e[3], o3);
  v[7] = csub(e[3], o3);
}

// Multiplication by a compile-time constant twiddle (c, s); quarter turns
// fold to swaps and negations.
template <class V, class T> __device__ __forceinline__ V cmul_k(V a, double c, double s) {
  if (c == 1.0 && s == 0.0) return a;
  if (c == 0.0 && s == -1.0) return V{a.y, -a.x};
  if (c == -1.0 && s == 0.0) return V{-a.x, -a.y};
  if (c == 0.0 && s == 1.0) return V{-a.y, a.x};
  const T tc = (T)c, ts = (T)s;
  return V{a.x * tc - a.y * ts, a.x * ts + a.y * tc};
}

template <class V, class T, int R> struct Dft;
template <class V, class T> struct Dft<V, T, 2> { static __device__ __forceinline__ void run(V* v) { dft2<V, T>(v); } };
template <class V, class T> struct Dft<V, T, 3> { static __device__ __forceinline__ void run(V* v) { dft3<V, T>(v); } };
template <class V, class T> struct Dft<V, T, 4> { static __device__ __forceinline__ void run(V* v) { dft4<V, T>(v); } };
template <class V, class T> struct Dft<V, T, 5> { static __device__ __forceinline__ void run(V* v) { dft5<V, T>(v); } };
template <class V, class T> struct Dft<V, T, 8> { static __device__ __forceinline__ void run(V* v) { dft8<V, T>(v); } };

// A DFT of R = A·B points in registers: B DFTs of A points on the inputs
// B apart, twiddles ω_R^{j2·k1}, then A DFTs of B points:
//   X[k1 + A·k2] = Σ_j2 ω_B^{j2·k2} ω_R^{j2·k1} Σ_j1 x[B·j1 + j2] ω_A^{j1·k1}
template <class V, class T, int A, int B> struct DftAB {
  static __device__ __forceinline__ void run(V* v) {
    constexpr int R = A * B;
    V y[R];
#pragma unroll
    for (int j2 = 0; j2 < B; j2++) {
      V u[A];
#pragma unroll
      for (int j1 = 0; j1 < A; j1++) u[j1] = v[B * j1 + j2];
      Dft<V, T, A>::run(u);
#pragma unroll
      for (int k1 = 0; k1 < A; k1++) {
        const int e = (j2 * k1) % R;
        y[j2 * A + k1] = cmul_k<V, T>(u[k1], DftW<R>::c(e), DftW<R>::s(e));
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < A; k1++) {
      V z[B];
#pragma unroll
      for (int j2 = 0; j2 < B; j2++) z[j2] = y[j2 * A + k1];
      Dft<V, T, B>::run(z);
#pragma unroll
      for (int k2 = 0; k2 < B; k2++) v[k1 + A * k2] = z[k2];
    }
  }
};
template <class V, class T> struct Dft<V, T, 6> : DftAB<V, T, 2, 3> {};
template <class V, class T> struct Dft<V, T, 9> : DftAB<V, T, 3, 3> {};
template <class V, class T> struct Dft<V, T, 10> : DftAB<V, T, 2, 5> {};
template <class V, class T> struct Dft<V, T, 12> : DftAB<V, T, 4, 3> {};
template <class V, class T> struct Dft<V, T, 15> : DftAB<V, T, 3, 5> {};
template <class V, class T> struct Dft<V, T, 16> : DftAB<V, T, 4, 4> {};

// The block's dynamic shared memory. The FFT buffers are addressed as
// offsets from this symbol, so the compiler emits shared-memory loads and
// stores with 32-bit addresses (a pointer chosen at run time between two
// buffers would fall back to generic 64-bit addressing).
extern __shared__ __align__(16) unsigned char psg_dyn_smem[];

// Where an FFT's two work buffers live: the block's dynamic shared memory,
// or (for transforms longer than it holds) a slice of global memory.
struct InShared {
  __device__ __forceinline__ unsigned char* base() const { return psg_dyn_smem; }
};
struct InGlobal {
  unsigned char* b;
  __device__ __forceinline__ unsigned char* base() const { return b; }
};

// One decimation-in-frequency Stockham pass of radix R over `s · sub`
// butterflies (fft/plan.nim:187-190):
//   y[q + s·(R·p + k)] = (Σ_j x[q + s·(p + j·sub)]·ω_R^{jk})·ω_cur^{pk}
// with cur = R·sub = m / s, so ω_cur^{pk} = tw[p·k·s] from the one table
// tw[e] = ω_m^e of the transform; x and y are element offsets into the
// buffer memory. Butterfly b = p·s + q: p = ⌊b / s⌋ from a multiply-high by
// magic = ⌈2^32 / s⌉ — ⌊b / s⌋ or one more for b < 2^31 — and one correction
// (magic = 0 marks s = 1).
// LAST: the transform's last pass (sub = 1, so p = 0 and every twiddle is 1).
template <int R, class T, int NT, bool LAST, class M>
__device__ __forceinline__ void fft_pass(const M& mem, int xo, int yo, int s, int sub, unsigned magic,
                                         const typename C2<T>::type* __restrict__ tw) {
  const int nt = NT ? NT : (int)blockDim.x;
  typedef typename C2<T>::type V;
  V* buf = reinterpret_cast<V*>(mem.base());
  const int total = s * sub;  // also the distance between a butterfly's inputs
  for (int b = threadIdx.x; b < total; b += nt) {
    int p = LAST ? 0 : (magic ? (int)__umulhi((unsigned)b, magic) : b);
    if (!LAST && p * s > b) p--;
    const int q = b - p * s;
    V v[R];
    const V* x = buf + (xo + q + s * p);
#pragma unroll
    for (int j = 0; j < R; j++) v[j] = x[j * total];
    Dft<V, T, R>::run(v);
    if (!LAST) {
      const int ps = p * s;
#pragma unroll
      for (int k = 1; k < R; k++) v[k] = cmul(v[k], __ldg(&tw[ps * k]));
    }
    V* y = buf + (yo + q + s * R * p);
#pragma unroll
    for (int k = 0; k < R; k++) y[s * k] = v[k];
  }
}

// The FFT passes of a plan, as the device reads them.
struct FftDesc {
  int m;          // complex length
  int npass;
  int radix[24];
  unsigned magic[24];  // ⌈2^32 / s⌉ of each pass, 0 for s = 1
};

// Runs f(std::integral_constant<int, R>) for the plan's radix r at run time;
// radices above MAXR are not compiled in (the plan never uses them).
template <int MAXR, class F> __device__ __forceinline__ void with_radix(int r, F&& f) {
  switch (r) {
    case 16: if constexpr (MAXR >= 16) f(std::integral_constant<int, 16>{}); break;
    case 15: if constexpr (MAXR >= 15) f(std::integral_constant<int, 15>{}); break;
    case 12: if constexpr (MAXR >= 12) f(std::integral_constant<int, 12>{}); break;
    case 10: if constexpr (MAXR >= 10) f(std::integral_constant<int, 10>{}); break;
    case 9: if constexpr (MAXR >= 9) f(std::integral_constant<int, 9>{}); break;
    case 8: f(std::integral_constant<int, 8>{}); break;
    case 6: f(std::integral_constant<int, 6>{}); break;
    case 5: f(std::integral_constant<int, 5>{}); break;
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 3: f(std::integral_constant<int, 3>{}); break;
    default: f(std::integral_constant<int, 2>{}); break;
  }
}

// The passes i0 .. npass − 1 of a transform, from the buffer at x (the
// other at y), `cur` points per sub-transform and stride s at pass i0.
// Returns the offset holding the result; each pass ends with a
// __syncthreads().
template <class T, int MAXR, int NT, class M>
__device__ __forceinline__ int cfft_passes(const M& mem, int x, int y, const FftDesc& d,
                                        const typename C2<T>::type* tw, int i0, int cur, int s) {
  for (int i = i0; i < d.npass; i++) {
    const int r = d.radix[i];
    const int sub = cur / r;
    const unsigned mg = d.magic[i];
    with_radix<MAXR>(r, [&](auto R) {
      if (sub == 1) fft_pass<decltype(R)::value, T, NT, true>(mem, x, y, s, sub, mg, tw);
      else fft_pass<decltype(R)::value, T, NT, false>(mem, x, y, s, sub, mg, tw);
    });
    __syncthreads();
    cur = sub;
    s *= r;
    const int tmp = x;
    x = y;
    y = tmp;
  }
  return x;
}

// Forward complex FFT of the m points at offset `ao`, `bo` the second
// buffer. Returns the offset holding the result; ends with a
// __syncthreads(). MAXR bounds the radices compiled in (and with them the
// registers a pass needs); the plan's factorization never uses a larger one.
// NT: the CTA's thread count when known at compile time (0: blockDim.x).
template <class T, int MAXR, int NT = 0, class M>
__device__ __forceinline__ int cfft_forward(const M& mem, int ao, int bo, const FftDesc& d,
                                         const typename C2<T>::type* tw) {
  return cfft_passes<T, MAXR, NT>(mem, ao, bo, d, tw, 0, d.m, 1);
}

// The first pass (stride 1) with its inputs from ld(c, j == 0), the c-th
// complex input of the transform (c = p + j·sub, so c = 0 only for j = 0),
// instead of a buffer: the pass that fuses its inputs' producer into its
// loads. The outputs go to the buffer at yo.
template <int R, class T, int NT, bool LAST, class M, class LD>
__device__ __forceinline__ void fft_pass_loaded(const M& mem, int yo, int sub, const typename C2<T>::type* __restrict__ tw,
                                                const LD& ld) {
  const int nt = NT ? NT : (int)blockDim.x;
  typedef typename C2<T>::type V;
  V* buf = reinterpret_cast<V*>(mem.base());
  for (int p = threadIdx.x; p < sub; p += nt) {
    V v[R];
#pragma unroll
    for (int j = 0; j < R; j++) v[j] = ld(p + j * sub, j == 0);
    Dft<V, T, R>::run(v);
    if (!LAST) {
#pragma unroll
      for (int k = 1; k < R; k++) v[k] = cmul(v[k], __ldg(&tw[p * k]));
    }
    V* y = buf + (yo + R * p);
#pragma unroll
    for (int k = 0; k < R; k++) y[k] = v[k];
  }
}

// Forward complex FFT whose m inputs come from ld (as fft_pass_loaded) rather
// than a buffer; `bo` and `ao` are the two work buffers (the first pass
// writes bo, so ld may read ao). Returns the offset holding the result.
template <class T, int MAXR, int NT, class M, class LD>
__device__ __forceinline__ int cfft_forward_loaded(const M& mem, int bo, int ao, const FftDesc& d,
                                                const typename C2<T>::type* tw, const LD& ld) {
  if (d.npass == 0) {
    // a transform of one point (no passes): the input itself, in bo
    typedef typename C2<T>::type V;
    V* buf = reinterpret_cast<V*>(mem.base());
    for (int c = threadIdx.x; c < d.m; c += (NT ? NT : (int)blockDim.x)) buf[bo + c] = ld(c, true);
    __syncthreads();
    return bo;
  }
  const int r = d.radix[0];
  const int sub = d.m / r;
  with_radix<MAXR>(r, [&](auto R) {
    if (sub == 1) fft_pass_loaded<decltype(R)::value, T, NT, true>(mem, bo, sub, tw, ld);
    else fft_pass_loaded<decltype(R)::value, T, NT, false>(mem, bo, sub, tw, ld);
  });
  __syncthreads();
  return cfft_passes<T, MAXR, NT>(mem, bo, ao, d, tw, 1, sub, r);
}

// Four values of T: a bin's pair of complex coefficients.
template <class T> struct alignas(4 * sizeof(T)) Quad { T x, y, z, w; };

// The real-FFT bridge between the forward and inverse complex transforms of
// a real trace of n = 2m samples packed as z[k] = x[2k] + i·x[2k+1]
// (fft/plan.nim:470-499): split into the spectrum X[k], multiply by the
// bin's factor M[k], un-split, scale by 1/n and swap re/im for the forward
// transform that inverts it. All of it is linear in (z[k], conj z[m − k]),
// so for each pair of bins it is one 2×2 map,
//   z'[k] = A'_k·conj(z[k]) + B'_k·z[m − k],
// with A'_k, B'_k computed on the host in float64 from ω^k = exp(−2πik/n),
// M[k], M[m − k] and 1/n (bridge_table). Bin 0 keeps the reference's real
// forms of the DC and Nyquist bins (the imaginary parts of M·X there are
// dropped): ab[0] = (Re M[0]/n, Re M[m]/n).
// z'[c] is computed where it is read: the first pass of the inverse transform
// loads its inputs through BridgeLoad instead of a buffer (a pass, a barrier
// and a store per bin fewer than bridging in place). Reads z at zo.
template <class T, class M> struct BridgeLoad {
  typedef typename C2<T>::type V;
  const M& mem;
  int zo, m;
  const Quad<T>* __restrict__ ab;
  __device__ __forceinline__ V operator()(int c, bool maybe_zero) const {
    const V* z = reinterpret_cast<const V*>(mem.base()) + zo;
    if (maybe_zero && c == 0) {
      const V z0 = z[0];
      const Quad<T> q = ab[0];
      const T x0 = (z0.x + z0.y) * q.x, xm = (z0.x - z0.y) * q.y;
      return V{x0 - xm, x0 + xm};
    }
    const V a = z[c], b = z[m - c];
    const Quad<T> q = ab[c];
    // A·conj(a) + B·b
    return V{q.x * a.x + q.y * a.y + q.z * b.x - q.w * b.y, q.y * a.x - q.x * a.y + q.z * b.y + q.w * b.x};
  }
};

// ------------------------------------------------- bulk copies (TMA, 1-D)
// A row moves from global into shared memory with one cp.async.bulk issued
// by one thread, completion tracked by an mbarrier carrying the byte count.
// Both addresses and the size are multiples of 16 bytes. No multicast: the
// destination is this CTA's own shared memory.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Orders this thread's earlier generic-proxy accesses of shared memory
// before later async-proxy (bulk copy) writes to it.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst_smem)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for a phase of `bar`, giving up after `limit` polls (each poll may
// suspend the thread for a while in hardware). Returns false on give-up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit) {
  for (long long i = 0; i < limit; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

}  // namespace psgd
