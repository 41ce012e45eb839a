// psg_device.cuh — device building blocks of libpsgcuda.so: complex helpers,
// block reductions and the shared-memory mixed-radix FFT.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

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
__device__ unsigned long long block_max_u64(unsigned long long v, unsigned long long* red) {
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

// One decimation-in-frequency Stockham pass of radix R over `s · sub`
// butterflies (fft/plan.nim:187-190):
//   y[q + s·(R·p + k)] = (Σ_j x[q + s·(p + j·sub)]·ω_R^{jk})·ω_cur^{pk}
// with the pass's twiddles tw[p·(R − 1) + k − 1] = ω_cur^{pk}.
template <int R, class T>
__device__ __forceinline__ void fft_pass(const typename C2<T>::type* __restrict__ x,
                                         typename C2<T>::type* __restrict__ y, int s, int sub,
                                         const typename C2<T>::type* __restrict__ tw) {
  typedef typename C2<T>::type V;
  const int total = s * sub;
  const float inv_s = 1.0f / (float)s;
  for (int b = threadIdx.x; b < total; b += blockDim.x) {
    int p = (int)((float)b * inv_s);
    if (p * s > b) p--;
    else if ((p + 1) * s <= b) p++;
    const int q = b - p * s;
    V v[R];
#pragma unroll
    for (int j = 0; j < R; j++) v[j] = x[q + s * (p + j * sub)];
    if (R == 2) dft2<V, T>(v);
    else if (R == 3) dft3<V, T>(v);
    else if (R == 4) dft4<V, T>(v);
    else if (R == 5) dft5<V, T>(v);
    else dft8<V, T>(v);
    const V* t = tw + p * (R - 1);
#pragma unroll
    for (int k = 1; k < R; k++) v[k] = cmul(v[k], __ldg(&t[k - 1]));
    V* o = y + q + s * R * p;
#pragma unroll
    for (int k = 0; k < R; k++) o[s * k] = v[k];
  }
}

// The FFT passes of a plan, as the device reads them.
struct FftDesc {
  int m;          // complex length
  int npass;
  int radix[24];
  int twoff[24];  // offset of each pass's twiddles
};

// Forward complex FFT of `a` (m points), `b` the second buffer. Returns the
// buffer holding the result. Ends with a __syncthreads().
template <class T>
__device__ typename C2<T>::type* cfft_forward(typename C2<T>::type* a, typename C2<T>::type* b,
                                              const FftDesc& d, const typename C2<T>::type* tw) {
  typedef typename C2<T>::type V;
  V* x = a;
  V* y = b;
  int cur = d.m, s = 1;
  for (int i = 0; i < d.npass; i++) {
    const int r = d.radix[i];
    const int sub = cur / r;
    const V* t = tw + d.twoff[i];
    switch (r) {
      case 8: fft_pass<8, T>(x, y, s, sub, t); break;
      case 4: fft_pass<4, T>(x, y, s, sub, t); break;
      case 2: fft_pass<2, T>(x, y, s, sub, t); break;
      case 3: fft_pass<3, T>(x, y, s, sub, t); break;
      default: fft_pass<5, T>(x, y, s, sub, t); break;
    }
    __syncthreads();
    cur = sub;
    s *= r;
    V* tmp = x;
    x = y;
    y = tmp;
  }
  return x;
}

// The real-FFT bridge between the forward and inverse complex transforms of
// a real trace of n = 2m samples packed as z[k] = x[2k] + i·x[2k+1]
// (fft/plan.nim:470-499), fused into one in-place pass over the pairs
// (k, m − k): split into the spectrum X[k], multiply by the bin's complex
// factor (a real gain: im = 0), and un-split into swap(Z'), scaled by 1/n,
// ready for the forward transform that inverts it.
template <class T, class MulFn>
__device__ void split_mul_unsplit(typename C2<T>::type* z, int m, const typename C2<T>::type* split,
                                  T scale, MulFn mul) {
  typedef typename C2<T>::type V;
  const T half = (T)0.5;
  for (int k = threadIdx.x; k <= m / 2; k += blockDim.x) {
    if (k == 0) {
      V z0 = z[0];
      V x0 = {z0.x + z0.y, (T)0}, xm = {z0.x - z0.y, (T)0};
      x0 = mul(x0, 0);
      xm = mul(xm, m);
      // ai[0] = (x0 + xm)·scale = Re Z'0, ar[0] = (x0 − xm)·scale = Im Z'0; stored swapped.
      z[0] = {(x0.x - xm.x) * scale, (x0.x + xm.x) * scale};
      continue;
    }
    const int j = m - k;
    V a = z[k], b = z[j];
    V wk = __ldg(&split[k]), wj = __ldg(&split[j]);
    // forward split at k (a = Z[k], b = Z[m−k]) and at m − k (roles swapped)
    V Xk, Xj;
    {
      T er = half * (a.x + b.x), ei = half * (a.y - b.y), orr = half * (a.y + b.y), oi = half * (b.x - a.x);
      Xk = {er + wk.x * orr - wk.y * oi, ei + wk.x * oi + wk.y * orr};
    }
    {
      T er = half * (b.x + a.x), ei = half * (b.y - a.y), orr = half * (b.y + a.y), oi = half * (a.x - b.x);
      Xj = {er + wj.x * orr - wj.y * oi, ei + wj.x * oi + wj.y * orr};
    }
    Xk = mul(Xk, k);
    Xj = mul(Xj, j);
    // inverse split at k (ar = X[k], br = X[m−k], ω = (wr, −wi)), stored as swap(Z')
    V Zk, Zj;
    {
      T wr = wk.x, wi = -wk.y;
      T er = Xk.x + Xj.x, ei = Xk.y - Xj.y, dr = Xk.x - Xj.x, di = Xk.y + Xj.y;
      T orr = dr * wr - di * wi, oi = dr * wi + di * wr;
      Zk = {(ei + orr) * scale, (er - oi) * scale};
    }
    {
      T wr = wj.x, wi = -wj.y;
      T er = Xj.x + Xk.x, ei = Xj.y - Xk.y, dr = Xj.x - Xk.x, di = Xj.y + Xk.y;
      T orr = dr * wr - di * wi, oi = dr * wi + di * wr;
      Zj = {(ei + orr) * scale, (er - oi) * scale};
    }
    z[k] = Zk;
    if (j != k) z[j] = Zj;
  }
  __syncthreads();
}

}  // namespace psgd
