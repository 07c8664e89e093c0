// Two complex64 values processed together with sm_100 packed FP32 arithmetic.
//
// cp2 holds the real parts of two complex numbers in one float2 and their
// imaginary parts in another, so every complex add, subtract or real-scaled
// rotation of the pair is one packed instruction per component (FADD2 /
// FMUL2 / FFMA2 on two lanes) instead of two scalar ones.  Two independent
// transforms of the same length share every twiddle, so the register FFT
// (fftreg.cuh) runs on cp2 elements unchanged: the codelets below are the
// forward DFTs of fft_core.cuh restated for this layout, written so that the
// multiplications by -i fold into the adds that follow them.  Each packed
// operation rounds its two lanes exactly as the scalar operation would.
#pragma once
#include "dda_common.cuh"

namespace dda {

struct cp2 {
  float2 re;   // (Re a, Re b)
  float2 im;   // (Im a, Im b)
};

__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b, exactly: -b * 1 + a rounds once
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

template <> __device__ __forceinline__ cp2 czero<cp2>() {
  cp2 c;
  c.re = make_float2(0.f, 0.f);
  c.im = make_float2(0.f, 0.f);
  return c;
}
__device__ __forceinline__ cp2 cadd(cp2 a, cp2 b) { return cp2{f2add(a.re, b.re), f2add(a.im, b.im)}; }
__device__ __forceinline__ cp2 csub(cp2 a, cp2 b) { return cp2{f2sub(a.re, b.re), f2sub(a.im, b.im)}; }
// t + (-i) d and t - (-i) d
__device__ __forceinline__ cp2 cadd_mi(cp2 t, cp2 d) { return cp2{f2add(t.re, d.im), f2sub(t.im, d.re)}; }
__device__ __forceinline__ cp2 csub_mi(cp2 t, cp2 d) { return cp2{f2sub(t.re, d.im), f2add(t.im, d.re)}; }
// swap(a + ib) = b + ia on both lanes: no instruction
__device__ __forceinline__ cp2 cswap(cp2 v) { return cp2{v.im, v.re}; }
// v * w for one complex64 w shared by both lanes (a twiddle)
__device__ __forceinline__ cp2 cmul(cp2 v, float2 w) {
  const float2 wr = f2(w.x), wi = f2(w.y), nwi = f2(-w.y);
  return cp2{f2fma(v.re, wr, f2mul(v.im, nwi)), f2fma(v.re, wi, f2mul(v.im, wr))};
}
// v * (c - i s) for real constants c, s: (c re + s im, c im - s re)
__device__ __forceinline__ cp2 crot(cp2 v, float c, float s) {
  return cp2{f2fma(v.re, f2(c), f2mul(v.im, f2(s))), f2fma(v.im, f2(c), f2mul(v.re, f2(-s)))};
}
// the two complex64 values of a pair, and a pair from two values
__device__ __forceinline__ cp2 cpack(float2 a, float2 b) { return cp2{make_float2(a.x, b.x), make_float2(a.y, b.y)}; }
__device__ __forceinline__ float2 clo(cp2 v) { return make_float2(v.re.x, v.im.x); }
__device__ __forceinline__ float2 chi(cp2 v) { return make_float2(v.re.y, v.im.y); }

// ---- forward DFT codelets on pairs (same outputs as fft_core.cuh's) ------
__device__ __forceinline__ void dft2(cp2& a0, cp2& a1) {
  const cp2 t = a0;
  a0 = cadd(t, a1);
  a1 = csub(t, a1);
}

// radix 4; with MI2 the third input enters multiplied by -i
template <bool MI2 = false>
__device__ __forceinline__ void dft4p(cp2& a0, cp2& a1, cp2& a2, cp2& a3) {
  const cp2 t0 = MI2 ? cadd_mi(a0, a2) : cadd(a0, a2);
  const cp2 t1 = MI2 ? csub_mi(a0, a2) : csub(a0, a2);
  const cp2 t2 = cadd(a1, a3), d = csub(a1, a3);
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd_mi(t1, d);
  a3 = csub_mi(t1, d);
}
__device__ __forceinline__ void dft4(cp2& a0, cp2& a1, cp2& a2, cp2& a3) { dft4p<false>(a0, a1, a2, a3); }

// radix 4 with a2 = a3 = 0
__device__ __forceinline__ void dft4_zh(cp2& a0, cp2& a1, cp2& a2, cp2& a3) {
  const cp2 x0 = a0, x1 = a1;
  a0 = cadd(x0, x1);
  a2 = csub(x0, x1);
  a1 = cadd_mi(x0, x1);
  a3 = csub_mi(x0, x1);
}

// radix 8 as two radix-4 halves after one radix-2 layer (decimation in
// frequency); zh: the upper four inputs are zero
template <bool ZH>
__device__ __forceinline__ void dft8p(cp2* a) {
  const float h = 0.7071067811865476f;
  cp2 b0, b1, b2, b3, c0, c1, c2, c3;
  if (ZH) {
    b0 = c0 = a[0]; b1 = c1 = a[1]; b2 = c2 = a[2]; b3 = c3 = a[3];
  } else {
    b0 = cadd(a[0], a[4]); b1 = cadd(a[1], a[5]); b2 = cadd(a[2], a[6]); b3 = cadd(a[3], a[7]);
    c0 = csub(a[0], a[4]); c1 = csub(a[1], a[5]); c2 = csub(a[2], a[6]); c3 = csub(a[3], a[7]);
  }
  // W8^1 = (h, -h), W8^2 = -i (folded into the radix 4), W8^3 = (-h, -h)
  c1 = cp2{f2mul(f2add(c1.re, c1.im), f2(h)), f2mul(f2sub(c1.im, c1.re), f2(h))};
  c3 = cp2{f2mul(f2sub(c3.im, c3.re), f2(h)), f2mul(f2add(c3.re, c3.im), f2(-h))};
  dft4(b0, b1, b2, b3);
  dft4p<true>(c0, c1, c2, c3);
  a[0] = b0; a[2] = b1; a[4] = b2; a[6] = b3;
  a[1] = c0; a[3] = c1; a[5] = c2; a[7] = c3;
}
__device__ __forceinline__ void dft8(cp2* a) { dft8p<false>(a); }
__device__ __forceinline__ void dft8_zh(cp2* a) { dft8p<true>(a); }

// radix 16 = 4 x 4 (zh: the upper eight inputs are zero)
template <bool ZH>
__device__ __forceinline__ void dft16p(cp2* a) {
  const float c1 = 0.9238795325112867f, s1 = 0.3826834323650898f, h = 0.7071067811865476f;
#pragma unroll
  for (int n1 = 0; n1 < 4; ++n1) {
    if (ZH) dft4_zh(a[n1], a[n1 + 4], a[n1 + 8], a[n1 + 12]);
    else dft4(a[n1], a[n1 + 4], a[n1 + 8], a[n1 + 12]);
  }
  // twiddles W16^(n1 k2); W16^4 = -i on a[10] is folded into its radix 4
  a[5] = crot(a[5], c1, s1);
  a[9] = crot(a[9], h, h);
  a[13] = crot(a[13], s1, c1);
  a[6] = crot(a[6], h, h);
  a[14] = crot(a[14], -h, h);
  a[7] = crot(a[7], s1, c1);
  a[11] = crot(a[11], -h, h);
  a[15] = crot(a[15], -c1, -s1);
  dft4(a[0], a[1], a[2], a[3]);
  dft4(a[4], a[5], a[6], a[7]);
  dft4p<true>(a[8], a[9], a[10], a[11]);
  dft4(a[12], a[13], a[14], a[15]);
  cp2 o[16];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) o[4 * k1 + k2] = a[4 * k2 + k1];
#pragma unroll
  for (int i = 0; i < 16; ++i) a[i] = o[i];
}
__device__ __forceinline__ void dft16(cp2* a) { dft16p<false>(a); }
__device__ __forceinline__ void dft16_zh(cp2* a) { dft16p<true>(a); }

}  // namespace dda
