// Shared-memory mixed-radix FFT engine used by every transform pass of the
// engine (Green's-tensor build, matvec, near field).
//
// A CTA holds a tile of W independent transforms of length L in shared memory
// in "column" layout: element (position j, transform w) lives at s[j*WS + w],
// WS >= W being a padded row stride.  The transform is a Stockham autosort
// sequence of radix-r stages (r in {2,3,4,5,7,8,16}); each stage stages its
// butterflies through registers so one buffer suffices.  Output is in natural
// order.  Forward uses exp(-2 pi i jk/L); inverse uses exp(+2 pi i jk/L) and is
// unnormalised.  Twiddles come from a per-length table tw[j] = exp(-2 pi i j/L)
// computed on the host in extended precision.
#pragma once
#include "dda_common.cuh"

namespace dda {

// ---- small DFT codelets (forward, in registers) ---------------------------
template <class C> __device__ __forceinline__ void dft2(C& a0, C& a1) {
  C t = a0; a0 = cadd(t, a1); a1 = csub(t, a1);
}

template <class C> __device__ __forceinline__ void dft4(C& a0, C& a1, C& a2, C& a3) {
  C t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = cmul_mi(csub(a1, a3));
  a0 = cadd(t0, t2); a2 = csub(t0, t2); a1 = cadd(t1, t3); a3 = csub(t1, t3);
}

template <class C> __device__ __forceinline__ void dft8(C* a) {
  typedef decltype(a[0].x) R;
  const R h = (R)0.7071067811865476;
  // radix-2 split over the two halves (decimation in frequency)
  C b0 = cadd(a[0], a[4]), b1 = cadd(a[1], a[5]), b2 = cadd(a[2], a[6]), b3 = cadd(a[3], a[7]);
  C c0 = csub(a[0], a[4]), c1 = csub(a[1], a[5]), c2 = csub(a[2], a[6]), c3 = csub(a[3], a[7]);
  // twiddles W8^k on the difference half: 1, (h,-h), -i, (-h,-h)
  C t;
  t = c1; c1.x = h * (t.x + t.y); c1.y = h * (t.y - t.x);
  c2 = cmul_mi(c2);
  t = c3; c3.x = h * (t.y - t.x); c3.y = -h * (t.x + t.y);
  dft4(b0, b1, b2, b3);
  dft4(c0, c1, c2, c3);
  a[0] = b0; a[2] = b1; a[4] = b2; a[6] = b3;
  a[1] = c0; a[3] = c1; a[5] = c2; a[7] = c3;
}

template <class C> __device__ __forceinline__ void dft16(C* a) {
  typedef decltype(a[0].x) R;
  // 16 = 4 x 4 in place: DFT4 over n2 (stride 4), twiddle W16^(n1*k2),
  // DFT4 over n1, then the index transpose X[4 k1 + k2] = a[4 k2 + k1]
  // (a register renaming once unrolled).
  const R c1 = (R)0.9238795325112867, s1 = (R)0.3826834323650898, h = (R)0.7071067811865476;
#pragma unroll
  for (int n1 = 0; n1 < 4; ++n1) dft4(a[n1], a[n1 + 4], a[n1 + 8], a[n1 + 12]);
  // now a[n1 + 4 k2]; twiddles
  C t;
  // n1=1: W^1, W^2, W^3
  t = a[5];  a[5].x = c1 * t.x + s1 * t.y;  a[5].y = c1 * t.y - s1 * t.x;
  t = a[9];  a[9].x = h * (t.x + t.y);      a[9].y = h * (t.y - t.x);
  t = a[13]; a[13].x = s1 * t.x + c1 * t.y; a[13].y = s1 * t.y - c1 * t.x;
  // n1=2: W^2, W^4, W^6
  t = a[6];  a[6].x = h * (t.x + t.y);      a[6].y = h * (t.y - t.x);
  a[10] = cmul_mi(a[10]);
  t = a[14]; a[14].x = h * (t.y - t.x);     a[14].y = -h * (t.x + t.y);
  // n1=3: W^3, W^6, W^9
  t = a[7];  a[7].x = s1 * t.x + c1 * t.y;  a[7].y = s1 * t.y - c1 * t.x;
  t = a[11]; a[11].x = h * (t.y - t.x);     a[11].y = -h * (t.x + t.y);
  t = a[15]; a[15].x = -c1 * t.x - s1 * t.y; a[15].y = -c1 * t.y + s1 * t.x;
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2) dft4(a[4 * k2], a[4 * k2 + 1], a[4 * k2 + 2], a[4 * k2 + 3]);
  // a[4 k2 + k1] holds X[4 k1 + k2]: transpose the 4x4 index
  C o[16];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) o[4 * k1 + k2] = a[4 * k2 + k1];
#pragma unroll
  for (int i = 0; i < 16; ++i) a[i] = o[i];
}

// DFTs whose upper half of inputs is zero (a[R/2..R-1] = 0), as the first
// stage of a transform of zero-padded data: the first radix-2 layer
// degenerates into copies.
template <class C> __device__ __forceinline__ void dft4_zh(C& a0, C& a1, C& a2, C& a3) {
  const C x0 = a0, x1 = a1, y1 = cmul_mi(a1);
  a0 = cadd(x0, x1); a2 = csub(x0, x1); a1 = cadd(x0, y1); a3 = csub(x0, y1);
}

template <class C> __device__ __forceinline__ void dft8_zh(C* a) {
  typedef decltype(a[0].x) R;
  const R h = (R)0.7071067811865476;
  C b0 = a[0], b1 = a[1], b2 = a[2], b3 = a[3];
  C c0 = a[0], c1 = a[1], c2 = a[2], c3 = a[3];
  C t;
  t = c1; c1.x = h * (t.x + t.y); c1.y = h * (t.y - t.x);
  c2 = cmul_mi(c2);
  t = c3; c3.x = h * (t.y - t.x); c3.y = -h * (t.x + t.y);
  dft4(b0, b1, b2, b3);
  dft4(c0, c1, c2, c3);
  a[0] = b0; a[2] = b1; a[4] = b2; a[6] = b3;
  a[1] = c0; a[3] = c1; a[5] = c2; a[7] = c3;
}

template <class C> __device__ __forceinline__ void dft16_zh(C* a) {
  typedef decltype(a[0].x) R;
  const R c1 = (R)0.9238795325112867, s1 = (R)0.3826834323650898, h = (R)0.7071067811865476;
#pragma unroll
  for (int n1 = 0; n1 < 4; ++n1) dft4_zh(a[n1], a[n1 + 4], a[n1 + 8], a[n1 + 12]);
  C t;
  t = a[5];  a[5].x = c1 * t.x + s1 * t.y;  a[5].y = c1 * t.y - s1 * t.x;
  t = a[9];  a[9].x = h * (t.x + t.y);      a[9].y = h * (t.y - t.x);
  t = a[13]; a[13].x = s1 * t.x + c1 * t.y; a[13].y = s1 * t.y - c1 * t.x;
  t = a[6];  a[6].x = h * (t.x + t.y);      a[6].y = h * (t.y - t.x);
  a[10] = cmul_mi(a[10]);
  t = a[14]; a[14].x = h * (t.y - t.x);     a[14].y = -h * (t.x + t.y);
  t = a[7];  a[7].x = s1 * t.x + c1 * t.y;  a[7].y = s1 * t.y - c1 * t.x;
  t = a[11]; a[11].x = h * (t.y - t.x);     a[11].y = -h * (t.x + t.y);
  t = a[15]; a[15].x = -c1 * t.x - s1 * t.y; a[15].y = -c1 * t.y + s1 * t.x;
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2) dft4(a[4 * k2], a[4 * k2 + 1], a[4 * k2 + 2], a[4 * k2 + 3]);
  C o[16];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) o[4 * k1 + k2] = a[4 * k2 + k1];
#pragma unroll
  for (int i = 0; i < 16; ++i) a[i] = o[i];
}

// odd radix via the conjugate-pair formulation:
// y_q = a0 + sum_k [cos(2 pi kq/R) (a_k + a_{R-k}) - i sin(2 pi kq/R) (a_k - a_{R-k})]
template <int R_> struct OddTab;
template <> struct OddTab<3> {
  static __device__ __forceinline__ double c(int k) { return -0.5; }
  static __device__ __forceinline__ double s(int k) { return 0.8660254037844386; }
};
template <> struct OddTab<5> {
  static __device__ __forceinline__ double c(int k) { return k == 1 ? 0.30901699437494745 : -0.8090169943749475; }
  static __device__ __forceinline__ double s(int k) { return k == 1 ? 0.9510565162951535 : 0.5877852522924731; }
};
template <> struct OddTab<7> {
  static __device__ __forceinline__ double c(int k) {
    return k == 1 ? 0.6234898018587335 : (k == 2 ? -0.2225209339563144 : -0.9009688679024191);
  }
  static __device__ __forceinline__ double s(int k) {
    return k == 1 ? 0.7818314824680298 : (k == 2 ? 0.9749279121818236 : 0.4338837391175581);
  }
};

template <int RAD, class C> __device__ __forceinline__ void dft_odd(C* a) {
  typedef decltype(a[0].x) R;
  constexpr int H = (RAD - 1) / 2;
  C t[H + 1], u[H + 1];
#pragma unroll
  for (int k = 1; k <= H; ++k) { t[k] = cadd(a[k], a[RAD - k]); u[k] = csub(a[k], a[RAD - k]); }
  C y0 = a[0];
#pragma unroll
  for (int k = 1; k <= H; ++k) y0 = cadd(y0, t[k]);
  C out[RAD];
  out[0] = y0;
#pragma unroll
  for (int q = 1; q <= H; ++q) {
    C re = a[0];
    C im = czero<C>();
#pragma unroll
    for (int k = 1; k <= H; ++k) {
      const int e = (k * q) % RAD;
      // cos/sin(2 pi e / RAD) from the half table with symmetry
      R cv, sv;
      if (e <= H) { cv = (R)OddTab<RAD>::c(e); sv = (R)OddTab<RAD>::s(e); }
      else { cv = (R)OddTab<RAD>::c(RAD - e); sv = -(R)OddTab<RAD>::s(RAD - e); }
      re.x += cv * t[k].x; re.y += cv * t[k].y;
      im.x += sv * u[k].x; im.y += sv * u[k].y;
    }
    // -i * im = (im.y, -im.x)
    out[q].x = re.x + im.y; out[q].y = re.y - im.x;
    out[RAD - q].x = re.x - im.y; out[RAD - q].y = re.y + im.x;
  }
#pragma unroll
  for (int q = 0; q < RAD; ++q) a[q] = out[q];
}

template <int RAD, class C> __device__ __forceinline__ void dft(C* a) {
  if constexpr (RAD == 2) dft2(a[0], a[1]);
  else if constexpr (RAD == 4) dft4(a[0], a[1], a[2], a[3]);
  else if constexpr (RAD == 8) dft8(a);
  else if constexpr (RAD == 16) dft16(a);
  else dft_odd<RAD>(a);
}

template <int RAD, class C> __device__ __forceinline__ void dft_zh(C* a) {
  static_assert(RAD % 2 == 0, "zero-half DFT needs an even radix");
  if constexpr (RAD == 2) { a[1] = a[0]; }
  else if constexpr (RAD == 4) dft4_zh(a[0], a[1], a[2], a[3]);
  else if constexpr (RAD == 8) dft8_zh(a);
  else dft16_zh(a);
}

// ---- compile-time FFT plans ----------------------------------------------
// L = 2^a 3^b 5^c 7^d.  The power of two uses radix-16 stages, with a tail of
// 8, 4, 2 or 8*4; then one stage per factor 3, 5, 7.
struct RadList {
  int n;
  int r[kMaxStages];
};

constexpr RadList make_radlist(int L) {
  RadList p{0, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}};
  int n = L, a = 0, b = 0, c = 0, d = 0;
  while (n > 1 && n % 2 == 0) { n /= 2; ++a; }
  while (n > 1 && n % 3 == 0) { n /= 3; ++b; }
  while (n > 1 && n % 5 == 0) { n /= 5; ++c; }
  while (n > 1 && n % 7 == 0) { n /= 7; ++d; }
  if (n != 1) return p;
  int q16 = a / 4, rem = a % 4;
  if (rem == 1 && q16 > 0) { q16 -= 1; rem = 5; }
  for (int i = 0; i < q16; ++i) p.r[p.n++] = 16;
  if (rem == 5) { p.r[p.n++] = 8; p.r[p.n++] = 4; }
  else if (rem == 3) p.r[p.n++] = 8;
  else if (rem == 2) p.r[p.n++] = 4;
  else if (rem == 1) p.r[p.n++] = 2;
  for (int i = 0; i < b; ++i) p.r[p.n++] = 3;
  for (int i = 0; i < c; ++i) p.r[p.n++] = 5;
  for (int i = 0; i < d; ++i) p.r[p.n++] = 7;
  return p;
}

// ---- shared-memory tile layouts -------------------------------------------
// Column layout: transform w, position j at s[j*WS + w]; consecutive threads
// take consecutive w.
struct LayCol {
  int W, WS;
  __device__ __forceinline__ int nw() const { return W; }
  template <int NB>
  __device__ __forceinline__ void decode(int idx, int& base, int& jb) const {
    const int w = idx % W;
    jb = idx / W;
    base = w;
  }
  __device__ __forceinline__ int js() const { return WS; }
};
// Line layout: NL lines of G interleaved transforms; transform (line, c),
// position j at s[line*LS + j*G + c]; consecutive threads take consecutive
// (c, j) so a line is walked contiguously.
template <int G>
struct LayLine {
  int NL, LS;
  __device__ __forceinline__ int nw() const { return NL * G; }
  template <int NB>
  __device__ __forceinline__ void decode(int idx, int& base, int& jb) const {
    const int c = idx % G;
    const int rest = idx / G;
    jb = rest % NB;
    const int line = rest / NB;
    base = line * LS + c;
  }
  __device__ __forceinline__ int js() const { return G; }
};

// ---- one Stockham stage over a shared-memory tile -------------------------
// Butterfly jb (0 <= jb < L/RAD) of a transform reads positions jb + m*L/RAD,
// applies twiddles exp(-+2 pi i m k/(NS RAD)) with k = jb mod NS, performs the
// RAD-point DFT and writes positions (jb - k)*RAD + k + q*NS.  All butterflies
// of the thread are read before the barrier and written after it, so the
// stage works in place.
template <int L, int RAD, int NS, bool INV, int EPT, int NT, class C, class Lay>
__device__ __forceinline__ void fft_stage(C* s, const Lay& lay, const C* __restrict__ tw) {
  constexpr int BPT = (EPT + RAD - 1) / RAD;
  constexpr int NB = L / RAD;
  const int total = NB * lay.nw();
  const int js = lay.js();
  C a[BPT][RAD];
  int bs[BPT], jbs[BPT];
#pragma unroll
  for (int b = 0; b < BPT; ++b) {
    const int idx = threadIdx.x + b * NT;
    if (idx < total) {
      lay.template decode<NB>(idx, bs[b], jbs[b]);
#pragma unroll
      for (int m = 0; m < RAD; ++m) a[b][m] = s[bs[b] + (jbs[b] + m * NB) * js];
    }
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < BPT; ++b) {
    const int idx = threadIdx.x + b * NT;
    if (idx < total) {
      const int jb = jbs[b];
      const int k = jb % NS;
      if (INV) {
#pragma unroll
        for (int m = 0; m < RAD; ++m) a[b][m].y = -a[b][m].y;
      }
      if (NS > 1) {
        constexpr int ST = L / (NS * RAD);
#pragma unroll
        for (int m = 1; m < RAD; ++m) a[b][m] = cmul(a[b][m], tw[m * k * ST]);
      }
      dft<RAD>(a[b]);
      if (INV) {
#pragma unroll
        for (int m = 0; m < RAD; ++m) a[b][m].y = -a[b][m].y;
      }
      const int o = (jb - k) * RAD + k;
#pragma unroll
      for (int q = 0; q < RAD; ++q) s[bs[b] + (o + q * NS) * js] = a[b][q];
    }
  }
  __syncthreads();
}

template <int L, bool INV, int EPT, int NT, int ST, int NS, class C, class Lay>
__device__ __forceinline__ void fft_stages(C* s, const Lay& lay, const C* __restrict__ tw) {
  constexpr RadList rl = make_radlist(L);
  if constexpr (ST < rl.n) {
    constexpr int RAD = rl.r[ST];
    fft_stage<L, RAD, NS, INV, EPT, NT>(s, lay, tw);
    fft_stages<L, INV, EPT, NT, ST + 1, NS * RAD>(s, lay, tw);
  }
}

// Full transform of a tile of L-point transforms.  Requires L*nw <= EPT*NT.
template <int L, bool INV, int EPT, int NT, class C, class Lay>
__device__ __forceinline__ void fft_tile(C* s, const Lay& lay, const C* __restrict__ tw) {
  static_assert(make_radlist(L).n > 0, "FFT length must factor into 2,3,5,7");
  fft_stages<L, INV, EPT, NT, 0, 1>(s, lay, tw);
}

}  // namespace dda
