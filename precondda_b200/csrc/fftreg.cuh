// Register-resident mixed-radix FFT for the transform passes.
//
// A transform of length L is worked on by T threads.  The radix plan
// (R_0, ..., R_{S-1}) has E = lcm(R_s) = L / T elements per thread: in stage s a
// thread owns butterflies jb = t + b*T (b < E/R_s).  Stage 0 inputs are read by
// the caller straight from global memory into registers, stage S-1 outputs are
// written straight back; stages exchange data through a padded shared-memory
// buffer (one exchange per stage boundary).  Stockham indexing: butterfly jb of
// stage s reads positions jb + m*L/R_s, multiplies by exp(-+2 pi i m k/(NS R))
// with NS = R_0...R_{s-1}, k = jb mod NS, and writes positions
// (jb - k)*R + k + q*NS, leaving the result in natural order.
//
// The last stage of a forward transform and the first stage of an inverse
// transform with the reversed plan own the same positions in the same thread,
// which lets pass 3 of the matvec apply the 3x3 tensor in registers between
// the two transforms.
#pragma once
#include "fft_core.cuh"

namespace dda {

// Values passed through an empty asm statement so the compiler cannot merge
// address arithmetic of different phases of a kernel (which would keep it
// live, in registers, across the whole kernel).
__device__ __forceinline__ int opaque(int v) {
  int r;
  asm volatile("mov.b32 %0, %1;" : "=r"(r) : "r"(v));
  return r;
}
// DDA_ASSUME_T=1: a kernel tells the compiler that its transform index t
// is below the plan's thread count (the launch guarantees it), so
// (t + 16 m) / 16 can fold into immediates of shared-memory addresses.
#ifndef DDA_ASSUME_T
#define DDA_ASSUME_T 1
#endif
template <int T> __device__ __forceinline__ void assume_t(int t) {
#if DDA_ASSUME_T
  __builtin_assume(t >= 0 && t < T);
#endif
}
template <class T> __device__ __forceinline__ T* opaque_ptr(T* p) {
  T* r;
  asm volatile("mov.b64 %0, %1;" : "=l"(r) : "l"(p));
  return r;
}

constexpr int cgcd(int a, int b) { return b == 0 ? a : cgcd(b, a % b); }
constexpr int clcm(int a, int b) { return a / cgcd(a, b) * b; }

template <int... Rs>
struct RPlan {
  static constexpr int S = sizeof...(Rs);
  static constexpr int r[S] = {Rs...};
  static constexpr int L = (Rs * ...);
  static constexpr int E = [] { int e = 1; for (int i = 0; i < S; ++i) e = clcm(e, r[i]); return e; }();
  static constexpr int T = L / E;
  static constexpr int ns(int s) { int p = 1; for (int i = 0; i < s; ++i) p *= r[i]; return p; }
};

// Reversed plan, used for the inverse transform in pass 3.
template <class P, class Seq> struct RevHelper;
template <class P, int... I> struct RevHelper<P, std::integer_sequence<int, I...>> {
  typedef RPlan<P::r[P::S - 1 - I]...> type;
};
template <class P> using RevPlan = typename RevHelper<P, std::make_integer_sequence<int, P::S>>::type;

// Plans of the compiled lengths (radices 2,3,4,5,8,16; E <= 24).  Complex128
// uses radices <= 8 where that keeps E small (register budget).
template <int L, typename R = float> struct PlanFor;
template <> struct PlanFor<8> { typedef RPlan<8> type; };
template <> struct PlanFor<12> { typedef RPlan<4, 3> type; };
template <> struct PlanFor<16> { typedef RPlan<16> type; };
template <> struct PlanFor<20> { typedef RPlan<4, 5> type; };
template <> struct PlanFor<24> { typedef RPlan<4, 2, 3> type; };
template <> struct PlanFor<32> { typedef RPlan<8, 4> type; };
template <> struct PlanFor<40> { typedef RPlan<4, 2, 5> type; };
template <> struct PlanFor<48> { typedef RPlan<4, 4, 3> type; };
template <> struct PlanFor<64> { typedef RPlan<8, 8> type; };
template <> struct PlanFor<72> { typedef RPlan<8, 3, 3> type; };
// DDA_C64_PLAN8=1 (an A/B build option): the radix-8 plans for the
// power-of-two lengths 128 and 256 too (E = 8: fewer registers per thread,
// one more exchange)
#if defined(DDA_C64_PLAN8) && DDA_C64_PLAN8
template <> struct PlanFor<128> { typedef RPlan<8, 4, 4> type; };
#else
template <> struct PlanFor<128> { typedef RPlan<16, 8> type; };
#endif
template <> struct PlanFor<144> { typedef RPlan<4, 4, 3, 3> type; };
#if defined(DDA_C64_PLAN8) && DDA_C64_PLAN8
template <> struct PlanFor<256> { typedef RPlan<8, 8, 4> type; };
#else
template <> struct PlanFor<256> { typedef RPlan<16, 16> type; };
#endif
template <> struct PlanFor<512> { typedef RPlan<8, 8, 8> type; };
template <> struct PlanFor<80> { typedef RPlan<4, 4, 5> type; };
template <> struct PlanFor<160> { typedef RPlan<4, 4, 2, 5> type; };
template <> struct PlanFor<320> { typedef RPlan<4, 4, 4, 5> type; };
// radix-3 lengths keep E = 24 (8, 8, 3 etc.): plans with E = 12 (one more
// exchange, half the registers) measured 12-23% slower on batched matvecs
template <> struct PlanFor<96> { typedef RPlan<8, 4, 3> type; };
template <> struct PlanFor<192> { typedef RPlan<8, 8, 3> type; };
template <> struct PlanFor<288> { typedef RPlan<8, 4, 3, 3> type; };
template <> struct PlanFor<384> { typedef RPlan<8, 8, 2, 3> type; };
// Plans with radices <= 8 (E <= 8 for powers of two): fewer registers per
// thread at the cost of one more exchange.
template <int L> struct Plan8 : PlanFor<L, float> {};
template <> struct Plan8<16> { typedef RPlan<4, 4> type; };
template <> struct Plan8<32> { typedef RPlan<8, 4> type; };
template <> struct Plan8<128> { typedef RPlan<8, 4, 4> type; };
template <> struct Plan8<256> { typedef RPlan<8, 8, 4> type; };
template <int L> struct PlanFor<L, double> : Plan8<L> {};


// shared-memory position padding: one spare slot every 16 positions
#ifndef DDA_PPAD
#define DDA_PPAD 1
#endif
__device__ __forceinline__ constexpr int ppad(int pos) { return DDA_PPAD ? pos + (pos >> 4) : pos; }
__host__ __device__ constexpr int ppad_len(int L) { return DDA_PPAD ? L + (L >> 4) + 1 : L; }

// A twiddle table: a global-memory pointer (read through the read-only
// path) or a copy of it in the CTA's shared memory.
template <class C> struct ShTw {
  const C* p;
};
template <class C> __device__ __forceinline__ C twget(const C* tw, int i) { return __ldg(tw + i); }
template <class C> __device__ __forceinline__ C twget(ShTw<C> tw, int i) { return tw.p[i]; }

// Copy a length-L table into shared memory (all threads of the CTA; the
// first exchange's barrier publishes it before any stage reads it).
template <class C> __device__ __forceinline__ ShTw<C> tw_to_shared(const C* __restrict__ tw, C* dst, int L) {
  for (int i = threadIdx.x; i < L; i += blockDim.x) dst[i] = __ldg(tw + i);
  return ShTw<C>{dst};
}

// Compute stage s of plan P on the thread's registers a[E] (twiddles for
// s > 0).  Always the forward transform: inverse transforms are run as
// swap(FFT(swap(x))), swap(a + ib) = b + ia, which costs no instructions.
// ZH (stage 0 only): the upper half of every butterfly's inputs is zero.
template <class P, int s, bool ZH = false, class C, class TW>
__device__ __forceinline__ void rstage(C* a, int t, TW tw) {
  static_assert(!ZH || s == 0, "zero-half inputs only at stage 0");
  constexpr int R = P::r[s];
  constexpr int NS = P::ns(s);
  constexpr int BPT = P::E / R;
#pragma unroll
  for (int b = 0; b < BPT; ++b) {
    C* v = a + b * R;
    if constexpr (NS > 1) {
      // twiddles w^m, w = exp(-2 pi i k/(NS R)), straight from the length-L
      // table (index m k L/(NS R) < L); the lanes of a warp mostly share k,
      // so the loads are broadcasts out of L1
      constexpr int ST = P::L / (NS * R);
      const int k = (t + b * P::T) % NS;
#pragma unroll
      for (int m = 1; m < R; ++m) v[m] = cmul(v[m], twget(tw, m * k * ST));
    }
    if constexpr (ZH) dft_zh<R>(v);
    else dft<R>(v);
  }
}

template <class C> __device__ __forceinline__ C cswap(C v) { C r; r.x = v.y; r.y = v.x; return r; }

// Positions touched by a thread: input of stage s (butterfly b, leg m) and
// output of stage s (butterfly b, leg q).
template <class P, int s>
__device__ __forceinline__ int rin_pos(int t, int b, int m) {
  constexpr int R = P::r[s];
  return t + b * P::T + m * (P::L / R);
}
template <class P, int s>
__device__ __forceinline__ int rout_pos(int t, int b, int q) {
  constexpr int R = P::r[s];
  constexpr int NS = P::ns(s);
  const int jb = t + b * P::T;
  const int k = jb % NS;
  return (jb - k) * R + k + q * NS;
}

// Exchange through shared memory between stage s and s+1 for NC interleaved
// components held by the thread (a[c*E + i]), then compute stage s+1.
// `sm(c, ppos)` returns the shared-memory slot of padded position ppos of
// component c of this thread's transform.  All threads of the CTA must call
// this together (it contains barriers).
template <class P, int NC, int s, class C, class SM, class TW>
__device__ __forceinline__ void rexchange(C* a, int t, const SM& sm, TW tw) {
  constexpr int R = P::r[s];
  constexpr int R2 = P::r[s + 1];
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int b = 0; b < P::E / R; ++b)
#pragma unroll
      for (int q = 0; q < R; ++q) sm(c, ppad(rout_pos<P, s>(t, b, q))) = a[c * P::E + b * R + q];
  __syncthreads();
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int b = 0; b < P::E / R2; ++b)
#pragma unroll
      for (int m = 0; m < R2; ++m) a[c * P::E + b * R2 + m] = sm(c, ppad(rin_pos<P, s + 1>(t, b, m)));
  __syncthreads();
#pragma unroll
  for (int c = 0; c < NC; ++c) rstage<P, s + 1>(a + c * P::E, t, tw);
}

// Stages s+1..S-1 (stage 0 is computed by the caller after its global load).
template <class P, int NC, int s, class C, class SM, class TW>
__device__ __forceinline__ void rrest(C* a, int t, const SM& sm, TW tw) {
  if constexpr (s + 1 < P::S) {
    rexchange<P, NC, s>(a, t, sm, tw);
    rrest<P, NC, s + 1>(a, t, sm, tw);
  }
}

// Stage-0 load: a[c*E + b*R0 + m] = ld(c, pos) for the thread's input positions.
// ZH: positions >= L/2 are known to be zero (they are exactly the legs
// m >= R0/2, because t + b*T < L/R0) and are not loaded.
template <class P, int NC, bool ZH = false, class C, class LD>
__device__ __forceinline__ void rload(C* a, int t, const LD& ld) {
  constexpr int R0 = P::r[0];
  static_assert(!ZH || R0 % 2 == 0, "zero-half load needs an even first radix");
#pragma unroll
  for (int m = 0; m < R0; ++m)
#pragma unroll
    for (int b = 0; b < P::E / R0; ++b)
#pragma unroll
      for (int c = 0; c < NC; ++c)
        a[c * P::E + b * R0 + m] = (ZH && m >= R0 / 2) ? czero<C>() : ld(c, rin_pos<P, 0>(t, b, m));
}

// Whether the last stage's outputs at positions >= L/2 are exactly the legs
// q >= R/2 (true for an even last radix: the output position is jb + q*NS
// with jb < NS and NS*R = L).
template <class P> constexpr bool half_store_ok() { return P::r[P::S - 1] % 2 == 0; }

// Last-stage store: st(c, pos, value) for the thread's output positions.
// DH: only positions < L/2 are wanted (requires half_store_ok<P>()).
template <class P, int NC, bool DH = false, class C, class ST>
__device__ __forceinline__ void rstore(const C* a, int t, const ST& st) {
  constexpr int RL = P::r[P::S - 1];
  static_assert(!DH || half_store_ok<P>(), "half store needs an even last radix");
#pragma unroll
  for (int q = 0; q < (DH ? RL / 2 : RL); ++q)
#pragma unroll
    for (int b = 0; b < P::E / RL; ++b)
#pragma unroll
      for (int c = 0; c < NC; ++c) st(c, rout_pos<P, P::S - 1>(t, b, q), a[c * P::E + b * RL + q]);
}

// Full transform of NC components: load, all stages, store.  INV: the
// inverse (unnormalised) transform, as swap(FFT(swap(x))).
// ZH / DH: zero upper half of the input / only the lower half of the output
// wanted (see rload / rstore).
template <class P, int NC, bool INV, bool ZH = false, bool DH = false, class C, class LD, class SM, class ST, class TW>
__device__ __forceinline__ void rfft(C* a, int t, const LD& ld, const SM& sm, const ST& st, TW tw) {
  if constexpr (INV) {
    rload<P, NC, ZH>(a, t, [&](int c, int pos) -> C { return cswap(ld(c, pos)); });
  } else {
    rload<P, NC, ZH>(a, t, ld);
  }
#pragma unroll
  for (int c = 0; c < NC; ++c) rstage<P, 0, ZH>(a + c * P::E, t, tw);
  rrest<P, NC, 0>(a, t, sm, tw);
  if constexpr (INV) {
    rstore<P, NC, DH>(a, opaque(t), [&](int c, int pos, C v) { st(c, pos, cswap(v)); });
  } else {
    rstore<P, NC, DH>(a, opaque(t), st);
  }
}

}  // namespace dda
