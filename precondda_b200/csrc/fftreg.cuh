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
template <> struct PlanFor<80> { typedef RPlan<4, 4, 5> type; };
template <> struct PlanFor<96> { typedef RPlan<8, 4, 3> type; };
template <> struct PlanFor<128> { typedef RPlan<16, 8> type; };
template <> struct PlanFor<144> { typedef RPlan<4, 4, 3, 3> type; };
template <> struct PlanFor<160> { typedef RPlan<4, 4, 2, 5> type; };
template <> struct PlanFor<192> { typedef RPlan<8, 8, 3> type; };
template <> struct PlanFor<256> { typedef RPlan<16, 16> type; };
template <> struct PlanFor<288> { typedef RPlan<8, 4, 3, 3> type; };
template <> struct PlanFor<320> { typedef RPlan<4, 4, 4, 5> type; };
template <> struct PlanFor<384> { typedef RPlan<8, 8, 2, 3> type; };
template <> struct PlanFor<512> { typedef RPlan<8, 8, 8> type; };
// Plans with radices <= 8 (E <= 8 for powers of two): fewer registers per
// thread at the cost of one more exchange.
template <int L> struct Plan8 : PlanFor<L, float> {};
template <> struct Plan8<16> { typedef RPlan<4, 4> type; };
template <> struct Plan8<32> { typedef RPlan<8, 4> type; };
template <> struct Plan8<128> { typedef RPlan<8, 4, 4> type; };
template <> struct Plan8<256> { typedef RPlan<8, 8, 4> type; };
template <int L> struct PlanFor<L, double> : Plan8<L> {};


// shared-memory position padding: one spare slot every 16 positions
__device__ __forceinline__ constexpr int ppad(int pos) { return pos + (pos >> 4); }
__host__ __device__ constexpr int ppad_len(int L) { return L + (L >> 4) + 1; }

// Compute stage s of plan P on the thread's registers a[E] (twiddles for s>0).
template <class P, int s, bool INV, class C>
__device__ __forceinline__ void rstage(C* a, int t, const C* __restrict__ tw) {
  constexpr int R = P::r[s];
  constexpr int NS = P::ns(s);
  constexpr int BPT = P::E / R;
#pragma unroll
  for (int b = 0; b < BPT; ++b) {
    C* v = a + b * R;
    if (INV) {
#pragma unroll
      for (int m = 0; m < R; ++m) v[m].y = -v[m].y;
    }
    if constexpr (NS > 1) {
      // twiddles w^m, w = exp(-2 pi i k/(NS R)): w^1, w^2, w^4, w^8 from the
      // table, the others as products of those (at most 3 roundings)
      constexpr int ST = P::L / (NS * R);
      const int k = (t + b * P::T) % NS;
      const C w1 = tw[k * ST];
      const C w2 = (R > 2) ? tw[2 * k * ST] : w1;
      const C w4 = (R > 4) ? tw[4 * k * ST] : w1;
      const C w8 = (R > 8) ? tw[8 * k * ST] : w1;
#pragma unroll
      for (int m = 1; m < R; ++m) {
        C w;
        bool set = false;
        if (m & 1) { w = w1; set = true; }
        if (m & 2) { w = set ? cmul(w, w2) : w2; set = true; }
        if (m & 4) { w = set ? cmul(w, w4) : w4; set = true; }
        if (m & 8) { w = set ? cmul(w, w8) : w8; set = true; }
        v[m] = cmul(v[m], w);
      }
    }
    dft<R>(v);
    if (INV) {
#pragma unroll
      for (int m = 0; m < R; ++m) v[m].y = -v[m].y;
    }
  }
}

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
template <class P, int NC, int s, bool INV, class C, class SM>
__device__ __forceinline__ void rexchange(C* a, int t, const SM& sm, const C* __restrict__ tw) {
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
  for (int c = 0; c < NC; ++c) rstage<P, s + 1, INV>(a + c * P::E, t, tw);
}

// Stages s+1..S-1 (stage 0 is computed by the caller after its global load).
template <class P, int NC, int s, bool INV, class C, class SM>
__device__ __forceinline__ void rrest(C* a, int t, const SM& sm, const C* __restrict__ tw) {
  if constexpr (s + 1 < P::S) {
    rexchange<P, NC, s, INV>(a, t, sm, tw);
    rrest<P, NC, s + 1, INV>(a, t, sm, tw);
  }
}

// Stage-0 load: a[c*E + b*R0 + m] = ld(c, pos) for the thread's input positions.
template <class P, int NC, class C, class LD>
__device__ __forceinline__ void rload(C* a, int t, const LD& ld) {
  constexpr int R0 = P::r[0];
#pragma unroll
  for (int m = 0; m < R0; ++m)
#pragma unroll
    for (int b = 0; b < P::E / R0; ++b)
#pragma unroll
      for (int c = 0; c < NC; ++c) a[c * P::E + b * R0 + m] = ld(c, rin_pos<P, 0>(t, b, m));
}

// Last-stage store: st(c, pos, value) for the thread's output positions.
template <class P, int NC, class C, class ST>
__device__ __forceinline__ void rstore(const C* a, int t, const ST& st) {
  constexpr int RL = P::r[P::S - 1];
#pragma unroll
  for (int q = 0; q < RL; ++q)
#pragma unroll
    for (int b = 0; b < P::E / RL; ++b)
#pragma unroll
      for (int c = 0; c < NC; ++c) st(c, rout_pos<P, P::S - 1>(t, b, q), a[c * P::E + b * RL + q]);
}

// Full transform of NC components: load, all stages, store.
template <class P, int NC, bool INV, class C, class LD, class SM, class ST>
__device__ __forceinline__ void rfft(C* a, int t, const LD& ld, const SM& sm, const ST& st,
                                     const C* __restrict__ tw) {
  rload<P, NC>(a, t, ld);
#pragma unroll
  for (int c = 0; c < NC; ++c) rstage<P, 0, INV>(a + c * P::E, t, tw);
  rrest<P, NC, 0, INV>(a, t, sm, tw);
  rstore<P, NC>(a, opaque(t), st);
}

}  // namespace dda
