// Deterministic block / grid reductions shared by the solver kernels.
// Each CTA publishes its partial sums; the last CTA of an instance (detected
// with an atomic ticket) adds the partials in a fixed order, so results do not
// depend on scheduling.
#pragma once
#include "dda_common.cuh"

namespace dda {

constexpr int KNT = 256;
constexpr int KNW = KNT / 32;
constexpr int KRED = 12;   // reduction slots per CTA (6 complex dots)

// Grid-stride loop over [start, n) that handles U elements per trip with
// their loads issued together (U independent memory requests in flight per
// thread), then the remainder one by one.  The element order of each
// thread's work is fixed, so reductions stay deterministic.
constexpr int KU = 4;
template <int U, class F>
__device__ __forceinline__ void grid_loop(long long n, long long start, long long stride, F&& f) {
  long long i = start;
  for (; i + (U - 1) * stride < n; i += U * stride) {
#pragma unroll
    for (int u = 0; u < U; ++u) f(i + u * stride);
  }
  for (; i < n; i += stride) f(i);
}

__device__ __forceinline__ int kinst(const int* act) { return act ? act[blockIdx.y] : (int)blockIdx.y; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-reduce K doubles, publish per-CTA partials, and return true in the
// last CTA of the instance, with `tot` holding the fixed-order grid total.
// Both stages spread their loads over the CTA's threads so that no thread
// walks a long dependent chain of L2 reads.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double (&sh)[K][KNW], double (&out)[K]) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const double s = warp_sum(v[k]);
    if (lane == 0) sh[k][wid] = s;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] = warp_sum(lane < KNW ? sh[k][lane] : 0.0);
  }
}

template <int K>
__device__ __forceinline__ bool reduce_last(double (&v)[K], double (&tot)[K], double* red, unsigned* cnt, int inst,
                                            int RB) {
  __shared__ double sh[K][KNW];
  __shared__ bool last;
  double part[K];
  block_sum<K>(v, sh, part);
  if (threadIdx.x == 0) {
    double* dst = red + ((size_t)inst * RB + blockIdx.x) * KRED;
#pragma unroll
    for (int k = 0; k < K; ++k) dst[k] = part[k];
    __threadfence();
    const unsigned prev = atomicAdd(&cnt[inst], 1u);
    last = (prev == (unsigned)RB - 1u);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  // every thread gathers a fixed subset of the CTAs' partials
  const double* src = red + (size_t)inst * RB * KRED;
  double g[K];
#pragma unroll
  for (int k = 0; k < K; ++k) g[k] = 0.0;
  for (int b = threadIdx.x; b < RB; b += KNT) {
    double t[K];
#pragma unroll
    for (int k = 0; k < K; ++k) t[k] = __ldcg(src + (size_t)b * KRED + k);
#pragma unroll
    for (int k = 0; k < K; ++k) g[k] += t[k];
  }
  block_sum<K>(g, sh, tot);
  if (threadIdx.x == 0) cnt[inst] = 0u;
  return true;   // only warp 0 holds valid totals
}

// last-CTA barrier without data (for kernels that only need "all done")
__device__ __forceinline__ bool finish_last(unsigned* cnt, int inst, int RB) {
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(&cnt[inst], 1u);
    last = (prev == (unsigned)RB - 1u);
    if (last) cnt[inst] = 0u;
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

}  // namespace dda
