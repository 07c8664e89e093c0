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

__device__ __forceinline__ int kinst(const int* act) { return act ? act[blockIdx.y] : (int)blockIdx.y; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-reduce K doubles, publish per-CTA partials, and return true in the
// last CTA of the instance, with `tot` holding the fixed-order grid total.
template <int K>
__device__ __forceinline__ bool reduce_last(double (&v)[K], double (&tot)[K], double* red, unsigned* cnt, int inst,
                                            int RB) {
  __shared__ double sh[K][KNW];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double s = warp_sum(v[k]);
    if (lane == 0) sh[k][wid] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double* dst = red + ((size_t)inst * RB + blockIdx.x) * KRED;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double s = 0.0;
      for (int w = 0; w < KNW; ++w) s += sh[k][w];
      dst[k] = s;
    }
    __threadfence();
    const unsigned prev = atomicAdd(&cnt[inst], 1u);
    last = (prev == (unsigned)RB - 1u);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  if (wid == 0) {
    const double* src = red + (size_t)inst * RB * KRED;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double s = 0.0;
      for (int b = lane; b < RB; b += 32) s += __ldcg(src + (size_t)b * KRED + k);
      s = warp_sum(s);
      tot[k] = s;
    }
    if (lane == 0) cnt[inst] = 0u;
  }
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
