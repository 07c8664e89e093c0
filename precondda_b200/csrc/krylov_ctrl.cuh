// Scalar steps of GPBiCGSTAB shared by the Krylov kernels and by the matvec
// passes that carry a fused dot product: alpha (Gpbicgstab.py:1019) and
// zeta / eta (Gpbicgstab.py:1038-1052, calculate_zeta_eta_twostep :239-380),
// plus a deterministic grid reduction for CTAs of any width.
#pragma once
#include "reduce.cuh"

namespace dda {

// zeta / eta dots of the general form: yy, tt, yt = conj(y) t, ys, ts
template <class C>
__device__ __forceinline__ void zeta_dots_acc(double (&acc)[8], const C& tv, const C& sv, const C& yv) {
  acc[0] += (double)yv.x * yv.x + (double)yv.y * yv.y;            // yy
  acc[1] += (double)tv.x * tv.x + (double)tv.y * tv.y;            // tt
  acc[2] += (double)yv.x * tv.x + (double)yv.y * tv.y;            // yt
  acc[3] += (double)yv.x * tv.y - (double)yv.y * tv.x;
  acc[4] += (double)yv.x * sv.x + (double)yv.y * sv.y;            // ys
  acc[5] += (double)yv.x * sv.y - (double)yv.y * sv.x;
  acc[6] += (double)tv.x * sv.x + (double)tv.y * sv.y;            // ts
  acc[7] += (double)tv.x * sv.y - (double)tv.y * sv.x;
}

// alpha = rho1 / <rhat, v>; tot = (Re, Im) of <rhat, v>
__device__ __forceinline__ void alpha_from_dot(InstState& S, const double* tot) {
  S.alpha = zdiv(S.rho1, make_double2(tot[0], tot[1]));
}

// first form: tot = (<t,t>, Re <t,s>, Im <t,s>); else the eight dots above
__device__ __forceinline__ void zeta_eta_from_dots(InstState& S, const double* tot, bool first) {
  if (first) {
    S.zeta = zdiv(make_double2(tot[1], tot[2]), make_double2(tot[0], 0.0));
    S.eta = make_double2(0.0, 0.0);
  } else {
    const double2 yy = make_double2(tot[0], 0.0), tt = make_double2(tot[1], 0.0);
    const double2 yt = make_double2(tot[2], tot[3]);
    const double2 ty = make_double2(tot[2], -tot[3]);   // conj(t) y = conj(conj(y) t)
    const double2 ys = make_double2(tot[4], tot[5]);
    const double2 ts = make_double2(tot[6], tot[7]);
    const double2 den = zsub(zmul(tt, yy), zmul(yt, ty));
    S.zeta = zdiv(zsub(zmul(yy, ts), zmul(ys, ty)), den);
    S.eta = zdiv(zsub(zmul(tt, ys), zmul(yt, ts)), den);
  }
}

// reduce_last for CTAs of up to MAXW warps (any blockDim): publish per-CTA
// partials at red[(inst*RB + blockIdx.x)*KRED], last CTA (atomic ticket)
// sums them in a fixed order; true in the last CTA, totals in warp 0.
template <int K, int MAXW = 32>
__device__ __forceinline__ bool reduce_last_n(double (&v)[K], double (&tot)[K], double* red, unsigned* cnt, int inst,
                                              int RB, int nthreads) {
  __shared__ double sh[K][MAXW];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (nthreads + 31) >> 5;
  auto bsum = [&](double (&x)[K], double (&out)[K]) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double s = warp_sum(x[k]);
      if (lane == 0) sh[k][wid] = s;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
      for (int k = 0; k < K; ++k) out[k] = warp_sum(lane < nw ? sh[k][lane] : 0.0);
    }
  };
  double part[K];
  bsum(v, part);
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
  const double* src = red + (size_t)inst * RB * KRED;
  double gsum[K];
#pragma unroll
  for (int k = 0; k < K; ++k) gsum[k] = 0.0;
  for (int b = threadIdx.x; b < RB; b += nthreads) {
    double tt[K];
#pragma unroll
    for (int k = 0; k < K; ++k) tt[k] = __ldcg(src + (size_t)b * KRED + k);
#pragma unroll
    for (int k = 0; k < K; ++k) gsum[k] += tt[k];
  }
  bsum(gsum, tot);
  if (threadIdx.x == 0) cnt[inst] = 0u;
  return true;
}

}  // namespace dda
