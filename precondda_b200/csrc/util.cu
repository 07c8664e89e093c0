// Small batched vector kernels around the solver: masked right-hand side,
// precision conversion and accumulation for iterative refinement, norms, and
// the FP64 cross-section reduction.
#include "dda_host.h"
#include "reduce.cuh"

namespace dda {

// b = mask * E  with mask = (inv_alpha != 0) (ddaforgit.py:1108; the
// reference forms E_inc * mask at Gpbicgstab.py:935, :1064)
template <typename R>
__global__ void __launch_bounds__(KNT) k_make_b(InstState* st, const int* act, long long nsite, int src_id,
                                                int dst_id) {
  typedef typename CT<R>::T C;
  InstState& S = st[kinst(act)];
  if (!S.active) return;
  const C* __restrict__ e = (const C*)S.vec[src_id];
  const C* __restrict__ ia = (const C*)S.inva;
  C* __restrict__ b = (C*)S.vec[dst_id];
  const int* __restrict__ cid = S.cidx;
  grid_loop<KU>(nsite * 3, (long long)blockIdx.x * KNT + threadIdx.x, (long long)gridDim.x * KNT, [&](long long i) {
    const long long site = i / 3;
    if (cid) {
      const int k = cid[site];
      if (k >= 0) b[3LL * k + (i - 3 * site)] = e[i];
    } else {
      const C a = ia[site];
      const bool m = (a.x != (R)0) || (a.y != (R)0);
      b[i] = m ? e[i] : czero<C>();
    }
  });
}

// dst(c64).vec[did] = (complex64) src(c128).vec[sid]
__global__ void __launch_bounds__(KNT) k_down(InstState* dst, int did, const InstState* src, int sid,
                                              const int* act, long long n3) {
  const int j = kinst(act);
  InstState& D = dst[j];
  if (!D.active) return;
  const double2* __restrict__ s = (const double2*)src[j].vec[sid];
  float2* __restrict__ d = (float2*)D.vec[did];
  const int* __restrict__ cid = D.cidx;
  for (long long i = (long long)blockIdx.x * KNT + threadIdx.x; i < n3; i += (long long)gridDim.x * KNT) {
    const float2 v = make_float2((float)s[i].x, (float)s[i].y);
    if (cid) {
      const long long site = i / 3;
      const int k = cid[site];
      if (k >= 0) d[3LL * k + (i - 3 * site)] = v;
    } else {
      d[i] = v;
    }
  }
}

// solution of a finished complex64 solve: the current iterate when it
// converged, else the best one, else zero (Gpbicgstab.py:1162-1201)
__device__ __forceinline__ const float2* sol64(const InstState& S) {
  if (S.status == ST_CONVERGED) return (const float2*)S.vec[V_X];
  if (S.best_x >= 0) return (const float2*)S.vec[V_XA + S.best_x];
  return nullptr;
}

// S.vec[V_TMP] := the iterate sol64 / k_store_solution read (the current one
// when no solution exists: it is never stored then), so a preconditioned
// solve can apply M to it in place before the store.
__global__ void k_pick_solution(InstState* st, const int* act, int nb) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nb) return;
  InstState& S = st[act ? act[j] : j];
  if (!S.active) return;
  void* e = S.vec[V_X];
  if (S.status != ST_CONVERGED && S.best_x >= 0) e = S.vec[V_XA + S.best_x];
  S.vec[V_TMP] = e;
}

void launch_pick_solution(InstState* st, int nb, cudaStream_t s, const int* act) {
  k_pick_solution<<<(nb + 127) / 128, 128, 0, s>>>(st, act, nb);
  note_launch(s, 1);
}

// x128 += solution(c64)
__global__ void __launch_bounds__(KNT) k_accum(InstState* st128, int xid, const InstState* st64, const int* act,
                                               long long n3) {
  const int j = kinst(act);
  const InstState& S = st64[j];
  if (!st128[j].active) return;
  const float2* __restrict__ e = sol64(S);
  if (!e) return;
  double2* __restrict__ x = (double2*)st128[j].vec[xid];
  const int* __restrict__ cid = S.cidx;
  grid_loop<KU>(n3, (long long)blockIdx.x * KNT + threadIdx.x, (long long)gridDim.x * KNT, [&](long long i) {
    long long src = i;
    if (cid) {
      const long long site = i / 3;
      const int k = cid[site];
      if (k < 0) return;
      src = 3LL * k + (i - 3 * site);
    }
    const float2 v = e[src];
    double2 a = x[i];
    a.x += (double)v.x; a.y += (double)v.y;
    x[i] = a;
  });
}

// P (dense, S.out) = solution of a finished solve: the current iterate when
// it converged, else the best one, else zero (Gpbicgstab.py:1162-1201);
// expanded from occupied-site storage when the instance uses it
template <typename R>
__global__ void __launch_bounds__(KNT) k_store_solution(const InstState* st, const int* act, long long n3) {
  typedef typename CT<R>::T C;
  const InstState& S = st[kinst(act)];
  if (!S.active || !S.out) return;
  const C* __restrict__ e = nullptr;
  if (S.status == ST_CONVERGED) e = (const C*)S.vec[V_X];
  else if (S.best_x >= 0) e = (const C*)S.vec[V_XA + S.best_x];
  C* __restrict__ out = (C*)S.out;
  const int* __restrict__ cid = S.cidx;
  grid_loop<KU>(n3, (long long)blockIdx.x * KNT + threadIdx.x, (long long)gridDim.x * KNT, [&](long long i) {
    C v = czero<C>();
    if (e) {
      if (cid) {
        const long long site = i / 3;
        const int k = cid[site];
        if (k >= 0) v = e[3LL * k + (i - 3 * site)];
      } else {
        v = e[i];
      }
    }
    out[i] = v;
  });
}

// ---------------------------------------------------------------------------
// occupied-site map: cidx[site] = rank of the site among the sites with
// inv_alpha != 0 (site order), -1 for an empty site; S.nv = 3 x count.
// Three passes over blocks of kSiteBlock sites: count, scan the block
// counts, write the ranks.  Every step has a fixed order (deterministic).
// ---------------------------------------------------------------------------
constexpr int kSitePer = 4;                      // sites per thread
constexpr int kSiteBlock = KNT * kSitePer;       // sites per CTA

template <typename R>
__device__ __forceinline__ int site_flags(const InstState& S, long long base, long long nsite, bool* f) {
  typedef typename CT<R>::T C;
  const C* __restrict__ ia = (const C*)S.inva;
  int n = 0;
#pragma unroll
  for (int j = 0; j < kSitePer; ++j) {
    const long long site = base + j;
    bool m = false;
    if (site < nsite) {
      const C a = ia[site];
      m = (a.x != (R)0) || (a.y != (R)0);
    }
    f[j] = m;
    n += m;
  }
  return n;
}

// exclusive prefix sum of v over the CTA (KNT threads); *total = CTA sum
__device__ __forceinline__ int block_excl_scan(int v, int* total) {
  __shared__ int wsum[KNW];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[wid] = x;
  __syncthreads();
  int woff = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < KNW; ++w) {
    if (w < wid) woff += wsum[w];
    tot += wsum[w];
  }
  __syncthreads();
  *total = tot;
  return woff + x - v;
}

template <typename R>
__global__ void __launch_bounds__(KNT) k_site_count(InstState* st, const int* act, long long nsite, int nblk,
                                                    int* bcount) {
  const int inst = kinst(act);
  const InstState& S = st[inst];
  if (!S.active || !S.cidx) return;
  bool f[kSitePer];
  const int n = site_flags<R>(S, (long long)blockIdx.x * kSiteBlock + (long long)threadIdx.x * kSitePer, nsite, f);
  int total;
  block_excl_scan(n, &total);
  if (threadIdx.x == 0) bcount[(size_t)inst * nblk + blockIdx.x] = total;
}

// one CTA per instance: block counts -> exclusive block offsets, nv = 3 M
__global__ void __launch_bounds__(KNT) k_site_scan(InstState* st, const int* act, int nblk, int* bcount) {
  const int inst = kinst(act);
  InstState& S = st[inst];
  if (!S.active || !S.cidx) return;
  int* bc = bcount + (size_t)inst * nblk;
  int carry = 0;
  for (int b0 = 0; b0 < nblk; b0 += KNT) {
    const int b = b0 + threadIdx.x;
    const int v = b < nblk ? bc[b] : 0;
    int total;
    const int ex = block_excl_scan(v, &total);
    if (b < nblk) bc[b] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) S.nv = 3LL * carry;
}

template <typename R>
__global__ void __launch_bounds__(KNT) k_site_index(InstState* st, const int* act, long long nsite, int nblk,
                                                    const int* bcount) {
  const int inst = kinst(act);
  const InstState& S = st[inst];
  if (!S.active || !S.cidx) return;
  const long long base = (long long)blockIdx.x * kSiteBlock + (long long)threadIdx.x * kSitePer;
  bool f[kSitePer];
  const int n = site_flags<R>(S, base, nsite, f);
  int total;
  int r = bcount[(size_t)inst * nblk + blockIdx.x] + block_excl_scan(n, &total);
  int* cid = const_cast<int*>(S.cidx);
#pragma unroll
  for (int j = 0; j < kSitePer; ++j) {
    if (base + j < nsite) cid[base + j] = f[j] ? r : -1;
    r += f[j];
  }
}

// out[inst] = ||vec[id]||^2 (FP64, deterministic)
template <typename R>
__global__ void __launch_bounds__(KNT) k_norm2(InstState* st, const int* act, int id, long long n3, double* red,
                                               unsigned* cnt, int RB, double* out) {
  typedef typename CT<R>::T C;
  const int inst = kinst(act);
  InstState& S = st[inst];
  if (!S.active) return;
  const C* __restrict__ v = (const C*)S.vec[id];
  double acc[1] = {0.0};
  grid_loop<KU>(n3, (long long)blockIdx.x * KNT + threadIdx.x, (long long)RB * KNT, [&](long long i) {
    const C a = v[i];
    acc[0] += (double)a.x * a.x + (double)a.y * a.y;
  });
  double tot[1];
  if (reduce_last<1>(acc, tot, red, cnt, inst, RB) && threadIdx.x == 0) out[inst] = tot[0];
}

// cross sections (Draine & Flatau 1994): sums reduced in FP64
template <typename R>
__global__ void __launch_bounds__(KNT) k_xsec(const typename CT<R>::T* __restrict__ P,
                                              const typename CT<R>::T* __restrict__ E,
                                              const typename CT<R>::T* __restrict__ ia, long long nsite, double k3,
                                              double* red, unsigned* cnt, int RB, double* out) {
  typedef typename CT<R>::T C;
  double acc[2] = {0.0, 0.0};
  for (long long j = (long long)blockIdx.x * KNT + threadIdx.x; j < nsite; j += (long long)RB * KNT) {
    const C a = ia[j];
    if (a.x == (R)0 && a.y == (R)0) continue;
    double p2 = 0.0, ext = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const C p = P[j * 3 + c], e = E[j * 3 + c];
      ext += (double)e.x * p.y - (double)e.y * p.x;       // Im(conj(e) p)
      p2 += (double)p.x * p.x + (double)p.y * p.y;
    }
    // Im(P . conj(ia) P*) = Im(conj(ia)) |P|^2 = -Im(ia) |P|^2
    acc[0] += ext;
    acc[1] += (-(double)a.y - (2.0 / 3.0) * k3) * p2;
  }
  double tot[2];
  if (reduce_last<2>(acc, tot, red, cnt, 0, RB) && threadIdx.x == 0) {
    out[0] = tot[0];
    out[1] = tot[1];
  }
}

// ---------------------------------------------------------------------------
int grid_for(long long n, int nb, int num_sms) {
  long long want = (n + KNT - 1) / KNT;
  long long cap = (4LL * num_sms + nb - 1) / nb;
  if (cap < 1) cap = 1;
  if (want > cap) want = cap;
  if (want < 1) want = 1;
  return (int)want;
}

template <typename R>
void launch_make_b(InstState* st, int nb, long long nsite, int src, int dst, int num_sms, cudaStream_t s,
                   const int* act) {
  k_make_b<R><<<dim3(grid_for(nsite * 3, nb, num_sms), nb), KNT, 0, s>>>(st, act, nsite, src, dst);
  note_launch(s, 1);
}
template void launch_make_b<float>(InstState*, int, long long, int, int, int, cudaStream_t, const int*);
template void launch_make_b<double>(InstState*, int, long long, int, int, int, cudaStream_t, const int*);

void launch_down(InstState* dst, int did, const InstState* src, int sid, int nb, long long n3, int num_sms,
                 cudaStream_t s, const int* act) {
  k_down<<<dim3(grid_for(n3, nb, num_sms), nb), KNT, 0, s>>>(dst, did, src, sid, act, n3);
  note_launch(s, 1);
}

void launch_accum(InstState* st128, int xid, const InstState* st64, int nb, long long n3, int num_sms,
                  cudaStream_t s, const int* act) {
  k_accum<<<dim3(grid_for(n3, nb, num_sms), nb), KNT, 0, s>>>(st128, xid, st64, act, n3);
  note_launch(s, 1);
}

int site_blocks(long long nsite) { return (int)((nsite + kSiteBlock - 1) / kSiteBlock); }

template <typename R>
void launch_site_map(InstState* st, int nb, long long nsite, int* bcount, cudaStream_t s, const int* act) {
  const int nblk = site_blocks(nsite);
  k_site_count<R><<<dim3(nblk, nb), KNT, 0, s>>>(st, act, nsite, nblk, bcount);
  k_site_scan<<<dim3(1, nb), KNT, 0, s>>>(st, act, nblk, bcount);
  k_site_index<R><<<dim3(nblk, nb), KNT, 0, s>>>(st, act, nsite, nblk, bcount);
  note_launch(s, 3);
}
template void launch_site_map<float>(InstState*, int, long long, int*, cudaStream_t, const int*);
template void launch_site_map<double>(InstState*, int, long long, int*, cudaStream_t, const int*);

template <typename R>
void launch_store_solution(InstState* st, int nb, long long n3, int num_sms, cudaStream_t s, const int* act) {
  k_store_solution<R><<<dim3(grid_for(n3, nb, num_sms), nb), KNT, 0, s>>>(st, act, n3);
  note_launch(s, 1);
}
template void launch_store_solution<float>(InstState*, int, long long, int, cudaStream_t, const int*);
template void launch_store_solution<double>(InstState*, int, long long, int, cudaStream_t, const int*);

template <typename R>
void launch_norm2(InstState* st, int id, int nb, long long n3, double* red, unsigned* cnt, int RB, double* out,
                  cudaStream_t s, const int* act) {
  k_norm2<R><<<dim3(RB, nb), KNT, 0, s>>>(st, act, id, n3, red, cnt, RB, out);
  note_launch(s, 1);
}
template void launch_norm2<float>(InstState*, int, int, long long, double*, unsigned*, int, double*, cudaStream_t,
                                  const int*);
template void launch_norm2<double>(InstState*, int, int, long long, double*, unsigned*, int, double*, cudaStream_t,
                                   const int*);

template <typename R>
void launch_xsec(const void* P, const void* E, const void* ia, long long nsite, double k, double* red, unsigned* cnt,
                 int RB, double* out, cudaStream_t s) {
  typedef typename CT<R>::T C;
  k_xsec<R><<<RB, KNT, 0, s>>>((const C*)P, (const C*)E, (const C*)ia, nsite, k * k * k, red, cnt, RB, out);
  note_launch(s, 1);
}
template void launch_xsec<float>(const void*, const void*, const void*, long long, double, double*, unsigned*, int,
                                 double*, cudaStream_t);
template void launch_xsec<double>(const void*, const void*, const void*, long long, double, double*, unsigned*, int,
                                  double*, cudaStream_t);

}  // namespace dda
