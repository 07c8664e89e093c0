// A.P matvec of the discrete-dipole approximation as five pruned FFT passes.
//
//   y = inv_alpha * x - mask * IFFT3[ Ghat (3x3) . FFT3( pad x ) ]   (cropped)
//
// x lives on the (nx,ny,nz) box, component index fastest.  The 3D transform
// over the (Lx,Ly,Lz) circulant grid (L >= 2n) is split so that no pass reads
// or writes the zero padding:
//   pass 1  z-FFT of each (x,y) line          x  (nx,ny,nz,3) -> T1 (nx,ny,Lz,3)
//   pass 2  y-FFT, zero rows y >= ny           T1               -> T2 (nx,Ly,Lz,3)
//   pass 3  x-FFT -> 3x3 tensor -> x-IFFT,     T2 in place, rows x < nx only
//           Ghat read from the reduced octant through the mirror rule
//   pass 4  y-IFFT, keep rows y < ny           T2               -> T1
//   pass 5  z-IFFT, keep z < nz, fused combine T1               -> y
// The reference computes the same product with separate padded cuFFT calls in
// x-chunks (Gpbicgstab.py:742-772) and the mirrored tensor kernel
// chunked_dot_product_reduced_kernel (Gpbicgstab.py:167-237).
#pragma once
#include "dda_host.h"
#include "fft_core.cuh"
#include "fft_sizes.h"

namespace dda {

template <typename R> struct KP;            // per-precision tile constants
template <> struct KP<float> { static constexpr int EPT = 24, NT = 256; };
template <> struct KP<double> { static constexpr int EPT = 12, NT = 256; };

__device__ __forceinline__ int inst_of(const int* act) { return act ? act[blockIdx.y] : (int)blockIdx.y; }

// ---------------------------------------------------------------------------
// pass 1: forward z on NL lines; input zero beyond nz
// ---------------------------------------------------------------------------
template <typename R, int LZ>
__global__ void __launch_bounds__(KP<R>::NT) k_mv_pass1(Geo g, const typename CT<R>::T* __restrict__ tw,
                                                        InstState* st, const int* act, int in_id, int cond, int NL) {
  typedef typename CT<R>::T C;
  constexpr int NT = KP<R>::NT;
  constexpr int LS = 3 * LZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  InstState& S = st[inst_of(act)];
  if (!cond_ok(S, cond)) return;
  const C* __restrict__ x = (const C*)S.vec[in_id];
  C* __restrict__ t1 = (C*)S.t1;
  const long long nlines = (long long)g.nx * g.ny;
  const long long line0 = (long long)blockIdx.x * NL;
  for (int idx = threadIdx.x; idx < NL * g.nz; idx += NT) {
    const int l = idx / g.nz, iz = idx - l * g.nz;
    const long long line = line0 + l;
    C v0 = czero<C>(), v1 = v0, v2 = v0;
    if (line < nlines) {
      const C* p = x + (line * g.nz + iz) * 3;
      v0 = p[0]; v1 = p[1]; v2 = p[2];
    }
    C* q = s + l * LS + iz * 3;
    q[0] = v0; q[1] = v1; q[2] = v2;
  }
  const int zc = 3 * (LZ - g.nz);
  for (int idx = threadIdx.x; idx < NL * zc; idx += NT) {
    const int l = idx / zc, r = idx - l * zc;
    s[l * LS + 3 * g.nz + r] = czero<C>();
  }
  __syncthreads();
  LayLine<3> lay{NL, LS};
  fft_tile<LZ, false, KP<R>::EPT, NT>(s, lay, tw);
  for (int idx = threadIdx.x; idx < NL * LS; idx += NT) {
    const int l = idx / LS, r = idx - l * LS;
    const long long line = line0 + l;
    if (line < nlines) t1[line * LS + r] = s[l * LS + r];
  }
}

// ---------------------------------------------------------------------------
// pass 2 / 4: y transforms on a (ix, kz-tile) slab.  INV=false: T1 -> T2 with
// rows y >= ny zero; INV=true: T2 -> T1 keeping rows y < ny.
// ---------------------------------------------------------------------------
template <typename R, bool INV, int LY>
__global__ void __launch_bounds__(KP<R>::NT) k_mv_pass_y(Geo g, const typename CT<R>::T* __restrict__ tw,
                                                         InstState* st, const int* act, int cond, int Tz, int ntz) {
  typedef typename CT<R>::T C;
  constexpr int NT = KP<R>::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  InstState& S = st[inst_of(act)];
  if (!cond_ok(S, cond)) return;
  C* __restrict__ t1 = (C*)S.t1;
  C* __restrict__ t2 = (C*)S.t2;
  const int ix = blockIdx.x / ntz, kzt = blockIdx.x - ix * ntz;
  const int kz0 = kzt * Tz;
  const int tzn = min(Tz, g.Lz - kz0);
  const int W = 3 * Tz, Wv = 3 * tzn;
  const int rows_in = INV ? LY : g.ny;
  const C* __restrict__ src = INV ? t2 : t1;
  const long long src_row0 = INV ? (long long)ix * LY : (long long)ix * g.ny;
  for (int idx = threadIdx.x; idx < rows_in * W; idx += NT) {
    const int r = idx / W, w = idx - r * W;
    C v = czero<C>();
    if (w < Wv) v = src[((src_row0 + r) * g.Lz + kz0) * 3 + w];
    s[r * W + w] = v;
  }
  if (!INV) {
    for (int idx = threadIdx.x; idx < (LY - g.ny) * W; idx += NT) s[g.ny * W + idx] = czero<C>();
  }
  __syncthreads();
  LayCol lay{W, W};
  fft_tile<LY, INV, KP<R>::EPT, NT>(s, lay, tw);
  const int rows_out = INV ? g.ny : LY;
  C* __restrict__ dst = INV ? t1 : t2;
  const long long dst_row0 = INV ? (long long)ix * g.ny : (long long)ix * LY;
  for (int idx = threadIdx.x; idx < rows_out * Wv; idx += NT) {
    const int r = idx / Wv, w = idx - r * Wv;
    dst[((dst_row0 + r) * g.Lz + kz0) * 3 + w] = s[r * W + w];
  }
}

// ---------------------------------------------------------------------------
// pass 3: x-pencils: forward x-FFT, symmetric 3x3 tensor product with the
// mirrored octant, inverse x-FFT, keep rows x < nx (in place in T2).
// Mirror rule (Gpbicgstab.py:192-211): an index i > L/2 maps to L - i, and the
// xy / xz / yz entries change sign when exactly one index of the pair is
// mirrored.
// ---------------------------------------------------------------------------
template <typename R, int LX>
__global__ void __launch_bounds__(KP<R>::NT) k_mv_pass3(Geo g, const typename CT<R>::T* __restrict__ tw,
                                                        InstState* st, const int* act, int cond, int Tz, int ntz,
                                                        R gscale) {
  typedef typename CT<R>::T C;
  constexpr int NT = KP<R>::NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  InstState& S = st[inst_of(act)];
  if (!cond_ok(S, cond)) return;
  C* __restrict__ t2 = (C*)S.t2;
  const C* __restrict__ gh = (const C*)S.ghat;
  // pencil order 0, 1, Ly-1, 2, Ly-2, ... keeps mirrored pencils (which read
  // the same octant rows) adjacent in time so the second read hits L2
  const int p = blockIdx.x / ntz, kzt = blockIdx.x - p * ntz;
  int ky;
  if (p == 0) ky = 0;
  else { const int pr = (p + 1) >> 1; ky = (p & 1) ? pr : g.Ly - pr; }
  const int kz0 = kzt * Tz;
  const int tzn = min(Tz, g.Lz - kz0);
  const int W = 3 * Tz, Wv = 3 * tzn;
  const long long rstride = (long long)g.Ly * g.Lz * 3;   // between x rows
  const long long base = ((long long)ky * g.Lz + kz0) * 3;
  for (int idx = threadIdx.x; idx < g.nx * W; idx += NT) {
    const int r = idx / W, w = idx - r * W;
    C v = czero<C>();
    if (w < Wv) v = t2[r * rstride + base + w];
    s[r * W + w] = v;
  }
  for (int idx = threadIdx.x; idx < (LX - g.nx) * W; idx += NT) s[g.nx * W + idx] = czero<C>();
  __syncthreads();
  LayCol lay{W, W};
  fft_tile<LX, false, KP<R>::EPT, NT>(s, lay, tw);
  const bool fy = ky > g.Ly / 2;
  const int my = fy ? g.Ly - ky : ky;
  for (int idx = threadIdx.x; idx < LX * tzn; idx += NT) {
    const int kx = idx / tzn, kzl = idx - kx * tzn;
    const int kz = kz0 + kzl;
    const bool fx = kx > LX / 2, fz = kz > g.Lz / 2;
    const int mx = fx ? LX - kx : kx;
    const int mz = fz ? g.Lz - kz : kz;
    const C* q = gh + (((long long)mx * g.hy + my) * g.hz + mz) * 6;
    C gxx = q[0], gxy = q[1], gxz = q[2], gyy = q[3], gyz = q[4], gzz = q[5];
    const R sxy = (fx != fy) ? -gscale : gscale;
    const R sxz = (fx != fz) ? -gscale : gscale;
    const R syz = (fy != fz) ? -gscale : gscale;
    gxx = cscale(gxx, gscale); gyy = cscale(gyy, gscale); gzz = cscale(gzz, gscale);
    gxy = cscale(gxy, sxy); gxz = cscale(gxz, sxz); gyz = cscale(gyz, syz);
    C* v = s + kx * W + 3 * kzl;
    const C a = v[0], b = v[1], c = v[2];
    v[0] = cadd(cadd(cmul(gxx, a), cmul(gxy, b)), cmul(gxz, c));
    v[1] = cadd(cadd(cmul(gxy, a), cmul(gyy, b)), cmul(gyz, c));
    v[2] = cadd(cadd(cmul(gxz, a), cmul(gyz, b)), cmul(gzz, c));
  }
  __syncthreads();
  fft_tile<LX, true, KP<R>::EPT, NT>(s, lay, tw);
  for (int idx = threadIdx.x; idx < g.nx * Wv; idx += NT) {
    const int r = idx / Wv, w = idx - r * Wv;
    t2[r * rstride + base + w] = s[r * W + w];
  }
}

// ---------------------------------------------------------------------------
// pass 5: inverse z on NL lines, keep z < nz, fused combine:
//   MV_AX           y = ia*x - mask*conv        (interaction_mult)
//   MV_RESIDUAL     y = b - (ia*x - mask*conv)  (b already masked)
//   MV_CONV         y = conv                    (E_field_solver)
//   MV_CONV_MASKED  y = mask*conv               (fft_matvec)
// mask = (inv_alpha != 0), the reference's alpha != 0 (ddaforgit.py:1108).
// ---------------------------------------------------------------------------
template <typename R, int LZ>
__global__ void __launch_bounds__(KP<R>::NT) k_mv_pass5(Geo g, const typename CT<R>::T* __restrict__ tw,
                                                        InstState* st, const int* act, int in_id, int out_id,
                                                        int mode, int cond, int NL) {
  typedef typename CT<R>::T C;
  constexpr int NT = KP<R>::NT;
  constexpr int LS = 3 * LZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  InstState& S = st[inst_of(act)];
  if (!cond_ok(S, cond)) return;
  const C* __restrict__ t1 = (const C*)S.t1;
  const long long nlines = (long long)g.nx * g.ny;
  const long long line0 = (long long)blockIdx.x * NL;
  for (int idx = threadIdx.x; idx < NL * LS; idx += NT) {
    const int l = idx / LS, r = idx - l * LS;
    const long long line = line0 + l;
    s[l * LS + r] = (line < nlines) ? t1[line * LS + r] : czero<C>();
  }
  __syncthreads();
  LayLine<3> lay{NL, LS};
  fft_tile<LZ, true, KP<R>::EPT, NT>(s, lay, tw);
  const C* __restrict__ x = (const C*)S.vec[in_id];
  C* __restrict__ y = (C*)S.vec[out_id];
  const C* __restrict__ ia = (const C*)S.inva;
  const C* __restrict__ b = (const C*)S.vec[V_B];
  for (int idx = threadIdx.x; idx < NL * g.nz; idx += NT) {
    const int l = idx / g.nz, iz = idx - l * g.nz;
    const long long line = line0 + l;
    if (line >= nlines) continue;
    const long long site = line * g.nz + iz;
    const C* q = s + l * LS + iz * 3;
    C c0 = q[0], c1 = q[1], c2 = q[2];
    C* yo = y + site * 3;
    if (mode == MV_CONV) {
      yo[0] = c0; yo[1] = c1; yo[2] = c2;
      continue;
    }
    const C a = ia[site];
    const bool m = (a.x != (R)0) || (a.y != (R)0);
    if (!m) { c0 = c1 = c2 = czero<C>(); }
    if (mode == MV_CONV_MASKED) {
      yo[0] = c0; yo[1] = c1; yo[2] = c2;
      continue;
    }
    const C* xi = x + site * 3;
    C r0 = csub(cmul(a, xi[0]), c0), r1 = csub(cmul(a, xi[1]), c1), r2 = csub(cmul(a, xi[2]), c2);
    if (mode == MV_RESIDUAL) {
      const C* bi = b + site * 3;
      r0 = csub(bi[0], r0); r1 = csub(bi[1], r1); r2 = csub(bi[2], r2);
    }
    yo[0] = r0; yo[1] = r1; yo[2] = r2;
  }
}

// ---------------------------------------------------------------------------
// host dispatch over the compiled lengths
// ---------------------------------------------------------------------------
template <typename R> struct MvKernels {
  typedef typename CT<R>::T C;
  typedef void (*P1)(Geo, const C*, InstState*, const int*, int, int, int);
  typedef void (*PY)(Geo, const C*, InstState*, const int*, int, int, int);
  typedef void (*P3)(Geo, const C*, InstState*, const int*, int, int, int, R);
  typedef void (*P5)(Geo, const C*, InstState*, const int*, int, int, int, int, int);
  static P1 p1(int L) {
    switch (L) {
#define DDA_K(n) case n: return k_mv_pass1<R, n>;
      DDA_FFT_SIZES(DDA_K)
#undef DDA_K
    }
    return nullptr;
  }
  static PY py(int L, bool inv) {
    switch (L) {
#define DDA_K(n) case n: return inv ? (PY)k_mv_pass_y<R, true, n> : (PY)k_mv_pass_y<R, false, n>;
      DDA_FFT_SIZES(DDA_K)
#undef DDA_K
    }
    return nullptr;
  }
  static P3 p3(int L) {
    switch (L) {
#define DDA_K(n) case n: return k_mv_pass3<R, n>;
      DDA_FFT_SIZES(DDA_K)
#undef DDA_K
    }
    return nullptr;
  }
  static P5 p5(int L) {
    switch (L) {
#define DDA_K(n) case n: return k_mv_pass5<R, n>;
      DDA_FFT_SIZES(DDA_K)
#undef DDA_K
    }
    return nullptr;
  }
};

template <typename R>
cudaError_t launch_matvec_impl(Ctx& ctx, const Geo& g, const PassCfg& pc, InstState* st, const int* act, int nb,
                               int in_id, int out_id, int mode, int cond, double gscale, cudaStream_t s) {
  typedef typename CT<R>::T C;
  constexpr bool dbl = sizeof(R) == 8;
  constexpr int NT = KP<R>::NT;
  auto k1 = MvKernels<R>::p1(g.Lz);
  auto k2 = MvKernels<R>::py(g.Ly, false);
  auto k3 = MvKernels<R>::p3(g.Lx);
  auto k4 = MvKernels<R>::py(g.Ly, true);
  auto k5 = MvKernels<R>::p5(g.Lz);
  if (!k1 || !k2 || !k3 || !k4 || !k5) return cudaErrorInvalidValue;
  const C* twx = (const C*)ctx.twiddles(g.Lx, dbl);
  const C* twy = (const C*)ctx.twiddles(g.Ly, dbl);
  const C* twz = (const C*)ctx.twiddles(g.Lz, dbl);
  if (!twx || !twy || !twz) return cudaErrorMemoryAllocation;
  const int mx = 200 * 1024;
  cudaError_t e;
  if ((e = cudaFuncSetAttribute((const void*)k1, cudaFuncAttributeMaxDynamicSharedMemorySize, mx))) return e;
  if ((e = cudaFuncSetAttribute((const void*)k2, cudaFuncAttributeMaxDynamicSharedMemorySize, mx))) return e;
  if ((e = cudaFuncSetAttribute((const void*)k3, cudaFuncAttributeMaxDynamicSharedMemorySize, mx))) return e;
  if ((e = cudaFuncSetAttribute((const void*)k4, cudaFuncAttributeMaxDynamicSharedMemorySize, mx))) return e;
  if ((e = cudaFuncSetAttribute((const void*)k5, cudaFuncAttributeMaxDynamicSharedMemorySize, mx))) return e;
  k1<<<dim3((unsigned)pc.grid1, nb), NT, pc.smem1, s>>>(g, twz, st, act, in_id, cond, pc.NL);
  k2<<<dim3((unsigned)pc.grid2, nb), NT, pc.smem2, s>>>(g, twy, st, act, cond, pc.Tz2, pc.ntz2);
  k3<<<dim3((unsigned)pc.grid3, nb), NT, pc.smem3, s>>>(g, twx, st, act, cond, pc.Tz3, pc.ntz3, (R)gscale);
  k4<<<dim3((unsigned)pc.grid2, nb), NT, pc.smem2, s>>>(g, twy, st, act, cond, pc.Tz2, pc.ntz2);
  k5<<<dim3((unsigned)pc.grid1, nb), NT, pc.smem1, s>>>(g, twz, st, act, in_id, out_id, mode, cond, pc.NL);
  note_launch(s, 5);
  return cudaGetLastError();
}

}  // namespace dda
