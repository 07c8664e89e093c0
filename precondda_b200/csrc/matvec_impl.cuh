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
// Each pass loads its first FFT stage straight from global memory into
// registers and stores its last stage straight back (fftreg.cuh), so a
// two-stage length costs one shared-memory exchange.  The reference computes
// the same product with separate padded cuFFT calls in x-chunks
// (Gpbicgstab.py:742-772) and the mirrored tensor kernel
// chunked_dot_product_reduced_kernel (Gpbicgstab.py:167-237).
#pragma once
#include "dda_host.h"
#include "fftreg.cuh"
#include "krylov_ctrl.cuh"
#include "fft_sizes.h"
#include "bulk.cuh"
#include "cpair.cuh"
#include <cooperative_groups.h>
#include <cstdlib>
#include <type_traits>

namespace dda {

namespace cg = cooperative_groups;

constexpr int kMvMaxThreads = 384;

// L2 prefetch of the input rows of another tile: `rows` row segments of
// `bytes` each, `stride` elements apart, issued by warp 0 as bulk prefetches.
template <class C>
__device__ __forceinline__ void prefetch_rows(const C* base, long long stride, int rows, int bytes) {
  if (threadIdx.x >= 32) return;
  for (int r = threadIdx.x; r < rows; r += 32) bulk_prefetch_l2(base + r * stride, (uint32_t)bytes);
}

// Twiddle tables in shared memory: the transform passes of a precision
// with the switch on copy their table there at entry (after the pass's
// exchange area) and read it from there instead of through the read-only
// global path.  B200, 128^3 matvec: complex128 1.434 -> 1.322 ms (on);
// complex64 0.5412 -> 0.5406 ms (off: no gain).  DDA_SMEM_TW_C64 /
// DDA_SMEM_TW_C128 override.
#ifndef DDA_SMEM_TW_C64
#define DDA_SMEM_TW_C64 0
#endif
#ifndef DDA_SMEM_TW_C128
#define DDA_SMEM_TW_C128 1
#endif
// whether the passes of complex elements of `bytes` bytes stage twiddles
__host__ __device__ constexpr bool smem_tw(int bytes) { return bytes == 16 ? DDA_SMEM_TW_C128 : DDA_SMEM_TW_C64; }
// The twiddle source of a pass: the global table, or its shared copy at
// `at` (n entries).
template <class C>
__device__ __forceinline__ auto pass_tw(const C* __restrict__ tw, void* at, int n) {
  if constexpr (smem_tw((int)sizeof(C))) {
    return tw_to_shared(tw, reinterpret_cast<C*>(at), n);
  } else {
    (void)at; (void)n;
    return tw;
  }
}

template <typename R, int L>
struct MvShape {
  typedef typename PlanFor<L, R>::type P;
  static constexpr int T = P::T, E = P::E, LP = ppad_len(L);
};

// Pass-3 variants (chosen by the launch configuration):
//   0: default plan, tensor product through shared memory
//   1: radix<=8 plan, three components per thread, tensor product in registers
//   2: radix<=8 plan, tensor product through shared memory
template <typename R, int L, int V>
struct P3Shape {
  typedef typename std::conditional<V == 0, typename PlanFor<L, R>::type, typename Plan8<L>::type>::type P;
  static constexpr int T = P::T, E = P::E, LP = ppad_len(L);
  static constexpr bool REG = (V == 1);
};
constexpr int kP3Variants = 3;

__device__ __forceinline__ int inst_of(const int* act) { return act ? act[blockIdx.y] : (int)blockIdx.y; }

// ---------------------------------------------------------------------------
// Tile sizes shared by the host configuration and the compile-time kernels:
// about 128 (complex64) or 64 (complex128) transforms' worth of threads per
// CTA.
// ---------------------------------------------------------------------------
// DDA_C128_LANES overrides the complex128 width (an A/B build option).
#ifndef DDA_C128_LANES
#define DDA_C128_LANES 64
#endif
// Complex128 transforms of 32 or more threads (the radix-8 plans of L >=
// 256) take twice the lanes: 4-column tiles, 192-byte row segments.  B200,
// 128^3 complex128 matvec 1.323 -> 1.255 ms; at L = 128 the wider tiles were
// slower (64^3: 0.150 -> 0.154 ms), so shorter transforms keep 64.
#ifndef DDA_C128_WIDE_LANES
#define DDA_C128_WIDE_LANES 128
#endif
template <typename R> constexpr int mv_lanes_t(int T) {
  return sizeof(R) == 4 ? 128 : (T >= 32 ? DDA_C128_WIDE_LANES : DDA_C128_LANES);
}
constexpr int cmin_i(int a, int b) { return a < b ? a : b; }
template <typename R, int T> constexpr int mv_tiles() { return mv_lanes_t<R>(T) / T > 1 ? mv_lanes_t<R>(T) / T : 1; }
// kz columns per CTA of the one-component x pass (k_mv_pass3s);
// DDA_P3_TZ128 > 0 sets it for complex64 L = 128 (an A/B build option)
#ifndef DDA_P3_TZ128
#define DDA_P3_TZ128 0
#endif
template <typename R, int LX, int T> constexpr int p3s_tiles() {
  return (sizeof(R) == 4 && LX == 128 && DDA_P3_TZ128 > 0) ? DDA_P3_TZ128 : mv_tiles<R, T>();
}

// NC > 0 selects the cubic specialisation of a pass: box NC^3 on the FFT
// grid (2 NC)^3, every size a compile-time constant, so shared-memory and
// global addresses become immediate offsets from per-thread bases, the zero
// half of each padded input is never loaded (and its first butterfly layer
// is pruned), and only the kept half of each inverse output is formed.
// NC = 0 reads the sizes from Geo.

// Register caps.  Each z / y pass exists twice: the plain kernel under
// __launch_bounds__(384) alone, and a `_cap` twin with __maxnreg__ (the same
// body, included from mv_pass*.inc); the dispatch takes the twin only for the
// instantiations a cap was measured to help.  __maxnreg__ 255 is not "no
// cap": ptxas then allocates more freely than under the launch bound alone
// (cubic L = 128 y pass 56 -> 87 registers, 128^3 complex64 matvec 7 %
// slower), and above 170 registers a 384-thread CTA cannot launch at all.
//
// Cubic complex64 z passes (1 and 5) of power-of-two lengths >= 128: 56
// registers, i.e. three CTAs of 384 threads per SM (a few bytes of spill;
// pass 5 otherwise takes 76 and fits two).  B200, 128^3 matvec 0.570 ->
// 0.538 ms, 64^3 unchanged.  DDA_Z_REGS / DDA_Z1_REGS override the cap of
// both passes / of pass 1.
#ifndef DDA_Z_REGS
#define DDA_Z_REGS 56
#endif
#ifndef DDA_Z1_REGS
#define DDA_Z1_REGS DDA_Z_REGS
#endif
// Mixed-radix lengths 40-192 (boxes 20^3-96^3): the x pass at two CTAs per
// SM (one CTA at 118-158 registers: 16-RHS matvecs 2-15 % slower); z passes
// plain (capped at 85 registers they were 5-9 % slower).  DDA_ZMR_REGS /
// DDA_P3MR_MINB override.
#ifndef DDA_ZMR_REGS
#define DDA_ZMR_REGS 0
#endif
#ifndef DDA_P3MR_MINB
#define DDA_P3MR_MINB 2
#endif
template <int NC> constexpr bool mixed_radix_mid() { return NC >= 20 && NC <= 96 && ((2 * NC) & (2 * NC - 1)) != 0; }
// General (runtime-size, NC = 0) complex64 kernels: the x pass at two CTAs
// per SM (one CTA: 16-RHS matvecs of non-cubic boxes 1-17 % slower); z and y
// passes plain (capped at 85 registers they were 5-16 % slower).
// DDA_GEN_REGS (z), DDA_GEN_Y_REGS (y) and DDA_GEN_P3_MINB override; a
// register cap of 0 selects the plain kernel.
#ifndef DDA_GEN_REGS
#define DDA_GEN_REGS 0
#endif
#ifndef DDA_GEN_Y_REGS
#define DDA_GEN_Y_REGS DDA_GEN_REGS
#endif
#ifndef DDA_GEN_P3_MINB
#define DDA_GEN_P3_MINB 2
#endif
// Complex128 z passes of power-of-two cubic lengths >= 128: at most 80
// registers (two CTAs of 384 threads per SM), the cap under which pass 5
// holds its batched combine operands (uncapped: 102).  At 56 registers
// (three CTAs) the 128^3 matvec took 1.403 against 1.428 ms plain, within
// noise.  DDA_ZD_REGS=0 leaves them uncapped.
#ifndef DDA_ZD_REGS
#define DDA_ZD_REGS 80
#endif
// Register cap of a z pass (0 = the plain kernel).
template <typename R, int NC, int CAP>
constexpr int z_regs() {
  if (sizeof(R) != 4) return (NC >= 64 && ((2 * NC) & (2 * NC - 1)) == 0) ? DDA_ZD_REGS : 0;
  if (NC >= 64 && ((2 * NC) & (2 * NC - 1)) == 0) return CAP;
  if (mixed_radix_mid<NC>()) return DDA_ZMR_REGS;
  return NC == 0 ? DDA_GEN_REGS : 0;
}
// Cubic complex64 y passes of power-of-two length: DDA_Y_REGS caps the
// forward (zero-half) pass, DDA_YI_REGS the inverse (0: plain kernels).
#ifndef DDA_Y_REGS
#define DDA_Y_REGS 0
#endif
#ifndef DDA_YI_REGS
#define DDA_YI_REGS 0
#endif
// Register cap of a y pass (0 = the plain kernel).
template <typename R, int NC, bool INV = false> constexpr int y_regs() {
  if (sizeof(R) == 4 && NC >= 64 && ((2 * NC) & (2 * NC - 1)) == 0) return INV ? DDA_YI_REGS : DDA_Y_REGS;
  return (sizeof(R) == 4 && NC == 0) ? DDA_GEN_Y_REGS : 0;
}

// ---------------------------------------------------------------------------
// pass 1: forward z on nl lines x 3 components; input zero beyond nz
// thread = (c fastest, t, line)
// ---------------------------------------------------------------------------
template <typename R, int LZ, int NC>
__global__ void __launch_bounds__(kMvMaxThreads)
    k_mv_pass1(Geo g, const typename CT<R>::T* __restrict__ tw, InstState* st, const int* act, int in_id,
               int cond, int nl_, int pre)
#include "mv_pass1.inc"
template <typename R, int LZ, int NC>
__global__ void __launch_bounds__(kMvMaxThreads) __maxnreg__((z_regs<R, NC, DDA_Z1_REGS>()))
    k_mv_pass1_cap(Geo g, const typename CT<R>::T* __restrict__ tw, InstState* st, const int* act, int in_id,
                   int cond, int nl_, int pre)
#include "mv_pass1.inc"

// ---------------------------------------------------------------------------
// pass 2 / 4: y transforms on a (ix, kz-tile) slab, W = 3 tz transforms;
// thread = (w fastest, t).  INV=false: T1 -> T2 (rows y >= ny are zero);
// INV=true: T2 -> T1 keeping rows y < ny.
// ---------------------------------------------------------------------------
template <typename R, bool INV, int LY, int NC>
__global__ void __launch_bounds__(kMvMaxThreads)
    k_mv_pass_y(Geo g, const typename CT<R>::T* __restrict__ tw, InstState* st, const int* act, int cond,
                int tz_, int ntz_)
#include "mv_pass_y.inc"
template <typename R, bool INV, int LY, int NC>
__global__ void __launch_bounds__(kMvMaxThreads) __maxnreg__((y_regs<R, NC, INV>()))
    k_mv_pass_y_cap(Geo g, const typename CT<R>::T* __restrict__ tw, InstState* st, const int* act, int cond,
                    int tz_, int ntz_)
#include "mv_pass_y.inc"

// ---------------------------------------------------------------------------
// pass 3: x-pencils: forward x-FFT, symmetric 3x3 tensor product with the
// mirrored octant, inverse x-FFT, keep rows x < nx (in place in T2).
// Mirror rule (Gpbicgstab.py:192-211): an index i > L/2 maps to L - i, and the
// xy / xz / yz entries change sign when exactly one index of the pair is
// mirrored.  The pencil row order 0, 1, Ly-1, 2, Ly-2, ... keeps mirrored
// pencils (which read the same octant rows) adjacent in time so the second
// read hits L2.
// ---------------------------------------------------------------------------
// Ghat is stored structure-of-arrays inside the engine: component c of octant
// point (mx,my,mz) at gh[c*H + (mx*hy + my)*hz + mz], H = hx*hy*hz, so the
// lanes of a warp (consecutive kz) read consecutive addresses.
__device__ __forceinline__ int pencil_ky(int p, int Ly) {
  if (p == 0) return 0;
  const int pr = (p + 1) >> 1;
  return (p & 1) ? pr : Ly - pr;
}

// variant with the three components of a pencil in one thread and the
// tensor product in registers: thread = (kzl fastest, t)
template <typename R, int LX, int V, int NC>
__global__ void __launch_bounds__(kMvMaxThreads) k_mv_pass3r(Geo g, const typename CT<R>::T* __restrict__ tw,
                                                             InstState* st, const int* act, int cond, int tz_,
                                                             int ntz_, R gscale, int op) {
  grid_dep_begin();
  typedef typename CT<R>::T C;
  typedef P3Shape<R, LX, V> SH;
  typedef typename SH::P P;
  typedef RevPlan<P> Q;
  constexpr bool CUBE = NC > 0;
  static_assert(!CUBE || LX == 2 * NC, "cubic kernels need L = 2n");
  constexpr int TZC = CUBE ? cmin_i(mv_tiles<R, SH::T>(), LX) : 1;
  constexpr int NTZC = (LX + TZC - 1) / TZC;
  constexpr bool ZH = CUBE && P::r[0] % 2 == 0;
  constexpr bool DH = CUBE && half_store_ok<Q>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  InstState& S = st[inst_of(act)];
  if (!cond_ok(S, cond)) return;
  C* __restrict__ t2 = (C*)S.t2;
  // op 0: the interaction octant; op 1: the preconditioner octant
  const C* __restrict__ gh = (const C*)(op ? S.pghat : S.ghat);
  const int tz = CUBE ? TZC : tz_;
  const int ntz = CUBE ? NTZC : ntz_;
  const int Ly = CUBE ? LX : g.Ly, Lz = CUBE ? LX : g.Lz;
  const int hy = CUBE ? LX / 2 + 1 : g.hy, hz = CUBE ? LX / 2 + 1 : g.hz;
  const int H = CUBE ? (LX / 2 + 1) * (LX / 2 + 1) * (LX / 2 + 1) : g.hx * g.hy * g.hz;
  const int nx = CUBE ? NC : g.nx;
  const int kzl = threadIdx.x % tz, t = threadIdx.x / tz;
  const int p = blockIdx.x / ntz, kzt = blockIdx.x - p * ntz;
  const int ky = pencil_ky(p, Ly);
  const int kz0 = kzt * tz;
  const int kz = kz0 + kzl;
  const bool ok = (CUBE && LX % TZC == 0) || kz < Lz;
  const long long rs = (long long)Ly * Lz * 3;          // x-row stride of T2
  C* col = t2 + ((long long)ky * Lz + kz) * 3;
  const int W = 3 * tz;
  C* sw = s + 3 * kzl;
  auto ld = [&](int c, int pos) -> C { return (ok && (ZH || pos < nx)) ? __ldcg(col + pos * rs + c) : czero<C>(); };
  auto sm = [&](int c, int pp) -> C& { return sw[pp * W + c]; };
  C a[3 * P::E];
  rload<P, 3, ZH>(a, t, ld);
#pragma unroll
  for (int c = 0; c < 3; ++c) rstage<P, 0, ZH>(a + c * P::E, t, tw);
  rrest<P, 3, 0>(a, t, sm, tw);
  // tensor product at the positions this thread owns after the last stage
  constexpr int RL = P::r[P::S - 1];
  const bool fy = ky > Ly / 2, fz = kz > Lz / 2;
  const int my = fy ? Ly - ky : ky;
  const int mz = fz ? Lz - kz : kz;
  const C* __restrict__ q0 = gh + my * hz + mz;
  if (ok) {
#pragma unroll
    for (int b = 0; b < P::E / RL; ++b)
#pragma unroll
      for (int q = 0; q < RL; ++q) {
        const int i = b * RL + q;
        const int kx = rout_pos<P, P::S - 1>(t, b, q);
        const bool fx = kx > LX / 2;
        const int mx = fx ? LX - kx : kx;
        const C* qp = q0 + mx * (hy * hz);
        const R sxy = (fx != fy) ? -gscale : gscale, sxz = (fx != fz) ? -gscale : gscale;
        const R syz = (fy != fz) ? -gscale : gscale;
        const C gxx = cscale(__ldg(qp), gscale), gxy = cscale(__ldg(qp + H), sxy);
        const C gxz = cscale(__ldg(qp + 2 * H), sxz), gyy = cscale(__ldg(qp + 3 * H), gscale);
        const C gyz = cscale(__ldg(qp + 4 * H), syz), gzz = cscale(__ldg(qp + 5 * H), gscale);
        const C a0 = a[i], a1 = a[P::E + i], a2 = a[2 * P::E + i];
        a[i] = cadd(cadd(cmul(gxx, a0), cmul(gxy, a1)), cmul(gxz, a2));
        a[P::E + i] = cadd(cadd(cmul(gxy, a0), cmul(gyy, a1)), cmul(gyz, a2));
        a[2 * P::E + i] = cadd(cadd(cmul(gxz, a0), cmul(gyz, a1)), cmul(gzz, a2));
      }
  }
  // inverse transform with the reversed plan: its stage 0 owns the same
  // positions; run as swap(FFT(swap(.)))
  const int ti = opaque(t);
  C* colo = opaque_ptr(col);
  auto stf = [&](int c, int pos, C v) { if (ok && (DH || pos < nx)) __stcg(colo + pos * rs + c, cswap(v)); };
#pragma unroll
  for (int i = 0; i < 3 * P::E; ++i) a[i] = cswap(a[i]);
#pragma unroll
  for (int c = 0; c < 3; ++c) rstage<Q, 0>(a + c * P::E, ti, tw);
  rrest<Q, 3, 0>(a, ti, sm, tw);
  rstore<Q, 3, DH>(a, ti, stf);
}

// variant with one component per thread and the tensor product through
// shared memory: thread = (w fastest, t)
// Cubic complex64 kernels of power-of-two length (E <= 16 per thread): three
// CTAs of 384 threads per SM (56 registers).  L = 128 (64^3 boxes) ran at
// two CTAs while its 56-register build spilled; with the transform-index
// range known to the compiler it no longer does, and three CTAs measured
// faster (B200, two-RHS 64^3 matvec 0.1270 -> 0.1208 ms, one RHS 0.0728 ->
// 0.0706 ms).  DDA_P3_MINB overrides all lengths.
// Complex128 cubic x passes of power-of-two length: at most 85 registers (two
// 384-thread CTAs; the 192-thread launches then fit four per SM).  ptxas
// settles at 80 without spills, against 100-108 uncapped: 64^3 two-RHS
// matvec 0.347 -> 0.323 ms, 128^3 1.636 -> 1.54 ms, preconditioned c128
// solve of the 64^3 sphere 39.2 -> 35.7 ms.  DDA_P3D_MINB overrides.
#ifndef DDA_P3D_MINB
#define DDA_P3D_MINB 2
#endif
// Complex128 x passes of every other length (general and mixed-radix
// cubic kernels): one CTA per SM.  At two, 4-RHS matvecs took 80^3 1.92
// against 1.38 ms, 48^3 0.42 against 0.27 ms, 96x64x96 2.55 against 1.42 ms
// (100x60x30 0.59 against 0.65 ms).  DDA_P3D_GEN_MINB overrides.
#ifndef DDA_P3D_GEN_MINB
#define DDA_P3D_GEN_MINB 1
#endif
template <typename R, int LX, int NC>
constexpr int p3_min_blocks() {
  if (NC > 0 && sizeof(R) == 8 && LX >= 64 && (LX & (LX - 1)) == 0) return DDA_P3D_MINB;
  if (sizeof(R) == 8) return DDA_P3D_GEN_MINB;
  if (sizeof(R) == 4 && mixed_radix_mid<NC>()) return DDA_P3MR_MINB;
  if (sizeof(R) == 4 && NC == 0) return DDA_GEN_P3_MINB;
#ifdef DDA_P3_MINB
  return (NC > 0 && sizeof(R) == 4 && LX >= 64 && (LX & (LX - 1)) == 0) ? DDA_P3_MINB : 1;
#else
  return (NC > 0 && sizeof(R) == 4 && LX >= 64 && (LX & (LX - 1)) == 0) ? 3 : 1;
#endif
}
template <typename R, int LX, int V, int NC>
__global__ void __launch_bounds__(kMvMaxThreads, p3_min_blocks<R, LX, NC>()) k_mv_pass3s(Geo g, const typename CT<R>::T* __restrict__ tw,
                                                             InstState* st, const int* act, int cond, int tz_,
                                                             int ntz_, R gscale, int op) {
  grid_dep_begin();
  typedef typename CT<R>::T C;
  typedef P3Shape<R, LX, V> SH;
  typedef typename SH::P P;
  typedef RevPlan<P> Q;
  constexpr bool CUBE = NC > 0;
  static_assert(!CUBE || LX == 2 * NC, "cubic kernels need L = 2n");
  constexpr int TZC = CUBE ? cmin_i(p3s_tiles<R, LX, SH::T>(), LX) : 1;
  constexpr int NTZC = (LX + TZC - 1) / TZC;
  constexpr bool ZH = CUBE && P::r[0] % 2 == 0;
  constexpr bool DH = CUBE && half_store_ok<Q>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  InstState& S = st[inst_of(act)];
  if (!cond_ok(S, cond)) return;
  C* __restrict__ t2 = (C*)S.t2;
  // op 0: the interaction octant; op 1: the preconditioner octant
  const C* __restrict__ gh = (const C*)(op ? S.pghat : S.ghat);
  const int tz = CUBE ? TZC : tz_;
  const int ntz = CUBE ? NTZC : ntz_;
  const int Ly = CUBE ? LX : g.Ly, Lz = CUBE ? LX : g.Lz;
  const int hy = CUBE ? LX / 2 + 1 : g.hy, hz = CUBE ? LX / 2 + 1 : g.hz;
  const int H = CUBE ? (LX / 2 + 1) * (LX / 2 + 1) * (LX / 2 + 1) : g.hx * g.hy * g.hz;
  const int nx = CUBE ? NC : g.nx;
  const int W = 3 * tz;
  const int w = threadIdx.x % W, t = threadIdx.x / W;
  assume_t<SH::T>(t);                   // blockDim.x = W T (make_pass_cfg)
  const int p = blockIdx.x / ntz, kzt = blockIdx.x - p * ntz;
  const int ky = pencil_ky(p, Ly);
  const int kz0 = kzt * tz;
  const int tzn = (CUBE && LX % TZC == 0) ? tz : min(tz, Lz - kz0);
  const bool ok = w < 3 * tzn;
  const long long rs = (long long)Ly * Lz * 3;
  C* col = t2 + ((long long)ky * Lz + kz0) * 3 + w;
  C* sw = s + w;
  const auto twk = pass_tw(tw, s + W * SH::LP, LX);
  if constexpr (CUBE && (3 * TZC * (int)sizeof(C)) % 16 == 0 && TZC % 2 == 0) {
    // the input rows of the tile g.pf3 CTAs ahead, into L2
    const int f = (int)blockIdx.x + g.pf3;
    if (g.pf3 > 0 && f < (int)gridDim.x) {
      const int fp = f / NTZC, fk = f - fp * NTZC;
      prefetch_rows(t2 + ((long long)pencil_ky(fp, Ly) * Lz + fk * TZC) * 3, rs, nx, 3 * TZC * (int)sizeof(C));
    }
  }
  auto ld = [&](int, int pos) -> C { return (ok && (ZH || pos < nx)) ? __ldcg(col + pos * rs) : czero<C>(); };
  auto sm = [&](int, int pp) -> C& { return sw[pp * W]; };
  C a[P::E];
  rload<P, 1, ZH>(a, t, ld);
  rstage<P, 0, ZH>(a, t, twk);
  rrest<P, 1, 0>(a, t, sm, twk);
  constexpr int RL = P::r[P::S - 1];
#pragma unroll
  for (int b = 0; b < P::E / RL; ++b)
#pragma unroll
    for (int q = 0; q < RL; ++q) sm(0, ppad(rout_pos<P, P::S - 1>(t, b, q))) = a[b * RL + q];
  __syncthreads();
  {
    // thread -> (kzl fastest, mirror pair j): pair j holds kx = j and
    // kx = LX - j, which read the same octant row (j = 0 and j = LX/2 stand
    // alone), so each octant entry is loaded once for two points
    const int kzl = threadIdx.x % tz, js = blockDim.x / tz;
    if (kzl < tzn) {
      const int kz = kz0 + kzl;
      const bool fy = ky > Ly / 2, fz = kz > Lz / 2;
      const int my = fy ? Ly - ky : ky;
      const int mz = fz ? Lz - kz : kz;
      // entry scales at kx <= LX/2 (mirror signs of y and z, tensor scale)
      const R sd = gscale;
      const R sxy = fy ? -gscale : gscale, sxz = fz ? -gscale : gscale;
      const R syz = (fy != fz) ? -gscale : gscale;
      const C* __restrict__ q0 = gh + my * hz + mz;
      for (int j = threadIdx.x / tz; j <= LX / 2; j += js) {
        const C* q = q0 + j * (hy * hz);
        const C gxx = cscale(__ldg(q), sd), gxy = cscale(__ldg(q + H), sxy), gxz = cscale(__ldg(q + 2 * H), sxz);
        const C gyy = cscale(__ldg(q + 3 * H), sd), gyz = cscale(__ldg(q + 4 * H), syz);
        const C gzz = cscale(__ldg(q + 5 * H), sd);
        {
          C* v = s + ppad(j) * W + 3 * kzl;
          const C a0 = v[0], a1 = v[1], a2 = v[2];
          v[0] = cadd(cadd(cmul(gxx, a0), cmul(gxy, a1)), cmul(gxz, a2));
          v[1] = cadd(cadd(cmul(gxy, a0), cmul(gyy, a1)), cmul(gyz, a2));
          v[2] = cadd(cadd(cmul(gxz, a0), cmul(gyz, a1)), cmul(gzz, a2));
        }
        if (j > 0 && j < LX / 2) {
          // kx = LX - j: the x mirror flips the xy and xz entries
          C* v = s + ppad(LX - j) * W + 3 * kzl;
          const C a0 = v[0], a1 = v[1], a2 = v[2];
          v[0] = csub(csub(cmul(gxx, a0), cmul(gxy, a1)), cmul(gxz, a2));
          v[1] = cadd(csub(cmul(gyy, a1), cmul(gxy, a0)), cmul(gyz, a2));
          v[2] = cadd(csub(cmul(gyz, a1), cmul(gxz, a0)), cmul(gzz, a2));
        }
      }
    }
  }
  __syncthreads();
  // inverse half: fresh copies of the index and pointers keep the compiler
  // from carrying the forward half's address arithmetic across the kernel
  const int ti = opaque(t);
  assume_t<SH::T>(ti);
  C* colo = opaque_ptr(col);
  C* swo = opaque_ptr(sw);
  auto smo = [&](int, int pp) -> C& { return swo[pp * W]; };
  auto stf = [&](int, int pos, C v) { if (ok && (DH || pos < nx)) __stcg(colo + pos * rs, cswap(v)); };
  constexpr int R0 = Q::r[0];
#pragma unroll
  for (int b = 0; b < Q::E / R0; ++b)
#pragma unroll
    for (int m = 0; m < R0; ++m) a[b * R0 + m] = cswap(smo(0, ppad(rin_pos<Q, 0>(ti, b, m))));
  __syncthreads();
  rstage<Q, 0>(a, ti, twk);
  rrest<Q, 1, 0>(a, ti, smo, twk);
  rstore<Q, 1, DH>(a, ti, stf);
}

// ---------------------------------------------------------------------------
// pass 3 on packed pairs (complex64 cubic boxes): every thread transforms two
// columns of the tile at once -- column p and column p + W/2, one per lane of
// the cp2 pair (cpair.cuh) -- so each butterfly add, twiddle product and
// exchange store / load covers two transforms in one packed FP32x2 or 128-bit
// shared-memory instruction.  Columns p and p + W/2 are the same component of
// the kz points kzl and kzl + TZ/2 (w = 3 kzl + c), so the tensor product
// also runs on pairs: the cp2 slot p = 3 kzl + c holds component c of both
// points, and each 3x3 product updates two points.  Tile shape, mirror rule
// and octant reads are those of k_mv_pass3s; results agree with it to
// complex64 rounding (the packed rotations round like the scalar ones, the
// grouping of a few sums differs).
// ---------------------------------------------------------------------------
template <int LX, int TZ>
struct P3Pair {
  typedef typename PlanFor<LX, float>::type P;
  static constexpr int W = 3 * TZ, WP = W / 2, T = P::T, TH = WP * T;
  static constexpr int LP = ppad_len(LX);
  static constexpr size_t smem = (size_t)LP * WP * sizeof(cp2) + (smem_tw(8) ? LX * sizeof(float2) : 0);
  static_assert(TZ % 2 == 0 && LX % TZ == 0, "pairs of kz columns");
  static_assert(TH <= 1024, "threads per CTA");
};

// A 3x3 entry of the octant for two points, scaled: (re, im, -re, -im).
struct G2 {
  float2 re, im, nre, nim;
};
__device__ __forceinline__ G2 g2_load(const float2* qa, const float2* qb, float2 s) {
  const cp2 g = cpack(__ldg(qa), __ldg(qb));
  G2 o;
  o.re = f2mul(g.re, s);
  o.im = f2mul(g.im, s);
  o.nre = f2mul(g.re, make_float2(-s.x, -s.y));
  o.nim = f2mul(g.im, make_float2(-s.x, -s.y));
  return o;
}
// sum of three products g_k a_k on pairs; NEG_k takes -g_k
template <bool N0, bool N1, bool N2>
__device__ __forceinline__ cp2 g2_dot3(const G2& g0, cp2 a0, const G2& g1, cp2 a1, const G2& g2, cp2 a2) {
  const float2 r0 = N0 ? g0.nre : g0.re, i0 = N0 ? g0.nim : g0.im, m0 = N0 ? g0.im : g0.nim;
  const float2 r1 = N1 ? g1.nre : g1.re, i1 = N1 ? g1.nim : g1.im, m1 = N1 ? g1.im : g1.nim;
  const float2 r2 = N2 ? g2.nre : g2.re, i2 = N2 ? g2.nim : g2.im, m2 = N2 ? g2.im : g2.nim;
  cp2 o;
  // re = sum r a.re - i a.im ; im = sum r a.im + i a.re   (m = -i)
  o.re = f2fma(r0, a0.re, f2fma(m0, a0.im, f2fma(r1, a1.re, f2fma(m1, a1.im, f2fma(r2, a2.re, f2mul(m2, a2.im))))));
  o.im = f2fma(r0, a0.im, f2fma(i0, a0.re, f2fma(r1, a1.im, f2fma(i1, a1.re, f2fma(r2, a2.im, f2mul(i2, a2.re))))));
  return o;
}

template <int LX, int NC, int TZ, int MINB>
__global__ void __launch_bounds__(P3Pair<LX, TZ>::TH, MINB)
    k_mv_pass3x(Geo g, const float2* __restrict__ tw, InstState* st, const int* act, int cond, int tz_, int ntz_,
                float gscale, int op) {
  grid_dep_begin();
  typedef float2 C;
  typedef P3Pair<LX, TZ> PS;
  typedef typename PS::P P;
  typedef RevPlan<P> Q;
  static_assert(NC == LX / 2, "cubic boxes on the (2n)^3 grid");
  constexpr bool ZH = P::r[0] % 2 == 0;
  constexpr bool DH = half_store_ok<Q>();
  static_assert(ZH && DH, "zero-half loads and half stores");
  constexpr int WP = PS::WP, NTZ = LX / TZ;
  constexpr long long rs = (long long)LX * LX * 3;
  constexpr int hy = LX / 2 + 1, hz = LX / 2 + 1, H = hy * hy * hz;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cp2* s = reinterpret_cast<cp2*>(smem_raw);
  InstState& S = st[inst_of(act)];
  if (!cond_ok(S, cond)) return;
  C* __restrict__ t2 = (C*)S.t2;
  const C* __restrict__ gh = (const C*)(op ? S.pghat : S.ghat);
  const int p = threadIdx.x % WP, t = threadIdx.x / WP;
  const int pen = blockIdx.x / NTZ, kzt = blockIdx.x - pen * NTZ;
  const int ky = pencil_ky(pen, LX);
  const int kz0 = kzt * TZ;
  C* col = t2 + ((long long)ky * LX + kz0) * 3;
  cp2* sw = s + p;
  const auto twk = pass_tw(tw, s + PS::LP * WP, LX);
  auto ld = [&](int, int pos) -> cp2 {
    const C* r = col + pos * rs;
    return cpack(__ldcg(r + p), __ldcg(r + p + WP));
  };
  auto sm = [&](int, int pp) -> cp2& { return sw[pp * WP]; };
  cp2 a[P::E];
  rload<P, 1, ZH>(a, t, ld);
  rstage<P, 0, ZH>(a, t, twk);
  rrest<P, 1, 0>(a, t, sm, twk);
  constexpr int RL = P::r[P::S - 1];
#pragma unroll
  for (int b = 0; b < P::E / RL; ++b)
#pragma unroll
    for (int q = 0; q < RL; ++q) sm(0, ppad(rout_pos<P, P::S - 1>(t, b, q))) = a[b * RL + q];
  __syncthreads();
  {
    // thread -> (kzl in [0, TZ/2), mirror pair j); lanes: kz0 + kzl, kz0 + kzl + TZ/2
    constexpr int TH2 = TZ / 2;
    constexpr int js = PS::TH / TH2;
    const int kzl = threadIdx.x % TH2;
    const int kza = kz0 + kzl, kzb = kza + TH2;
    const bool fy = ky > LX / 2, fza = kza > LX / 2, fzb = kzb > LX / 2;
    const int my = fy ? LX - ky : ky;
    const int mza = fza ? LX - kza : kza, mzb = fzb ? LX - kzb : kzb;
    const float2 sd = f2(gscale);
    const float2 sxy = f2(fy ? -gscale : gscale);
    const float2 sxz = make_float2(fza ? -gscale : gscale, fzb ? -gscale : gscale);
    const float2 syz = make_float2((fy != fza) ? -gscale : gscale, (fy != fzb) ? -gscale : gscale);
    const C* __restrict__ qa0 = gh + my * hz + mza;
    const C* __restrict__ qb0 = gh + my * hz + mzb;
    for (int j = threadIdx.x / TH2; j <= LX / 2; j += js) {
      const C* qa = qa0 + j * (hy * hz);
      const C* qb = qb0 + j * (hy * hz);
      const G2 gxx = g2_load(qa, qb, sd), gxy = g2_load(qa + H, qb + H, sxy);
      const G2 gxz = g2_load(qa + 2 * H, qb + 2 * H, sxz), gyy = g2_load(qa + 3 * H, qb + 3 * H, sd);
      const G2 gyz = g2_load(qa + 4 * H, qb + 4 * H, syz), gzz = g2_load(qa + 5 * H, qb + 5 * H, sd);
      {
        cp2* v = s + ppad(j) * WP + 3 * kzl;
        const cp2 a0 = v[0], a1 = v[1], a2 = v[2];
        v[0] = g2_dot3<false, false, false>(gxx, a0, gxy, a1, gxz, a2);
        v[1] = g2_dot3<false, false, false>(gxy, a0, gyy, a1, gyz, a2);
        v[2] = g2_dot3<false, false, false>(gxz, a0, gyz, a1, gzz, a2);
      }
      if (j > 0 && j < LX / 2) {
        // kx = LX - j: the x mirror flips the xy and xz entries
        cp2* v = s + ppad(LX - j) * WP + 3 * kzl;
        const cp2 a0 = v[0], a1 = v[1], a2 = v[2];
        v[0] = g2_dot3<false, true, true>(gxx, a0, gxy, a1, gxz, a2);
        v[1] = g2_dot3<true, false, false>(gxy, a0, gyy, a1, gyz, a2);
        v[2] = g2_dot3<true, false, false>(gxz, a0, gyz, a1, gzz, a2);
      }
    }
  }
  __syncthreads();
  const int ti = opaque(t);
  C* colo = opaque_ptr(col);
  cp2* swo = opaque_ptr(sw);
  auto smo = [&](int, int pp) -> cp2& { return swo[pp * WP]; };
  auto stf = [&](int, int pos, cp2 v) {
    v = cswap(v);
    C* r = colo + pos * rs;
    __stcg(r + p, clo(v));
    __stcg(r + p + WP, chi(v));
  };
  constexpr int R0 = Q::r[0];
#pragma unroll
  for (int b = 0; b < Q::E / R0; ++b)
#pragma unroll
    for (int m = 0; m < R0; ++m) a[b * R0 + m] = cswap(smo(0, ppad(rin_pos<Q, 0>(ti, b, m))));
  __syncthreads();
  rstage<Q, 0>(a, ti, twk);
  rrest<Q, 1, 0>(a, ti, smo, twk);
  rstore<Q, 1, DH>(a, ti, stf);
}

// ---------------------------------------------------------------------------
// pass 3, staged and persistent (cubic boxes, one component per thread):
// the same arithmetic as k_mv_pass3s, but every CTA loops over tiles (one
// pencil row ky x TZ kz columns) and its input tile -- the NC kept x rows of
// 3 TZ complex each, contiguous in T2 -- arrives in shared memory through
// bulk async copies issued one tile ahead, so the transform of tile i runs
// while tile i+1 is in flight.  Two input buffers alternate; the exchange /
// tensor area is that of k_mv_pass3s.  Outputs go straight to T2 from the
// inverse transform's last stage (rows x < NC).
// ---------------------------------------------------------------------------
template <typename R, int LX, int V, int TZ>
struct P3Pipe {
  typedef typename CT<R>::T C;
  typedef P3Shape<R, LX, V> SH;
  static constexpr int NC = LX / 2;              // kept x rows (box edge)
  static constexpr int W = 3 * TZ;               // complex per row segment
  static constexpr int TH = W * SH::T;           // threads
  static constexpr int ROWB = W * (int)sizeof(C);
  static constexpr size_t XS = (size_t)W * SH::LP * sizeof(C);     // exchange / tensor area
  static constexpr size_t IB = (size_t)NC * W * sizeof(C);         // one input buffer
  static constexpr size_t smem = XS + 2 * IB + 16;                 // + two mbarriers
  static_assert(ROWB % 16 == 0, "bulk copies move multiples of 16 bytes");
  static_assert(XS % 16 == 0 && IB % 16 == 0, "16-byte aligned buffers");
  static_assert(TH <= 1024, "threads per CTA");
};

template <typename R, int LX, int V, int NC, int TZ, int MINB>
__global__ void __launch_bounds__(P3Pipe<R, LX, V, TZ>::TH, MINB)
    k_mv_pass3p(Geo g, const typename CT<R>::T* __restrict__ tw, InstState* st, const int* act, int cond, int tz_,
                int ntz_, R gscale, int op) {
  grid_dep_begin();
  typedef typename CT<R>::T C;
  typedef P3Pipe<R, LX, V, TZ> PP;
  typedef typename PP::SH::P P;
  typedef RevPlan<P> Q;
  static_assert(NC == LX / 2 && NC > 0, "cubic boxes on the (2n)^3 grid");
  static_assert(LX % TZ == 0, "whole kz tiles");
  constexpr bool ZH = P::r[0] % 2 == 0;
  constexpr bool DH = half_store_ok<Q>();
  static_assert(ZH && DH, "zero-half loads and half stores");
  constexpr int W = PP::W, NTZ = LX / TZ, NT = LX * NTZ;
  constexpr long long rs = (long long)LX * LX * 3;          // x-row stride of T2
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  // input buffer b at smem_raw + XS + b IB
  auto ibuf = [&](int b) -> C* { return reinterpret_cast<C*>(smem_raw + PP::XS + (size_t)b * PP::IB); };
  uint64_t* mb = reinterpret_cast<uint64_t*>(smem_raw + PP::XS + 2 * PP::IB);
  InstState& S = st[inst_of(act)];
  if (!cond_ok(S, cond)) return;
  C* __restrict__ t2 = (C*)S.t2;
  const C* __restrict__ gh = (const C*)(op ? S.pghat : S.ghat);
  constexpr int H = (LX / 2 + 1) * (LX / 2 + 1) * (LX / 2 + 1);
  constexpr int hy = LX / 2 + 1, hz = LX / 2 + 1;
  const int w = threadIdx.x % W, t = threadIdx.x / W;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    mbar_init(&mb[0], 1);
    mbar_init(&mb[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  // bulk copies of tile `tile` into buffer b by warp 0 (one row per copy)
  auto issue = [&](int tile, int b) {
    const int ky = pencil_ky(tile / NTZ, LX), kz0 = (tile % NTZ) * TZ;
    if (lane == 0) mbar_arrive_expect_tx(&mb[b], (uint32_t)(NC * PP::ROWB));
    __syncwarp();
    const C* src = t2 + ((long long)ky * LX + kz0) * 3;
    C* dst = ibuf(b);
    for (int pos = lane; pos < NC; pos += 32) bulk_g2s(dst + pos * W, src + pos * rs, PP::ROWB, &mb[b]);
  };
  int tile = blockIdx.x;
  if (warp == 0 && tile < NT) issue(tile, 0);
  for (int it = 0; tile < NT; ++it, tile += gridDim.x) {
    const int b = it & 1;
    const int next = tile + gridDim.x;
    // the other buffer was last read by tile it-1, which has passed several
    // CTA barriers since
    if (warp == 0 && next < NT) issue(next, b ^ 1);
    const bool ok_wait = mbar_wait_bounded(&mb[b], (uint32_t)((it >> 1) & 1), 2000000000LL);
    if (__syncthreads_or(!ok_wait)) {
      // give up on this instance: flag it, let the other buffer's copies
      // (if any) land before the CTA's shared memory goes away
      if (threadIdx.x == 0) {
        atomicExch(&S.fault, 1);
        if (next < NT) mbar_wait_bounded(&mb[b ^ 1], (uint32_t)(((it + 1) >> 1) & 1), 2000000000LL);
      }
      return;
    }
    const int ky = pencil_ky(tile / NTZ, LX), kz0 = (tile % NTZ) * TZ;
    const C* in = ibuf(b) + w;
    C* col = t2 + ((long long)ky * LX + kz0) * 3 + w;
    C* sw = s + w;
    auto ld = [&](int, int pos) -> C { return in[pos * W]; };
    auto sm = [&](int, int pp) -> C& { return sw[pp * W]; };
    C a[P::E];
    rload<P, 1, ZH>(a, t, ld);
    rstage<P, 0, ZH>(a, t, tw);
    rrest<P, 1, 0>(a, t, sm, tw);
    constexpr int RL = P::r[P::S - 1];
#pragma unroll
    for (int bb = 0; bb < P::E / RL; ++bb)
#pragma unroll
      for (int q = 0; q < RL; ++q) sm(0, ppad(rout_pos<P, P::S - 1>(t, bb, q))) = a[bb * RL + q];
    __syncthreads();
    {
      // thread -> (kzl fastest, mirror pair j), as in k_mv_pass3s
      const int kzl = threadIdx.x % TZ;
      constexpr int js = PP::TH / TZ;
      const int kz = kz0 + kzl;
      const bool fy = ky > LX / 2, fz = kz > LX / 2;
      const int my = fy ? LX - ky : ky;
      const int mz = fz ? LX - kz : kz;
      const R sd = gscale;
      const R sxy = fy ? -gscale : gscale, sxz = fz ? -gscale : gscale;
      const R syz = (fy != fz) ? -gscale : gscale;
      const C* __restrict__ q0 = gh + my * hz + mz;
      for (int j = threadIdx.x / TZ; j <= LX / 2; j += js) {
        const C* q = q0 + j * (hy * hz);
        const C gxx = cscale(__ldg(q), sd), gxy = cscale(__ldg(q + H), sxy), gxz = cscale(__ldg(q + 2 * H), sxz);
        const C gyy = cscale(__ldg(q + 3 * H), sd), gyz = cscale(__ldg(q + 4 * H), syz);
        const C gzz = cscale(__ldg(q + 5 * H), sd);
        {
          C* v = s + ppad(j) * W + 3 * kzl;
          const C a0 = v[0], a1 = v[1], a2 = v[2];
          v[0] = cadd(cadd(cmul(gxx, a0), cmul(gxy, a1)), cmul(gxz, a2));
          v[1] = cadd(cadd(cmul(gxy, a0), cmul(gyy, a1)), cmul(gyz, a2));
          v[2] = cadd(cadd(cmul(gxz, a0), cmul(gyz, a1)), cmul(gzz, a2));
        }
        if (j > 0 && j < LX / 2) {
          C* v = s + ppad(LX - j) * W + 3 * kzl;
          const C a0 = v[0], a1 = v[1], a2 = v[2];
          v[0] = csub(csub(cmul(gxx, a0), cmul(gxy, a1)), cmul(gxz, a2));
          v[1] = cadd(csub(cmul(gyy, a1), cmul(gxy, a0)), cmul(gyz, a2));
          v[2] = cadd(csub(cmul(gyz, a1), cmul(gxz, a0)), cmul(gzz, a2));
        }
      }
    }
    __syncthreads();
    const int ti = opaque(t);
    C* colo = opaque_ptr(col);
    C* swo = opaque_ptr(sw);
    auto smo = [&](int, int pp) -> C& { return swo[pp * W]; };
    auto stf = [&](int, int pos, C v) { __stcg(colo + pos * rs, cswap(v)); };
    constexpr int R0 = Q::r[0];
#pragma unroll
    for (int bb = 0; bb < Q::E / R0; ++bb)
#pragma unroll
      for (int m = 0; m < R0; ++m) a[bb * R0 + m] = cswap(smo(0, ppad(rin_pos<Q, 0>(ti, bb, m))));
    __syncthreads();
    rstage<Q, 0>(a, ti, tw);
    rrest<Q, 1, 0>(a, ti, smo, tw);
    rstore<Q, 1, DH>(a, ti, stf);
  }
}

// ---------------------------------------------------------------------------
// passes 2 / 4 on packed pairs (complex64 cubic boxes): as k_mv_pass_y, with
// each thread transforming columns p and p + W/2 of the tile in the two
// lanes of a cp2 (FP32x2 butterflies, 128-bit exchanges).
// ---------------------------------------------------------------------------
template <int LY, int TZ>
struct PYPair {
  typedef typename PlanFor<LY, float>::type P;
  static constexpr int W = 3 * TZ, WP = W / 2, T = P::T, TH = WP * T;
  static constexpr int LP = ppad_len(LY);
  static constexpr size_t smem = (size_t)LP * WP * sizeof(cp2) + (smem_tw(8) ? LY * sizeof(float2) : 0);
  static_assert(TZ % 2 == 0 && LY % TZ == 0, "pairs of kz columns");
};

template <bool INV, int LY, int NC, int TZ, int MINB>
__global__ void __launch_bounds__(PYPair<LY, TZ>::TH, MINB)
    k_mv_pass_yx(Geo g, const float2* __restrict__ tw, InstState* st, const int* act, int cond, int tz_,
                 int ntz_) {
  grid_dep_begin();
  typedef float2 C;
  typedef PYPair<LY, TZ> PS;
  typedef typename PS::P P;
  static_assert(NC == LY / 2, "cubic boxes on the (2n)^3 grid");
  constexpr bool ZH = !INV && P::r[0] % 2 == 0;
  constexpr bool DH = INV && half_store_ok<P>();
  static_assert(INV ? DH : ZH, "zero-half loads / half stores");
  constexpr int WP = PS::WP, NTZ = LY / TZ;
  constexpr long long rs = (long long)LY * 3;                 // row stride of T1/T2 (Lz = LY)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cp2* s = reinterpret_cast<cp2*>(smem_raw);
  InstState& S = st[inst_of(act)];
  if (!cond_ok(S, cond)) return;
  C* __restrict__ t1 = (C*)S.t1;
  C* __restrict__ t2 = (C*)S.t2;
  const int p = threadIdx.x % WP, t = threadIdx.x / WP;
  const int ix = blockIdx.x / NTZ, kzt = blockIdx.x - ix * NTZ;
  const int kz0 = kzt * TZ;
  const C* src = (INV ? t2 + (long long)ix * LY * rs : t1 + (long long)ix * NC * rs) + kz0 * 3 + p;
  C* dst = (INV ? t1 + (long long)ix * NC * rs : t2 + (long long)ix * LY * rs) + kz0 * 3 + p;
  cp2* sw = s + p;
  const auto twk = pass_tw(tw, s + PS::LP * WP, LY);
  auto ld = [&](int, int pos) -> cp2 { return cpack(__ldcg(src + pos * rs), __ldcg(src + pos * rs + WP)); };
  auto sm = [&](int, int pp) -> cp2& { return sw[pp * WP]; };
  auto stf = [&](int, int pos, cp2 v) {
    __stcg(dst + pos * rs, clo(v));
    __stcg(dst + pos * rs + WP, chi(v));
  };
  cp2 a[P::E];
  rfft<P, 1, INV, ZH, DH>(a, t, ld, sm, stf, twk);
}

// ---------------------------------------------------------------------------
// passes 1 / 5 on packed pairs (complex64 cubic boxes, no Krylov step fused
// into the pass): as k_mv_pass1 / k_mv_pass5, with each thread transforming
// component c of lines l and l + NL/2 of the tile in the two lanes of a cp2.
// Pass 5 runs its combine per lane, as the scalar kernel does.
// ---------------------------------------------------------------------------
template <int LZ>
struct PZPair {
  typedef typename PlanFor<LZ, float>::type P;
  static constexpr int NC = LZ / 2;
  static constexpr int NL = cmin_i(mv_tiles<float, P::T>(), NC * NC);   // lines per CTA
  static constexpr int NLP = NL / 2, T = P::T, TH = 3 * T * NLP;
  static constexpr int LP = ppad_len(LZ);
  static constexpr size_t smem = (size_t)NLP * 3 * LP * sizeof(cp2) + (smem_tw(8) ? LZ * sizeof(float2) : 0);
  static_assert(NL % 2 == 0 && (NC * NC) % NL == 0, "pairs of lines");
};

template <int LZ, int MINB>
__global__ void __launch_bounds__(PZPair<LZ>::TH, MINB)
    k_mv_pass1x(Geo g, const float2* __restrict__ tw, InstState* st, const int* act, int in_id, int cond, int nl_,
                int pre) {
  grid_dep_begin();
  typedef float2 C;
  typedef PZPair<LZ> PS;
  typedef typename PS::P P;
  constexpr int NC = PS::NC, NL = PS::NL, NLP = PS::NLP;
  constexpr bool ZH = P::r[0] % 2 == 0;
  static_assert(ZH, "zero-half loads");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cp2* s = reinterpret_cast<cp2*>(smem_raw);
  InstState& S = st[inst_of(act)];
  if (!cond_ok(S, cond)) return;
  const C* __restrict__ x = (const C*)S.vec[in_id];
  C* __restrict__ t1 = (C*)S.t1;
  const int c = threadIdx.x % 3, rest = threadIdx.x / 3;
  const int t = rest % PS::T, lp = rest / PS::T;
  const long long la = (long long)blockIdx.x * NL + lp, lb = la + NLP;
  const int* __restrict__ cid = S.cidx;
  auto eidx = [&](long long line, int pos) -> long long {
    if (!cid) return (line * NC + pos) * 3 + c;
    const int k = cid[line * NC + pos];
    return k < 0 ? -1 : 3LL * k + c;
  };
  auto ld = [&](int, int pos) -> cp2 {
    const long long ia = eidx(la, pos), ib = eidx(lb, pos);
    return cpack(ia < 0 ? czero<C>() : __ldcg(x + ia), ib < 0 ? czero<C>() : __ldcg(x + ib));
  };
  const auto twk = pass_tw(tw, s + NLP * 3 * PS::LP, LZ);
  cp2* sl = s + lp * 3 * PS::LP + c;
  auto sm = [&](int, int pp) -> cp2& { return sl[pp * 3]; };
  C* ta = t1 + la * (long long)LZ * 3 + c;
  C* tb = t1 + lb * (long long)LZ * 3 + c;
  auto stf = [&](int, int pos, cp2 v) {
    __stcg(ta + pos * 3, clo(v));
    __stcg(tb + pos * 3, chi(v));
  };
  cp2 a[P::E];
  rfft<P, 1, false, ZH, false>(a, t, ld, sm, stf, twk);
}

template <int LZ, int MINB>
__global__ void __launch_bounds__(PZPair<LZ>::TH, MINB)
    k_mv_pass5x(Geo g, const float2* __restrict__ tw, InstState* st, const int* act, int in_id, int out_id,
                int mode, int cond, int nl_, int post, double* red, unsigned* cnt) {
  grid_dep_begin();
  typedef float2 C;
  typedef PZPair<LZ> PS;
  typedef typename PS::P P;
  constexpr int NC = PS::NC, NL = PS::NL, NLP = PS::NLP;
  constexpr bool DH = half_store_ok<P>();
  static_assert(DH, "half stores");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cp2* s = reinterpret_cast<cp2*>(smem_raw);
  InstState& S = st[inst_of(act)];
  if (!cond_ok(S, cond)) return;
  const C* __restrict__ t1 = (const C*)S.t1;
  const int c = threadIdx.x % 3, rest = threadIdx.x / 3;
  const int t = rest % PS::T, lp = rest / PS::T;
  const long long la = (long long)blockIdx.x * NL + lp, lb = la + NLP;
  const C* tla = t1 + la * (long long)LZ * 3 + c;
  const C* tlb = t1 + lb * (long long)LZ * 3 + c;
  const C* __restrict__ xg = (const C*)S.vec[in_id];
  C* __restrict__ yg = (C*)S.vec[out_id];
  const C* __restrict__ iag = (const C*)S.inva;
  const C* __restrict__ bg = (mode == MV_RESIDUAL) ? (const C*)S.vec[V_B] : nullptr;
  const int* __restrict__ cid = S.cidx;
  auto ld = [&](int, int pos) -> cp2 { return cpack(__ldcg(tla + pos * 3), __ldcg(tlb + pos * 3)); };
  const auto twk = pass_tw(tw, s + NLP * 3 * PS::LP, LZ);
  cp2* sl = s + lp * 3 * PS::LP + c;
  auto sm = [&](int, int pp) -> cp2& { return sl[pp * 3]; };
  // the combine of pass 5 for one element of one line
  auto comb = [&](long long line, int pos, C v) {
    const long long site = line * NC + pos;
    long long e = site * 3 + c;
    if (cid) {
      const int k = cid[site];
      if (k < 0) return;
      e = 3LL * k + c;
    }
    C r;
    if (mode == MV_CONV) {
      r = v;
    } else {
      const C a_ = __ldg(iag + site);
      const bool msk = (a_.x != 0.f) || (a_.y != 0.f);
      if (!msk) v = czero<C>();
      if (mode == MV_CONV_MASKED) {
        r = v;
      } else {
        r = csub(cmul(a_, __ldcg(xg + e)), v);
        if (mode == MV_RESIDUAL) r = csub(__ldcg(bg + e), r);
      }
    }
    __stcg(yg + e, r);
  };
  auto stf = [&](int, int pos, cp2 v) {
    comb(la, pos, clo(v));
    comb(lb, pos, chi(v));
  };
  cp2 a[P::E];
  rfft<P, 1, true, false, DH>(a, t, ld, sm, stf, twk);
}

// ---------------------------------------------------------------------------
// pass 5: inverse z on nl lines, keep z < nz, fused combine:
//   MV_AX           y = ia*x - mask*conv        (interaction_mult)
//   MV_RESIDUAL     y = b - (ia*x - mask*conv)  (b already masked)
//   MV_CONV         y = conv                    (E_field_solver)
//   MV_CONV_MASKED  y = mask*conv               (fft_matvec)
// mask = (inv_alpha != 0), the reference's alpha != 0 (ddaforgit.py:1108).
// In the cubic kernels of power-of-two length (64^3 boxes and up) the
// combine's operands are loaded DDA_P5_EB outputs at a time, before those
// outputs' stores.  B200, 128^3 complex64 matvec: 0.560 ms one at a time,
// 0.538 ms by two, 0.544 by four, 0.554 by eight (more registers, spills
// under the z passes' cap).  Complex128 by two under an 80-register cap:
// 128^3 1.259 -> 1.225 ms, 64^3 0.1485 -> 0.1444 ms (uncapped it took 102
// registers and was slower, 1.283 ms).  The other kernels load at each
// output (batched, they take 10-30 more registers).
// ---------------------------------------------------------------------------
#ifndef DDA_P5_EB
#define DDA_P5_EB 2
#endif
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
// ia x - v with a fixed rounding (explicit fused multiply-adds), so every
// kernel that forms the combine gives the same bits
template <class C> __device__ __forceinline__ C combine_ax(C ia, C x, C v) {
  C r;
  r.x = fma_rn(ia.x, x.x, fma_rn(-ia.y, x.y, -v.x));
  r.y = fma_rn(ia.x, x.y, fma_rn(ia.y, x.x, -v.y));
  return r;
}

// The combine of pass 5 on one thread's inverse-z outputs: a[] holds the
// last stage of plan P (swapped: the inverse runs as swap(FFT(swap(.)))),
// thread ti; outputs at positions >= nz (or all beyond L/2 with DH) and
// empty sites of occupied-site vectors are not stored.  The operands of a
// batch of EB outputs (inv_alpha, x) are loaded before the batch's first
// store: a cache-hinted store is a compiler memory barrier and the hinted
// loads keep their order, so loads written between the stores would each
// wait for the store before them, one memory latency per output.
// post(e, r) runs after the store of element e (fused dot products).
template <class P, bool DH, int EB0, typename R, class C, class POST>
__device__ __forceinline__ void mv_combine_out(const C* a, int ti, bool ok, int nz, long long site0, int c,
                                               const int* __restrict__ cid, const C* __restrict__ iag,
                                               const C* __restrict__ xg, const C* __restrict__ bg,
                                               C* __restrict__ yg, int mode, const POST& post) {
  constexpr int RL = P::r[P::S - 1];
  constexpr int NQ = DH ? RL / 2 : RL;
  constexpr int NB = P::E / RL;
  constexpr int K = NQ * NB;
  constexpr int EB = K < EB0 ? K : EB0;
  const bool need_ia = mode != MV_CONV;
  const bool need_x = mode == MV_AX || mode == MV_RESIDUAL;
#pragma unroll
  for (int k0 = 0; k0 < K; k0 += EB) {
    int ee[EB];             // element index in the instance's vectors (< 2^31: n^3 <= 512^3)
    C iav[EB], xv[EB];
#pragma unroll
    for (int j = 0; j < EB; ++j) {
      const int q = (k0 + j) / NB, b = (k0 + j) % NB;
      const int pos = rout_pos<P, P::S - 1>(ti, b, q);
      int e = -1;
      if (k0 + j < K && ok && (DH || pos < nz)) {
        e = (int)((site0 + pos) * 3 + c);
        if (cid) {
          const int kk = cid[pos];
          e = kk < 0 ? -1 : 3 * kk + c;
        }
      }
      ee[j] = e;
      iav[j] = (need_ia && e >= 0) ? __ldg(iag + pos) : czero<C>();   // shared by the 3 component lanes
      xv[j] = (need_x && e >= 0) ? __ldcg(xg + e) : czero<C>();
    }
#pragma unroll
    for (int j = 0; j < EB; ++j) {
      const int q = (k0 + j) / NB, b = (k0 + j) % NB;
      const int e = ee[j];
      if (e < 0) continue;
      C v = cswap(a[b * RL + q]);
      C r;
      if (mode == MV_CONV) {
        r = v;
      } else {
        const C ia = iav[j];
        if (ia.x == (R)0 && ia.y == (R)0) v = czero<C>();
        if (mode == MV_CONV_MASKED) {
          r = v;
        } else {
          r = combine_ax(ia, xv[j], v);
          if (mode == MV_RESIDUAL) r = csub(__ldcg(bg + e), r);
        }
      }
      __stcg(yg + e, r);
      post(e, r);
    }
  }
}
template <typename R, int LZ, int NC>
__global__ void __launch_bounds__(kMvMaxThreads)
    k_mv_pass5(Geo g, const typename CT<R>::T* __restrict__ tw, InstState* st, const int* act, int in_id,
               int out_id, int mode, int cond, int nl_, int post, double* red, unsigned* cnt)
#include "mv_pass5.inc"
template <typename R, int LZ, int NC>
__global__ void __launch_bounds__(kMvMaxThreads) __maxnreg__((z_regs<R, NC, DDA_Z_REGS>()))
    k_mv_pass5_cap(Geo g, const typename CT<R>::T* __restrict__ tw, InstState* st, const int* act, int in_id,
                   int out_id, int mode, int cond, int nl_, int post, double* red, unsigned* cnt)
#include "mv_pass5.inc"

// ---------------------------------------------------------------------------
// pass 5 of M (MV_CONV_MASKED) + pass 1 of A on the same z lines, for the
// product A M of a preconditioned solve whose preconditioner grid is the
// operator's (mv_pass51.inc).  Plain kernels (DDA_Z51_REGS sets a cap where
// the z passes have one): under the z passes' 56-register cap the L = 128
// kernel spilled 88 bytes; uncapped it takes 77 registers (L = 256: 56, no
// spill).  B200, preconditioned mixed solves: 64^3 x 2 RHS 108.3 solves/s
// with the separate passes, 110.4 capped, 111.9 uncapped; 128^3 x 2 RHS
// 14.72, 15.04, 15.06.
// ---------------------------------------------------------------------------
#ifndef DDA_Z51_REGS
#define DDA_Z51_REGS 0
#endif
template <typename R, int LZ, int NC>
__global__ void __launch_bounds__(kMvMaxThreads)
    k_mv_pass51(Geo g, const typename CT<R>::T* __restrict__ tw, InstState* st, const int* act, int mid_id,
                int cond, int nl_)
#include "mv_pass51.inc"
template <typename R, int LZ, int NC>
__global__ void __launch_bounds__(kMvMaxThreads) __maxnreg__((z_regs<R, NC, DDA_Z51_REGS>()))
    k_mv_pass51_cap(Geo g, const typename CT<R>::T* __restrict__ tw, InstState* st, const int* act, int mid_id,
                    int cond, int nl_)
#include "mv_pass51.inc"

// ---------------------------------------------------------------------------
// Passes 1+2 and 4+5 fused over a thread-block cluster (cubic boxes; the
// z/y transforms keep T1 on chip).  The CL CTAs of a cluster share one x
// slab ix:
//   forward  CTA r runs the z transforms of rows y in [r YR, (r+1) YR) and
//            writes each output kz into the shared memory of the CTA owning
//            kz's block (kz / KB) through distributed shared memory; after the
//            cluster barrier every CTA runs the y transforms of its KB kz
//            columns straight from that buffer into T2.
//   inverse  CTA r runs the y inverse transforms of its kz block from T2 and
//            writes each kept row y into the buffer of row owner y / YR;
//            after the barrier every CTA runs the z inverse transforms of its
//            YR rows with the pass-5 combine.
// T1 is neither written nor read and one launch replaces two.  Every value
// goes through the same arithmetic as in the separate passes, so the results
// are equal bit for bit.  All CTAs of a cluster share blockIdx.y (the
// instance), so the condition test exits whole clusters or none.
// ---------------------------------------------------------------------------
template <typename R, int L>
struct FusedZY {
  typedef MvShape<R, L> SH;
  typedef typename SH::P P;
  // CTAs per cluster (one x slab) and CTAs per SM: 4 and 2 for L = 128
  // (64^3), 8 and 1 for L = 256 (128^3; about 200 KB of shared memory each)
  static constexpr int CL = L >= 256 ? 8 : 4;
  static constexpr int MINB = L >= 256 ? 1 : 2;
  static constexpr int NC = L / 2;              // box edge
  static constexpr int YR = NC / CL;            // z lines (rows y) per CTA
  static constexpr int KB = L / CL;             // kz columns per CTA
  static constexpr int TH = 3 * SH::T * YR;     // z phase: thread = (c, t, row)
  static constexpr int TZ = YR;                 // y phase: kz columns per round, thread = (3 kz + c, t)
  static constexpr int ROUNDS = KB / TZ;
  static constexpr int BWF = 3 * KB;            // forward buffer: NC rows of KB kz x 3
  static constexpr int BWI = 3 * L + 1;         // inverse buffer: YR rows of L kz x 3 (+1 bank pad)
  static constexpr int XS = 3 * YR * SH::LP;    // exchange scratch of either phase
  typedef typename CT<R>::T C;
  static constexpr size_t smem_fwd = (size_t)(NC * BWF + XS) * sizeof(C);
  static constexpr size_t smem_inv = (size_t)(YR * BWI + XS) * sizeof(C);
  static_assert(NC % CL == 0 && KB % TZ == 0 && TH <= 1024, "cluster tiling");
  static_assert(P::r[0] % 2 == 0 && half_store_ok<P>(), "zero-half loads and half stores");
  // MINB CTAs per SM: shared memory for all of them, registers capped by the launch bounds
  static_assert(smem_fwd <= (MINB == 2 ? 110 : 226) * 1024 && smem_inv <= (MINB == 2 ? 110 : 226) * 1024,
                "CTAs per SM");
};

template <typename R, int L>
__global__ void __launch_bounds__(FusedZY<R, L>::TH, FusedZY<R, L>::MINB) k_mv_fwd_zy(Geo g, const typename CT<R>::T* __restrict__ tw,
                                                                 InstState* st, const int* act, int in_id,
                                                                 int cond) {
  grid_dep_begin();
  typedef typename CT<R>::T C;
  typedef FusedZY<R, L> F;
  typedef typename F::P P;
  constexpr int NC = F::NC, LP = F::SH::LP, T = F::SH::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);     // [NC][BWF], filled by the whole cluster
  C* xs = buf + NC * F::BWF;                    // exchange scratch
  InstState& S = st[inst_of(act)];
  if (!cond_ok(S, cond)) return;
  cg::cluster_group cluster = cg::this_cluster();
  const int r = (int)cluster.block_rank();
  const int ix = (int)blockIdx.x / F::CL;
  cluster.sync();                               // every peer runs before its buffer is written
  {
    const C* __restrict__ x = (const C*)S.vec[in_id];
    const int c = threadIdx.x % 3, rest = threadIdx.x / 3;
    const int t = rest % T, l = rest / T;
    const int y = r * F::YR + l;
    const long long line = (long long)ix * NC + y;
    const long long base = line * NC * 3 + c;
    const int* __restrict__ cid = S.cidx ? S.cidx + line * NC : nullptr;
    auto ld = [&](int, int pos) -> C {
      long long i = base + (long long)pos * 3;
      if (cid) {
        const int k = cid[pos];
        if (k < 0) return czero<C>();
        i = 3LL * k + c;
      }
      return __ldcg(x + i);
    };
    C* sl = xs + l * 3 * LP + c;
    auto sm = [&](int, int pp) -> C& { return sl[pp * 3]; };
    C* brow = buf + y * F::BWF + c;
    auto stf = [&](int, int kz, C v) { *cluster.map_shared_rank(brow + 3 * (kz % F::KB), kz / F::KB) = v; };
    C a[P::E];
    rfft<P, 1, false, true, false>(a, t, ld, sm, stf, tw);
  }
  cluster.sync();                               // all NC rows of this CTA's kz block are in
  {
    C* __restrict__ t2 = (C*)S.t2;
    constexpr int W = 3 * F::TZ;
    constexpr long long rs = (long long)L * 3;
    const int w = threadIdx.x % W, t = threadIdx.x / W;
    C* sw = xs + w;
    auto sm = [&](int, int pp) -> C& { return sw[pp * W]; };
#pragma unroll 1
    for (int q = 0; q < F::ROUNDS; ++q) {
      const C* src = buf + q * W + w;
      C* dst = t2 + (long long)ix * L * rs + (r * F::KB + q * F::TZ) * 3 + w;
      auto ld = [&](int, int pos) -> C { return src[pos * F::BWF]; };
      auto stf = [&](int, int pos, C v) { __stcg(dst + pos * rs, v); };
      C a[P::E];
      rfft<P, 1, false, true, false>(a, t, ld, sm, stf, tw);
    }
  }
}

template <typename R, int L>
__global__ void __launch_bounds__(FusedZY<R, L>::TH, FusedZY<R, L>::MINB) k_mv_inv_yz(Geo g, const typename CT<R>::T* __restrict__ tw,
                                                                 InstState* st, const int* act, int in_id,
                                                                 int out_id, int mode, int cond) {
  grid_dep_begin();
  typedef typename CT<R>::T C;
  typedef FusedZY<R, L> F;
  typedef typename F::P P;
  constexpr int NC = F::NC, LP = F::SH::LP, T = F::SH::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);     // [YR][BWI], filled by the whole cluster
  C* xs = buf + F::YR * F::BWI;                 // exchange scratch
  InstState& S = st[inst_of(act)];
  if (!cond_ok(S, cond)) return;
  cg::cluster_group cluster = cg::this_cluster();
  const int r = (int)cluster.block_rank();
  const int ix = (int)blockIdx.x / F::CL;
  cluster.sync();
  {
    const C* __restrict__ t2 = (const C*)S.t2;
    constexpr int W = 3 * F::TZ;
    constexpr long long rs = (long long)L * 3;
    const int w = threadIdx.x % W, t = threadIdx.x / W;
    C* sw = xs + w;
    auto sm = [&](int, int pp) -> C& { return sw[pp * W]; };
#pragma unroll 1
    for (int q = 0; q < F::ROUNDS; ++q) {
      const int col = (r * F::KB + q * F::TZ) * 3 + w;
      const C* src = t2 + (long long)ix * L * rs + col;
      C* bcol = buf + col;
      auto ld = [&](int, int pos) -> C { return __ldcg(src + pos * rs); };
      auto stf = [&](int, int y, C v) { *cluster.map_shared_rank(bcol + (y % F::YR) * F::BWI, y / F::YR) = v; };
      C a[P::E];
      rfft<P, 1, true, false, true>(a, t, ld, sm, stf, tw);
    }
  }
  cluster.sync();                               // all L kz of this CTA's rows are in
  {
    // fresh copies keep the y phase's address arithmetic out of this one
    const int tid = opaque((int)threadIdx.x);
    const int c = tid % 3, rest = tid / 3;
    const int t = rest % T, l = rest / T;
    const long long line = (long long)opaque(ix * NC + r * F::YR) + l;
    buf = opaque_ptr(buf);
    xs = opaque_ptr(xs);
    const long long site0 = line * NC;
    const C* __restrict__ xg = (const C*)S.vec[in_id];
    C* __restrict__ yg = (C*)S.vec[out_id];
    const C* __restrict__ iag = (const C*)S.inva + site0;
    const C* __restrict__ bg = (mode == MV_RESIDUAL) ? (const C*)S.vec[V_B] : nullptr;
    const int* __restrict__ cid = S.cidx ? S.cidx + site0 : nullptr;
    const C* brow = buf + l * F::BWI + c;
    auto ld = [&](int, int pos) -> C { return brow[pos * 3]; };
    C* sl = xs + l * 3 * LP + c;
    auto sm = [&](int, int pp) -> C& { return sl[pp * 3]; };
    // the combine of pass 5 (y = ia x - mask conv and its variants)
    C a[P::E];
    rload<P, 1, false>(a, t, [&](int, int pos) -> C { return cswap(ld(0, pos)); });
    rstage<P, 0, false>(a, t, tw);
    rrest<P, 1, 0>(a, t, sm, tw);
    mv_combine_out<P, true, DDA_P5_EB, R>(a, opaque(t), true, NC, site0, c, cid, iag, xg, bg, yg, mode,
                                          [](int, C) {});
  }
}

// ---------------------------------------------------------------------------
// host dispatch over the compiled lengths
// ---------------------------------------------------------------------------
template <typename R> struct MvSet {
  typedef typename CT<R>::T C;
  typedef void (*P1)(Geo, const C*, InstState*, const int*, int, int, int, int);
  typedef void (*PY)(Geo, const C*, InstState*, const int*, int, int, int);
  typedef void (*P3)(Geo, const C*, InstState*, const int*, int, int, int, R, int);
  typedef void (*P5)(Geo, const C*, InstState*, const int*, int, int, int, int, int, int, double*, unsigned*);
  typedef void (*PF)(Geo, const C*, InstState*, const int*, int, int);
  typedef void (*PI)(Geo, const C*, InstState*, const int*, int, int, int, int);
  typedef void (*P51)(Geo, const C*, InstState*, const int*, int, int, int);
  P1 k1 = nullptr; PY k2 = nullptr; P3 k3 = nullptr; PY k4 = nullptr; P5 k5 = nullptr;
  P51 k51 = nullptr;   // pass 5 of M + pass 1 of A (launch_amul_impl)
  // tile sizes the kernels were compiled for (cubic set only; 0 = any)
  int nl = 0, tz2 = 0, tz3 = 0;
  // cluster-fused passes 1+2 (kf) and 4+5 (ki), cubic sets only: cluster
  // size, threads, CTAs per instance and dynamic shared memory
  PF kf = nullptr; PI ki = nullptr;
  int cl = 0, thf = 0, gridf = 0;
  size_t smemf = 0, smemi = 0;
  bool fused_any = false;        // fused passes also in batched launches
  // staged persistent x pass (cubic sets only): threads, tiles per
  // instance, dynamic shared memory, CTAs per SM it is built for
  P3 k3p = nullptr;
  int th3p = 0, nt3p = 0, minb3p = 1;
  size_t smem3p = 0;
  // packed-pair x pass (complex64 cubic sets): threads, CTAs per instance,
  // dynamic shared memory
  P3 k3x = nullptr;
  int th3x = 0, grid3x = 0;
  size_t smem3x = 0;
  // packed-pair y passes (complex64 cubic sets)
  PY k2x = nullptr, k4x = nullptr;
  int th2x = 0, grid2x = 0;
  size_t smem2x = 0;
  // packed-pair z passes (complex64 cubic sets)
  P1 k1x = nullptr;
  P5 k5x = nullptr;
  int th1x = 0, grid1x = 0;
  size_t smem1x = 0;
};

// General kernels (sizes from Geo), defined with the instantiations.
template <typename R> bool mv_general_set(int Lx, int Ly, int Lz, int p3var, MvSet<R>& out);
// Cubic kernels for the FFT length L = 2n (box n^3): complex64 with pass-3
// variant 0, complex128 with variant 2 (matvec_cube_f32.cu / _f64.cu).
template <typename R> bool mv_cube_set(int L, int p3var, MvSet<R>& out);
template <> bool mv_general_set<float>(int, int, int, int, MvSet<float>&);
template <> bool mv_general_set<double>(int, int, int, int, MvSet<double>&);
template <> bool mv_cube_set<float>(int, int, MvSet<float>&);
template <> bool mv_cube_set<double>(int, int, MvSet<double>&);

// The z / y pass kernels of an instantiation: the `_cap` twin where a
// register cap applies, else the plain kernel.
template <typename R, int L, int NC>
auto pick_pass1() {
  if constexpr (z_regs<R, NC, DDA_Z1_REGS>() > 0) return k_mv_pass1_cap<R, L, NC>;
  else return k_mv_pass1<R, L, NC>;
}
template <typename R, int L, int NC>
auto pick_pass5() {
  if constexpr (z_regs<R, NC, DDA_Z_REGS>() > 0) return k_mv_pass5_cap<R, L, NC>;
  else return k_mv_pass5<R, L, NC>;
}
template <typename R, int L, int NC>
auto pick_pass51() {
  if constexpr (z_regs<R, NC, DDA_Z51_REGS>() > 0) return k_mv_pass51_cap<R, L, NC>;
  else return k_mv_pass51<R, L, NC>;
}
template <typename R, bool INV, int L, int NC>
auto pick_pass_y() {
  if constexpr (y_regs<R, NC, INV>() > 0) return k_mv_pass_y_cap<R, INV, L, NC>;
  else return k_mv_pass_y<R, INV, L, NC>;
}

template <typename R>
bool mv_general_set_impl(int Lx, int Ly, int Lz, int p3var, MvSet<R>& o) {
  typedef MvSet<R> M;
  switch (Lz) {
#define DDA_K(n) case n: o.k1 = pick_pass1<R, n, 0>(); o.k5 = pick_pass5<R, n, 0>(); o.k51 = pick_pass51<R, n, 0>(); break;
    DDA_FFT_SIZES(DDA_K)
#undef DDA_K
    default: return false;
  }
  switch (Ly) {
#define DDA_K(n)                                                                                   \
  case n:                                                                                          \
    o.k2 = (typename M::PY)pick_pass_y<R, false, n, 0>();                                          \
    o.k4 = (typename M::PY)pick_pass_y<R, true, n, 0>();                                           \
    break;
    DDA_FFT_SIZES(DDA_K)
#undef DDA_K
    default: return false;
  }
  switch (Lx) {
#define DDA_K(n)                                                                                   \
  case n:                                                                                          \
    o.k3 = p3var == 1 ? (typename M::P3)k_mv_pass3r<R, n, 1, 0>                                    \
                      : (p3var == 2 ? (typename M::P3)k_mv_pass3s<R, n, 2, 0>                      \
                                    : (typename M::P3)k_mv_pass3s<R, n, 0, 0>);                    \
    break;
    DDA_FFT_SIZES(DDA_K)
#undef DDA_K
    default: return false;
  }
  return true;
}

template <typename R, int L, int V>
void mv_cube_fill(MvSet<R>& o) {
  typedef MvSet<R> M;
  constexpr int NC = L / 2;
  o.k1 = pick_pass1<R, L, NC>();
  o.k2 = (typename M::PY)pick_pass_y<R, false, L, NC>();
  if constexpr (V == 1) o.k3 = (typename M::P3)k_mv_pass3r<R, L, V, NC>;
  else o.k3 = (typename M::P3)k_mv_pass3s<R, L, V, NC>;
  o.k4 = (typename M::PY)pick_pass_y<R, true, L, NC>();
  o.k5 = pick_pass5<R, L, NC>();
  o.k51 = pick_pass51<R, L, NC>();
  o.nl = cmin_i(mv_tiles<R, MvShape<R, L>::T>(), NC * NC);
  o.tz2 = cmin_i(mv_tiles<R, MvShape<R, L>::T>(), L);
  o.tz3 = cmin_i(V == 1 ? mv_tiles<R, P3Shape<R, L, V>::T>() : p3s_tiles<R, L, P3Shape<R, L, V>::T>(), L);
  if constexpr (sizeof(R) == 4 && V == 0 && (L == 128 || L == 256)) {
    // complex64 64^3 / 128^3: the staged persistent x pass, same tile shape
    constexpr int TZ = cmin_i(mv_tiles<R, P3Shape<R, L, V>::T>(), L);
    typedef P3Pipe<R, L, V, TZ> PP;
    o.k3p = (typename M::P3)k_mv_pass3p<R, L, V, NC, TZ, 2>;
    o.th3p = PP::TH;
    o.nt3p = L * (L / TZ);
    o.minb3p = 2;
    o.smem3p = PP::smem;
  }
  if constexpr (sizeof(R) == 4 && V == 0 && (L == 128 || L == 256)) {
    // the packed-pair x pass on the same tiles (192 threads; 4 CTAs per SM
    // at L = 256, 3 at L = 128, where the 16 x 8 plan needs more registers)
    constexpr int TZ = cmin_i(mv_tiles<R, P3Shape<R, L, V>::T>(), L);
    typedef P3Pair<L, TZ> PX;
    o.k3x = (typename M::P3)k_mv_pass3x<L, NC, TZ, (L == 256 ? 4 : 3)>;
    o.th3x = PX::TH;
    o.grid3x = L * (L / TZ);
    o.smem3x = PX::smem;
    constexpr int TY = cmin_i(mv_tiles<R, MvShape<R, L>::T>(), L);
    typedef PYPair<L, TY> PY2;
    o.k2x = (typename M::PY)k_mv_pass_yx<false, L, NC, TY, (L == 256 ? 4 : 3)>;
    o.k4x = (typename M::PY)k_mv_pass_yx<true, L, NC, TY, (L == 256 ? 4 : 3)>;
    o.th2x = PY2::TH;
    o.grid2x = NC * (L / TY);
    o.smem2x = PY2::smem;
    typedef PZPair<L> PZ2;
    o.k1x = k_mv_pass1x<L, (L == 256 ? 4 : 3)>;
    o.k5x = k_mv_pass5x<L, (L == 256 ? 4 : 3)>;
    o.th1x = PZ2::TH;
    o.grid1x = NC * NC / PZ2::NL;
    o.smem1x = PZ2::smem;
  }
  if constexpr (sizeof(R) == 8 && V == 2 && (L == 128 || L == 256)) {
    // complex128 64^3 / 128^3: tiles of 8 kz columns (384-byte row
    // segments against 96 bytes in the one-tile kernel's 2-column tiles)
    constexpr int TZ = 8;
    constexpr int MB = L == 256 ? 1 : 2;
    typedef P3Pipe<R, L, V, TZ> PP;
    o.k3p = (typename M::P3)k_mv_pass3p<R, L, V, NC, TZ, MB>;
    o.th3p = PP::TH;
    o.nt3p = L * (L / TZ);
    o.minb3p = MB;
    o.smem3p = PP::smem;
  }
  if constexpr (sizeof(R) == 4 && (L == 128 || (L == 256 && MvShape<R, L>::T <= 16))) {
    // complex64 64^3: both fused buffers fit two CTAs per SM; 128^3: one CTA
    // per SM in clusters of eight (T1, 151 MB and beyond L2, is neither
    // written nor read), for launches of any width, but only where the
    // tuning table selects them (DDA_TUNE_FUSED): B200, 128^3 matvec 0.679
    // against 0.542 ms with the separate passes
    typedef FusedZY<R, L> F;
    o.fused_any = L == 256;
    o.kf = k_mv_fwd_zy<R, L>;
    o.ki = k_mv_inv_yz<R, L>;
    o.cl = F::CL;
    o.thf = F::TH;
    o.gridf = NC * F::CL;
    o.smemf = F::smem_fwd;
    o.smemi = F::smem_inv;
  }
}

// The kernel set for a geometry: the cubic one when the box is n^3 on a
// (2n)^3 grid and its tile sizes match the configuration, else the general.
template <typename R>
bool mv_select(const Geo& g, const PassCfg& pc, MvSet<R>& o) {
  const bool cube = g.nx == g.ny && g.ny == g.nz && g.Lx == g.Ly && g.Ly == g.Lz && g.Lx == 2 * g.nx;
  if (cube && !getenv("DDA_NO_CUBE") && mv_cube_set<R>(g.Lx, pc.p3var, o) && o.nl == pc.nl &&
      o.tz2 == pc.tz2 && o.tz3 == pc.tz3)
    return true;
  o = MvSet<R>();
  return mv_general_set<R>(g.Lx, g.Ly, g.Lz, pc.p3var, o);
}

// Raise the dynamic shared-memory limit of each kernel once per device
// (null entries are skipped).
cudaError_t mv_prepare(const void* const* ks, int n);
// Whether the cluster-fused z/y passes run (DDA_NO_FUSED_ZY=1 turns both
// off, DDA_NO_FUSED_INV=1 the inverse one only); read at every launch.
bool fused_zy_enabled(bool inverse);
// Whether the staged persistent x pass is forced where compiled
// (DDA_P3PIPE=1; otherwise it runs only where the tuning table selects
// it: on B200 it measured slower than the one-tile kernel at 64^3 and
// 128^3); read at every launch.
bool p3_pipe_forced();
// Whether the packed-pair x pass is forced where compiled (DDA_P3PAIR=1;
// otherwise DDA_TUNE_P3PAIR in the tuning table selects it).
bool p3_pair_forced();
// Likewise for the packed-pair y passes (DDA_YPAIR=1 / DDA_TUNE_YPAIR).
bool y_pair_forced();
// Likewise for the packed-pair z passes (DDA_ZPAIR=1 / DDA_TUNE_ZPAIR).
bool z_pair_forced();
// Streaming multiprocessors of the current device (cached per device).
int device_sms();
// CTAs of kernel k resident per SM at this block size and shared memory
// (occupancy query, cached per kernel and shape).
int resident_ctas(const void* k, int threads, size_t smem);
// Whether the x / y passes prefetch the input rows of the tiles one
// resident wave ahead into L2 (DDA_PREFETCH=1 forces it; otherwise
// DDA_TUNE_PREFETCH in the tuning table).  B200: slower at every size
// measured (128^3 c64 0.587 against 0.558 ms, c128 1.363 against 1.269;
// 64^3 c64 0.083 against 0.078), so nothing selects it by default.
bool prefetch_forced();


// Launch on clusters of `cl` CTAs along x, with programmatic stream
// serialization unless DDA_NO_PDL=1.
template <typename... KArgs, typename... Args>
cudaError_t launch_cluster(void (*k)(KArgs...), int cl, dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                           Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)cl;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = (pdl_enabled() && stream_pdl(s)) ? 2 : 1;
  return cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}

template <typename R>
cudaError_t launch_mv_set(const MvSet<R>& k, const Geo& g, const PassCfg& pc, InstState* st, const int* act, int nb,
                          const typename CT<R>::T* twx, const typename CT<R>::T* twy, const typename CT<R>::T* twz,
                          int in_id, int out_id, int mode, int cond, double gscale, cudaStream_t s,
                          const MvFuse& fz = MvFuse()) {
  const void* ks[13] = {(const void*)k.k1, (const void*)k.k2, (const void*)k.k3, (const void*)k.k4,
                        (const void*)k.k5, (const void*)k.kf, (const void*)k.ki, (const void*)k.k3p,
                        (const void*)k.k3x, (const void*)k.k2x, (const void*)k.k4x, (const void*)k.k1x,
                        (const void*)k.k5x};
  cudaError_t e = mv_prepare(ks, 13);
  if (e != cudaSuccess) return e;
  // The fused z/y kernels take the place of passes 1+2 / 4+5 in launches of
  // one instance with no Krylov step fused into those passes (cubic sets use
  // one twiddle table).  Measured on B200 at 64^3 complex64: one instance
  // 0.0768 -> 0.0748 ms per matvec; two instances in one launch 0.132 ->
  // 0.138 ms (the separate passes already fill the GPU there and the fused
  // kernels hold two CTAs per SM), so batched launches keep the separate
  // passes.
  const int tf = tune_flags(sizeof(R) == 8 ? DDA_C128 : DDA_C64, g, nb);
  const bool one = k.fused_any ? (tf & DDA_TUNE_FUSED) != 0 : nb == 1;
  const bool skip1 = (fz.skip & 1) != 0, skip5 = (fz.skip & 2) != 0;
  const bool ff = !skip1 && one && k.kf && fz.pre == MV_PRE_NONE && fused_zy_enabled(false) &&
                  !(tf & DDA_TUNE_NO_FUSED_ZY);
  const bool fi = !skip5 && one && k.ki && fz.post == MV_POST_NONE && fused_zy_enabled(true) &&
                  !(tf & DDA_TUNE_NO_FUSED_INV);
  const bool ypair = k.k2x && (y_pair_forced() || (tf & DDA_TUNE_YPAIR));
  const bool zpair = k.k1x && (z_pair_forced() || (tf & DDA_TUNE_ZPAIR));
  Geo gq = g;
  if (prefetch_forced() || (tf & DDA_TUNE_PREFETCH)) {
    gq.pf3 = resident_ctas((const void*)k.k3, pc.th3, pc.smem3) * device_sms();
    gq.pf2 = resident_ctas((const void*)k.k2, pc.th2, pc.smem2) * device_sms();
  }
  if (ff) {
    if ((e = launch_cluster(k.kf, k.cl, dim3((unsigned)k.gridf, nb), dim3(k.thf), k.smemf, s, g, twz, st, act,
                            in_id, cond)))
      return e;
  } else {
    if (skip1) {
      // T1 already holds the forward z transform (k_mv_pass51)
    } else if (zpair && fz.pre == MV_PRE_NONE) {
      if ((e = launch_pdl(k.k1x, dim3((unsigned)k.grid1x, nb), dim3(k.th1x), k.smem1x, s, g, twz, st, act, in_id,
                          cond, pc.nl, fz.pre)))
        return e;
    } else if ((e = launch_pdl(k.k1, dim3((unsigned)pc.grid1, nb), dim3(pc.th1), pc.smem1, s, g, twz, st, act,
                               in_id, cond, pc.nl, fz.pre))) {
      return e;
    }
    if (ypair) {
      if ((e = launch_pdl(k.k2x, dim3((unsigned)k.grid2x, nb), dim3(k.th2x), k.smem2x, s, g, twy, st, act, cond,
                          pc.tz2, pc.ntz2)))
        return e;
    } else if ((e = launch_pdl(k.k2, dim3((unsigned)pc.grid2, nb), dim3(pc.th2), pc.smem2, s, gq, twy, st, act, cond,
                               pc.tz2, pc.ntz2))) {
      return e;
    }
  }
  if (k.k3x && (p3_pair_forced() || (tf & DDA_TUNE_P3PAIR))) {
    if ((e = launch_pdl(k.k3x, dim3((unsigned)k.grid3x, nb), dim3(k.th3x), k.smem3x, s, g, twx, st, act, cond,
                        pc.tz3, pc.ntz3, (R)gscale, fz.tensor)))
      return e;
  } else if (k.k3p && (p3_pipe_forced() || (tf & (DDA_TUNE_P3PIPE | DDA_TUNE_P3PIPE_1SM)))) {
    // persistent: about minb3p resident CTAs per SM over all instances (one
    // per SM when tuned so)
    const int per_sm = (tf & DDA_TUNE_P3PIPE_1SM) ? 1 : k.minb3p;
    const int want = (per_sm * device_sms() + nb - 1) / nb;
    const int gx = std::max(1, std::min(k.nt3p, want));
    if ((e = launch_pdl(k.k3p, dim3((unsigned)gx, nb), dim3(k.th3p), k.smem3p, s, g, twx, st, act, cond, pc.tz3,
                        pc.ntz3, (R)gscale, fz.tensor)))
      return e;
  } else if ((e = launch_pdl(k.k3, dim3((unsigned)pc.grid3, nb), dim3(pc.th3), pc.smem3, s, gq, twx, st, act, cond,
                             pc.tz3, pc.ntz3, (R)gscale, fz.tensor))) {
    return e;
  }
  if (fi) {
    if ((e = launch_cluster(k.ki, k.cl, dim3((unsigned)k.gridf, nb), dim3(k.thf), k.smemi, s, g, twz, st, act,
                            in_id, out_id, mode, cond)))
      return e;
  } else {
    if (ypair) {
      if ((e = launch_pdl(k.k4x, dim3((unsigned)k.grid2x, nb), dim3(k.th2x), k.smem2x, s, g, twy, st, act, cond,
                          pc.tz2, pc.ntz2)))
        return e;
    } else if ((e = launch_pdl(k.k4, dim3((unsigned)pc.grid2, nb), dim3(pc.th2), pc.smem2, s, gq, twy, st, act, cond,
                               pc.tz2, pc.ntz2))) {
      return e;
    }
    if (skip5) {
      // T1 is left for the next product's first pass (k_mv_pass51)
    } else if (zpair && fz.post == MV_POST_NONE) {
      if ((e = launch_pdl(k.k5x, dim3((unsigned)k.grid1x, nb), dim3(k.th1x), k.smem1x, s, g, twz, st, act, in_id,
                          out_id, mode, cond, pc.nl, fz.post, fz.red, fz.cnt)))
        return e;
    } else if ((e = launch_pdl(k.k5, dim3((unsigned)pc.grid1, nb), dim3(pc.th1), pc.smem1, s, g, twz, st, act,
                               in_id, out_id, mode, cond, pc.nl, fz.post, fz.red, fz.cnt))) {
      return e;
    }
  }
  note_launch(s, 5 - (ff ? 1 : 0) - (fi ? 1 : 0) - (skip1 ? 1 : 0) - (skip5 ? 1 : 0));
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_matvec_impl(Ctx& ctx, const Geo& g, const PassCfg& pc, InstState* st, const int* act, int nb,
                               int in_id, int out_id, int mode, int cond, double gscale, cudaStream_t s,
                               const MvFuse& fz) {
  typedef typename CT<R>::T C;
  constexpr bool dbl = sizeof(R) == 8;
  MvSet<R> k;
  if (!mv_select<R>(g, pc, k)) return cudaErrorInvalidValue;
  const C* twx = (const C*)ctx.twiddles(g.Lx, dbl);
  const C* twy = (const C*)ctx.twiddles(g.Ly, dbl);
  const C* twz = (const C*)ctx.twiddles(g.Lz, dbl);
  if (!twx || !twy || !twz) return cudaErrorMemoryAllocation;
  const int K = mv_split_ways(nb);
  if (K <= 1 || (!act && nb > Ctx::kIota))
    return launch_mv_set<R>(k, g, pc, st, act, nb, twx, twy, twz, in_id, out_id, mode, cond, gscale, s, fz);
  // K concurrent branches, each a launch sequence over nb/K instances: the
  // first on s, the others on the context's auxiliary streams, forked from
  // and joined back into s by events (graph branches under capture), so one
  // branch's passes fill the SMs another's wave tails leave idle
  std::lock_guard<std::mutex> lk(ctx.fork_mu);
  cudaError_t e = cudaEventRecord(ctx.ev_fork, s);
  if (e != cudaSuccess) return e;
  for (int j = 1; j < K; ++j)
    if ((e = cudaStreamWaitEvent(ctx.aux[j - 1], ctx.ev_fork, 0)) != cudaSuccess) return e;
  cudaError_t first = cudaSuccess;
  for (int j = 0; j < K; ++j) {
    const int o = j * nb / K, n = (j + 1) * nb / K - o;
    const int* a = (act ? act : ctx.iota) + o;
    e = launch_mv_set<R>(k, g, pc, st, a, n, twx, twy, twz, in_id, out_id, mode, cond, gscale,
                         j ? ctx.aux[j - 1] : s, fz);
    if (e != cudaSuccess && first == cudaSuccess) first = e;
  }
  for (int j = 1; j < K; ++j) {
    if ((e = cudaEventRecord(ctx.ev_join[j - 1], ctx.aux[j - 1])) == cudaSuccess)
      e = cudaStreamWaitEvent(s, ctx.ev_join[j - 1], 0);
    if (e != cudaSuccess && first == cudaSuccess) first = e;
  }
  return first;
}

// out = A M in for a preconditioned product whose preconditioner grid is the
// operator's (gp = g): M's passes 1-4 (octant pghat), k_mv_pass51 (M's pass 5
// with its mask into mid_id, then A's pass 1 from shared memory), A's passes
// 2-5 (its combine reads mid_id).  A's first pass reads no vector.  fz: M's pass 1 takes fz.pre, A's pass 5
// fz.post (fused Krylov steps).
template <typename R>
cudaError_t launch_amul_impl(Ctx& ctx, const Geo& g, const PassCfg& pc, InstState* st, const int* act, int nb,
                             int in_id, int mid_id, int out_id, int mode, int cond, double gscale, double pscale,
                             cudaStream_t s, const MvFuse& fz) {
  typedef typename CT<R>::T C;
  constexpr bool dbl = sizeof(R) == 8;
  MvSet<R> k;
  if (!mv_select<R>(g, pc, k) || !k.k51) return cudaErrorInvalidValue;
  const C* twx = (const C*)ctx.twiddles(g.Lx, dbl);
  const C* twy = (const C*)ctx.twiddles(g.Ly, dbl);
  const C* twz = (const C*)ctx.twiddles(g.Lz, dbl);
  if (!twx || !twy || !twz) return cudaErrorMemoryAllocation;
  const void* ks[1] = {(const void*)k.k51};
  cudaError_t e = mv_prepare(ks, 1);
  if (e != cudaSuccess) return e;
  MvFuse fm;
  fm.tensor = 1;
  fm.pre = fz.pre;
  fm.skip = 2;
  if ((e = launch_mv_set<R>(k, g, pc, st, act, nb, twx, twy, twz, in_id, mid_id, MV_CONV_MASKED, cond, pscale, s,
                            fm)))
    return e;
  if ((e = launch_pdl(k.k51, dim3((unsigned)pc.grid1, nb), dim3(pc.th1), pc.smem1, s, g, twz, st, act, mid_id,
                      cond, pc.nl)))
    return e;
  note_launch(s, 1);
  MvFuse fa = fz;
  fa.pre = MV_PRE_NONE;
  fa.tensor = 0;
  fa.skip = 1;
  // A's combine reads its x (the M vector) from mid_id
  return launch_mv_set<R>(k, g, pc, st, act, nb, twx, twy, twz, mid_id, out_id, mode, cond, gscale, s, fa);
}

// Same five launches with caller-provided twiddle tables (used by the
// allocation-free entry point, whose tables live in its own static buffer).
template <typename R>
cudaError_t launch_matvec_tw_impl(const Geo& g, const PassCfg& pc, InstState* st, const typename CT<R>::T* twx,
                                  const typename CT<R>::T* twy, const typename CT<R>::T* twz, int in_id,
                                  int out_id, int mode, double gscale, cudaStream_t s) {
  MvSet<R> k;
  if (!mv_select<R>(g, pc, k)) return cudaErrorInvalidValue;
  return launch_mv_set<R>(k, g, pc, st, nullptr, 1, twx, twy, twz, in_id, out_id, mode, C_ALWAYS, gscale, s);
}

// Tile shapes: about 128 (complex64) or 64 (complex128) transforms' worth of
// threads per CTA, at most one tile dimension's extent.

template <typename R>
static bool tile_dims(int L, int& T, int& LP) {
  switch (L) {
#define DDA_K(n) case n: T = MvShape<R, n>::T; LP = MvShape<R, n>::LP; return true;
    DDA_FFT_SIZES(DDA_K)
#undef DDA_K
  }
  return false;
}

template <typename R>
static bool tile_dims3(int L, int v, int& T, int& LP) {
  switch (L) {
#define DDA_K(n)                                                                      \
  case n:                                                                             \
    if (v == 0) { T = P3Shape<R, n, 0>::T; LP = P3Shape<R, n, 0>::LP; }               \
    else { T = P3Shape<R, n, 1>::T; LP = P3Shape<R, n, 1>::LP; }                      \
    return true;
    DDA_FFT_SIZES(DDA_K)
#undef DDA_K
  }
  return false;
}

// Pass-3 variant: DDA_P3_VARIANT overrides; default 0 for complex64 and 2
// for complex128 (both one component per thread, coalesced columns).
template <typename R>
static int p3_variant() {
  const char* e = getenv("DDA_P3_VARIANT");
  if (e && *e >= '0' && *e < '0' + kP3Variants) return *e - '0';
  return sizeof(R) == 4 ? 0 : 2;
}

template <typename R>
PassCfg make_pass_cfg_impl(const Geo& g) {
  PassCfg c{};
  const size_t esz = sizeof(R) * 2;
  int T, LP;
  // z passes: nl lines x 3 components, 3*T threads per line
  tile_dims<R>(g.Lz, T, LP);
  const long long nlines = (long long)g.nx * g.ny;
  c.nl = (int)std::min<long long>(std::max(1, mv_lanes_t<R>(T) / T), nlines);
  c.th1 = 3 * T * c.nl;
  c.smem1 = (size_t)c.nl * 3 * LP * esz + (smem_tw((int)esz) ? (size_t)g.Lz * esz : 0);
  c.grid1 = (nlines + c.nl - 1) / c.nl;
  // y passes: tz kz columns, 3*tz transforms of T threads
  tile_dims<R>(g.Ly, T, LP);
  c.tz2 = std::min(std::max(1, mv_lanes_t<R>(T) / T), g.Lz);
  c.th2 = 3 * c.tz2 * T;
  c.smem2 = (size_t)3 * c.tz2 * LP * esz + (smem_tw((int)esz) ? (size_t)g.Ly * esz : 0);
  c.ntz2 = (g.Lz + c.tz2 - 1) / c.tz2;
  c.grid2 = (long long)g.nx * c.ntz2;
  // x pass
  c.p3var = p3_variant<R>();
  tile_dims3<R>(g.Lx, c.p3var, T, LP);
  c.p3reg = c.p3var == 1;
  c.tz3 = std::min(std::max(1, mv_lanes_t<R>(T) / T), g.Lz);
  if (sizeof(R) == 4 && g.Lx == 128 && DDA_P3_TZ128 > 0 && !c.p3reg) c.tz3 = std::min(DDA_P3_TZ128, g.Lz);
  c.th3 = (c.p3reg ? 1 : 3) * c.tz3 * T;
  c.smem3 = (size_t)3 * c.tz3 * LP * esz + (smem_tw((int)esz) ? (size_t)g.Lx * esz : 0);
  c.ntz3 = (g.Lz + c.tz3 - 1) / c.tz3;
  c.grid3 = (long long)g.Ly * c.ntz3;
  return c;
}

}  // namespace dda
