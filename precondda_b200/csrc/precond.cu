// Preconditioner builder for the right-preconditioned GPBiCGSTAB (the
// reference's precon=True path, Gpbicgstab.py:1002-1199).  The reference
// applies an octant P with the interaction octant's mirror rule,
//   M x = mask * IFFT[ P . FFT(pad x) ]   on the grid 2 (octant extent - 1)
// (fft_matvec3 + optimized_dot_product_reduced_kernel, Gpbicgstab.py:36-103,
// :633-668), but the builders it calls are not defined anywhere
// (ddaforgit.py:1118-1136).  This file builds one for that format:
//
//   P(q) = [abar I - FFT_L(-c)(q)]^-1,    c(t) = sum_{j = t mod L} w(j) G(j)
//
// abar = mean inverse polarizability of the occupied sites; G(j) the lattice
// Green tensor at offsets j in (-n, n)^3 (zero at j = 0); w(j) the fraction
// of occupied sites whose neighbour at offset j is occupied (occupancy
// autocorrelation R(j)/R(0), averaged over the 8 axis reflections of j so the
// weighted kernel keeps G's per-axis parity and the octant format stays
// exact).  c is T. Chan's optimal circulant approximation of the masked
// interaction operator (Frobenius-nearest circulant), folded onto the
// L-periodic grid (L >= n per axis; L = n is the cheapest to apply), and P is
// its inverse.  Everything is computed in FP64.
//
// Steps: abar (one-CTA reduction); R by two forward FFTs of the padded
// occupancy on a grid >= 2n (the second transforms |F|^2, which is real and
// even); the weighted, folded G evaluated inside a z-FFT pass; the y and x
// passes of the Green build (green_yx); a 3x3 complex symmetric inverse per
// octant point.
#include <cmath>
#include <string>

#include "dda_host.h"
#include "fft_core.cuh"
#include "fft_sizes.h"

namespace dda {

constexpr int PEPT = 12, PNT = 256;   // FP64 tiles: L * transforms <= 3072

// ---------------------------------------------------------------------------
// mean inverse polarizability of the occupied sites and their count:
// meta[0..1] = abar, meta[2] = count (fixed-order, one CTA)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_pre_abar(const double2* __restrict__ ia, long long n, double* meta) {
  __shared__ double sh[3][32];
  double sx = 0.0, sy = 0.0, cnt = 0.0;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) {
    const double2 v = ia[i];
    if (v.x != 0.0 || v.y != 0.0) { sx += v.x; sy += v.y; cnt += 1.0; }
  }
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_down_sync(0xffffffffu, sx, o);
    sy += __shfl_down_sync(0xffffffffu, sy, o);
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { sh[0][wid] = sx; sh[1][wid] = sy; sh[2][wid] = cnt; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0, c = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { a += sh[0][w]; b += sh[1][w]; c += sh[2][w]; }
    meta[0] = c > 0 ? a / c : 1.0;
    meta[1] = c > 0 ? b / c : 0.0;
    meta[2] = c;
  }
}

// occupancy (1 where inv_alpha != 0) padded into the (Ax,Ay,Az) grid
__global__ void k_pre_occ(const double2* __restrict__ ia, int nx, int ny, int nz, int Ax, int Ay, int Az,
                          double2* __restrict__ A) {
  const long long tot = (long long)Ax * Ay * Az;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(i % Az);
    const long long r = i / Az;
    const int iy = (int)(r % Ay), ix = (int)(r / Ay);
    double o = 0.0;
    if (ix < nx && iy < ny && iz < nz) {
      const double2 v = ia[((long long)ix * ny + iy) * nz + iz];
      o = (v.x != 0.0 || v.y != 0.0) ? 1.0 : 0.0;
    }
    A[i] = make_double2(o, 0.0);
  }
}

__global__ void k_pre_abs2(double2* __restrict__ A, long long tot) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const double2 v = A[i];
    A[i] = make_double2(v.x * v.x + v.y * v.y, 0.0);
  }
}

// in-place forward FFT along z of NL lines of length L per CTA
template <int L>
__global__ void __launch_bounds__(PNT) k_pre_fft_z(double2* __restrict__ A, long long nlines, int NL,
                                                   const double2* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* s = reinterpret_cast<double2*>(smem_raw);
  const long long line0 = (long long)blockIdx.x * NL;
  for (int idx = threadIdx.x; idx < NL * L; idx += PNT) {
    const int l = idx / L;
    s[idx] = (line0 + l < nlines) ? A[line0 * L + idx] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  LayLine<1> lay{NL, L};
  fft_tile<L, false, PEPT, PNT>(s, lay, tw);
  for (int idx = threadIdx.x; idx < NL * L; idx += PNT) {
    const int l = idx / L;
    if (line0 + l < nlines) A[line0 * L + idx] = s[idx];
  }
}

// in-place forward FFT along y (AX = 1) or x (AX = 0) of Tz columns per CTA
template <int AX, int L>
__global__ void __launch_bounds__(PNT) k_pre_fft_col(double2* __restrict__ A, int Ax, int Ay, int Az, int Tz, int ntz,
                                                     const double2* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* s = reinterpret_cast<double2*>(smem_raw);
  const int o = blockIdx.x / ntz, kzt = blockIdx.x - o * ntz;   // o = ix (AX 1) or iy (AX 0)
  const int kz0 = kzt * Tz;
  const int tzn = min(Tz, Az - kz0);
  auto at = [&](int r, int w) -> long long {
    return (AX == 1 ? ((long long)o * Ay + r) : ((long long)r * Ay + o)) * Az + kz0 + w;
  };
  for (int idx = threadIdx.x; idx < L * Tz; idx += PNT) {
    const int r = idx / Tz, w = idx - r * Tz;
    s[idx] = w < tzn ? A[at(r, w)] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  LayCol lay{Tz, Tz};
  fft_tile<L, false, PEPT, PNT>(s, lay, tw);
  for (int idx = threadIdx.x; idx < L * Tz; idx += PNT) {
    const int r = idx / Tz, w = idx - r * Tz;
    if (w < tzn) A[at(r, w)] = s[idx];
  }
}

// signed offsets j in (-n, n) that fold onto grid index i of an L-point axis
// (L >= n): j = i and j = i - L where in range; returns how many
__device__ __forceinline__ int fold_offsets(int i, int n, int L, int* j) {
  int c = 0;
  if (i <= n - 1) j[c++] = i;
  if (i - L >= -(n - 1)) j[c++] = i - L;
  return c;
}

// z pass of the weighted, folded Green tensor on the (Lx,Ly,Lz) grid: NL
// lines per CTA, G evaluated in place, z-FFT, kz < hz kept -> b1
// (Lx,Ly,hz,6), the input format of green_yx.  R holds N_A R(j) (the second
// FFT of |F|^2) on the (Ax,Ay,Az) grid.
template <int LZ>
__global__ void __launch_bounds__(PNT) k_pre_z(Geo g, const double2* __restrict__ tw, double k, double d, int NL,
                                               const double2* __restrict__ R, int Ax, int Ay, int Az,
                                               double2* __restrict__ b1) {
  constexpr int LS = 6 * LZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* s = reinterpret_cast<double2*>(smem_raw);
  const long long nlines = (long long)g.Lx * g.Ly;
  const long long line0 = (long long)blockIdx.x * NL;
  const double r0 = R[0].x;
  const double inv8r0 = r0 > 0.0 ? 0.125 / r0 : 0.0;
  auto ridx = [&](int jx, int jy, int jz) -> long long {
    const int ax = jx < 0 ? jx + Ax : jx, ay = jy < 0 ? jy + Ay : jy, az = jz < 0 ? jz + Az : jz;
    return ((long long)ax * Ay + ay) * Az + az;
  };
  for (int idx = threadIdx.x; idx < NL * LZ; idx += PNT) {
    const int l = idx / LZ, iz = idx - l * LZ;
    const long long line = line0 + l;
    double2 v[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) v[c] = make_double2(0.0, 0.0);
    if (line < nlines) {
      const int ix = (int)(line / g.Ly), iy = (int)(line - (long long)ix * g.Ly);
      int ox[2], oy[2], oz[2];
      const int cx = fold_offsets(ix, g.nx, g.Lx, ox);
      const int cy = fold_offsets(iy, g.ny, g.Ly, oy);
      const int cz = fold_offsets(iz, g.nz, g.Lz, oz);
      for (int a = 0; a < cx; ++a)
        for (int b = 0; b < cy; ++b)
          for (int e = 0; e < cz; ++e) {
            const int jx = ox[a], jy = oy[b], jz = oz[e];
            if (jx == 0 && jy == 0 && jz == 0) continue;
            // occupancy weight, averaged over the 8 axis reflections
            double wsum = 0.0;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              const double rr = R[ridx((q & 1) ? -jx : jx, (q & 2) ? -jy : jy, (q & 4) ? -jz : jz)].x;
              wsum += rr > 0.0 ? rr : 0.0;
            }
            const double wgt = wsum * inv8r0;
            if (wgt == 0.0) continue;
            const double X = jx * d, Y = jy * d, Z = jz * d;
            const double r2 = X * X + Y * Y + Z * Z;
            const double r = sqrt(r2);
            const double ir = 1.0 / r;
            const double n0 = X * ir, n1 = Y * ir, n2 = Z * ir;
            const double kr = k * r;
            double sn, cs;
            sincos(kr, &sn, &cs);
            const double2 ex = make_double2(wgt * cs * ir, wgt * sn * ir);   // w e^{ikr}/r
            const double2 f2 = make_double2(-1.0 / r2, kr / r2);             // (ikr - 1)/r^2
            const double nn[6] = {n0 * n0, n0 * n1, n0 * n2, n1 * n1, n1 * n2, n2 * n2};
            const double dl[6] = {1.0, 0.0, 0.0, 1.0, 0.0, 1.0};
#pragma unroll
            for (int c = 0; c < 6; ++c) {
              const double t1 = k * k * (nn[c] - dl[c]);
              const double aa = 3.0 * nn[c] - dl[c];
              const double2 t = make_double2(t1 + aa * f2.x, aa * f2.y);
              v[c] = cadd(v[c], cmul(ex, t));
            }
          }
    }
    double2* q = s + l * LS + iz * 6;
#pragma unroll
    for (int c = 0; c < 6; ++c) q[c] = v[c];
  }
  __syncthreads();
  LayLine<6> lay{NL, LS};
  fft_tile<LZ, false, PEPT, PNT>(s, lay, tw);
  for (int idx = threadIdx.x; idx < NL * g.hz * 6; idx += PNT) {
    const int l = idx / (g.hz * 6), rem = idx - l * g.hz * 6;
    const int kz = rem / 6, c = rem - kz * 6;
    const long long line = line0 + l;
    if (line < nlines) b1[(line * g.hz + kz) * 6 + c] = s[l * LS + kz * 6 + c];
  }
}

// P = (abar I - Gw)^-1 per octant point; Gw (6,H) FP64 engine layout.
// Output: engine (6,H) or reference (H,6) layout, complex128 and/or complex64.
__global__ void k_pre_invert(const double2* __restrict__ gw, long long H, const double* __restrict__ meta, int soa,
                             double2* __restrict__ o128, float2* __restrict__ o64) {
  const double2 ab = make_double2(meta[0], meta[1]);
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < H; p += (long long)gridDim.x * blockDim.x) {
    double2 t[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) t[c] = make_double2(-gw[c * H + p].x, -gw[c * H + p].y);
    t[0] = cadd(t[0], ab); t[3] = cadd(t[3], ab); t[5] = cadd(t[5], ab);
    // symmetric [[a b c] [b d e] [c e f]]: inverse = cofactors / det
    const double2 a = t[0], b = t[1], c = t[2], dd = t[3], e = t[4], f = t[5];
    const double2 c00 = csub(cmul(dd, f), cmul(e, e));
    const double2 c01 = csub(cmul(c, e), cmul(b, f));
    const double2 c02 = csub(cmul(b, e), cmul(c, dd));
    const double2 c11 = csub(cmul(a, f), cmul(c, c));
    const double2 c12 = csub(cmul(b, c), cmul(a, e));
    const double2 c22 = csub(cmul(a, dd), cmul(b, b));
    const double2 det = cadd(cadd(cmul(a, c00), cmul(b, c01)), cmul(c, c02));
    const double den = det.x * det.x + det.y * det.y;
    const double2 id = make_double2(det.x / den, -det.y / den);
    const double2 r[6] = {cmul(c00, id), cmul(c01, id), cmul(c02, id), cmul(c11, id), cmul(c12, id), cmul(c22, id)};
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const long long off = soa ? (long long)q * H + p : p * 6 + q;
      if (o128) o128[off] = r[q];
      if (o64) o64[off] = make_float2((float)r[q].x, (float)r[q].y);
    }
  }
}

typedef void (*PZ)(double2*, long long, int, const double2*);
typedef void (*PC)(double2*, int, int, int, int, int, const double2*);
typedef void (*PG)(Geo, const double2*, double, double, int, const double2*, int, int, int, double2*);

static PZ pre_fft_z(int L) {
  switch (L) {
#define DDA_K(n) case n: return k_pre_fft_z<n>;
    DDA_FFT_SIZES(DDA_K)
#undef DDA_K
  }
  return nullptr;
}
static PC pre_fft_col(int L, int ax) {
  switch (L) {
#define DDA_K(n) case n: return ax == 1 ? (PC)k_pre_fft_col<1, n> : (PC)k_pre_fft_col<0, n>;
    DDA_FFT_SIZES(DDA_K)
#undef DDA_K
  }
  return nullptr;
}
static PG pre_green_z(int L) {
  switch (L) {
#define DDA_K(n) case n: return k_pre_z<n>;
    DDA_FFT_SIZES(DDA_K)
#undef DDA_K
  }
  return nullptr;
}

static int next_compiled(int n) {
  int best = 0;
#define DDA_K(m) if ((m) >= n && (best == 0 || (m) < best)) best = (m);
  DDA_FFT_SIZES(DDA_K)
#undef DDA_K
  return best;
}

// forward 3D FFT in place of the (Ax,Ay,Az) complex FP64 field A
static cudaError_t fft3(Ctx& ctx, double2* A, int Ax, int Ay, int Az, cudaStream_t s) {
  const int cap = PEPT * PNT;
  PZ kz = pre_fft_z(Az);
  PC ky = pre_fft_col(Ay, 1), kx = pre_fft_col(Ax, 0);
  if (!kz || !ky || !kx) return cudaErrorInvalidValue;
  const double2* twx = (const double2*)ctx.twiddles(Ax, true);
  const double2* twy = (const double2*)ctx.twiddles(Ay, true);
  const double2* twz = (const double2*)ctx.twiddles(Az, true);
  if (!twx || !twy || !twz) return cudaErrorMemoryAllocation;
  cudaError_t e;
  if ((e = cudaFuncSetAttribute((const void*)kz, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024))) return e;
  if ((e = cudaFuncSetAttribute((const void*)ky, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024))) return e;
  if ((e = cudaFuncSetAttribute((const void*)kx, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024))) return e;
  const long long nlines = (long long)Ax * Ay;
  const int NL = cap / Az;
  kz<<<(unsigned)((nlines + NL - 1) / NL), PNT, (size_t)NL * Az * sizeof(double2), s>>>(A, nlines, NL, twz);
  int Tz = std::min(cap / Ay, Az), ntz = (Az + Tz - 1) / Tz;
  ky<<<(unsigned)(Ax * ntz), PNT, (size_t)Ay * Tz * sizeof(double2), s>>>(A, Ax, Ay, Az, Tz, ntz, twy);
  Tz = std::min(cap / Ax, Az);
  ntz = (Az + Tz - 1) / Tz;
  kx<<<(unsigned)(Ay * ntz), PNT, (size_t)Ax * Tz * sizeof(double2), s>>>(A, Ax, Ay, Az, Tz, ntz, twx);
  note_launch(s, 3);
  return cudaGetLastError();
}

int precond_build(Ctx& ctx, const Geo& g, double k, double d, const void* inv_alpha128, int layout, void* out128,
                  void* out64, cudaStream_t s) {
  const int cap = PEPT * PNT;
  const int Ax = next_compiled(2 * g.nx), Ay = next_compiled(2 * g.ny), Az = next_compiled(2 * g.nz);
  if (!Ax || !Ay || !Az) {
    set_error("preconditioner: box too large for the occupancy autocorrelation (2n <= 512)");
    return DDA_ERR_BAD_SHAPE;
  }
  PG kz = pre_green_z(g.Lz);
  if (!kz || 6 * g.Lz > cap) {
    set_error("preconditioner: FFT length has no compiled kernel");
    return DDA_ERR_BAD_SHAPE;
  }
  const long long nA = (long long)Ax * Ay * Az;
  const long long H = (long long)g.hx * g.hy * g.hz;
  const size_t n1 = (size_t)g.Lx * g.Ly * g.hz * 6;
  double2 *A = nullptr, *b1 = nullptr, *gw = nullptr;
  double* meta = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&A, nA * sizeof(double2), s);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&b1, n1 * sizeof(double2), s);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&gw, (size_t)H * 6 * sizeof(double2), s);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&meta, 4 * sizeof(double), s);
  auto release = [&]() {
    if (A) cudaFreeAsync(A, s);
    if (b1) cudaFreeAsync(b1, s);
    if (gw) cudaFreeAsync(gw, s);
    if (meta) cudaFreeAsync(meta, s);
  };
  if (e != cudaSuccess) {
    cudaGetLastError();
    release();
    set_error("preconditioner: out of device memory");
    return DDA_ERR_OOM;
  }
  const double2* ia = (const double2*)inv_alpha128;
  k_pre_abar<<<1, 1024, 0, s>>>(ia, g.nsite, meta);
  const int gb = (int)std::min<long long>((nA + 255) / 256, 8 * ctx.num_sms);
  k_pre_occ<<<gb, 256, 0, s>>>(ia, g.nx, g.ny, g.nz, Ax, Ay, Az, A);
  note_launch(s, 2);
  if ((e = fft3(ctx, A, Ax, Ay, Az, s)) == cudaSuccess) {
    k_pre_abs2<<<gb, 256, 0, s>>>(A, nA);
    note_launch(s, 1);
    e = fft3(ctx, A, Ax, Ay, Az, s);
  }
  int rc = DDA_OK;
  if (e == cudaSuccess) {
    const double2* twz = (const double2*)ctx.twiddles(g.Lz, true);
    e = twz ? cudaFuncSetAttribute((const void*)kz, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024)
            : cudaErrorMemoryAllocation;
    if (e == cudaSuccess) {
      const int NL = cap / (6 * g.Lz);
      const long long grid1 = ((long long)g.Lx * g.Ly + NL - 1) / NL;
      kz<<<(unsigned)grid1, PNT, (size_t)NL * 6 * g.Lz * sizeof(double2), s>>>(g, twz, k, d, NL, A, Ax, Ay, Az, b1);
      note_launch(s, 1);
      e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess) {
    rc = green_yx(ctx, g, b1, 1.0, gw, nullptr, 1, s);
    if (rc == DDA_OK) {
      const int gi = (int)std::min<long long>((H + 255) / 256, 8 * ctx.num_sms);
      k_pre_invert<<<gi, 256, 0, s>>>(gw, H, meta, layout == DDA_GHAT_ENGINE ? 1 : 0, (double2*)out128,
                                     (float2*)out64);
      note_launch(s, 1);
      e = cudaGetLastError();
    }
  }
  release();
  if (rc != DDA_OK) return rc;
  if (e != cudaSuccess) {
    set_error(std::string("preconditioner: ") + cudaGetErrorString(e));
    return DDA_ERR_CUDA;
  }
  return DDA_OK;
}

}  // namespace dda
