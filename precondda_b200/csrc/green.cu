// Green's-tensor build: the 6 unique entries of the symmetric 3x3 block
//   G(r) = e^{ikr}/r [ k^2 (rr - I) + (ikr - 1)/r^2 (3 rr - I) ]
// on the (Lx,Ly,Lz) circulant embedding of the (nx,ny,nz) box, transformed
// once by three FFT passes and cropped to the reduced octant (hx,hy,hz,6),
// hn = Ln/2 + 1, stored as scale * FFT(-G).  G is evaluated on the fly inside
// the first pass, so the full embedded tensor is never materialised.
//
// Follows ddaforgit.py:939-1080 (greens_kernel_* + generate_interaction_row):
// origin zero (:955-958), wrap of indices >= n to negative offsets (:951-953),
// zero planes at the unused offsets (:983), FFT of the negated component and
// the octant crop (:1074-1077).  Everything is computed in FP64; the complex64
// copy is a rounding of the FP64 result.
#include "dda_host.h"
#include "fft_core.cuh"
#include "fft_sizes.h"

namespace dda {

constexpr int GEPT = 12, GNT = 256;   // FP64 tiles: L*W <= 3072

__device__ __forceinline__ double axis_pos(int i, int n, int L, bool& valid) {
  valid = (i <= n - 1) || (i >= L - n + 1);
  return (double)(i < n ? i : i - L);
}

// G1: z-FFT of NL full lines (ix,iy) with G computed in place; keeps kz < hz.
template <int LZ>
__global__ void __launch_bounds__(GNT) k_green_z(Geo g, const double2* __restrict__ tw, double k, double d, int NL,
                                                 double2* __restrict__ b1) {
  constexpr int LS = 6 * LZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* s = reinterpret_cast<double2*>(smem_raw);
  const long long nlines = (long long)g.Lx * g.Ly;
  const long long line0 = (long long)blockIdx.x * NL;
  for (int idx = threadIdx.x; idx < NL * g.Lz; idx += GNT) {
    const int l = idx / g.Lz, iz = idx - l * g.Lz;
    const long long line = line0 + l;
    double2 v[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) v[c] = make_double2(0.0, 0.0);
    if (line < nlines) {
      const int ix = (int)(line / g.Ly), iy = (int)(line - (long long)ix * g.Ly);
      bool vx, vy, vz;
      const double X = axis_pos(ix, g.nx, g.Lx, vx) * d;
      const double Y = axis_pos(iy, g.ny, g.Ly, vy) * d;
      const double Z = axis_pos(iz, g.nz, g.Lz, vz) * d;
      const double r2 = X * X + Y * Y + Z * Z;
      if (vx && vy && vz && r2 > 0.0) {
        const double r = sqrt(r2);
        const double ir = 1.0 / r;
        const double n0 = X * ir, n1 = Y * ir, n2 = Z * ir;
        const double kr = k * r;
        double sn, cs;
        sincos(kr, &sn, &cs);
        const double2 ex = make_double2(cs * ir, sn * ir);          // e^{ikr}/r
        const double2 f2 = make_double2(-1.0 / r2, kr / r2);        // (ikr - 1)/r^2
        const double nn[6] = {n0 * n0, n0 * n1, n0 * n2, n1 * n1, n1 * n2, n2 * n2};
        const double dl[6] = {1.0, 0.0, 0.0, 1.0, 0.0, 1.0};
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          const double t1 = k * k * (nn[c] - dl[c]);
          const double a = 3.0 * nn[c] - dl[c];
          const double2 t = make_double2(t1 + a * f2.x, a * f2.y);
          v[c] = cmul(ex, t);
        }
      }
    }
    double2* q = s + l * LS + iz * 6;
#pragma unroll
    for (int c = 0; c < 6; ++c) q[c] = v[c];
  }
  __syncthreads();
  LayLine<6> lay{NL, LS};
  fft_tile<LZ, false, GEPT, GNT>(s, lay, tw);
  for (int idx = threadIdx.x; idx < NL * g.hz * 6; idx += GNT) {
    const int l = idx / (g.hz * 6), rem = idx - l * g.hz * 6;
    const int kz = rem / 6, c = rem - kz * 6;
    const long long line = line0 + l;
    if (line < nlines) b1[(line * g.hz + kz) * 6 + c] = s[l * LS + kz * 6 + c];
  }
}

// G2 / G3: FFT along y (G2) or x (G3) of a column tile of W = 6*Tz entries.
// G2: src rows (ix, iy) of B1 -> B2 rows (ix, ky < hy)
// G3: src rows (ix, ky) of B2 -> octant rows (kx < hx, ky), negated and scaled
template <int AX, int L>
__global__ void __launch_bounds__(GNT) k_green_col(Geo g, const double2* __restrict__ tw, int Tz, int ntz,
                                                   const double2* __restrict__ src,
                                                   double2* __restrict__ dst128, float2* __restrict__ dst64,
                                                   double scale, int soa) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* s = reinterpret_cast<double2*>(smem_raw);
  const int o = blockIdx.x / ntz, kzt = blockIdx.x - o * ntz;   // o = ix (G2) or ky (G3)
  const int kz0 = kzt * Tz;
  const int tzn = min(Tz, g.hz - kz0);
  const int W = 6 * Tz, Wv = 6 * tzn;
  for (int idx = threadIdx.x; idx < L * W; idx += GNT) {
    const int r = idx / W, w = idx - r * W;
    double2 v = make_double2(0.0, 0.0);
    if (w < Wv) {
      long long row = (AX == 1) ? (long long)o * g.Ly + r : (long long)r * g.hy + o;
      v = src[(row * g.hz + kz0) * 6 + w];
    }
    s[r * W + w] = v;
  }
  __syncthreads();
  LayCol lay{W, W};
  fft_tile<L, false, GEPT, GNT>(s, lay, tw);
  const int hout = (AX == 1) ? g.hy : g.hx;
  for (int idx = threadIdx.x; idx < hout * Wv; idx += GNT) {
    const int r = idx / Wv, w = idx - r * Wv;
    const double2 v = s[r * W + w];
    if (AX == 1) {
      dst128[(((long long)o * g.hy + r) * g.hz + kz0) * 6 + w] = v;
    } else {
      // AoS (reference layout): (kx,ky,kz,6); SoA (engine layout): (6,kx,ky,kz)
      const long long pt = ((long long)r * g.hy + o) * g.hz + kz0 + w / 6;
      const long long off = soa ? (long long)(w % 6) * g.hx * g.hy * g.hz + pt : pt * 6 + (w % 6);
      const double2 u = make_double2(-scale * v.x, -scale * v.y);
      if (dst128) dst128[off] = u;
      if (dst64) dst64[off] = make_float2((float)u.x, (float)u.y);
    }
  }
}

typedef void (*GZ)(Geo, const double2*, double, double, int, double2*);
typedef void (*GC)(Geo, const double2*, int, int, const double2*, double2*, float2*, double, int);

static GZ green_z_kernel(int L) {
  switch (L) {
#define DDA_K(n) case n: return k_green_z<n>;
    DDA_FFT_SIZES(DDA_K)
#undef DDA_K
  }
  return nullptr;
}
static GC green_col_kernel(int L, int ax) {
  switch (L) {
#define DDA_K(n) case n: return ax == 1 ? (GC)k_green_col<1, n> : (GC)k_green_col<0, n>;
    DDA_FFT_SIZES(DDA_K)
#undef DDA_K
  }
  return nullptr;
}

// Reference (AoS) octant -> engine (SoA) octant, same precision.
template <class C>
__global__ void k_ghat_aos_to_soa(const C* __restrict__ src, C* __restrict__ dst, long long H) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < H * 6; i += (long long)gridDim.x * blockDim.x) {
    const long long p = i / 6;
    const int c = (int)(i - p * 6);
    dst[c * H + p] = src[i];
  }
}

int ghat_to_soa(const void* src, void* dst, long long H, bool dbl, cudaStream_t s) {
  const int blocks = (int)std::min<long long>((H * 6 + 255) / 256, 4096);
  if (dbl) k_ghat_aos_to_soa<double2><<<blocks, 256, 0, s>>>((const double2*)src, (double2*)dst, H);
  else k_ghat_aos_to_soa<float2><<<blocks, 256, 0, s>>>((const float2*)src, (float2*)dst, H);
  note_launch(s, 1);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int green_yx(Ctx& ctx, const Geo& g, const void* b1v, double scale, void* out128, void* out64, int soa,
             cudaStream_t s) {
  const int cap = GEPT * GNT;
  if (6 * g.Ly > cap || 6 * g.Lx > cap) {
    set_error("green_build: FFT length too large (max 512)");
    return 7;
  }
  GC ky = green_col_kernel(g.Ly, 1), kx = green_col_kernel(g.Lx, 0);
  if (!ky || !kx) {
    set_error("green_build: FFT length has no compiled kernel");
    return 7;
  }
  DDA_CUDA_OK(cudaFuncSetAttribute((const void*)ky, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  DDA_CUDA_OK(cudaFuncSetAttribute((const void*)kx, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  const double2* twx = (const double2*)ctx.twiddles(g.Lx, true);
  const double2* twy = (const double2*)ctx.twiddles(g.Ly, true);
  if (!twx || !twy) { set_error("green_build: twiddle allocation failed"); return 2; }
  const double2* b1 = (const double2*)b1v;
  const size_t n2 = (size_t)g.Lx * g.hy * g.hz * 6;
  double2* b2 = nullptr;
  if (cudaMallocAsync((void**)&b2, n2 * sizeof(double2), s) != cudaSuccess) {
    cudaGetLastError();
    set_error("green_build: out of memory");
    return 2;
  }
  // G2: y
  int Tz = cap / (6 * g.Ly);
  if (Tz > g.hz) Tz = g.hz;
  int ntz = (g.hz + Tz - 1) / Tz;
  ky<<<(unsigned)(g.Lx * ntz), GNT, (size_t)g.Ly * 6 * Tz * sizeof(double2), s>>>(g, twy, Tz, ntz, b1, b2, nullptr,
                                                                                  1.0, 0);
  // G3: x, negate, scale, crop to the octant
  Tz = cap / (6 * g.Lx);
  if (Tz > g.hz) Tz = g.hz;
  ntz = (g.hz + Tz - 1) / Tz;
  kx<<<(unsigned)(g.hy * ntz), GNT, (size_t)g.Lx * 6 * Tz * sizeof(double2), s>>>(g, twx, Tz, ntz, b2,
                                                                                  (double2*)out128, (float2*)out64,
                                                                                  scale, soa);
  note_launch(s, 2);
  const cudaError_t e = cudaGetLastError();
  cudaFreeAsync(b2, s);
  if (e != cudaSuccess) { set_error(std::string("green_build: ") + cudaGetErrorString(e)); return 6; }
  return 0;
}

int green_build(Ctx& ctx, const Geo& g, double k, double d, double scale, void* out128, void* out64, int soa,
                cudaStream_t s) {
  const int cap = GEPT * GNT;
  if (6 * g.Lz > cap) {
    set_error("green_build: FFT length too large (max 512)");
    return 7;
  }
  GZ kz = green_z_kernel(g.Lz);
  if (!kz) {
    set_error("green_build: FFT length has no compiled kernel");
    return 7;
  }
  DDA_CUDA_OK(cudaFuncSetAttribute((const void*)kz, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  const double2* twz = (const double2*)ctx.twiddles(g.Lz, true);
  if (!twz) { set_error("green_build: twiddle allocation failed"); return 2; }
  const size_t n1 = (size_t)g.Lx * g.Ly * g.hz * 6;
  double2* b1 = nullptr;
  if (cudaMallocAsync((void**)&b1, n1 * sizeof(double2), s) != cudaSuccess) {
    cudaGetLastError();
    set_error("green_build: out of memory");
    return 2;
  }
  // G1: z with G evaluated in place
  const int NL = cap / (6 * g.Lz);
  const long long grid1 = ((long long)g.Lx * g.Ly + NL - 1) / NL;
  kz<<<(unsigned)grid1, GNT, (size_t)NL * 6 * g.Lz * sizeof(double2), s>>>(g, twz, k, d, NL, b1);
  note_launch(s, 1);
  cudaError_t e = cudaGetLastError();
  int rc = 0;
  if (e != cudaSuccess) {
    set_error(std::string("green_build: ") + cudaGetErrorString(e));
    rc = 6;
  } else {
    rc = green_yx(ctx, g, b1, scale, out128, out64, soa, s);
  }
  cudaFreeAsync(b1, s);
  return rc;
}

}  // namespace dda
