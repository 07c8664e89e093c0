// Far-field scattering amplitude of a dipole lattice (not in the reference;
// the standard DDA far field, Draine 1988, in the reference's Gaussian units):
//
//   F(n) = k^2 sum_j [P_j - n (n . P_j)] exp(-i k n . r_j),   r_j = (i, j, k) d
//
// so the scattered field is E_sca = F(n) exp(ikr) / r, dC_sca/dOmega =
// |F|^2 / |E0|^2, and F at the incidence direction gives C_ext through the
// optical theorem.  The origin of r_j is the one the incident field uses
// (ddaforgit.py:1626-1632), so phases are consistent with E_inc.
//
// Work is (sites x directions): CTA (b, d) sums site block b for direction d
// in FP64 (phase from FP64 sincos), the partials of a direction are then added
// in a fixed order (deterministic).
#include <cmath>
#include <string>
#include <vector>

#include "../../include/dda_b200.h"
#include "dda_host.h"
#include "reduce.cuh"

namespace dda {

constexpr int kFFSites = KNT * 8;     // sites per CTA

template <typename R>
__global__ void __launch_bounds__(KNT) k_farfield_part(const typename CT<R>::T* __restrict__ P, int nx, int ny, int nz,
                                                       double d, double k, const double* __restrict__ dirs,
                                                       int nblk, double* __restrict__ part) {
  typedef typename CT<R>::T C;
  const int dir = blockIdx.y;
  const double ux = dirs[3 * dir], uy = dirs[3 * dir + 1], uz = dirs[3 * dir + 2];
  const long long nsite = (long long)nx * ny * nz;
  double acc[6] = {0, 0, 0, 0, 0, 0};   // sum_j P_j exp(-i k n.r_j), 3 complex
  const long long b0 = (long long)blockIdx.x * kFFSites;
  for (int q = threadIdx.x; q < kFFSites; q += KNT) {
    const long long site = b0 + q;
    if (site >= nsite) break;
    const C p0 = P[site * 3], p1 = P[site * 3 + 1], p2 = P[site * 3 + 2];
    if (p0.x == (R)0 && p0.y == (R)0 && p1.x == (R)0 && p1.y == (R)0 && p2.x == (R)0 && p2.y == (R)0) continue;
    const int iz = (int)(site % nz);
    const long long r = site / nz;
    const int iy = (int)(r % ny), ix = (int)(r / ny);
    const double ph = -k * d * (ux * ix + uy * iy + uz * iz);
    double sn, cs;
    sincos(ph, &sn, &cs);
    acc[0] += p0.x * cs - p0.y * sn; acc[1] += p0.x * sn + p0.y * cs;
    acc[2] += p1.x * cs - p1.y * sn; acc[3] += p1.x * sn + p1.y * cs;
    acc[4] += p2.x * cs - p2.y * sn; acc[5] += p2.x * sn + p2.y * cs;
  }
  __shared__ double sh[6][KNW];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    const double s = warp_sum(acc[c]);
    if (lane == 0) sh[c][wid] = s;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double s = 0.0;
    for (int w = 0; w < KNW; ++w) s += sh[threadIdx.x][w];
    part[((size_t)dir * nblk + blockIdx.x) * 6 + threadIdx.x] = s;
  }
}

// fixed-order sum of the partials, transverse projection and k^2 factor:
// out[dir*6 + 2c + {0,1}] = (Re, Im) F_c(n)
__global__ void k_farfield_sum(const double* __restrict__ part, int nblk, int ndir, const double* __restrict__ dirs,
                               double k, double* __restrict__ out) {
  const int dir = blockIdx.x * blockDim.x + threadIdx.x;
  if (dir >= ndir) return;
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (int b = 0; b < nblk; ++b)
    for (int c = 0; c < 6; ++c) s[c] += part[((size_t)dir * nblk + b) * 6 + c];
  const double u[3] = {dirs[3 * dir], dirs[3 * dir + 1], dirs[3 * dir + 2]};
  const double dre = u[0] * s[0] + u[1] * s[2] + u[2] * s[4];
  const double dim = u[0] * s[1] + u[1] * s[3] + u[2] * s[5];
  const double k2 = k * k;
  for (int c = 0; c < 3; ++c) {
    out[dir * 6 + 2 * c] = k2 * (s[2 * c] - u[c] * dre);
    out[dir * 6 + 2 * c + 1] = k2 * (s[2 * c + 1] - u[c] * dim);
  }
}

}  // namespace dda

using namespace dda;

struct dda_ctx {
  Ctx c;
};

extern "C" int dda_far_field(dda_ctx* ctx, int dtype, int nx, int ny, int nz, double d, double k, const void* p,
                             int ndir, const double* dirs3, double* out6, void* stream) {
  if (!ctx || !p || !dirs3 || !out6 || ndir < 1 || ndir > 65535 || nx < 1 || ny < 1 || nz < 1) {
    set_error("far field: bad arguments");
    return DDA_ERR_ARG;
  }
  if (dtype != DDA_C64 && dtype != DDA_C128) { set_error("far field: bad dtype"); return DDA_ERR_ARG; }
  cudaSetDevice(ctx->c.device);
  cudaStream_t s = ctx->c.stream;
  cudaStream_t user = (cudaStream_t)stream;
  DDA_CUDA_OK(cudaEventRecord(ctx->c.ev_user, user));
  DDA_CUDA_OK(cudaStreamWaitEvent(s, ctx->c.ev_user, 0));
  // unit directions
  std::vector<double> u(3 * (size_t)ndir);
  for (int i = 0; i < ndir; ++i) {
    const double x = dirs3[3 * i], y = dirs3[3 * i + 1], z = dirs3[3 * i + 2];
    const double n = std::sqrt(x * x + y * y + z * z);
    if (!(n > 0)) { set_error("far field: zero direction"); return DDA_ERR_ARG; }
    u[3 * i] = x / n; u[3 * i + 1] = y / n; u[3 * i + 2] = z / n;
  }
  const long long nsite = (long long)nx * ny * nz;
  const int nblk = (int)((nsite + kFFSites - 1) / kFFSites);
  double *d_dirs = nullptr, *d_part = nullptr, *d_out = nullptr;
  DDA_CUDA_OK(cudaMallocAsync((void**)&d_dirs, u.size() * sizeof(double), s));
  cudaError_t e = cudaMallocAsync((void**)&d_part, (size_t)ndir * nblk * 6 * sizeof(double), s);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&d_out, (size_t)ndir * 6 * sizeof(double), s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_dirs, u.data(), u.size() * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    if (dtype == DDA_C64)
      k_farfield_part<float><<<dim3(nblk, ndir), KNT, 0, s>>>((const float2*)p, nx, ny, nz, d, k, d_dirs, nblk,
                                                              d_part);
    else
      k_farfield_part<double><<<dim3(nblk, ndir), KNT, 0, s>>>((const double2*)p, nx, ny, nz, d, k, d_dirs, nblk,
                                                               d_part);
    k_farfield_sum<<<(ndir + 127) / 128, 128, 0, s>>>(d_part, nblk, ndir, d_dirs, k, d_out);
    note_launch(s, 2);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out6, d_out, (size_t)ndir * 6 * sizeof(double), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(d_dirs, s);
  if (d_part) cudaFreeAsync(d_part, s);
  if (d_out) cudaFreeAsync(d_out, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) { set_error(std::string("far field: ") + cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  return DDA_OK;
}
