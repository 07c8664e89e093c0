// Lattice setup on the device: voxelisation of shapes into the inverse
// polarizability array, and plane-wave incident fields.
//
// Membership tests follow the reference's Numba functions (ddaforgit.py:
// sphere :439-448, ellipsoid :450-459, rectangle :461-475, cylinder :477-509,
// prism :511-572) evaluated at voxel centres origin + (i+0.5) d
// (ddaforgit.py:617, :643-647); later shapes overwrite earlier ones as in
// mark_shapes (:656-661), and a shape with DDA_SHAPE_WINDOW marks only the
// index window mark_shapes evaluates it on (:626-649).  The reference's
// cylinder takes its radial distance in the (x, y) plane for every axis and,
// for the x and y axes, tests the signed z offset against height/2; that is
// the default here too (DDA_SHAPE_GEOMETRIC_AXES selects the perpendicular
// split).  The cylinder arithmetic uses round-to-nearest intrinsics, so no
// multiply-add is contracted and each operation rounds as the reference's
// does.  Extensions: an ellipsoid may carry a rotation (body -> lab matrix),
// and a sphere list expresses aggregates.
// The incident field is e exp(i k.r) with r = (i,j,k) d, no half-voxel offset
// (ddaforgit.py:1626-1632).
#include <algorithm>

#include "../../include/dda_b200.h"
#include "dda_host.h"

namespace dda {

constexpr double kEps = 1e-7;

__device__ bool inside(const dda_shape& s, double x, double y, double z) {
  const double dx = x - s.center[0], dy = y - s.center[1], dz = z - s.center[2];
  switch (s.type) {
    case DDA_SHAPE_SPHERE: {
      const double r = s.p[0];
      const double dist = sqrt(dx * dx + dy * dy + dz * dz);
      return (dist < r) || (fabs(dist - r) < kEps);
    }
    case DDA_SHAPE_ELLIPSOID: {
      // body-frame offset = R^T (lab offset)
      const double* R = s.rot;
      const double bx = R[0] * dx + R[3] * dy + R[6] * dz;
      const double by = R[1] * dx + R[4] * dy + R[7] * dz;
      const double bz = R[2] * dx + R[5] * dy + R[8] * dz;
      const double qx = bx / s.p[0], qy = by / s.p[1], qz = bz / s.p[2];
      return sqrt(qx * qx + qy * qy + qz * qz) <= 1.0 + kEps;
    }
    case DDA_SHAPE_RECTANGLE: {
      const double hx = s.p[0] / 2, hy = s.p[1] / 2, hz = s.p[2] / 2;
      const double ax = fabs(dx), ay = fabs(dy), az = fabs(dz);
      const bool in = ax <= hx && ay <= hy && az <= hz;
      const bool edge = (fabs(ax - hx) < kEps && ay <= hy && az <= hz) ||
                        (fabs(ay - hy) < kEps && ax <= hx && az <= hz) ||
                        (fabs(az - hz) < kEps && ax <= hx && ay <= hy);
      return in || edge;
    }
    case DDA_SHAPE_CYLINDER:
      if (!(s.flags & DDA_SHAPE_GEOMETRIC_AXES)) {
        const double r = s.p[0], hh = s.p[1] / 2;
        const double rd = sqrt(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
        const double h = s.axis == 2 ? fabs(dz) : dz;
        const bool inr = rd <= r, onr = fabs(rd - r) < kEps, inh = h <= hh, cap = fabs(h - hh) < kEps;
        return (inr && inh) || (onr && inh) || (inr && cap);
      }
      [[fallthrough]];
    case DDA_SHAPE_PRISM: {
      double u, v, h;      // in-plane offsets and axial distance
      if (s.axis == 0) { u = dy; v = dz; h = fabs(dx); }
      else if (s.axis == 1) { u = dx; v = dz; h = fabs(dy); }
      else { u = dx; v = dy; h = fabs(dz); }
      const double hh = s.p[1] / 2;
      if (s.type == DDA_SHAPE_CYLINDER) {
        const double r = s.p[0];
        const double rd = sqrt(u * u + v * v);
        const bool inr = rd <= r, onr = fabs(rd - r) < kEps, inh = h <= hh, cap = fabs(h - hh) < kEps;
        return (inr && inh) || (onr && inh) || (inr && cap);
      }
      // regular polygon of `sides` vertices at radius p[0]: even-odd rule,
      // points on an edge count as inside
      const int n = s.sides;
      const double r = s.p[0];
      bool in = false, edge = false;
      for (int j = 0; j < n && !edge; ++j) {
        const double a0 = 2.0 * M_PI * j / n, a1 = 2.0 * M_PI * ((j + 1) % n) / n;
        const double xi = r * cos(a0), yi = r * sin(a0), xj = r * cos(a1), yj = r * sin(a1);
        const double ex = xj - xi, ey = yj - yi;
        const double ln = sqrt(ex * ex + ey * ey);
        if (ln > kEps) {
          const double ux = ex / ln, uy = ey / ln, wx = u - xi, wy = v - yi;
          const double proj = wx * ux + wy * uy, dist = fabs(wx * uy - wy * ux);
          if (dist < kEps && proj >= -kEps && proj <= ln + kEps) { edge = true; break; }
        }
        if (((yi > v) != (yj > v)) && (u < (xj - xi) * (v - yi) / (yj - yi) + xi)) in = !in;
      }
      return (in || edge) && (h <= hh || fabs(h - hh) < kEps);
    }
  }
  return false;
}

template <typename R>
__global__ void k_voxelize(const dda_shape* __restrict__ shapes, int nshape, int nx, int ny, int nz, double d,
                           double ox, double oy, double oz, typename CT<R>::T* __restrict__ ia) {
  typedef typename CT<R>::T C;
  const long long n = (long long)nx * ny * nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(i % nz);
    const long long r = i / nz;
    const int iy = (int)(r % ny), ix = (int)(r / ny);
    const double x = ox + (ix + 0.5) * d, y = oy + (iy + 0.5) * d, z = oz + (iz + 0.5) * d;
    C v = czero<C>();
    for (int s = 0; s < nshape; ++s) {
      const dda_shape& sh = shapes[s];
      if ((sh.flags & DDA_SHAPE_WINDOW) && (ix < sh.win[0] || ix >= sh.win[1] || iy < sh.win[2] ||
                                            iy >= sh.win[3] || iz < sh.win[4] || iz >= sh.win[5]))
        continue;
      if (inside(sh, x, y, z)) v = mk<C>(sh.inv_alpha[0], sh.inv_alpha[1]);
    }
    ia[i] = v;
  }
}

template <typename R>
__global__ void k_plane_wave(int nx, int ny, int nz, double d, double kx, double ky, double kz, double e0r,
                             double e0i, double e1r, double e1i, double e2r, double e2i,
                             typename CT<R>::T* __restrict__ E) {
  typedef typename CT<R>::T C;
  const long long n = (long long)nx * ny * nz;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(i % nz);
    const long long r = i / nz;
    const int iy = (int)(r % ny), ix = (int)(r / ny);
    const double ph = kx * (ix * d) + ky * (iy * d) + kz * (iz * d);
    double sn, cs;
    sincos(ph, &sn, &cs);
    E[i * 3 + 0] = mk<C>(e0r * cs - e0i * sn, e0r * sn + e0i * cs);
    E[i * 3 + 1] = mk<C>(e1r * cs - e1i * sn, e1r * sn + e1i * cs);
    E[i * 3 + 2] = mk<C>(e2r * cs - e2i * sn, e2r * sn + e2i * cs);
  }
}

int voxelize(const dda_shape* shapes_dev, int nshape, int nx, int ny, int nz, double d, const double* origin,
             bool dbl, void* out, int num_sms, cudaStream_t s) {
  const long long n = (long long)nx * ny * nz;
  const int blocks = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 8LL * num_sms));
  if (dbl)
    k_voxelize<double><<<blocks, 256, 0, s>>>(shapes_dev, nshape, nx, ny, nz, d, origin[0], origin[1], origin[2],
                                              (double2*)out);
  else
    k_voxelize<float><<<blocks, 256, 0, s>>>(shapes_dev, nshape, nx, ny, nz, d, origin[0], origin[1], origin[2],
                                             (float2*)out);
  note_launch(s, 1);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

int plane_wave(int nx, int ny, int nz, double d, const double* kvec, const double* pol, bool dbl, void* out,
               int num_sms, cudaStream_t s) {
  const long long n = (long long)nx * ny * nz;
  const int blocks = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 8LL * num_sms));
  if (dbl)
    k_plane_wave<double><<<blocks, 256, 0, s>>>(nx, ny, nz, d, kvec[0], kvec[1], kvec[2], pol[0], pol[1], pol[2],
                                                pol[3], pol[4], pol[5], (double2*)out);
  else
    k_plane_wave<float><<<blocks, 256, 0, s>>>(nx, ny, nz, d, kvec[0], kvec[1], kvec[2], pol[0], pol[1], pol[2],
                                               pol[3], pol[4], pol[5], (float2*)out);
  note_launch(s, 1);
  return cudaGetLastError() == cudaSuccess ? 0 : 6;
}

}  // namespace dda
