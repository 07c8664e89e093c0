// Common device helpers for the B200 DDA engine: complex arithmetic on
// float2 / double2, the per-instance solver state, and launch constants.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace dda {

// ---------------------------------------------------------------------------
// complex type traits: R = float -> float2 (complex64), double -> double2
// ---------------------------------------------------------------------------
template <typename R> struct CT;
template <> struct CT<float> { typedef float2 T; };
template <> struct CT<double> { typedef double2 T; };

template <class C> __host__ __device__ __forceinline__ C mk(double re, double im) {
  C c; c.x = (decltype(c.x))re; c.y = (decltype(c.y))im; return c;
}
template <class C> __device__ __forceinline__ C cadd(C a, C b) { C c; c.x = a.x + b.x; c.y = a.y + b.y; return c; }
template <class C> __device__ __forceinline__ C csub(C a, C b) { C c; c.x = a.x - b.x; c.y = a.y - b.y; return c; }
template <class C> __device__ __forceinline__ C cmul(C a, C b) {
  C c; c.x = a.x * b.x - a.y * b.y; c.y = a.x * b.y + a.y * b.x; return c;
}
// conj(a) * b
template <class C> __device__ __forceinline__ C cmulc(C a, C b) {
  C c; c.x = a.x * b.x + a.y * b.y; c.y = a.x * b.y - a.y * b.x; return c;
}
template <class C, typename S> __device__ __forceinline__ C cscale(C a, S s) { C c; c.x = a.x * s; c.y = a.y * s; return c; }
template <class C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
// multiply by -i
template <class C> __device__ __forceinline__ C cmul_mi(C a) { C c; c.x = a.y; c.y = -a.x; return c; }
template <class C> __device__ __forceinline__ C czero() { C c; c.x = 0; c.y = 0; return c; }

// complex64 add / subtract / real scale as single packed sm_100 float2
// instructions (round-to-nearest, bitwise the same results as the two scalar
// operations they replace); off by default (see DDA_PACKED_F32).
#ifndef DDA_PACKED_F32
#define DDA_PACKED_F32 0
#endif
#if DDA_PACKED_F32 && defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
#endif

// Programmatic dependent launch: a kernel launched with the
// programmatic-stream-serialization attribute may start while its
// predecessor drains; grid_dep_begin() waits until the predecessor has
// completed and its memory is visible, then lets this kernel's own successor
// start launching (every CTA of this grid is resident by then).  Without the
// attribute both instructions return at once.
__device__ __forceinline__ void grid_dep_begin() {
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 900)
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}

// complex double helpers used by the scalar control logic
__device__ __forceinline__ double2 zmul(double2 a, double2 b) { return cmul(a, b); }
__device__ __forceinline__ double2 zdiv(double2 a, double2 b) {
  // plain complex division; scalars here are O(1) so no scaling is needed
  double den = b.x * b.x + b.y * b.y;
  double2 c; c.x = (a.x * b.x + a.y * b.y) / den; c.y = (a.y * b.x - a.x * b.y) / den; return c;
}
__device__ __forceinline__ double2 zsub(double2 a, double2 b) { return csub(a, b); }

// convert complex between precisions
template <class D, class S> __device__ __forceinline__ D ccvt(S s) {
  D d; d.x = (decltype(d.x))s.x; d.y = (decltype(d.y))s.y; return d;
}

// ---------------------------------------------------------------------------
// geometry of one batch bucket: box (nx,ny,nz) and FFT lengths (Lx,Ly,Lz)
// ---------------------------------------------------------------------------
struct Geo {
  int nx, ny, nz;
  int Lx, Ly, Lz;
  int hx, hy, hz;     // octant extents L/2+1
  long long nsite;    // nx*ny*nz
  // L2 prefetch distance, in CTAs, of the x pass and of the y passes (each
  // CTA prefetches the input rows of the CTA that far ahead; 0 = none)
  int pf3 = 0, pf2 = 0;
};

// Largest number of Stockham stages a length may need (L <= 4096).
constexpr int kMaxStages = 12;


// ---------------------------------------------------------------------------
// Logical vectors of one GPBiCGSTAB instance.  Kernels address vectors by
// these ids through InstState::vec, so the control logic can rotate buffers
// (s <-> s_prev, current / best iterate) on the device without copies.
// ---------------------------------------------------------------------------
enum VecId {
  V_R = 0, V_RHAT, V_P, V_V, V_T, V_S, V_SPREV, V_U, V_Z, V_W, V_Y,
  V_X, V_B, V_TMP, V_XA, V_XB, V_XC,
  V_MH,             // preconditioned vector M p / M s / M x (preconditioned solves only)
  kNumVec
};

// control condition under which a (matvec / update) kernel does work
enum Cond { C_ALWAYS = 0, C_ACTIVE = 1, C_TRUE_RES = 2, C_RESET_RES = 3, C_RESET = 4, C_LIVE = 5 };

// solver status codes (mirrors the sign convention of the reference's
// iteration return value)
enum SolveStatus { ST_RUNNING = 0, ST_CONVERGED = 1, ST_MAXITER = 2, ST_NAN = 3, ST_STAGNATED = 4 };

struct InstState {
  // vector table (device pointers, element type given by the batch dtype)
  void* vec[kNumVec];
  const void* ghat;    // octant of FFT(-G), engine layout (6,hx,hy,hz)
  const void* pghat;   // preconditioner octant, engine layout, on its own grid (or null)
  const void* inva;    // inverse polarizability per site (N complex)
  void* t1;            // scratch (nx,ny,Lz,3)
  void* t2;            // scratch (nx,Ly,Lz,3)
  // Occupied-site storage: when cidx is set, every vector of the instance
  // holds only the M sites with inv_alpha != 0 (site-major, component
  // fastest) and cidx[site] is the site's rank among them, -1 for an empty
  // site.  Empty sites carry zero in every Krylov vector of the reference's
  // recurrence (the right-hand side and every operator row are masked), so
  // dropping them changes no value.  nv = vector length in complex elements
  // (3M, or 3N when cidx is null).
  const int* cidx;
  long long nv;
  void* out;           // solution destination (dense (nx,ny,nz,3))
  // scalars (complex double)
  double2 rho1, rho0, alpha, beta, zeta, eta;
  double initial_norm, lowest, current, prev_lowest, first, target, ratio;
  double bnorm;        // ||b|| for reporting
  int iter;            // current iteration index i
  int max_iter;
  int last_change;
  int was_reset;
  int reset_count;
  int done;            // 1 once the reference's loop would have exited
  int status;          // SolveStatus
  int ret_iters;       // reference-style return code (iterations / -(i+1))
  int flag_true_res;   // r := b - A x needed this iteration (i == 1)
  int flag_reset;      // reset branch taken this iteration
  int flag_reset_res;  // reset branch recomputes the true residual
  int cur_x;           // which of XA/XB/XC holds the current iterate (0..2)
  int best_x;          // which holds the best iterate (0..2), -1 = none yet
  int active;          // 1 while the instance takes part in the batch
  int fault;           // set by a kernel whose bounded wait for its staged input gave up
  int pad_[2];
};

__device__ __forceinline__ bool cond_ok(const InstState& s, int cond) {
  switch (cond) {
    case C_ALWAYS: return true;
    case C_ACTIVE: return s.active && !s.done;
    case C_TRUE_RES: return s.active && !s.done && s.flag_true_res;
    case C_RESET_RES: return s.active && !s.done && s.flag_reset && s.flag_reset_res;
    case C_RESET: return s.active && !s.done;
    case C_LIVE: return s.active != 0;
  }
  return false;
}

}  // namespace dda
