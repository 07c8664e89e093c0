// Host-side internal declarations of the B200 DDA engine (not part of the
// public C ABI, which lives in include/dda_b200.h).
#pragma once
#include <cuda_runtime.h>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "dda_common.cuh"
#include "../../include/dda_b200.h"

namespace dda {

void set_error(const std::string& msg);

// Launch with programmatic stream serialization (the kernel must begin with
// grid_dep_begin()); DDA_NO_PDL=1 launches plainly.  Streams registered
// with set_stream_pdl(s, false) launch plainly too: slot pools run several
// streams at once, and a kernel launched early holds SM resources while it
// waits for its predecessor, which other streams' work could use.
bool pdl_enabled();
// Branches a batched matvec launch sequence of nb instances is split into
// (DDA_MV_SPLIT; 1 = one launch sequence over all instances).
int mv_split_ways(int nb);
bool stream_pdl(cudaStream_t s);
void set_stream_pdl(cudaStream_t s, bool on);
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = (pdl_enabled() && stream_pdl(s)) ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}
// Counts kernels this library enqueues (launches made while a stream is being
// captured into a graph are counted when the graph is launched instead).
void note_launch(cudaStream_t s, long long n);
long long launch_count();
const std::string& get_error();

#define DDA_CUDA_OK(expr)                                                        \
  do {                                                                           \
    cudaError_t e_ = (expr);                                                     \
    if (e_ != cudaSuccess) {                                                     \
      ::dda::set_error(std::string(#expr) + ": " + cudaGetErrorString(e_));      \
      return DDA_ERR_CUDA;                                                       \
    }                                                                            \
  } while (0)

// status codes shared with include/dda_b200.h
enum {
  DDA_OK_ = 0
};

// Twiddle tables per FFT length, in both precisions, resident on one device.
struct TwTable {
  void* d64 = nullptr;    // float2[L]
  void* d128 = nullptr;   // double2[L]
};

struct BatchWs;

struct Ctx {
  int device = 0;
  int num_sms = 148;
  std::mutex mu;
  std::map<int, TwTable> tw;
  std::map<std::string, BatchWs*> ws;
  cudaStream_t stream = nullptr;     // internal non-blocking stream
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaEvent_t ev_user = nullptr, ev_done = nullptr;
  // small reduction scratch for one-off reductions (cross sections)
  double* xred = nullptr;      // [xrb * 12]
  unsigned* xcnt = nullptr;
  double* xout = nullptr;      // [4] device
  double* xout_h = nullptr;    // [4] pinned
  int xrb = 1;
  // Concurrent branches of one batched launch sequence (mv_split): auxiliary
  // streams, fork / join events and instance indices 0..kIota-1 for launches
  // without an active list.  Made at context creation, so a fork needs no
  // allocation (it may be recorded into a graph).
  static constexpr int kMaxSplit = 4;
  static constexpr int kIota = 4096;
  cudaStream_t aux[kMaxSplit - 1] = {};
  cudaEvent_t ev_fork = nullptr;
  cudaEvent_t ev_join[kMaxSplit - 1] = {};
  int* iota = nullptr;
  std::mutex fork_mu;
  // returns device twiddles for length L (builds on first use)
  const void* twiddles(int L, bool dbl);
  // cached solver workspace for (dtype, geometry, batch size)
  // (tag separates workspaces of different users of the same shape)
  BatchWs* workspace(int dtype, const Geo& g, int nb, bool full, int* err, int tag = 0, const Geo* gp = nullptr);
  void trim();
  ~Ctx();
};

// Recycled pinned host blocks (cudaFreeHost would synchronise the device).
void* pinned_get(size_t bytes);
void pinned_put(void* p, size_t bytes);

// Launch geometry of the five matvec passes for one (Geo, dtype).
struct PassCfg {
  int nl = 1, th1 = 0;           // z passes: lines per CTA, threads
  int tz2 = 1, th2 = 0, ntz2 = 1;  // y passes: kz columns per CTA
  int tz3 = 1, th3 = 0, ntz3 = 1;  // x pass
  int p3reg = 0;                 // x pass keeps 3 components per thread
  int p3var = 0;                 // x pass kernel variant
  size_t smem1 = 0, smem2 = 0, smem3 = 0;
  long long grid1 = 0, grid2 = 0, grid3 = 0;
};

PassCfg make_pass_cfg(const Geo& g, bool dbl);

// Launch tuning table (DDA_TUNE_* flags of include/dda_b200.h) keyed by
// dtype, geometry and batch-width class (1, 2-3, 4-7, 8-15, 16+).
int nb_class(int nb);
int tune_flags(int dtype, const Geo& g, int nb);
void tune_set(int dtype, const Geo& g, int nb, int flags);
bool tune_get(int dtype, const Geo& g, int nb, int* flags);

// Preconditioner of a batched solve (the reference's right-preconditioned
// GPBiCGSTAB, precon=True): per-instance octants (engine layout) on the grid
// g.Lx/Ly/Lz (box g.nx/ny/nz, the solve's), applied as
//   M x = mask * scale * IFFT[ P . FFT(pad x) ]   (cropped to the box)
// i.e. the matvec passes in MV_CONV_MASKED mode with the x pass on
// InstState::pghat.
struct PreSpec {
  Geo g{};
  double scale = 1.0;
  const void* const* phat = nullptr;
};

// Device memory of a batch of solver instances sharing one geometry.
struct BatchWs {
  int dtype = 0, nb = 0, nslot = 0, RB = 1;
  bool full = true;
  bool pre = false;              // preconditioned solve: gp / pcp / pscale and the V_MH slot
  Geo g{};
  PassCfg pc{};
  Geo gp{};
  PassCfg pcp{};
  double pscale = 1.0, graph_pscale = 0.0;
  size_t esz = 8, n3 = 0, t1n = 0, t2n = 0;
  void* vecs = nullptr;          // nb * nslot * n3 complex
  void* scratch = nullptr;       // nb * (t1n + t2n) complex
  InstState* d_st = nullptr;
  InstState* h_st[2] = {nullptr, nullptr};   // pinned status buffers
  double* red = nullptr;
  unsigned* cnt = nullptr;
  int* cidx = nullptr;           // nb * nsite occupied-site maps (full workspaces)
  int* bcount = nullptr;         // nb * site_blocks(nsite) block offsets
  double* d_out = nullptr;
  double* h_out = nullptr;
  cudaGraphExec_t gexec = nullptr;
  double graph_gscale = 0.0;
  long long graph_kernels = 0;
  // set before alloc: device buffers come from the stream-ordered pool on
  // this stream and are freed on it (no device-wide synchronisation)
  cudaStream_t astream = nullptr;
  size_t pin_bytes = 0, pin_out = 0;
  int alloc(Ctx& c, int dtype, const Geo& g, int nb, bool full, const Geo* gp = nullptr);
  // frees everything (idempotent; the destructor calls it)
  void release();
  // vector slots the workspace allocates, in storage order
  const int* slots() const;
  // state of instance j: vector slots and scratch; with `sites` the
  // instance stores occupied sites only (its map is built on the device)
  void base_state(int j, InstState& S, bool sites = false) const;
  ~BatchWs();
};

enum MvMode { MV_AX = 0, MV_RESIDUAL = 1, MV_CONV = 2, MV_CONV_MASKED = 3 };

// Krylov steps fused into a matvec: before the first pass (the input is
// formed on the fly) and after the last pass (a dot product of the output
// reduced across the grid, the scalar step run by the last CTA).
enum MvPre { MV_PRE_NONE = 0, MV_PRE_SY = 1 };                 // s = r - alpha v, y = s_prev - s - alpha w
enum MvPost { MV_POST_NONE = 0, MV_POST_ALPHA = 1, MV_POST_ZETA = 2 };
struct MvFuse {
  int pre = MV_PRE_NONE, post = MV_POST_NONE;
  double* red = nullptr;      // >= nb * grid1 * KRED doubles
  unsigned* cnt = nullptr;    // per-instance tickets
  int tensor = 0;             // octant of the x pass: 0 InstState::ghat, 1 InstState::pghat
  int skip = 0;               // 1: no pass 1 (T1 already holds it), 2: no pass 5 (T1 left for the next product)
};

// Enqueue the 5-pass matvec for a batch of instances that share Geo.
// Instance slots: st[act ? act[j] : j], j < nb.
template <typename R>
cudaError_t launch_matvec(Ctx& ctx, const Geo& g, const PassCfg& pc, InstState* st, const int* act, int nb,
                          int in_id, int out_id, int mode, int cond, double gscale, cudaStream_t s,
                          const MvFuse& fz = MvFuse());

// out = A M in over a preconditioner grid equal to the operator's, M in
// stored in mid_id, with M's last pass and A's first fused (launch_amul_impl
// in matvec_impl.cuh).
template <typename R>
cudaError_t launch_amul(Ctx& ctx, const Geo& g, const PassCfg& pc, InstState* st, const int* act, int nb,
                        int in_id, int mid_id, int out_id, int mode, int cond, double gscale, double pscale,
                        cudaStream_t s, const MvFuse& fz = MvFuse());
// Whether products A M use launch_amul (DDA_NO_MA_FUSE=1 turns it off).
bool ma_fuse_enabled();
// Inner (complex64) target of a mixed solve's later sweeps: what the FP64
// tolerance still needs from the current true relative residual, times a
// safety factor (0.8; DDA_SWEEP_SAFETY overrides), within [inner_tol, 0.5].
// B200, preconditioned mixed solves to 1e-6, factor 0.3 / 0.6 / 0.8 / 0.9:
// 64^3 sphere 29 / 28 / 26 / 26 inner iterations, 128^3 ellipsoid 26 / 25 /
// - / 24, every solve in two sweeps with true residual <= 1e-6.
double mixed_sweep_target(double inner_tol, double tol, double relres);
// Reset ratio of a mixed solve's complex64 sweeps.  The plain solves keep
// the reference's rule (reset at the third iteration and whenever the
// residual fell by `ratio` since the last reset, Gpbicgstab.py:1125-1158);
// the sweeps keep it with the ratio raised to at least 1000 (0 still
// means no resets; DDA_INNER_RATIO overrides): a reset restarts the
// recurrence, and the FP64 refinement around the sweeps is what guards the
// accuracy.  B200, preconditioned mixed solves to 1e-6, ratio 100 / 1000 /
// 0: 64^3 m = 1.7+0.1i 26 / 21 / 21 inner iterations (19.3 / 15.5 / 14.6
// ms for two RHS), m = 2.5+0.1i 57 / 54 / 49, m = 3.5+0.05i 829 / 777 / 909,
// 48^3 m = 3.5+0.5i 58 / 58 / 47, 96^3 m = 2+0.3i 21 / 19 / 16; all in two
// sweeps to true residual <= 1e-6.
double mixed_inner_ratio(double ratio);

// One matvec with explicit twiddle tables (allocation-free entry point).
template <typename R>
cudaError_t launch_matvec_tw(const Geo& g, const PassCfg& pc, InstState* st, const void* twx, const void* twy,
                             const void* twz, int in_id, int out_id, int mode, double gscale, cudaStream_t s);

// Batched GPBiCGSTAB kernels (krylov.cu); RB CTAs per instance.
struct KrylovLaunch {
  InstState* st; const int* act; int nb; double* red; unsigned* cnt; long long n3; int RB;
  // graph conditional handles set by the control code (0: none): the
  // true-residual matvec at i == 1 and the reset branch's residual matvec
  unsigned long long cond_true = 0, cond_reset = 0;
};
template <typename R> void launch_init(const KrylovLaunch& k, cudaStream_t s);
template <typename R> void launch_alpha(const KrylovLaunch& k, cudaStream_t s);
template <typename R> void launch_sy(const KrylovLaunch& k, cudaStream_t s);
template <typename R> void launch_zeta(const KrylovLaunch& k, cudaStream_t s);
template <typename R> void launch_uzrx(const KrylovLaunch& k, cudaStream_t s);
template <typename R> void launch_norm(const KrylovLaunch& k, cudaStream_t s);
template <typename R> void launch_fin(const KrylovLaunch& k, cudaStream_t s);

// One GPBiCGSTAB iteration for every instance of a workspace (solver.cu).
template <typename R>
cudaError_t enqueue_iteration(Ctx& c, BatchWs& w, double gscale, cudaStream_t s);
// The iteration as a CUDA graph whose two residual matvecs (i == 1, resets)
// sit in conditional nodes the control kernels switch on; falls back to the
// plain captured sequence where conditional nodes are unavailable.
template <typename R>
cudaError_t capture_iteration(Ctx& c, BatchWs& w, double gscale, cudaStream_t s, cudaGraph_t* out,
                              long long* kernels);

template <typename R>
int solve_batch(Ctx& c, const Geo& g, double gscale, const struct dda_instance* inst, int nb, double target,
                int max_iter, double ratio, struct dda_result* res, cudaStream_t user, const PreSpec* pre = nullptr);
// pre (optional) preconditions the complex64 sweeps; its octants are complex64
int solve_mixed(Ctx& c, const Geo& g, double gscale, const struct dda_instance* i64,
                const struct dda_instance* i128, int nb, double tol, double inner_tol, int max_iter, int max_outer,
                double ratio, struct dda_result* res, cudaStream_t user, const PreSpec* pre = nullptr);
template <typename R>
void launch_xsec(const void* P, const void* E, const void* ia, long long nsite, double k, double* red, unsigned* cnt,
                 int RB, double* out, cudaStream_t s);

// Batched helper kernels (util.cu); act = instance list (null: all nb).
template <typename R>
void launch_make_b(InstState* st, int nb, long long nsite, int src, int dst, int num_sms, cudaStream_t s,
                   const int* act);
void launch_down(InstState* dst, int did, const InstState* src, int sid, int nb, long long n3, int num_sms,
                 cudaStream_t s, const int* act);
void launch_accum(InstState* st128, int xid, const InstState* st64, int nb, long long n3, int num_sms,
                  cudaStream_t s, const int* act);
template <typename R>
void launch_norm2(InstState* st, int id, int nb, long long n3, double* red, unsigned* cnt, int RB, double* out,
                  cudaStream_t s, const int* act);
int grid_for(long long n, int nb, int num_sms);
// occupied-site maps of the instances (S.cidx set on the host beforehand)
int site_blocks(long long nsite);
template <typename R>
void launch_site_map(InstState* st, int nb, long long nsite, int* bcount, cudaStream_t s, const int* act);
// dense solution of each finished instance into S.out
template <typename R>
void launch_store_solution(InstState* st, int nb, long long n3, int num_sms, cudaStream_t s, const int* act);
// S.vec[V_TMP] := the iterate the solution store / refinement accumulate
// reads (converged: x; else the best iterate; else x)
void launch_pick_solution(InstState* st, int nb, cudaStream_t s, const int* act);

// Preconditioner builder (precond.cu): octant (engine or reference layout)
// of the occupancy-weighted circulant inverse on the grid g.Lx/Ly/Lz; see
// dda_precond_build.
int precond_build(Ctx& ctx, const Geo& g, double k, double d, const void* inv_alpha128, int layout, void* out128,
                  void* out64, cudaStream_t s);
// The y and x passes of the Green build from the z pass's output b1
// (Lx,Ly,hz,6) FP64: octant of -scale * FFT (green.cu).
int green_yx(Ctx& ctx, const Geo& g, const void* b1, double scale, void* out128, void* out64, int soa,
             cudaStream_t s);
// whether solver workspaces store occupied sites only (DDA_NO_COMPRESS=1: dense)
bool compress_sites();

// Lattice setup kernels (lattice.cu).
int voxelize(const dda_shape* shapes_dev, int nshape, int nx, int ny, int nz, double d, const double* origin,
             bool dbl, void* out, int num_sms, cudaStream_t s);
int plane_wave(int nx, int ny, int nz, double d, const double* kvec, const double* pol, bool dbl, void* out,
               int num_sms, cudaStream_t s);

// Green's tensor build: FFT(-G) octant (hx,hy,hz,6) scaled by `scale`.
// Writes complex128 to out128 (if non-null) and complex64 to out64 (if non-null).
// soa = 0: reference layout (hx,hy,hz,6); soa = 1: engine layout (6,hx,hy,hz).
int green_build(Ctx& ctx, const Geo& g, double k, double d, double scale, void* out128, void* out64, int soa,
                cudaStream_t s);
// Reference-layout octant -> engine layout (H = hx*hy*hz points).
int ghat_to_soa(const void* src, void* dst, long long H, bool dbl, cudaStream_t s);

}  // namespace dda
