// Host side of the engine: FFT plans and twiddles, solver workspaces, the
// batched GPBiCGSTAB driver (graph-captured iterations, pipelined status
// polling) and the mixed-precision iterative-refinement driver.
#include <algorithm>
#include <map>
#include <mutex>
#include <atomic>
#include <cmath>
#include <vector>
#include <cstring>
#include <string>

#include "../../include/dda_b200.h"
#include "dda_host.h"
#include "reduce.cuh"

namespace dda {

static thread_local std::string g_err;
void set_error(const std::string& m) { g_err = m; }

static std::atomic<long long> g_launches{0};
// kernels this thread enqueued into a stream capture (counted per captured
// segment by capture_iteration)
static thread_local long long g_captured = 0;
void note_launch(cudaStream_t s, long long n) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
    g_captured += n;
    return;
  }
  g_launches.fetch_add(n, std::memory_order_relaxed);
}
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }
const std::string& get_error() { return g_err; }



const void* Ctx::twiddles(int L, bool dbl) {
  std::lock_guard<std::mutex> g(mu);
  auto it = tw.find(L);
  if (it == tw.end()) {
    std::vector<double2> h(L);
    std::vector<float2> hf(L);
    const long double tau = 6.283185307179586476925286766559005768L;
    for (int j = 0; j < L; ++j) {
      const long double a = tau * (long double)j / (long double)L;
      const double c = (double)cosl(a), s = (double)-sinl(a);
      h[j] = make_double2(c, s);
      hf[j] = make_float2((float)c, (float)s);
    }
    TwTable t;
    if (cudaMalloc(&t.d128, L * sizeof(double2)) != cudaSuccess) return nullptr;
    if (cudaMalloc(&t.d64, L * sizeof(float2)) != cudaSuccess) { cudaFree(t.d128); return nullptr; }
    cudaMemcpy(t.d128, h.data(), L * sizeof(double2), cudaMemcpyHostToDevice);
    cudaMemcpy(t.d64, hf.data(), L * sizeof(float2), cudaMemcpyHostToDevice);
    it = tw.emplace(L, t).first;
  }
  return dbl ? it->second.d128 : it->second.d64;
}

Ctx::~Ctx() {
  for (auto& kv : tw) { cudaFree(kv.second.d64); cudaFree(kv.second.d128); }
}

// ---------------------------------------------------------------------------
// workspaces
// ---------------------------------------------------------------------------
static const int kFullSlots[] = {V_R, V_RHAT, V_P, V_V, V_T, V_S, V_SPREV, V_U, V_Z, V_W, V_Y, V_B, V_TMP,
                                 V_XA, V_XB, V_XC};
static const int kPreSlots[] = {V_R, V_RHAT, V_P, V_V, V_T, V_S, V_SPREV, V_U, V_Z, V_W, V_Y, V_B, V_TMP,
                                V_XA, V_XB, V_XC, V_MH};
static const int kLightSlots[] = {V_R, V_B};

const int* BatchWs::slots() const { return full ? (pre ? kPreSlots : kFullSlots) : kLightSlots; }

// Pinned host blocks are recycled by size instead of returned to the
// driver: cudaFreeHost synchronises the whole device, which would stall every
// other stream each time a short-lived workspace (a slot pool) goes away.
namespace {
std::mutex g_pin_mu;
std::multimap<size_t, void*> g_pin_free;
}  // namespace

void* pinned_get(size_t bytes) {
  {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    auto it = g_pin_free.find(bytes);
    if (it != g_pin_free.end()) {
      void* p = it->second;
      g_pin_free.erase(it);
      return p;
    }
  }
  void* p = nullptr;
  if (cudaMallocHost(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

void pinned_put(void* p, size_t bytes) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(g_pin_mu);
  g_pin_free.emplace(bytes, p);
}

// Device buffers come from the stream-ordered pool when the workspace has a
// stream of its own (slot pools): freeing them then orders after that
// stream's work instead of synchronising the device.
static cudaError_t ws_malloc(void** p, size_t bytes, cudaStream_t as) {
  return as ? cudaMallocAsync(p, bytes, as) : cudaMalloc(p, bytes);
}
static void ws_free(void* p, cudaStream_t as) {
  if (!p) return;
  if (as) cudaFreeAsync(p, as);
  else cudaFree(p);
}

void BatchWs::release() {
  if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
  ws_free(vecs, astream); ws_free(scratch, astream); ws_free(d_st, astream);
  ws_free(red, astream); ws_free(cnt, astream); ws_free(d_out, astream);
  ws_free(cidx, astream); ws_free(bcount, astream);
  vecs = scratch = nullptr; d_st = nullptr; red = nullptr; cnt = nullptr; d_out = nullptr;
  cidx = nullptr; bcount = nullptr;
  pinned_put(h_st[0], pin_bytes); pinned_put(h_st[1], pin_bytes); pinned_put(h_out, pin_out);
  h_st[0] = h_st[1] = nullptr; h_out = nullptr;
}

BatchWs::~BatchWs() { release(); }

int BatchWs::alloc(Ctx& c, int dtype_, const Geo& g_, int nb_, bool full_, const Geo* gp_) {
  dtype = dtype_; g = g_; nb = nb_; full = full_;
  pre = full && gp_ != nullptr;
  esz = dtype == DDA_C128 ? 16 : 8;
  n3 = (size_t)g.nsite * 3;
  nslot = full ? (pre ? (int)(sizeof(kPreSlots) / sizeof(int)) : (int)(sizeof(kFullSlots) / sizeof(int)))
               : (int)(sizeof(kLightSlots) / sizeof(int));
  pc = make_pass_cfg(g, dtype == DDA_C128);
  RB = grid_for((long long)n3, nb, c.num_sms);
  t1n = (size_t)g.nx * g.ny * g.Lz * 3;
  t2n = (size_t)g.nx * g.Ly * g.Lz * 3;
  if (pre) {
    // the preconditioner passes share the transform scratch
    gp = *gp_;
    pcp = make_pass_cfg(gp, dtype == DDA_C128);
    t1n = std::max(t1n, (size_t)gp.nx * gp.ny * gp.Lz * 3);
    t2n = std::max(t2n, (size_t)gp.nx * gp.Ly * gp.Lz * 3);
  }
  pin_bytes = (size_t)nb * sizeof(InstState);
  pin_out = (size_t)nb * sizeof(double);
  cudaStream_t as = astream;
  h_st[0] = (InstState*)pinned_get(pin_bytes);
  h_st[1] = (InstState*)pinned_get(pin_bytes);
  h_out = (double*)pinned_get(pin_out);
  if (ws_malloc(&vecs, (size_t)nb * nslot * n3 * esz, as) != cudaSuccess ||
      ws_malloc(&scratch, (size_t)nb * (t1n + t2n) * esz, as) != cudaSuccess ||
      ws_malloc((void**)&d_st, nb * sizeof(InstState), as) != cudaSuccess || !h_st[0] || !h_st[1] || !h_out ||
      ws_malloc((void**)&red, (size_t)nb * std::max<long long>(RB, pc.grid1) * KRED * sizeof(double), as) !=
          cudaSuccess ||
      ws_malloc((void**)&cnt, nb * sizeof(unsigned), as) != cudaSuccess ||
      ws_malloc((void**)&d_out, nb * sizeof(double), as) != cudaSuccess ||
      (full && (ws_malloc((void**)&cidx, (size_t)nb * g.nsite * sizeof(int), as) != cudaSuccess ||
                ws_malloc((void**)&bcount, (size_t)nb * site_blocks(g.nsite) * sizeof(int), as) != cudaSuccess))) {
    cudaGetLastError();
    set_error("solver workspace: out of device memory");
    return DDA_ERR_OOM;
  }
  if (as) cudaMemsetAsync(cnt, 0, nb * sizeof(unsigned), as);
  else cudaMemset(cnt, 0, nb * sizeof(unsigned));
  std::memset(h_st[0], 0, nb * sizeof(InstState));
  return DDA_OK;
}

bool compress_sites() {
  const char* e = getenv("DDA_NO_COMPRESS");
  return !(e && *e == '1');
}

// base InstState of instance j: vector slots and scratch
void BatchWs::base_state(int j, InstState& S, bool sites) const {
  std::memset(&S, 0, sizeof(S));
  S.nv = (long long)n3;
  S.cidx = (sites && cidx) ? cidx + (size_t)j * g.nsite : nullptr;
  const int* sl = slots();
  char* v0 = (char*)vecs + (size_t)j * nslot * n3 * esz;
  for (int q = 0; q < nslot; ++q) S.vec[sl[q]] = v0 + (size_t)q * n3 * esz;
  if (full) S.vec[V_X] = S.vec[V_XA];
  char* sc = (char*)scratch + (size_t)j * (t1n + t2n) * esz;
  S.t1 = sc;
  S.t2 = sc + t1n * esz;
  S.best_x = -1;
}

BatchWs* Ctx::workspace(int dtype, const Geo& g, int nb, bool full, int* err, int tag, const Geo* gp) {
  char key[200];
  snprintf(key, sizeof(key), "%d:%d,%d,%d:%d,%d,%d:%d:%d:%d:p%d,%d,%d", dtype, g.nx, g.ny, g.nz, g.Lx, g.Ly, g.Lz,
           nb, full ? 1 : 0, tag, gp ? gp->Lx : 0, gp ? gp->Ly : 0, gp ? gp->Lz : 0);
  std::lock_guard<std::mutex> lk(mu);
  auto it = ws.find(key);
  if (it != ws.end()) return it->second;
  BatchWs* w = new BatchWs();
  const int e = w->alloc(*this, dtype, g, nb, full, gp);
  if (e != DDA_OK) { delete w; *err = e; return nullptr; }
  ws[key] = w;
  return w;
}

void Ctx::trim() {
  std::lock_guard<std::mutex> lk(mu);
  for (auto& kv : ws) delete kv.second;
  ws.clear();
}

// ---------------------------------------------------------------------------
// one GPBiCGSTAB iteration for every instance of the workspace
// ---------------------------------------------------------------------------
// DDA_FUSE_KRYLOV=1 lets the Krylov steps alpha (<rhat, v>), s / y and
// zeta / eta ride on the two matvecs (dot products in the last pass, s and y
// formed in the first -- M's first pass in a preconditioned solve) instead of
// three separate kernels.  Measured on B200 it is no faster overall: with
// the preconditioner's last pass fused into A's first (launch_amul),
// preconditioned 64^3 x 2 RHS mixed 112.3 against 111.7 solves/s and 128^3
// x 2 RHS 14.05 against 15.22; before that fusion, 64^3 108.7 against
// 108.4, c128 60.8 against 61.6, 128^3 x 16 RHS 15.76 against 15.66, plain
// c128 32^3 197.6 against 189.0.  The separate kernels are the default.
static bool fuse_krylov() {
  const char* e = getenv("DDA_FUSE_KRYLOV");
  return e && *e == '1';
}

// out = A in, or A M in for a preconditioned workspace (M in goes to V_MH):
// Gpbicgstab.py:1008-1015, :1026-1033 and the residuals :1061-1064, :1143-1144.
// fz carries the fused Krylov steps: `pre` goes to the first product (M when
// preconditioned, so s and y are formed by M's first pass), `post` to A.
template <typename R>
static cudaError_t amul(Ctx& c, BatchWs& w, int in, int out, int mode, int cond, double gscale, cudaStream_t s,
                        const MvFuse& fz = MvFuse()) {
  MvFuse fa = fz;
  if (w.pre && ma_fuse_enabled() && w.gp.nx == w.g.nx && w.gp.ny == w.g.ny && w.gp.nz == w.g.nz &&
      w.gp.Lx == w.g.Lx && w.gp.Ly == w.g.Ly && w.gp.Lz == w.g.Lz) {
    // M's last pass and A's first in one kernel: A's first pass reads no vector
    return launch_amul<R>(c, w.g, w.pc, w.d_st, nullptr, w.nb, in, V_MH, out, mode, cond, gscale, w.pscale, s, fz);
  }
  if (w.pre) {
    MvFuse fm;
    fm.tensor = 1;
    fm.pre = fz.pre;
    cudaError_t e = launch_matvec<R>(c, w.gp, w.pcp, w.d_st, nullptr, w.nb, in, V_MH, MV_CONV_MASKED, cond, w.pscale,
                                     s, fm);
    if (e != cudaSuccess) return e;
    in = V_MH;
    fa.pre = MV_PRE_NONE;
  }
  return launch_matvec<R>(c, w.g, w.pc, w.d_st, nullptr, w.nb, in, out, mode, cond, gscale, s, fa);
}

template <typename R>
static cudaError_t enqueue_front(Ctx& c, BatchWs& w, double gscale, cudaStream_t s, const KrylovLaunch& k) {
  cudaError_t e;
  if (fuse_krylov()) {
    MvFuse f1, f2;
    f1.post = MV_POST_ALPHA; f1.red = w.red; f1.cnt = w.cnt;
    f2.pre = MV_PRE_SY; f2.post = MV_POST_ZETA; f2.red = w.red; f2.cnt = w.cnt;
    if ((e = amul<R>(c, w, V_P, V_V, MV_AX, C_ACTIVE, gscale, s, f1))) return e;
    if ((e = amul<R>(c, w, V_S, V_T, MV_AX, C_ACTIVE, gscale, s, f2))) return e;
  } else {
    if ((e = amul<R>(c, w, V_P, V_V, MV_AX, C_ACTIVE, gscale, s))) return e;
    launch_alpha<R>(k, s);
    launch_sy<R>(k, s);
    if ((e = amul<R>(c, w, V_S, V_T, MV_AX, C_ACTIVE, gscale, s))) return e;
    launch_zeta<R>(k, s);
  }
  launch_uzrx<R>(k, s);
  return cudaGetLastError();
}

template <typename R>
cudaError_t enqueue_iteration(Ctx& c, BatchWs& w, double gscale, cudaStream_t s) {
  KrylovLaunch k{w.d_st, nullptr, w.nb, w.red, w.cnt, (long long)w.n3, w.RB};
  cudaError_t e;
  if ((e = enqueue_front<R>(c, w, gscale, s, k))) return e;
  if ((e = amul<R>(c, w, V_X, V_R, MV_RESIDUAL, C_TRUE_RES, gscale, s))) return e;
  launch_norm<R>(k, s);
  if ((e = amul<R>(c, w, V_X, V_R, MV_RESIDUAL, C_RESET_RES, gscale, s))) return e;
  launch_fin<R>(k, s);
  return cudaGetLastError();
}

template cudaError_t enqueue_iteration<float>(Ctx&, BatchWs&, double, cudaStream_t);
template cudaError_t enqueue_iteration<double>(Ctx&, BatchWs&, double, cudaStream_t);

namespace {
// Capture launches issued by `fn` on stream s into graph G after `deps`;
// returns the capture's final dependencies (the segment's sink nodes).
template <class F>
cudaError_t capture_segment(cudaStream_t s, cudaGraph_t G, const std::vector<cudaGraphNode_t>& deps,
                            std::vector<cudaGraphNode_t>& sinks, F fn) {
  cudaError_t e = cudaStreamBeginCaptureToGraph(s, G, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                                cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  cudaError_t ef = fn();
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t* d = nullptr;
  size_t nd = 0;
  cudaError_t ei = cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &d, &nd);
  if (ei == cudaSuccess) sinks.assign(d, d + nd);
  cudaGraph_t g2 = nullptr;
  cudaError_t ee = cudaStreamEndCapture(s, &g2);
  return ef != cudaSuccess ? ef : (ei != cudaSuccess ? ei : ee);
}

// IF node on handle h after `deps`; its body is captured from `fn`.
template <class F>
cudaError_t add_if(cudaStream_t s, cudaGraph_t G, cudaGraphConditionalHandle h,
                   const std::vector<cudaGraphNode_t>& deps, cudaGraphNode_t* node, F fn) {
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  cudaError_t e = cudaGraphAddNode(node, G, deps.data(), deps.size(), &cp);
  if (e != cudaSuccess) return e;
  std::vector<cudaGraphNode_t> none, sinks;
  return capture_segment(s, cp.conditional.phGraph_out[0], none, sinks, fn);
}
}  // namespace

template <typename R>
cudaError_t capture_iteration(Ctx& c, BatchWs& w, double gscale, cudaStream_t s, cudaGraph_t* out,
                              long long* kernels) {
  *out = nullptr;
  cudaGraph_t G = nullptr;
  cudaError_t e = cudaGraphCreate(&G, 0);
  if (e != cudaSuccess) return e;
  cudaGraphConditionalHandle hT = 0, hR = 0;
  bool cond = !getenv("DDA_NO_GRAPH_COND") &&
              cudaGraphConditionalHandleCreate(&hT, G, 0, cudaGraphCondAssignDefault) == cudaSuccess &&
              cudaGraphConditionalHandleCreate(&hR, G, 0, cudaGraphCondAssignDefault) == cudaSuccess;
  if (cond) {
    KrylovLaunch k{w.d_st, nullptr, w.nb, w.red, w.cnt, (long long)w.n3, w.RB};
    k.cond_true = hT;
    k.cond_reset = hR;
    std::vector<cudaGraphNode_t> none, d1, d2, d3;
    cudaGraphNode_t n1 = nullptr, n2 = nullptr;
    // kernels every launch of the graph runs: the three unconditional
    // segments (the bodies of the IF nodes are not counted)
    long long nk = 0, c0 = 0;
    c0 = g_captured;
    e = capture_segment(s, G, none, d1, [&]() -> cudaError_t { return enqueue_front<R>(c, w, gscale, s, k); });
    nk += g_captured - c0;
    if (e == cudaSuccess)
      e = add_if(s, G, hT, d1, &n1, [&]() -> cudaError_t {
        return amul<R>(c, w, V_X, V_R, MV_RESIDUAL, C_TRUE_RES, gscale, s);
      });
    c0 = g_captured;
    if (e == cudaSuccess)
      e = capture_segment(s, G, std::vector<cudaGraphNode_t>{n1}, d2, [&]() -> cudaError_t {
        launch_norm<R>(k, s);
        return cudaGetLastError();
      });
    nk += g_captured - c0;
    if (e == cudaSuccess)
      e = add_if(s, G, hR, d2, &n2, [&]() -> cudaError_t {
        return amul<R>(c, w, V_X, V_R, MV_RESIDUAL, C_RESET_RES, gscale, s);
      });
    c0 = g_captured;
    if (e == cudaSuccess)
      e = capture_segment(s, G, std::vector<cudaGraphNode_t>{n2}, d3, [&]() -> cudaError_t {
        launch_fin<R>(k, s);
        return cudaGetLastError();
      });
    nk += g_captured - c0;
    if (e == cudaSuccess) {
      *out = G;
      *kernels = nk;
      return cudaSuccess;
    }
    cudaGetLastError();
  }
  // plain capture: both residual matvecs are launched every iteration and
  // return at once when no instance needs them
  cudaGraphDestroy(G);
  G = nullptr;
  if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return e;
  const long long c1 = g_captured;
  cudaError_t e1 = enqueue_iteration<R>(c, w, gscale, s);
  const long long nk = g_captured - c1;
  e = cudaStreamEndCapture(s, &G);
  if (e1 != cudaSuccess || e != cudaSuccess) {
    if (G) cudaGraphDestroy(G);
    return e1 != cudaSuccess ? e1 : e;
  }
  *kernels = nk;
  *out = G;
  return cudaSuccess;
}

template cudaError_t capture_iteration<float>(Ctx&, BatchWs&, double, cudaStream_t, cudaGraph_t*, long long*);
template cudaError_t capture_iteration<double>(Ctx&, BatchWs&, double, cudaStream_t, cudaGraph_t*, long long*);

template <typename R>
static int build_graph(Ctx& c, BatchWs& w, double gscale) {
  if (w.gexec && w.graph_gscale == gscale && w.graph_pscale == w.pscale) return DDA_OK;
  if (w.gexec) { cudaGraphExecDestroy(w.gexec); w.gexec = nullptr; }
  // make sure lazily created resources exist before capture
  c.twiddles(w.g.Lx, sizeof(R) == 8); c.twiddles(w.g.Ly, sizeof(R) == 8); c.twiddles(w.g.Lz, sizeof(R) == 8);
  if (w.pre) {
    c.twiddles(w.gp.Lx, sizeof(R) == 8); c.twiddles(w.gp.Ly, sizeof(R) == 8); c.twiddles(w.gp.Lz, sizeof(R) == 8);
  }
  cudaGraph_t graph = nullptr;
  long long nk = 0;
  cudaError_t e = capture_iteration<R>(c, w, gscale, c.stream, &graph, &nk);
  if (e != cudaSuccess) {
    set_error(std::string("graph capture: ") + cudaGetErrorString(e));
    return DDA_ERR_CUDA;
  }
  w.graph_kernels = nk;
  e = cudaGraphInstantiate(&w.gexec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) { set_error(std::string("graph instantiate: ") + cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  w.graph_gscale = gscale;
  w.graph_pscale = w.pscale;
  return DDA_OK;
}

// Preconditioned solves iterate on y with x = M y (Gpbicgstab.py:1171-1199):
// M is applied in place to the iterate the store / accumulate step reads.
template <typename R>
static cudaError_t finish_pre(Ctx& c, BatchWs& w, cudaStream_t s) {
  if (!w.pre) return cudaSuccess;
  launch_pick_solution(w.d_st, w.nb, s, nullptr);
  MvFuse f;
  f.tensor = 1;
  return launch_matvec<R>(c, w.gp, w.pcp, w.d_st, nullptr, w.nb, V_TMP, V_TMP, MV_CONV_MASKED, C_LIVE, w.pscale, s,
                          f);
}

// Run iterations until every active instance is done.  Status is polled
// through two pinned buffers so the GPU keeps iterating while the host checks.
// Iterations per graph-launch chunk between status checks (two chunks are in
// flight; a finished solve runs at most one chunk and a partial one of
// early-exit iterations).  Measured on B200, 64^3 two-RHS preconditioned
// mixed solve: chunk 4 19.76 ms, 2 19.43 ms, 1 19.34 ms (but the
// unpreconditioned solve slows at 1).  DDA_CHUNK overrides.
static int solve_chunk() {
  static const int ch = [] {
    const char* e = getenv("DDA_CHUNK");
    const int v = e ? atoi(e) : 0;
    return (v >= 1 && v <= 64) ? v : 2;
  }();
  return ch;
}

template <typename R>
static int run_iterations(Ctx& c, BatchWs& w, double gscale, int chunk) {
  int rc = build_graph<R>(c, w, gscale);
  if (rc) return rc;
  cudaStream_t s = c.stream;
  auto enqueue_chunk = [&](int buf) -> cudaError_t {
    for (int q = 0; q < chunk; ++q) {
      cudaError_t e = cudaGraphLaunch(w.gexec, s);
      if (e != cudaSuccess) return e;
      note_launch(s, w.graph_kernels);
    }
    cudaError_t e = cudaMemcpyAsync(w.h_st[buf], w.d_st, w.nb * sizeof(InstState), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return e;
    return cudaEventRecord(c.ev[buf], s);
  };
  DDA_CUDA_OK(enqueue_chunk(0));
  DDA_CUDA_OK(enqueue_chunk(1));
  for (int it = 0;; ++it) {
    const int buf = it & 1;
    DDA_CUDA_OK(cudaEventSynchronize(c.ev[buf]));
    bool all = true;
    for (int j = 0; j < w.nb; ++j) {
      const InstState& S = w.h_st[buf][j];
      if (S.active && !S.done) { all = false; break; }
    }
    if (all) break;
    DDA_CUDA_OK(enqueue_chunk(buf));
  }
  DDA_CUDA_OK(cudaStreamSynchronize(s));
  DDA_CUDA_OK(cudaMemcpy(w.h_st[0], w.d_st, w.nb * sizeof(InstState), cudaMemcpyDeviceToHost));
  return DDA_OK;
}

static void fill_result(const InstState& S, dda_result& r) {
  r.iters = S.ret_iters;
  r.status = S.status == ST_CONVERGED ? DDA_OK : (S.status == ST_MAXITER ? DDA_NOT_CONVERGED : DDA_ERR_NAN);
  r.lowest_rel = S.initial_norm > 0 ? S.lowest / S.initial_norm : NAN;
  r.first_rel = S.initial_norm > 0 ? S.first / S.initial_norm : NAN;
  r.true_relres = -1.0;
  r.outer = 0;
  r.resets = S.reset_count;
}

template <typename R>
int solve_batch(Ctx& c, const Geo& g, double gscale, const dda_instance* inst, int nb, double target, int max_iter,
                double ratio, dda_result* res, cudaStream_t user, const PreSpec* pre) {
  int err = DDA_OK;
  const int dtype = sizeof(R) == 8 ? DDA_C128 : DDA_C64;
  BatchWs* w = c.workspace(dtype, g, nb, true, &err, 0, pre ? &pre->g : nullptr);
  if (!w) return err;
  if (pre) w->pscale = pre->scale;
  InstState* H = w->h_st[0];
  const bool sites = compress_sites();
  for (int j = 0; j < nb; ++j) {
    w->base_state(j, H[j], sites);
    H[j].ghat = inst[j].ghat;
    H[j].pghat = pre ? pre->phat[j] : nullptr;
    H[j].inva = inst[j].inv_alpha;
    H[j].vec[V_TMP] = (void*)inst[j].e_inc;
    H[j].out = inst[j].p_out;
    H[j].target = target;
    H[j].ratio = ratio;
    H[j].max_iter = max_iter;
    H[j].active = 1;
  }
  cudaStream_t s = c.stream;
  DDA_CUDA_OK(cudaEventRecord(c.ev_user, user));
  DDA_CUDA_OK(cudaStreamWaitEvent(s, c.ev_user, 0));
  DDA_CUDA_OK(cudaMemcpyAsync(w->d_st, H, nb * sizeof(InstState), cudaMemcpyHostToDevice, s));
  if (sites) launch_site_map<R>(w->d_st, nb, g.nsite, w->bcount, s, nullptr);
  launch_make_b<R>(w->d_st, nb, g.nsite, V_TMP, V_B, c.num_sms, s, nullptr);
  KrylovLaunch k{w->d_st, nullptr, nb, w->red, w->cnt, (long long)w->n3, w->RB};
  launch_init<R>(k, s);
  DDA_CUDA_OK(cudaGetLastError());
  int rc = run_iterations<R>(c, *w, gscale, solve_chunk());
  if (rc) return rc;
  DDA_CUDA_OK(finish_pre<R>(c, *w, s));
  launch_store_solution<R>(w->d_st, nb, (long long)w->n3, c.num_sms, s, nullptr);
  DDA_CUDA_OK(cudaGetLastError());
  for (int j = 0; j < nb; ++j)
    if (res) fill_result(w->h_st[0][j], res[j]);
  DDA_CUDA_OK(cudaEventRecord(c.ev_done, s));
  DDA_CUDA_OK(cudaStreamWaitEvent(user, c.ev_done, 0));
  return DDA_OK;
}
template int solve_batch<float>(Ctx&, const Geo&, double, const dda_instance*, int, double, int, double, dda_result*,
                                cudaStream_t, const PreSpec*);
template int solve_batch<double>(Ctx&, const Geo&, double, const dda_instance*, int, double, int, double,
                                 dda_result*, cudaStream_t, const PreSpec*);

// ---------------------------------------------------------------------------
// mixed precision: complex64 sweeps inside FP64 iterative refinement
// ---------------------------------------------------------------------------
int solve_mixed(Ctx& c, const Geo& g, double gscale, const dda_instance* i64, const dda_instance* i128, int nb,
                double tol, double inner_tol, int max_iter, int max_outer, double ratio, dda_result* res,
                cudaStream_t user, const PreSpec* pre) {
  int err = DDA_OK;
  BatchWs* w64 = c.workspace(DDA_C64, g, nb, true, &err, 0, pre ? &pre->g : nullptr);
  if (!w64) return err;
  if (pre) w64->pscale = pre->scale;
  BatchWs* w128 = c.workspace(DDA_C128, g, nb, false, &err);
  if (!w128) return err;
  cudaStream_t s = c.stream;
  DDA_CUDA_OK(cudaEventRecord(c.ev_user, user));
  DDA_CUDA_OK(cudaStreamWaitEvent(s, c.ev_user, 0));
  // FP64 side: b = mask*E, x = 0, r = b
  InstState* H = w128->h_st[0];
  const size_t bytes128 = w128->n3 * 16;
  for (int j = 0; j < nb; ++j) {
    w128->base_state(j, H[j]);
    H[j].ghat = i128[j].ghat;
    H[j].inva = i128[j].inv_alpha;
    H[j].vec[V_TMP] = (void*)i128[j].e_inc;
    H[j].vec[V_X] = i128[j].p_out;
    H[j].active = 1;
    DDA_CUDA_OK(cudaMemsetAsync(i128[j].p_out, 0, bytes128, s));
  }
  DDA_CUDA_OK(cudaMemcpyAsync(w128->d_st, H, nb * sizeof(InstState), cudaMemcpyHostToDevice, s));
  launch_make_b<double>(w128->d_st, nb, g.nsite, V_TMP, V_B, c.num_sms, s, nullptr);
  launch_norm2<double>(w128->d_st, V_B, nb, (long long)w128->n3, w128->red, w128->cnt, w128->RB, w128->d_out, s,
                       nullptr);
  DDA_CUDA_OK(cudaMemcpyAsync(w128->h_out, w128->d_out, nb * sizeof(double), cudaMemcpyDeviceToHost, s));
  DDA_CUDA_OK(cudaStreamSynchronize(s));
  std::vector<double> bnorm(nb), relres(nb, 1.0);
  std::vector<int> active(nb, 1), total(nb, 0), outer(nb, 0), resets(nb, 0), last_status(nb, ST_RUNNING);
  std::vector<double> first_rel(nb, NAN), lowest_rel(nb, NAN);
  for (int j = 0; j < nb; ++j) {
    bnorm[j] = std::sqrt(w128->h_out[j]);
    // a zero right-hand side is solved by P = 0; a NaN or infinite one ends
    // at once with the NaN status (the reference returns -1 there: its first
    // residual norm is NaN)
    if (!std::isfinite(bnorm[j])) { active[j] = 0; relres[j] = NAN; total[j] = 1; }
    else if (!(bnorm[j] > 0)) { active[j] = 0; relres[j] = 0.0; }
  }
  // residual r = b (x = 0)
  for (int j = 0; j < nb; ++j)
    DDA_CUDA_OK(cudaMemcpyAsync(H[j].vec[V_R], H[j].vec[V_B], bytes128, cudaMemcpyDeviceToDevice, s));
  InstState* H64 = w64->h_st[0];
  const bool sites = compress_sites();
  for (int sweep = 0; sweep < max_outer; ++sweep) {
    int nact = 0;
    for (int j = 0; j < nb; ++j) nact += active[j];
    if (!nact) break;
    for (int j = 0; j < nb; ++j) {
      w64->base_state(j, H64[j], sites);
      H64[j].ghat = i64[j].ghat;
      H64[j].pghat = pre ? pre->phat[j] : nullptr;
      H64[j].inva = i64[j].inv_alpha;
      // inner target: inner_tol, relaxed on later sweeps to what the FP64
      // target still needs (mixed_sweep_target)
      const double tj = sweep > 0 ? mixed_sweep_target(inner_tol, tol, relres[j]) : inner_tol;
      H64[j].target = tj;
      H64[j].ratio = mixed_inner_ratio(ratio);
      H64[j].max_iter = max_iter;
      H64[j].active = active[j];
      H[j].active = active[j];
    }
    DDA_CUDA_OK(cudaMemcpyAsync(w64->d_st, H64, nb * sizeof(InstState), cudaMemcpyHostToDevice, s));
    DDA_CUDA_OK(cudaMemcpyAsync(w128->d_st, H, nb * sizeof(InstState), cudaMemcpyHostToDevice, s));
    if (sites) launch_site_map<float>(w64->d_st, nb, g.nsite, w64->bcount, s, nullptr);
    launch_down(w64->d_st, V_B, w128->d_st, V_R, nb, (long long)w64->n3, c.num_sms, s, nullptr);
    KrylovLaunch k{w64->d_st, nullptr, nb, w64->red, w64->cnt, (long long)w64->n3, w64->RB};
    launch_init<float>(k, s);
    int rc = run_iterations<float>(c, *w64, gscale, solve_chunk());
    if (rc) return rc;
    DDA_CUDA_OK(finish_pre<float>(c, *w64, s));
    for (int j = 0; j < nb; ++j) {
      if (!active[j]) continue;
      const InstState& S = w64->h_st[0][j];
      total[j] += S.ret_iters < 0 ? -S.ret_iters : S.ret_iters;
      resets[j] += S.reset_count;
      outer[j] += 1;
      last_status[j] = S.status;
      if (sweep == 0) {
        first_rel[j] = S.initial_norm > 0 ? S.first / S.initial_norm : NAN;
        lowest_rel[j] = S.initial_norm > 0 ? S.lowest / S.initial_norm : NAN;
      }
    }
    launch_accum(w128->d_st, V_X, w64->d_st, nb, (long long)w64->n3, c.num_sms, s, nullptr);
    cudaError_t e = launch_matvec<double>(c, g, w128->pc, w128->d_st, nullptr, nb, V_X, V_R, MV_RESIDUAL, C_ACTIVE,
                                          gscale, s);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
    launch_norm2<double>(w128->d_st, V_R, nb, (long long)w128->n3, w128->red, w128->cnt, w128->RB, w128->d_out, s,
                         nullptr);
    DDA_CUDA_OK(cudaMemcpyAsync(w128->h_out, w128->d_out, nb * sizeof(double), cudaMemcpyDeviceToHost, s));
    DDA_CUDA_OK(cudaStreamSynchronize(s));
    for (int j = 0; j < nb; ++j) {
      if (!active[j]) continue;
      relres[j] = std::sqrt(w128->h_out[j]) / bnorm[j];
      if (relres[j] <= tol || std::isnan(relres[j])) active[j] = 0;
    }
  }
  for (int j = 0; j < nb; ++j) {
    if (!res) break;
    dda_result& r = res[j];
    r.status = (relres[j] <= tol) ? DDA_OK : (std::isnan(relres[j]) ? DDA_ERR_NAN : DDA_NOT_CONVERGED);
    // the reference's sign convention: -(iterations) when the solve ended on NaN
    r.iters = r.status == DDA_ERR_NAN ? -total[j] : total[j];
    r.lowest_rel = lowest_rel[j];
    r.first_rel = first_rel[j];
    r.true_relres = relres[j];
    r.outer = outer[j];
    r.resets = resets[j];
  }
  DDA_CUDA_OK(cudaEventRecord(c.ev_done, s));
  DDA_CUDA_OK(cudaStreamWaitEvent(user, c.ev_done, 0));
  return DDA_OK;
}

}  // namespace dda
