// Slot pool for continuous batching.
//
// A pool owns a fixed number of solver instance slots sharing one box / FFT
// size.  Every slot carries its own device-side GPBiCGSTAB state (the state
// machine of krylov.cu), so the pool iterates all occupied slots together in
// one captured graph while requests enter and leave at any time:
//   admit   -> fill a free slot (right-hand side, operator pointers) and
//              initialise it while the other slots keep their state;
//   run     -> enqueue n iterations of the whole pool on its own stream;
//   poll    -> read every slot's status; finished complex64 sweeps of a
//              mixed-precision slot are accumulated into its FP64 solution,
//              its FP64 true residual is formed with a complex128 matvec, and
//              the slot either completes or is re-armed for another sweep;
//              completed slots are reported and become free.
// Pools on different streams overlap on the device.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/dda_b200.h"
#include "dda_host.h"

using namespace dda;

struct dda_ctx {
  Ctx c;
};

namespace {
struct SlotInfo {
  int state = 0;          // 0 free, 1 running
  void* p_out = nullptr;  // result destination (single-precision pools)
  double tol = 1e-5, inner_tol = 1e-4, ratio = 100.0;
  int max_iter = 1000, max_outer = 10;
  int outer = 0, resets = 0;
  long long iters = 0;
  double bnorm = 0.0, relres = 1.0, first_rel = NAN, lowest_rel = NAN;
};
}  // namespace

struct dda_slots {
  dda_ctx* ctx = nullptr;
  int prec = DDA_PREC_C64;
  Geo g{};
  double gscale = 1.0;
  bool pre = false;   // preconditioned slots (precon=True): octant per slot, grid p->w.gp
  int n = 0;
  BatchWs w;      // solver workspace (complex64 for C64 / MIXED, complex128 for C128)
  BatchWs w128;   // MIXED: FP64 right-hand side and residual per slot
  double* d_bnorm = nullptr;
  double* h_norm = nullptr;   // pinned [2n]: residual norms, then b norms
  int* d_act = nullptr;       // two active lists of n entries
  cudaStream_t s = nullptr;
  cudaEvent_t ev = nullptr;
  std::vector<SlotInfo> info;
};

static int set_act(dda_slots* p, int which, const std::vector<int>& ids) {
  cudaError_t e = cudaMemcpyAsync(p->d_act + which * p->n, ids.data(), ids.size() * sizeof(int),
                                  cudaMemcpyHostToDevice, p->s);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  return DDA_OK;
}

static int put_state(dda_slots* p, BatchWs& w, int j, const InstState& S) {
  cudaError_t e = cudaMemcpyAsync(w.d_st + j, &S, sizeof(InstState), cudaMemcpyHostToDevice, p->s);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  return DDA_OK;
}

// (Re)initialise the complex64 / complex128 Krylov state of slot j from its
// right-hand side (already in V_B for mixed pools, in V_TMP otherwise).
static int arm_solver(dda_slots* p, int j, const void* ghat, const void* pghat, const void* inva, const void* e_inc,
                      double target, int max_iter, double ratio, bool from_tmp, void* out) {
  InstState S;
  p->w.base_state(j, S, compress_sites());
  S.out = out;
  S.ghat = ghat;
  S.pghat = pghat;
  S.inva = inva;
  if (from_tmp) S.vec[V_TMP] = (void*)e_inc;
  S.target = target;
  S.ratio = ratio;
  S.max_iter = max_iter;
  S.active = 1;
  return put_state(p, p->w, j, S);
}

extern "C" {

static int slots_create(dda_ctx* ctx, int precision, int nx, int ny, int nz, int Lx, int Ly, int Lz, double gscale,
                        const Geo* gp, double pscale, int nslots, dda_slots** out);

int dda_slots_create(dda_ctx* ctx, int precision, int nx, int ny, int nz, int Lx, int Ly, int Lz, double gscale,
                     int nslots, dda_slots** out) {
  return slots_create(ctx, precision, nx, ny, nz, Lx, Ly, Lz, gscale, nullptr, 1.0, nslots, out);
}

int dda_slots_create_pre(dda_ctx* ctx, int precision, int nx, int ny, int nz, int Lx, int Ly, int Lz, double gscale,
                         int Px, int Py, int Pz, double pscale, int nslots, dda_slots** out) {
  const int dt = precision == DDA_PREC_C128 ? DDA_C128 : DDA_C64;
  if (Px < nx || Py < ny || Pz < nz || !dda_fft_length_ok(Px, dt) || !dda_fft_length_ok(Py, dt) ||
      !dda_fft_length_ok(Pz, dt)) {
    set_error("slot pool: bad preconditioner grid");
    return DDA_ERR_BAD_SHAPE;
  }
  Geo gp;
  gp.nx = nx; gp.ny = ny; gp.nz = nz; gp.Lx = Px; gp.Ly = Py; gp.Lz = Pz;
  gp.hx = Px / 2 + 1; gp.hy = Py / 2 + 1; gp.hz = Pz / 2 + 1;
  gp.nsite = (long long)nx * ny * nz;
  return slots_create(ctx, precision, nx, ny, nz, Lx, Ly, Lz, gscale, &gp, pscale, nslots, out);
}

static int slots_create(dda_ctx* ctx, int precision, int nx, int ny, int nz, int Lx, int Ly, int Lz, double gscale,
                        const Geo* gp, double pscale, int nslots, dda_slots** out) {
  if (!ctx || !out || nslots < 1) { set_error("bad slot-pool arguments"); return DDA_ERR_ARG; }
  if (precision < DDA_PREC_C64 || precision > DDA_PREC_MIXED) { set_error("bad precision"); return DDA_ERR_ARG; }
  *out = nullptr;
  cudaError_t e = cudaSetDevice(ctx->c.device);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  if (!dda_fft_length_ok(Lx, precision == DDA_PREC_C64 ? DDA_C64 : DDA_C128) ||
      !dda_fft_length_ok(Ly, precision == DDA_PREC_C64 ? DDA_C64 : DDA_C128) ||
      !dda_fft_length_ok(Lz, precision == DDA_PREC_C64 ? DDA_C64 : DDA_C128) || Lx < 2 * nx || Ly < 2 * ny ||
      Lz < 2 * nz || nx < 1 || ny < 1 || nz < 1) {
    set_error("slot pool: bad box or FFT lengths");
    return DDA_ERR_BAD_SHAPE;
  }
  dda_slots* p = new dda_slots();
  p->ctx = ctx;
  p->prec = precision;
  Geo& g = p->g;
  g.nx = nx; g.ny = ny; g.nz = nz; g.Lx = Lx; g.Ly = Ly; g.Lz = Lz;
  g.hx = Lx / 2 + 1; g.hy = Ly / 2 + 1; g.hz = Lz / 2 + 1;
  g.nsite = (long long)nx * ny * nz;
  p->gscale = gscale;
  p->n = nslots;
  p->info.resize(nslots);
  p->pre = gp != nullptr;
  // the pool's memory is ordered on its own stream: creating and destroying
  // pools does not synchronise the device (other pools keep running)
  int rc = DDA_OK;
  if (cudaStreamCreateWithFlags(&p->s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&p->ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    set_error("slot pool: stream creation failed");
    rc = DDA_ERR_CUDA;
  }
  p->w.astream = p->s;
  p->w128.astream = p->s;
  // pools run side by side on their own streams: their kernels launch
  // without programmatic serialization (B200, the 64-geometry batched
  // workload measured 86-84 solves/s with it, 117 without; DDA_POOL_PDL=1
  // keeps it)
  if (p->s) {
    const char* pe = getenv("DDA_POOL_PDL");
    if (!(pe && *pe == '1')) set_stream_pdl(p->s, false);
  }
  if (!rc) rc = p->w.alloc(ctx->c, precision == DDA_PREC_C128 ? DDA_C128 : DDA_C64, g, nslots, true, gp);
  p->w.pscale = pscale;
  if (!rc && precision == DDA_PREC_MIXED) rc = p->w128.alloc(ctx->c, DDA_C128, g, nslots, false);
  if (!rc) {
    p->h_norm = (double*)pinned_get(2 * nslots * sizeof(double));
    if (cudaMallocAsync((void**)&p->d_bnorm, nslots * sizeof(double), p->s) != cudaSuccess ||
        cudaMallocAsync((void**)&p->d_act, 2 * nslots * sizeof(int), p->s) != cudaSuccess || !p->h_norm) {
      cudaGetLastError();
      set_error("slot pool: out of device memory");
      rc = DDA_ERR_OOM;
    }
  }
  if (!rc) {
    // inactive slots: all kernels of the graph skip them
    std::vector<InstState> H(nslots);
    for (int j = 0; j < nslots; ++j) p->w.base_state(j, H[j]);
    if (cudaMemcpyAsync(p->w.d_st, H.data(), nslots * sizeof(InstState), cudaMemcpyHostToDevice, p->s) !=
            cudaSuccess ||
        cudaStreamSynchronize(p->s) != cudaSuccess) {
      set_error("slot pool: state upload failed");
      rc = DDA_ERR_CUDA;
    }
  }
  if (!rc) {
    const bool dbl = precision == DDA_PREC_C128;
    ctx->c.twiddles(Lx, dbl); ctx->c.twiddles(Ly, dbl); ctx->c.twiddles(Lz, dbl);
    if (gp) { ctx->c.twiddles(gp->Lx, dbl); ctx->c.twiddles(gp->Ly, dbl); ctx->c.twiddles(gp->Lz, dbl); }
    if (precision == DDA_PREC_MIXED) { ctx->c.twiddles(Lx, true); ctx->c.twiddles(Ly, true); ctx->c.twiddles(Lz, true); }
    cudaGraph_t graph = nullptr;
    long long nk = 0;
    cudaError_t e1 = dbl ? capture_iteration<double>(ctx->c, p->w, gscale, p->s, &graph, &nk)
                         : capture_iteration<float>(ctx->c, p->w, gscale, p->s, &graph, &nk);
    if (e1 != cudaSuccess) {
      set_error(std::string("slot pool graph capture: ") + cudaGetErrorString(e1));
      rc = DDA_ERR_CUDA;
    } else {
      p->w.graph_kernels = nk;
      if (cudaGraphInstantiate(&p->w.gexec, graph, 0) != cudaSuccess) {
        set_error("slot pool graph instantiate failed");
        rc = DDA_ERR_CUDA;
      }
      cudaGraphDestroy(graph);
    }
  }
  if (rc) {
    dda_slots_destroy(p);
    return rc;
  }
  *out = p;
  return DDA_OK;
}

void dda_slots_destroy(dda_slots* p) {
  if (!p) return;
  cudaSetDevice(p->ctx->c.device);
  // the pool's own work completes first (its pinned blocks are then free to
  // reuse); device memory returns to the stream-ordered pool on its stream
  if (p->s) cudaStreamSynchronize(p->s);
  p->w.release();
  p->w128.release();
  if (p->s) {
    if (p->d_bnorm) cudaFreeAsync(p->d_bnorm, p->s);
    if (p->d_act) cudaFreeAsync(p->d_act, p->s);
  }
  pinned_put(p->h_norm, 2 * p->n * sizeof(double));
  if (p->ev) cudaEventDestroy(p->ev);
  if (p->s) {
    set_stream_pdl(p->s, true);
    cudaStreamDestroy(p->s);
  }
  cudaGetLastError();
  delete p;
}

int dda_slots_capacity(const dda_slots* p) { return p ? p->n : 0; }

int dda_slots_free_slot(const dda_slots* p) {
  if (!p) return -1;
  for (int j = 0; j < p->n; ++j)
    if (p->info[j].state == 0) return j;
  return -1;
}

static int slots_admit(dda_slots* p, int slot, const dda_instance* lo, const dda_instance* hi, const void* phat,
                       double tol, double inner_tol, int max_iter, int max_outer, double ratio, void* stream);

int dda_slots_admit(dda_slots* p, int slot, const dda_instance* lo, const dda_instance* hi, double tol,
                    double inner_tol, int max_iter, int max_outer, double ratio, void* stream) {
  if (p && p->pre) { set_error("a preconditioned pool admits with dda_slots_admit_pre"); return DDA_ERR_ARG; }
  return slots_admit(p, slot, lo, hi, nullptr, tol, inner_tol, max_iter, max_outer, ratio, stream);
}

int dda_slots_admit_pre(dda_slots* p, int slot, const dda_instance* lo, const dda_instance* hi, const void* phat,
                        double tol, double inner_tol, int max_iter, int max_outer, double ratio, void* stream) {
  if (!p || !p->pre) { set_error("dda_slots_admit_pre needs a pool made by dda_slots_create_pre"); return DDA_ERR_ARG; }
  if (!phat) { set_error("null preconditioner octant"); return DDA_ERR_ARG; }
  return slots_admit(p, slot, lo, hi, phat, tol, inner_tol, max_iter, max_outer, ratio, stream);
}

static int slots_admit(dda_slots* p, int slot, const dda_instance* lo, const dda_instance* hi, const void* phat,
                       double tol, double inner_tol, int max_iter, int max_outer, double ratio, void* stream) {
  if (!p || slot < 0 || slot >= p->n) { set_error("bad slot"); return DDA_ERR_ARG; }
  if (p->info[slot].state != 0) { set_error("slot is occupied"); return DDA_ERR_ARG; }
  const dda_instance* in = p->prec == DDA_PREC_C128 ? hi : lo;
  if (!in || !in->ghat || !in->inv_alpha) { set_error("null instance"); return DDA_ERR_ARG; }
  if (p->prec == DDA_PREC_MIXED && (!hi || !hi->ghat || !hi->inv_alpha || !hi->e_inc || !hi->p_out)) {
    set_error("mixed pools need the complex128 instance");
    return DDA_ERR_ARG;
  }
  if (p->prec != DDA_PREC_MIXED && (!in->e_inc || !in->p_out)) { set_error("null vectors"); return DDA_ERR_ARG; }
  cudaSetDevice(p->ctx->c.device);
  cudaEventRecord(p->ev, (cudaStream_t)stream);
  cudaStreamWaitEvent(p->s, p->ev, 0);
  SlotInfo& I = p->info[slot];
  I = SlotInfo();
  I.state = 1;
  I.tol = tol; I.inner_tol = inner_tol; I.max_iter = max_iter; I.max_outer = max_outer; I.ratio = ratio;
  const std::vector<int> one{slot};
  int rc = set_act(p, 0, one);
  if (rc) return rc;
  const int* act = p->d_act;
  Ctx& c = p->ctx->c;
  if (p->prec != DDA_PREC_MIXED) {
    I.p_out = in->p_out;
    if ((rc = arm_solver(p, slot, in->ghat, phat, in->inv_alpha, in->e_inc, tol, max_iter, ratio, true, in->p_out)))
      return rc;
    KrylovLaunch k{p->w.d_st, act, 1, p->w.red, p->w.cnt, (long long)p->w.n3, p->w.RB};
    const bool sites = compress_sites();
    if (p->prec == DDA_PREC_C128) {
      if (sites) launch_site_map<double>(p->w.d_st, 1, p->g.nsite, p->w.bcount, p->s, act);
      launch_make_b<double>(p->w.d_st, 1, p->g.nsite, V_TMP, V_B, c.num_sms, p->s, act);
      launch_init<double>(k, p->s);
    } else {
      if (sites) launch_site_map<float>(p->w.d_st, 1, p->g.nsite, p->w.bcount, p->s, act);
      launch_make_b<float>(p->w.d_st, 1, p->g.nsite, V_TMP, V_B, c.num_sms, p->s, act);
      launch_init<float>(k, p->s);
    }
  } else {
    InstState H;
    p->w128.base_state(slot, H);
    H.ghat = hi->ghat;
    H.inva = hi->inv_alpha;
    H.vec[V_TMP] = (void*)hi->e_inc;
    H.vec[V_X] = hi->p_out;
    H.active = 1;
    if ((rc = put_state(p, p->w128, slot, H))) return rc;
    const size_t bytes = p->w128.n3 * 16;
    cudaMemsetAsync(hi->p_out, 0, bytes, p->s);
    launch_make_b<double>(p->w128.d_st, 1, p->g.nsite, V_TMP, V_B, c.num_sms, p->s, act);
    launch_norm2<double>(p->w128.d_st, V_B, 1, (long long)p->w128.n3, p->w128.red, p->w128.cnt, p->w128.RB,
                         p->d_bnorm, p->s, act);
    cudaMemcpyAsync(H.vec[V_R], H.vec[V_B], bytes, cudaMemcpyDeviceToDevice, p->s);
    if ((rc = arm_solver(p, slot, lo->ghat, phat, lo->inv_alpha, nullptr, inner_tol, max_iter,
                         mixed_inner_ratio(ratio), false, nullptr)))
      return rc;
    if (compress_sites()) launch_site_map<float>(p->w.d_st, 1, p->g.nsite, p->w.bcount, p->s, act);
    launch_down(p->w.d_st, V_B, p->w128.d_st, V_R, 1, (long long)p->w.n3, c.num_sms, p->s, act);
    KrylovLaunch k{p->w.d_st, act, 1, p->w.red, p->w.cnt, (long long)p->w.n3, p->w.RB};
    launch_init<float>(k, p->s);
    I.p_out = hi->p_out;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  return DDA_OK;
}

int dda_slots_run(dda_slots* p, int niter) {
  if (!p || niter < 0) { set_error("bad arguments"); return DDA_ERR_ARG; }
  cudaSetDevice(p->ctx->c.device);
  for (int i = 0; i < niter; ++i) {
    cudaError_t e = cudaGraphLaunch(p->w.gexec, p->s);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
    note_launch(p->s, p->w.graph_kernels);
  }
  return DDA_OK;
}

int dda_slots_ready(const dda_slots* p) {
  if (!p) { set_error("null pool"); return -DDA_ERR_ARG; }
  cudaSetDevice(p->ctx->c.device);
  const cudaError_t e = cudaStreamQuery(p->s);
  if (e == cudaSuccess) return 1;
  if (e == cudaErrorNotReady) { cudaGetLastError(); return 0; }
  set_error(cudaGetErrorString(e));
  return -DDA_ERR_CUDA;
}

int dda_slots_poll(dda_slots* p, int* finished, dda_result* results, int* nfinished, int* nrunning) {
  if (!p || !finished || !nfinished) { set_error("bad arguments"); return DDA_ERR_ARG; }
  cudaSetDevice(p->ctx->c.device);
  Ctx& c = p->ctx->c;
  *nfinished = 0;
  cudaError_t e = cudaStreamSynchronize(p->s);
  if (e == cudaSuccess) e = cudaMemcpy(p->w.h_st[1], p->w.d_st, p->n * sizeof(InstState), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  std::vector<int> done;
  for (int j = 0; j < p->n; ++j)
    if (p->info[j].state == 1 && p->w.h_st[1][j].active && p->w.h_st[1][j].done) done.push_back(j);
  auto finish = [&](int j, int status) {
    SlotInfo& I = p->info[j];
    dda_result r{};
    r.iters = (int)I.iters;
    r.status = status;
    r.lowest_rel = I.lowest_rel;
    r.first_rel = I.first_rel;
    r.true_relres = p->prec == DDA_PREC_MIXED ? I.relres : -1.0;
    r.outer = I.outer;
    r.resets = I.resets;
    finished[*nfinished] = j;
    if (results) results[*nfinished] = r;
    ++*nfinished;
    I.state = 0;
  };
  // preconditioned slots iterate on y with x = M y: M goes in place onto the
  // iterate the store / accumulate below reads (Gpbicgstab.py:1171-1199)
  auto apply_pre = [&](int m, const int* act) -> cudaError_t {
    if (!p->pre) return cudaSuccess;
    launch_pick_solution(p->w.d_st, m, p->s, act);
    MvFuse f;
    f.tensor = 1;
    if (p->prec == DDA_PREC_C128)
      return launch_matvec<double>(c, p->w.gp, p->w.pcp, p->w.d_st, act, m, V_TMP, V_TMP, MV_CONV_MASKED, C_LIVE,
                                   p->w.pscale, p->s, f);
    return launch_matvec<float>(c, p->w.gp, p->w.pcp, p->w.d_st, act, m, V_TMP, V_TMP, MV_CONV_MASKED, C_LIVE,
                                p->w.pscale, p->s, f);
  };
  if (p->prec != DDA_PREC_MIXED) {
    if (!done.empty()) {
      int rc = set_act(p, 0, done);
      if (rc) return rc;
      if ((e = apply_pre((int)done.size(), p->d_act)) != cudaSuccess) {
        set_error(cudaGetErrorString(e));
        return DDA_ERR_CUDA;
      }
      if (p->prec == DDA_PREC_C128)
        launch_store_solution<double>(p->w.d_st, (int)done.size(), (long long)p->w.n3, c.num_sms, p->s, p->d_act);
      else
        launch_store_solution<float>(p->w.d_st, (int)done.size(), (long long)p->w.n3, c.num_sms, p->s, p->d_act);
    }
    for (int j : done) {
      const InstState& S = p->w.h_st[1][j];
      SlotInfo& I = p->info[j];
      I.iters = S.ret_iters;
      I.resets = S.reset_count;
      I.first_rel = S.initial_norm > 0 ? S.first / S.initial_norm : NAN;
      I.lowest_rel = S.initial_norm > 0 ? S.lowest / S.initial_norm : NAN;
      finish(j, S.status == ST_CONVERGED ? DDA_OK : (S.status == ST_MAXITER ? DDA_NOT_CONVERGED : DDA_ERR_NAN));
    }
    if (!done.empty()) cudaStreamSynchronize(p->s);
  } else if (!done.empty()) {
    const int m = (int)done.size();
    int rc = set_act(p, 0, done);
    if (rc) return rc;
    const int* act = p->d_act;
    if ((e = apply_pre(m, act)) != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
    launch_accum(p->w128.d_st, V_X, p->w.d_st, m, (long long)p->w.n3, c.num_sms, p->s, act);
    e = launch_matvec<double>(c, p->g, p->w128.pc, p->w128.d_st, act, m, V_X, V_R, MV_RESIDUAL, C_ACTIVE,
                              p->gscale, p->s);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
    launch_norm2<double>(p->w128.d_st, V_R, m, (long long)p->w128.n3, p->w128.red, p->w128.cnt, p->w128.RB,
                         p->w128.d_out, p->s, act);
    cudaMemcpyAsync(p->h_norm, p->w128.d_out, p->n * sizeof(double), cudaMemcpyDeviceToHost, p->s);
    cudaMemcpyAsync(p->h_norm + p->n, p->d_bnorm, p->n * sizeof(double), cudaMemcpyDeviceToHost, p->s);
    if ((e = cudaStreamSynchronize(p->s)) != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
    std::vector<int> rearm;
    for (int j : done) {
      const InstState& S = p->w.h_st[1][j];
      SlotInfo& I = p->info[j];
      I.iters += S.ret_iters < 0 ? -S.ret_iters : S.ret_iters;
      I.resets += S.reset_count;
      if (I.outer == 0) {
        I.first_rel = S.initial_norm > 0 ? S.first / S.initial_norm : NAN;
        I.lowest_rel = S.initial_norm > 0 ? S.lowest / S.initial_norm : NAN;
      }
      I.outer += 1;
      I.bnorm = std::sqrt(p->h_norm[p->n + j]);
      // zero right-hand side: P = 0 solves it; NaN / infinite: NaN status
      I.relres = !std::isfinite(I.bnorm) ? NAN : (I.bnorm > 0 ? std::sqrt(p->h_norm[j]) / I.bnorm : 0.0);
      if (std::isnan(I.relres)) {
        I.iters = -I.iters;        // the reference's sign convention for a NaN exit
        finish(j, DDA_ERR_NAN);
      } else if (I.relres <= I.tol) finish(j, DDA_OK);
      else if (I.outer >= I.max_outer) finish(j, DDA_NOT_CONVERGED);
      else rearm.push_back(j);
    }
    if (!rearm.empty()) {
      for (int j : rearm) {
        SlotInfo& I = p->info[j];
        const InstState& S = p->w.h_st[1][j];
        const double tj = mixed_sweep_target(I.inner_tol, I.tol, I.relres);
        if ((rc = arm_solver(p, j, S.ghat, S.pghat, S.inva, nullptr, tj, I.max_iter, mixed_inner_ratio(I.ratio),
                             false, nullptr)))
          return rc;
      }
      if ((rc = set_act(p, 1, rearm))) return rc;
      const int* act2 = p->d_act + p->n;
      const int r = (int)rearm.size();
      if (compress_sites()) launch_site_map<float>(p->w.d_st, r, p->g.nsite, p->w.bcount, p->s, act2);
      launch_down(p->w.d_st, V_B, p->w128.d_st, V_R, r, (long long)p->w.n3, c.num_sms, p->s, act2);
      KrylovLaunch k{p->w.d_st, act2, r, p->w.red, p->w.cnt, (long long)p->w.n3, p->w.RB};
      launch_init<float>(k, p->s);
    }
  }
  if (nrunning) {
    int nr = 0;
    for (int j = 0; j < p->n; ++j) nr += p->info[j].state == 1;
    *nrunning = nr;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  return DDA_OK;
}

int dda_slots_release(dda_slots* p, int slot) {
  if (!p || slot < 0 || slot >= p->n) { set_error("bad slot"); return DDA_ERR_ARG; }
  cudaSetDevice(p->ctx->c.device);
  InstState S;
  p->w.base_state(slot, S);          // inactive
  int rc = put_state(p, p->w, slot, S);
  if (rc) return rc;
  p->info[slot].state = 0;
  return cudaStreamSynchronize(p->s) == cudaSuccess ? DDA_OK : DDA_ERR_CUDA;
}

}  // extern "C"
