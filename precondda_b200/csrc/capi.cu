// extern "C" entry points of include/dda_b200.h.
#include <cmath>
#include <cstring>
#include <vector>
#include <new>

#include "../../include/dda_b200.h"
#include "dda_host.h"
#include "reduce.cuh"
#include "fft_sizes.h"

using namespace dda;

struct dda_ctx {
  Ctx c;
};

struct dda_op {
  dda_ctx* ctx = nullptr;
  int dtype = 0;
  Geo g{};
  PassCfg pc{};
  double gscale = 1.0;
  const void* ghat = nullptr;
  const void* inva = nullptr;
  void* scratch = nullptr;
  InstState* d_st = nullptr;
};

static int check_ctx(dda_ctx* ctx) {
  if (!ctx) { set_error("null context"); return DDA_ERR_ARG; }
  cudaError_t e = cudaSetDevice(ctx->c.device);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  return DDA_OK;
}

static int fft_cap(int dtype) { return dtype == DDA_C128 ? 12 * 256 : 24 * 256; }

static bool length_ok(int L, int dtype) {
  if (L < 2 || (L & 1)) return false;
  if (3 * L > fft_cap(dtype)) return false;
  return fft_size_compiled(L);
}

// minmul = 2: an operator's grid (linear convolution, L >= 2n); 1: a
// preconditioner's grid (the reference places x at the origin of any grid
// L >= n and crops, Gpbicgstab.py:636-666)
static int make_geo(int nx, int ny, int nz, int Lx, int Ly, int Lz, int dtype, Geo* g, int minmul = 2) {
  if (nx < 1 || ny < 1 || nz < 1) { set_error("box dimensions must be >= 1"); return DDA_ERR_BAD_SHAPE; }
  if (Lx < minmul * nx || Ly < minmul * ny || Lz < minmul * nz) {
    set_error(minmul == 2 ? "FFT lengths must be >= twice the box dimensions"
                          : "preconditioner FFT lengths must be >= the box dimensions");
    return DDA_ERR_BAD_SHAPE;
  }
  if (!length_ok(Lx, dtype) || !length_ok(Ly, dtype) || !length_ok(Lz, dtype)) {
    set_error("FFT lengths must be one of the compiled sizes (even, 2^a 3^b 5^c 7^d, <= 512)");
    return DDA_ERR_BAD_SHAPE;
  }
  g->nx = nx; g->ny = ny; g->nz = nz;
  g->Lx = Lx; g->Ly = Ly; g->Lz = Lz;
  g->hx = Lx / 2 + 1; g->hy = Ly / 2 + 1; g->hz = Lz / 2 + 1;
  g->nsite = (long long)nx * ny * nz;
  return DDA_OK;
}

extern "C" {

int dda_version(void) { return 100; }

long long dda_kernel_launches(void) { return launch_count(); }

const char* dda_last_error(void) { return get_error().c_str(); }

int dda_ctx_create(int device, dda_ctx** out) {
  if (!out) { set_error("null output pointer"); return DDA_ERR_ARG; }
  *out = nullptr;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  dda_ctx* c = new (std::nothrow) dda_ctx();
  if (!c) { set_error("host allocation failed"); return DDA_ERR_OOM; }
  c->c.device = device;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0)
    c->c.num_sms = sms;
  if ((e = cudaStreamCreateWithFlags(&c->c.stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&c->c.ev[0], cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&c->c.ev[1], cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&c->c.ev_user, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&c->c.ev_done, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaMalloc((void**)&c->c.xred, (size_t)4 * c->c.num_sms * 12 * sizeof(double))) != cudaSuccess ||
      (e = cudaMalloc((void**)&c->c.xcnt, sizeof(unsigned))) != cudaSuccess ||
      (e = cudaMalloc((void**)&c->c.xout, 4 * sizeof(double))) != cudaSuccess ||
      (e = cudaMallocHost((void**)&c->c.xout_h, 4 * sizeof(double))) != cudaSuccess ||
      (e = cudaMemset(c->c.xcnt, 0, sizeof(unsigned))) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&c->c.ev_fork, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaMalloc((void**)&c->c.iota, Ctx::kIota * sizeof(int))) != cudaSuccess) {
    set_error(cudaGetErrorString(e));
    delete c;
    return DDA_ERR_CUDA;
  }
  for (int j = 0; j < Ctx::kMaxSplit - 1; ++j) {
    if ((e = cudaStreamCreateWithFlags(&c->c.aux[j], cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->c.ev_join[j], cudaEventDisableTiming)) != cudaSuccess) {
      set_error(cudaGetErrorString(e));
      delete c;
      return DDA_ERR_CUDA;
    }
  }
  {
    std::vector<int> h(Ctx::kIota);
    for (int j = 0; j < Ctx::kIota; ++j) h[j] = j;
    if ((e = cudaMemcpy(c->c.iota, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess) {
      set_error(cudaGetErrorString(e));
      delete c;
      return DDA_ERR_CUDA;
    }
  }
  // transient buffers (Green-build transforms, voxeliser shape lists) come
  // from the device's stream-ordered pool; keep freed blocks in the pool
  // instead of unmapping them at every synchronisation (dda_ctx_trim
  // returns them)
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    unsigned long long keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  *out = c;
  return DDA_OK;
}

void dda_ctx_destroy(dda_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->c.device);
  cudaStreamSynchronize(ctx->c.stream);
  ctx->c.trim();
  cudaEventDestroy(ctx->c.ev[0]); cudaEventDestroy(ctx->c.ev[1]);
  cudaEventDestroy(ctx->c.ev_user); cudaEventDestroy(ctx->c.ev_done);
  cudaStreamDestroy(ctx->c.stream);
  for (int j = 0; j < Ctx::kMaxSplit - 1; ++j) {
    if (ctx->c.aux[j]) { cudaStreamSynchronize(ctx->c.aux[j]); cudaStreamDestroy(ctx->c.aux[j]); }
    if (ctx->c.ev_join[j]) cudaEventDestroy(ctx->c.ev_join[j]);
  }
  if (ctx->c.ev_fork) cudaEventDestroy(ctx->c.ev_fork);
  cudaFree(ctx->c.iota);
  cudaFree(ctx->c.xred); cudaFree(ctx->c.xcnt); cudaFree(ctx->c.xout); cudaFreeHost(ctx->c.xout_h);
  delete ctx;
}

int dda_ctx_trim(dda_ctx* ctx) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  cudaStreamSynchronize(ctx->c.stream);
  ctx->c.trim();
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, ctx->c.device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
  cudaGetLastError();
  return DDA_OK;
}

int dda_fft_length_ok(int L, int dtype) { return length_ok(L, dtype) ? 1 : 0; }

int dda_tuning_set(int dtype, int nx, int ny, int nz, int Lx, int Ly, int Lz, int nb, int flags) {
  if (dtype != DDA_C64 && dtype != DDA_C128) { set_error("bad dtype"); return DDA_ERR_ARG; }
  if (nb < 1) { set_error("nb must be >= 1"); return DDA_ERR_ARG; }
  if (flags > (DDA_TUNE_P3PIPE | DDA_TUNE_P3PIPE_1SM | DDA_TUNE_NO_FUSED_ZY | DDA_TUNE_NO_FUSED_INV |
                DDA_TUNE_P3PAIR | DDA_TUNE_YPAIR | DDA_TUNE_ZPAIR | DDA_TUNE_FUSED | DDA_TUNE_PREFETCH)) {
    set_error("unknown tuning flags");
    return DDA_ERR_ARG;
  }
  Geo g;
  int rc = make_geo(nx, ny, nz, Lx, Ly, Lz, dtype, &g, 1);
  if (rc) return rc;
  tune_set(dtype, g, nb, flags);
  return DDA_OK;
}

int dda_tuning_get(int dtype, int nx, int ny, int nz, int Lx, int Ly, int Lz, int nb, int* flags) {
  if (!flags || nb < 1) { set_error("null flags or nb < 1"); return DDA_ERR_ARG; }
  Geo g;
  int rc = make_geo(nx, ny, nz, Lx, Ly, Lz, dtype, &g, 1);
  if (rc) return rc;
  if (!tune_get(dtype, g, nb, flags)) { set_error("no tuning entry"); return DDA_ERR_ARG; }
  return DDA_OK;
}

int dda_green_build(dda_ctx* ctx, int nx, int ny, int nz, int Lx, int Ly, int Lz, double k, double d, double scale,
                    int layout, void* out_c128, void* out_c64, void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  Geo g;
  if ((rc = make_geo(nx, ny, nz, Lx, Ly, Lz, DDA_C128, &g))) return rc;
  if (!(k > 0) || !(d > 0)) { set_error("k and d must be positive"); return DDA_ERR_ARG; }
  if (!out_c128 && !out_c64) { set_error("no output"); return DDA_ERR_ARG; }
  if (layout != DDA_GHAT_REFERENCE && layout != DDA_GHAT_ENGINE) { set_error("bad octant layout"); return DDA_ERR_ARG; }
  return green_build(ctx->c, g, k, d, scale, out_c128, out_c64, layout == DDA_GHAT_ENGINE ? 1 : 0,
                     (cudaStream_t)stream);
}

int dda_ghat_to_engine(dda_ctx* ctx, int dtype, int hx, int hy, int hz, const void* src, void* dst, void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!src || !dst || src == dst) { set_error("octant conversion needs distinct src and dst"); return DDA_ERR_ARG; }
  if (hx < 1 || hy < 1 || hz < 1) { set_error("bad octant extents"); return DDA_ERR_BAD_SHAPE; }
  if (dtype != DDA_C64 && dtype != DDA_C128) { set_error("bad dtype"); return DDA_ERR_ARG; }
  if (ghat_to_soa(src, dst, (long long)hx * hy * hz, dtype == DDA_C128, (cudaStream_t)stream)) {
    set_error("octant conversion launch failed");
    return DDA_ERR_CUDA;
  }
  return DDA_OK;
}

int dda_op_create(dda_ctx* ctx, int dtype, int nx, int ny, int nz, int Lx, int Ly, int Lz, const void* ghat,
                  double gscale, const void* inv_alpha, dda_op** out) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!out || !ghat || !inv_alpha) { set_error("null argument"); return DDA_ERR_ARG; }
  if (dtype != DDA_C64 && dtype != DDA_C128) { set_error("bad dtype"); return DDA_ERR_ARG; }
  *out = nullptr;
  Geo g;
  if ((rc = make_geo(nx, ny, nz, Lx, Ly, Lz, dtype, &g))) return rc;
  dda_op* op = new (std::nothrow) dda_op();
  if (!op) { set_error("host allocation failed"); return DDA_ERR_OOM; }
  op->ctx = ctx; op->dtype = dtype; op->g = g; op->gscale = gscale; op->ghat = ghat; op->inva = inv_alpha;
  op->pc = make_pass_cfg(g, dtype == DDA_C128);
  // transform scratch is allocated on the first dda_matvec (solves use the
  // context's workspaces instead)
  *out = op;
  return DDA_OK;
}

static int op_scratch(dda_op* op) {
  if (op->scratch) return DDA_OK;
  const size_t esz = op->dtype == DDA_C128 ? 16 : 8;
  const size_t t1n = (size_t)op->g.nx * op->g.ny * op->g.Lz * 3, t2n = (size_t)op->g.nx * op->g.Ly * op->g.Lz * 3;
  if (cudaMalloc(&op->scratch, (t1n + t2n) * esz) != cudaSuccess ||
      cudaMalloc((void**)&op->d_st, sizeof(InstState)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(op->scratch);
    op->scratch = nullptr;
    set_error("operator scratch: out of device memory");
    return DDA_ERR_OOM;
  }
  return DDA_OK;
}

void dda_op_destroy(dda_op* op) {
  if (!op) return;
  cudaSetDevice(op->ctx->c.device);
  if (op->scratch) cudaFree(op->scratch);     // cudaFree waits for work using it
  if (op->d_st) cudaFree(op->d_st);
  delete op;
}

int dda_matvec(dda_op* op, int mode, const void* x, void* y, const void* b, void* stream) {
  if (!op) { set_error("null operator"); return DDA_ERR_ARG; }
  int rc = check_ctx(op->ctx);
  if (rc) return rc;
  if (!x || !y || (mode == DDA_MV_RESIDUAL && !b)) { set_error("null vector"); return DDA_ERR_ARG; }
  if (mode < 0 || mode > 3) { set_error("bad matvec mode"); return DDA_ERR_ARG; }
  if (x == y) { set_error("x and y must not alias"); return DDA_ERR_ARG; }
  if ((rc = op_scratch(op))) return rc;
  InstState S;
  std::memset(&S, 0, sizeof(S));
  S.vec[V_R] = (void*)x;
  S.vec[V_RHAT] = y;
  S.vec[V_B] = (void*)b;
  S.ghat = op->ghat;
  S.inva = op->inva;
  const size_t esz = op->dtype == DDA_C128 ? 16 : 8;
  S.t1 = op->scratch;
  S.t2 = (char*)op->scratch + (size_t)op->g.nx * op->g.ny * op->g.Lz * 3 * esz;
  S.active = 1;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(op->d_st, &S, sizeof(S), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  if (op->dtype == DDA_C128)
    e = launch_matvec<double>(op->ctx->c, op->g, op->pc, op->d_st, nullptr, 1, V_R, V_RHAT, mode, C_ALWAYS,
                              op->gscale, s);
  else
    e = launch_matvec<float>(op->ctx->c, op->g, op->pc, op->d_st, nullptr, 1, V_R, V_RHAT, mode, C_ALWAYS,
                             op->gscale, s);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  return DDA_OK;
}

int dda_matvec_batch(dda_op* const* ops, int nb, int mode, const void* const* x, void* const* y,
                     const void* const* b, void* stream) {
  if (!ops || nb < 1 || !x || !y) { set_error("bad batch arguments"); return DDA_ERR_ARG; }
  if (mode < 0 || mode > 3 || (mode == DDA_MV_RESIDUAL && !b)) { set_error("bad matvec mode"); return DDA_ERR_ARG; }
  const dda_op* o0 = ops[0];
  if (!o0) { set_error("null operator"); return DDA_ERR_ARG; }
  int rc = check_ctx(o0->ctx);
  if (rc) return rc;
  for (int j = 0; j < nb; ++j) {
    const dda_op* o = ops[j];
    if (!o || o->ctx != o0->ctx || o->dtype != o0->dtype || o->gscale != o0->gscale || o->g.nx != o0->g.nx ||
        o->g.ny != o0->g.ny || o->g.nz != o0->g.nz || o->g.Lx != o0->g.Lx || o->g.Ly != o0->g.Ly ||
        o->g.Lz != o0->g.Lz) {
      set_error("batched operators must share context, dtype, box, FFT lengths and tensor scale");
      return DDA_ERR_ARG;
    }
    if (!x[j] || !y[j] || x[j] == y[j] || (mode == DDA_MV_RESIDUAL && !b[j])) {
      set_error("null or aliased vector");
      return DDA_ERR_ARG;
    }
  }
  Ctx& c = o0->ctx->c;
  cudaSetDevice(c.device);
  int err = DDA_OK;
  BatchWs* w = c.workspace(o0->dtype, o0->g, nb, false, &err, 1);
  if (!w) return err;
  std::vector<InstState> H(nb);
  for (int j = 0; j < nb; ++j) {
    w->base_state(j, H[j]);
    H[j].vec[V_R] = (void*)x[j];
    H[j].vec[V_RHAT] = y[j];
    H[j].vec[V_B] = b ? (void*)b[j] : nullptr;
    H[j].ghat = ops[j]->ghat;
    H[j].inva = ops[j]->inva;
    H[j].active = 1;
  }
  cudaStream_t s = (cudaStream_t)stream;
  // pageable source: the copy is staged before the call returns
  cudaError_t e = cudaMemcpyAsync(w->d_st, H.data(), nb * sizeof(InstState), cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  if (o0->dtype == DDA_C128)
    e = launch_matvec<double>(c, o0->g, w->pc, w->d_st, nullptr, nb, V_R, V_RHAT, mode, C_ALWAYS, o0->gscale, s);
  else
    e = launch_matvec<float>(c, o0->g, w->pc, w->d_st, nullptr, nb, V_R, V_RHAT, mode, C_ALWAYS, o0->gscale, s);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  return DDA_OK;
}

int dda_precond_build(dda_ctx* ctx, int nx, int ny, int nz, int Lx, int Ly, int Lz, double k, double d,
                      const void* inv_alpha128, int layout, void* out_c128, void* out_c64, void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  Geo g;
  if ((rc = make_geo(nx, ny, nz, Lx, Ly, Lz, DDA_C128, &g, 1))) return rc;
  if (!(k > 0) || !(d > 0)) { set_error("k and d must be positive"); return DDA_ERR_ARG; }
  if (!inv_alpha128) { set_error("null inverse polarizability"); return DDA_ERR_ARG; }
  if (!out_c128 && !out_c64) { set_error("no output"); return DDA_ERR_ARG; }
  if (layout != DDA_GHAT_REFERENCE && layout != DDA_GHAT_ENGINE) { set_error("bad octant layout"); return DDA_ERR_ARG; }
  return precond_build(ctx->c, g, k, d, inv_alpha128, layout, out_c128, out_c64, (cudaStream_t)stream);
}

int dda_precond_op_create(dda_ctx* ctx, int dtype, int nx, int ny, int nz, int Lx, int Ly, int Lz, const void* phat,
                          double scale, const void* inv_alpha, dda_op** out) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!out || !phat || !inv_alpha) { set_error("null argument"); return DDA_ERR_ARG; }
  if (dtype != DDA_C64 && dtype != DDA_C128) { set_error("bad dtype"); return DDA_ERR_ARG; }
  *out = nullptr;
  Geo g;
  if ((rc = make_geo(nx, ny, nz, Lx, Ly, Lz, dtype, &g, 1))) return rc;
  dda_op* op = new (std::nothrow) dda_op();
  if (!op) { set_error("host allocation failed"); return DDA_ERR_OOM; }
  op->ctx = ctx; op->dtype = dtype; op->g = g; op->gscale = scale; op->ghat = phat; op->inva = inv_alpha;
  op->pc = make_pass_cfg(g, dtype == DDA_C128);
  *out = op;
  return DDA_OK;
}

static int pre_spec(const dda_ctx* ctx, int nx, int ny, int nz, int Px, int Py, int Pz, double pscale,
                    const void* const* phat, int nb, int dtype, PreSpec* ps) {
  (void)ctx;
  if (!phat) { set_error("null preconditioner list"); return DDA_ERR_ARG; }
  for (int j = 0; j < nb; ++j)
    if (!phat[j]) { set_error("null preconditioner octant"); return DDA_ERR_ARG; }
  int rc = make_geo(nx, ny, nz, Px, Py, Pz, dtype, &ps->g, 1);
  if (rc) return rc;
  ps->scale = pscale;
  ps->phat = phat;
  return DDA_OK;
}

int dda_gpbicgstab_pre(dda_op* op, const dda_op* pre, const void* e_inc, double target, int max_iter, double ratio,
                       void* p_out, dda_result* res, void* stream) {
  if (!op || !pre) { set_error("null operator"); return DDA_ERR_ARG; }
  if (pre->ctx != op->ctx || pre->dtype != op->dtype || pre->g.nx != op->g.nx || pre->g.ny != op->g.ny ||
      pre->g.nz != op->g.nz) {
    set_error("preconditioner must share the operator's context, dtype and box");
    return DDA_ERR_ARG;
  }
  dda_instance in{op->ghat, op->inva, e_inc, p_out};
  const void* ph[1] = {pre->ghat};
  return dda_solve_batch_pre(op->ctx, op->dtype, op->g.nx, op->g.ny, op->g.nz, op->g.Lx, op->g.Ly, op->g.Lz,
                             op->gscale, pre->g.Lx, pre->g.Ly, pre->g.Lz, pre->gscale, ph, &in, 1, target, max_iter,
                             ratio, res, stream);
}

int dda_gpbicgstab(dda_op* op, const void* e_inc, double target, int max_iter, double ratio, void* p_out,
                   dda_result* res, void* stream) {
  if (!op) { set_error("null operator"); return DDA_ERR_ARG; }
  dda_instance in{op->ghat, op->inva, e_inc, p_out};
  return dda_solve_batch(op->ctx, op->dtype, op->g.nx, op->g.ny, op->g.nz, op->g.Lx, op->g.Ly, op->g.Lz, op->gscale,
                         &in, 1, target, max_iter, ratio, res, stream);
}

int dda_solve_batch(dda_ctx* ctx, int dtype, int nx, int ny, int nz, int Lx, int Ly, int Lz, double gscale,
                    const dda_instance* inst, int nb, double target, int max_iter, double ratio, dda_result* res,
                    void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!inst || nb < 1) { set_error("no instances"); return DDA_ERR_ARG; }
  if (dtype != DDA_C64 && dtype != DDA_C128) { set_error("bad dtype"); return DDA_ERR_ARG; }
  Geo g;
  if ((rc = make_geo(nx, ny, nz, Lx, Ly, Lz, dtype, &g))) return rc;
  for (int j = 0; j < nb; ++j)
    if (!inst[j].ghat || !inst[j].inv_alpha || !inst[j].e_inc || !inst[j].p_out) {
      set_error("null instance pointer");
      return DDA_ERR_ARG;
    }
  if (dtype == DDA_C128)
    return solve_batch<double>(ctx->c, g, gscale, inst, nb, target, max_iter, ratio, res, (cudaStream_t)stream);
  return solve_batch<float>(ctx->c, g, gscale, inst, nb, target, max_iter, ratio, res, (cudaStream_t)stream);
}

int dda_solve_batch_pre(dda_ctx* ctx, int dtype, int nx, int ny, int nz, int Lx, int Ly, int Lz, double gscale,
                        int Px, int Py, int Pz, double pscale, const void* const* phat, const dda_instance* inst,
                        int nb, double target, int max_iter, double ratio, dda_result* res, void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!inst || nb < 1) { set_error("no instances"); return DDA_ERR_ARG; }
  if (dtype != DDA_C64 && dtype != DDA_C128) { set_error("bad dtype"); return DDA_ERR_ARG; }
  Geo g;
  if ((rc = make_geo(nx, ny, nz, Lx, Ly, Lz, dtype, &g))) return rc;
  PreSpec ps;
  if ((rc = pre_spec(ctx, nx, ny, nz, Px, Py, Pz, pscale, phat, nb, dtype, &ps))) return rc;
  for (int j = 0; j < nb; ++j)
    if (!inst[j].ghat || !inst[j].inv_alpha || !inst[j].e_inc || !inst[j].p_out) {
      set_error("null instance pointer");
      return DDA_ERR_ARG;
    }
  if (dtype == DDA_C128)
    return solve_batch<double>(ctx->c, g, gscale, inst, nb, target, max_iter, ratio, res, (cudaStream_t)stream, &ps);
  return solve_batch<float>(ctx->c, g, gscale, inst, nb, target, max_iter, ratio, res, (cudaStream_t)stream, &ps);
}

int dda_solve_mixed_batch_pre(dda_ctx* ctx, int nx, int ny, int nz, int Lx, int Ly, int Lz, double gscale, int Px,
                              int Py, int Pz, double pscale, const void* const* phat64, const dda_instance* inst64,
                              const dda_instance* inst128, int nb, double tol, double inner_tol, int max_iter,
                              int max_outer, double ratio, dda_result* res, void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!inst64 || !inst128 || nb < 1) { set_error("no instances"); return DDA_ERR_ARG; }
  Geo g;
  if ((rc = make_geo(nx, ny, nz, Lx, Ly, Lz, DDA_C128, &g))) return rc;
  PreSpec ps;
  if ((rc = pre_spec(ctx, nx, ny, nz, Px, Py, Pz, pscale, phat64, nb, DDA_C64, &ps))) return rc;
  for (int j = 0; j < nb; ++j)
    if (!inst64[j].ghat || !inst64[j].inv_alpha || !inst128[j].ghat || !inst128[j].inv_alpha || !inst128[j].e_inc ||
        !inst128[j].p_out) {
      set_error("null instance pointer");
      return DDA_ERR_ARG;
    }
  return solve_mixed(ctx->c, g, gscale, inst64, inst128, nb, tol, inner_tol, max_iter, max_outer, ratio, res,
                     (cudaStream_t)stream, &ps);
}

int dda_solve_mixed_batch(dda_ctx* ctx, int nx, int ny, int nz, int Lx, int Ly, int Lz, double gscale,
                          const dda_instance* inst64, const dda_instance* inst128, int nb, double tol,
                          double inner_tol, int max_iter, int max_outer, double ratio, dda_result* res,
                          void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!inst64 || !inst128 || nb < 1) { set_error("no instances"); return DDA_ERR_ARG; }
  Geo g;
  if ((rc = make_geo(nx, ny, nz, Lx, Ly, Lz, DDA_C128, &g))) return rc;
  for (int j = 0; j < nb; ++j)
    if (!inst64[j].ghat || !inst64[j].inv_alpha || !inst128[j].ghat || !inst128[j].inv_alpha || !inst128[j].e_inc ||
        !inst128[j].p_out) {
      set_error("null instance pointer");
      return DDA_ERR_ARG;
    }
  return solve_mixed(ctx->c, g, gscale, inst64, inst128, nb, tol, inner_tol, max_iter, max_outer, ratio, res,
                     (cudaStream_t)stream);
}

int dda_voxelize(dda_ctx* ctx, int dtype, const dda_shape* shapes, int nshape, int nx, int ny, int nz, double d,
                 const double* origin3, void* inv_alpha_out, void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!shapes || nshape < 1 || !inv_alpha_out || !(d > 0)) { set_error("bad voxelize arguments"); return DDA_ERR_ARG; }
  if (nx < 1 || ny < 1 || nz < 1) { set_error("box dimensions must be >= 1"); return DDA_ERR_BAD_SHAPE; }
  if (dtype != DDA_C64 && dtype != DDA_C128) { set_error("bad dtype"); return DDA_ERR_ARG; }
  for (int i = 0; i < nshape; ++i)
    if (shapes[i].type < DDA_SHAPE_SPHERE || shapes[i].type > DDA_SHAPE_PRISM ||
        (shapes[i].type == DDA_SHAPE_PRISM && shapes[i].sides < 3) || shapes[i].axis < 0 || shapes[i].axis > 2) {
      set_error("bad shape description");
      return DDA_ERR_ARG;
    }
  const double zero[3] = {0, 0, 0};
  cudaStream_t s = (cudaStream_t)stream;
  dda_shape* dev = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&dev, sizeof(dda_shape) * nshape, s);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_OOM; }
  e = cudaMemcpyAsync(dev, shapes, sizeof(dda_shape) * nshape, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && voxelize(dev, nshape, nx, ny, nz, d, origin3 ? origin3 : zero, dtype == DDA_C128,
                                   inv_alpha_out, ctx->c.num_sms, s))
    e = cudaErrorLaunchFailure;
  cudaFreeAsync(dev, s);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return DDA_ERR_CUDA; }
  return DDA_OK;
}

int dda_incident_field(dda_ctx* ctx, int dtype, int nx, int ny, int nz, double d, const double* k3,
                       const double* pol6, void* e_out, void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!k3 || !pol6 || !e_out) { set_error("null argument"); return DDA_ERR_ARG; }
  if (nx < 1 || ny < 1 || nz < 1) { set_error("box dimensions must be >= 1"); return DDA_ERR_BAD_SHAPE; }
  if (dtype != DDA_C64 && dtype != DDA_C128) { set_error("bad dtype"); return DDA_ERR_ARG; }
  if (plane_wave(nx, ny, nz, d, k3, pol6, dtype == DDA_C128, e_out, ctx->c.num_sms, (cudaStream_t)stream)) {
    set_error("incident field launch failed");
    return DDA_ERR_CUDA;
  }
  return DDA_OK;
}

int dda_cross_sections(dda_ctx* ctx, int dtype, long long nsite, const void* p, const void* e_inc,
                       const void* inv_alpha, double k, double e0, double* out3, void* stream) {
  int rc = check_ctx(ctx);
  if (rc) return rc;
  if (!p || !e_inc || !inv_alpha || !out3 || nsite < 0) { set_error("null argument"); return DDA_ERR_ARG; }
  if (!(e0 != 0.0)) { set_error("E0 must be non-zero"); return DDA_ERR_ARG; }
  Ctx& c = ctx->c;
  cudaStream_t s = c.stream;
  cudaError_t e;
  if ((e = cudaEventRecord(c.ev_user, (cudaStream_t)stream)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(s, c.ev_user, 0)) != cudaSuccess) {
    set_error(cudaGetErrorString(e));
    return DDA_ERR_CUDA;
  }
  long long want = (nsite + 255) / 256;
  int RB = (int)std::max<long long>(1, std::min<long long>(want, 4LL * c.num_sms));
  if (dtype == DDA_C128) launch_xsec<double>(p, e_inc, inv_alpha, nsite, k, c.xred, c.xcnt, RB, c.xout, s);
  else launch_xsec<float>(p, e_inc, inv_alpha, nsite, k, c.xred, c.xcnt, RB, c.xout, s);
  if ((e = cudaMemcpyAsync(c.xout_h, c.xout, 2 * sizeof(double), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess) {
    set_error(cudaGetErrorString(e));
    return DDA_ERR_CUDA;
  }
  const double* h = c.xout_h;
  const double pref = 4.0 * M_PI * k / (std::fabs(e0) * std::fabs(e0));
  out3[0] = pref * h[0];
  out3[1] = pref * h[1];
  out3[2] = out3[0] - out3[1];
  return DDA_OK;
}

}  // extern "C"
