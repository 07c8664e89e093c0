// GPBiCGSTAB on the device: fused vector updates, deterministic reductions
// and the reference's control logic, for a batch of independent instances.
//
// The recurrence, restarts, true-residual replacement, best-iterate tracking
// and return codes follow Gpbicgstab.py:957-1201 (precon=False, so M = I,
// Gpbicgstab.py:634-635).  All decisions the reference takes on the host after
// its per-iteration `.get()` (Gpbicgstab.py:1076) are taken here by the last
// CTA of a reduction, so an iteration needs no host round trip:
//
//   MV(p -> v)                                  5 transform passes
//   k_alpha  : <rhat, v>          -> alpha = rho1 / <rhat, v>
//   k_sy     : s = r - alpha v ;  y = s_prev - s - alpha w
//   MV(s -> t)
//   k_zeta   : <t,s>,<t,t> (first form) or the six dots of y,t,s -> zeta, eta
//   k_uzrx   : u, z, r, x updates ; ||r||^2, <rhat, r>  -> control (i != 1)
//   MV_res(x -> r), k_norm            only at i == 1    -> control
//   MV_res(x -> r)                    on a reset with i % 100 != 0
//   k_fin    : reset: rhat = r, p = r ; else w = t + beta v, p = r + beta(p-u)
//              swap s / s_prev, i += 1
//
// Dots and norms accumulate in FP64 whatever the vector precision.
#include "dda_host.h"
#include "krylov_ctrl.cuh"

namespace dda {

template <class C> __device__ __forceinline__ C tocr(double2 z) { return mk<C>(z.x, z.y); }

// ---------------------------------------------------------------------------
// control: the body of the reference loop after the residual norm
// (Gpbicgstab.py:1076-1158).  Runs in one thread.
// ---------------------------------------------------------------------------
__device__ void ctrl_check(InstState& S, double norm2, double2 rho_new) {
  const double cur = sqrt(norm2);
  const int i = S.iter;
  S.current = cur;
  if (i == 0) S.first = cur;
  S.last_change += 1;
  if (!isnan(cur) && (isnan(S.lowest) || cur < S.lowest)) {
    S.last_change = 0;
    S.lowest = cur;
    S.best_x = S.cur_x;
  }
  if (isnan(cur) || S.last_change >= 5000) {
    S.done = 1;
    S.status = isnan(cur) ? ST_NAN : ST_STAGNATED;
    S.ret_iters = -(i + 1);
    return;
  }
  if (cur < S.target * S.initial_norm) {
    S.done = 1;
    S.status = ST_CONVERGED;
    S.ret_iters = i + 1;
    return;
  }
  bool reset = false;
  S.rho0 = S.rho1;
  S.rho1 = rho_new;
  if (S.ratio != 0.0) {
    if (i == 2 || (i > 2 && cur < S.prev_lowest / S.ratio)) {
      reset = true;
      S.prev_lowest = cur;
      S.last_change = 0;
    }
  }
  S.flag_reset = reset ? 1 : 0;
  S.flag_reset_res = (reset && (i % 100 != 0)) ? 1 : 0;
  if (!reset) S.beta = zmul(zdiv(S.alpha, S.zeta), zdiv(S.rho1, S.rho0));
}

// ---------------------------------------------------------------------------
// initialisation: r = rhat = p = b, x = 0, other vectors 0
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(KNT) k_init(InstState* st, const int* act, double* red, unsigned* cnt, long long n3,
                                              int RB) {
  grid_dep_begin();
  typedef typename CT<R>::T C;
  const int inst = kinst(act);
  InstState& S = st[inst];
  if (!S.active) return;
  const C* __restrict__ b = (const C*)S.vec[V_B];
  C* r = (C*)S.vec[V_R]; C* rh = (C*)S.vec[V_RHAT]; C* p = (C*)S.vec[V_P];
  C* xa = (C*)S.vec[V_XA];
  C* zs[7] = {(C*)S.vec[V_V], (C*)S.vec[V_T], (C*)S.vec[V_S], (C*)S.vec[V_SPREV], (C*)S.vec[V_U], (C*)S.vec[V_Z],
              (C*)S.vec[V_W]};
  double acc[1] = {0.0};
  grid_loop<KU>(S.nv, (long long)blockIdx.x * KNT + threadIdx.x, (long long)RB * KNT, [&](long long i) {
    const C bv = b[i];
    r[i] = bv; rh[i] = bv; p[i] = bv;
    xa[i] = czero<C>();
#pragma unroll
    for (int j = 0; j < 7; ++j) zs[j][i] = czero<C>();
    acc[0] += (double)bv.x * bv.x + (double)bv.y * bv.y;
  });
  double tot[1];
  if (reduce_last<1>(acc, tot, red, cnt, inst, RB) && threadIdx.x == 0) {
    const double nrm = sqrt(tot[0]);
    S.initial_norm = nrm; S.bnorm = nrm;
    S.lowest = nrm; S.current = nrm; S.prev_lowest = nrm; S.first = 0.0;
    S.rho1 = make_double2(tot[0], 0.0);
    S.rho0 = S.rho1;
    S.alpha = S.beta = S.zeta = S.eta = make_double2(0.0, 0.0);
    S.iter = 0; S.last_change = 0; S.was_reset = 0; S.reset_count = 0;
    S.done = 0; S.status = ST_RUNNING; S.ret_iters = 0;
    S.flag_true_res = 0; S.flag_reset = 0; S.flag_reset_res = 0;
    S.cur_x = 0; S.best_x = -1;
    S.vec[V_X] = S.vec[V_XA];
    if (S.max_iter <= 0) { S.done = 1; S.status = ST_MAXITER; S.ret_iters = S.max_iter; }
  }
}

// alpha = rho1 / <rhat, v>   (Gpbicgstab.py:1019)
template <typename R>
__global__ void __launch_bounds__(KNT) k_alpha(InstState* st, const int* act, double* red, unsigned* cnt, long long n3,
                                               int RB) {
  grid_dep_begin();
  typedef typename CT<R>::T C;
  const int inst = kinst(act);
  InstState& S = st[inst];
  if (!cond_ok(S, C_ACTIVE)) return;
  const C* __restrict__ rh = (const C*)S.vec[V_RHAT];
  const C* __restrict__ v = (const C*)S.vec[V_V];
  double acc[2] = {0.0, 0.0};
  grid_loop<KU>(S.nv, (long long)blockIdx.x * KNT + threadIdx.x, (long long)RB * KNT, [&](long long i) {
    const C a = rh[i], b = v[i];
    acc[0] += (double)a.x * b.x + (double)a.y * b.y;
    acc[1] += (double)a.x * b.y - (double)a.y * b.x;
  });
  double tot[2];
  if (reduce_last<2>(acc, tot, red, cnt, inst, RB) && threadIdx.x == 0) alpha_from_dot(S, tot);
}

// s = r - alpha v ; y = s_prev - s - alpha w   (Gpbicgstab.py:1020-1021)
template <typename R>
__global__ void __launch_bounds__(KNT) k_sy(InstState* st, const int* act, long long n3) {
  grid_dep_begin();
  typedef typename CT<R>::T C;
  const int inst = kinst(act);
  InstState& S = st[inst];
  if (!cond_ok(S, C_ACTIVE)) return;
  const C* __restrict__ r = (const C*)S.vec[V_R];
  const C* __restrict__ v = (const C*)S.vec[V_V];
  const C* __restrict__ sp = (const C*)S.vec[V_SPREV];
  const C* __restrict__ w = (const C*)S.vec[V_W];
  C* __restrict__ s = (C*)S.vec[V_S];
  C* __restrict__ y = (C*)S.vec[V_Y];
  const C al = tocr<C>(S.alpha);
  grid_loop<KU>(S.nv, (long long)blockIdx.x * KNT + threadIdx.x, (long long)gridDim.x * KNT, [&](long long i) {
    const C sv = csub(r[i], cmul(al, v[i]));
    s[i] = sv;
    y[i] = csub(csub(sp[i], sv), cmul(al, w[i]));
  });
}

// zeta, eta  (Gpbicgstab.py:1038-1052, calculate_zeta_eta_twostep :239-380)
template <typename R>
__global__ void __launch_bounds__(KNT) k_zeta(InstState* st, const int* act, double* red, unsigned* cnt, long long n3,
                                              int RB) {
  grid_dep_begin();
  typedef typename CT<R>::T C;
  const int inst = kinst(act);
  InstState& S = st[inst];
  if (!cond_ok(S, C_ACTIVE)) return;
  const bool first = (S.iter == 0) || S.was_reset;
  const C* __restrict__ t = (const C*)S.vec[V_T];
  const C* __restrict__ s = (const C*)S.vec[V_S];
  const C* __restrict__ y = (const C*)S.vec[V_Y];
  double acc[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) acc[k] = 0.0;
  if (first) {
    grid_loop<KU>(S.nv, (long long)blockIdx.x * KNT + threadIdx.x, (long long)RB * KNT, [&](long long i) {
      const C tv = t[i], sv = s[i];
      acc[0] += (double)tv.x * tv.x + (double)tv.y * tv.y;            // <t,t>
      acc[1] += (double)tv.x * sv.x + (double)tv.y * sv.y;            // <t,s>
      acc[2] += (double)tv.x * sv.y - (double)tv.y * sv.x;
    });
  } else {
    grid_loop<KU>(S.nv, (long long)blockIdx.x * KNT + threadIdx.x, (long long)RB * KNT, [&](long long i) {
      const C tv = t[i], sv = s[i], yv = y[i];
      zeta_dots_acc(acc, tv, sv, yv);
    });
  }
  double tot[8];
  if (reduce_last<8>(acc, tot, red, cnt, inst, RB) && threadIdx.x == 0) zeta_eta_from_dots(S, tot, first);
}

// u, z, r, x updates (Gpbicgstab.py:1038-1057) and ||r||^2, <rhat, r>
// SETC: the kernel switches the graph's conditional residual matvecs (a
// separate instantiation, so the plain one stays visible to profilers)
template <typename R, bool SETC>
__global__ void __launch_bounds__(KNT) k_uzrx(InstState* st, const int* act, double* red, unsigned* cnt, long long n3,
                                              int RB, unsigned long long cond_true, unsigned long long cond_reset) {
  grid_dep_begin();
  typedef typename CT<R>::T C;
  const int inst = kinst(act);
  InstState& S = st[inst];
  if (!cond_ok(S, C_ACTIVE)) return;
  const bool first = (S.iter == 0) || S.was_reset;
  const int cur = S.cur_x;
  int nxt = 0;
  while (nxt == cur || nxt == S.best_x) ++nxt;
  const C* __restrict__ v = (const C*)S.vec[V_V];
  const C* __restrict__ sp = (const C*)S.vec[V_SPREV];
  const C* __restrict__ s = (const C*)S.vec[V_S];
  const C* __restrict__ y = (const C*)S.vec[V_Y];
  const C* __restrict__ t = (const C*)S.vec[V_T];
  const C* __restrict__ p = (const C*)S.vec[V_P];
  const C* __restrict__ rh = (const C*)S.vec[V_RHAT];
  const C* __restrict__ xo = (const C*)S.vec[V_XA + cur];
  C* __restrict__ xn = (C*)S.vec[V_XA + nxt];
  C* __restrict__ r = (C*)S.vec[V_R];
  C* __restrict__ u = (C*)S.vec[V_U];
  C* __restrict__ z = (C*)S.vec[V_Z];
  const C ze = tocr<C>(S.zeta), et = tocr<C>(S.eta), al = tocr<C>(S.alpha), be = tocr<C>(S.beta);
  double acc[3] = {0.0, 0.0, 0.0};
  grid_loop<KU>(S.nv, (long long)blockIdx.x * KNT + threadIdx.x, (long long)RB * KNT, [&](long long i) {
    C un, zn, rn;
    if (first) {
      un = cmul(ze, v[i]);
      zn = cmul(ze, s[i]);
      rn = csub(s[i], cmul(ze, t[i]));
    } else {
      const C ro = r[i];
      un = cadd(cmul(ze, v[i]), cmul(et, cadd(csub(sp[i], ro), cmul(be, u[i]))));
      zn = csub(cadd(cmul(ze, ro), cmul(et, z[i])), cmul(al, un));
      rn = csub(csub(s[i], cmul(et, y[i])), cmul(ze, t[i]));
    }
    u[i] = un; z[i] = zn; r[i] = rn;
    xn[i] = cadd(cadd(xo[i], cmul(al, p[i])), zn);
    const C h = rh[i];
    acc[0] += (double)rn.x * rn.x + (double)rn.y * rn.y;
    acc[1] += (double)h.x * rn.x + (double)h.y * rn.y;
    acc[2] += (double)h.x * rn.y - (double)h.y * rn.x;
  });
  double tot[3];
  if (reduce_last<3>(acc, tot, red, cnt, inst, RB) && threadIdx.x == 0) {
    S.cur_x = nxt;
    S.vec[V_X] = S.vec[V_XA + nxt];
    if (!S.flag_true_res) ctrl_check(S, tot[0], make_double2(tot[1], tot[2]));
    if constexpr (SETC) {
      if (S.flag_true_res && !S.done) cudaGraphSetConditional(cond_true, 1);
      if (S.flag_reset && S.flag_reset_res && !S.done) cudaGraphSetConditional(cond_reset, 1);
    }
  }
}

// ||r||^2, <rhat, r> after the i == 1 true residual (Gpbicgstab.py:1059-1076)
template <typename R, bool SETC>
__global__ void __launch_bounds__(KNT) k_norm(InstState* st, const int* act, double* red, unsigned* cnt, long long n3,
                                              int RB, unsigned long long cond_reset) {
  grid_dep_begin();
  typedef typename CT<R>::T C;
  const int inst = kinst(act);
  InstState& S = st[inst];
  if (!cond_ok(S, C_TRUE_RES)) return;
  const C* __restrict__ r = (const C*)S.vec[V_R];
  const C* __restrict__ rh = (const C*)S.vec[V_RHAT];
  double acc[3] = {0.0, 0.0, 0.0};
  grid_loop<KU>(S.nv, (long long)blockIdx.x * KNT + threadIdx.x, (long long)RB * KNT, [&](long long i) {
    const C rn = r[i], h = rh[i];
    acc[0] += (double)rn.x * rn.x + (double)rn.y * rn.y;
    acc[1] += (double)h.x * rn.x + (double)h.y * rn.y;
    acc[2] += (double)h.x * rn.y - (double)h.y * rn.x;
  });
  double tot[3];
  if (reduce_last<3>(acc, tot, red, cnt, inst, RB) && threadIdx.x == 0) {
    ctrl_check(S, tot[0], make_double2(tot[1], tot[2]));
    if constexpr (SETC) {
      if (S.flag_reset && S.flag_reset_res && !S.done) cudaGraphSetConditional(cond_reset, 1);
    }
  }
}

// end of iteration: reset copies or the w / p updates; buffer swap; i += 1
// (Gpbicgstab.py:1139-1158)
template <typename R>
__global__ void __launch_bounds__(KNT) k_fin(InstState* st, const int* act, unsigned* cnt, long long n3, int RB) {
  grid_dep_begin();
  typedef typename CT<R>::T C;
  const int inst = kinst(act);
  InstState& S = st[inst];
  if (!cond_ok(S, C_ACTIVE)) return;
  const bool reset = S.flag_reset;
  const C* __restrict__ r = (const C*)S.vec[V_R];
  C* __restrict__ p = (C*)S.vec[V_P];
  if (reset) {
    C* __restrict__ rh = (C*)S.vec[V_RHAT];
    grid_loop<KU>(S.nv, (long long)blockIdx.x * KNT + threadIdx.x, (long long)RB * KNT, [&](long long i) {
      const C rv = r[i];
      rh[i] = rv; p[i] = rv;
    });
  } else {
    const C* __restrict__ t = (const C*)S.vec[V_T];
    const C* __restrict__ v = (const C*)S.vec[V_V];
    const C* __restrict__ u = (const C*)S.vec[V_U];
    C* __restrict__ w = (C*)S.vec[V_W];
    const C be = tocr<C>(S.beta);
    grid_loop<KU>(S.nv, (long long)blockIdx.x * KNT + threadIdx.x, (long long)RB * KNT, [&](long long i) {
      w[i] = cadd(t[i], cmul(be, v[i]));
      p[i] = cadd(r[i], cmul(be, csub(p[i], u[i])));
    });
  }
  if (finish_last(cnt, inst, RB) && threadIdx.x == 0) {
    void* tmp = S.vec[V_S]; S.vec[V_S] = S.vec[V_SPREV]; S.vec[V_SPREV] = tmp;
    S.was_reset = reset ? 1 : 0;
    if (reset) { S.beta = make_double2(0.0, 0.0); S.reset_count += 1; }
    S.flag_reset = 0; S.flag_reset_res = 0;
    S.iter += 1;
    S.flag_true_res = (S.iter == 1) ? 1 : 0;
    if (S.iter >= S.max_iter && !S.done) {
      S.done = 1; S.status = ST_MAXITER; S.ret_iters = S.max_iter;
    }
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------


template <typename R> void launch_init(const KrylovLaunch& k, cudaStream_t s) {
  launch_pdl(k_init<R>, dim3(k.RB, k.nb), dim3(KNT), 0, s, k.st, k.act, k.red, k.cnt, k.n3, k.RB);
  note_launch(s, 1);
}
template <typename R> void launch_alpha(const KrylovLaunch& k, cudaStream_t s) {
  launch_pdl(k_alpha<R>, dim3(k.RB, k.nb), dim3(KNT), 0, s, k.st, k.act, k.red, k.cnt, k.n3, k.RB);
  note_launch(s, 1);
}
template <typename R> void launch_sy(const KrylovLaunch& k, cudaStream_t s) {
  launch_pdl(k_sy<R>, dim3(k.RB, k.nb), dim3(KNT), 0, s, k.st, k.act, k.n3);
  note_launch(s, 1);
}
template <typename R> void launch_zeta(const KrylovLaunch& k, cudaStream_t s) {
  launch_pdl(k_zeta<R>, dim3(k.RB, k.nb), dim3(KNT), 0, s, k.st, k.act, k.red, k.cnt, k.n3, k.RB);
  note_launch(s, 1);
}
template <typename R> void launch_uzrx(const KrylovLaunch& k, cudaStream_t s) {
  if (k.cond_true && k.cond_reset)
    launch_pdl(k_uzrx<R, true>, dim3(k.RB, k.nb), dim3(KNT), 0, s, k.st, k.act, k.red, k.cnt, k.n3, k.RB, k.cond_true,
               k.cond_reset);
  else
    launch_pdl(k_uzrx<R, false>, dim3(k.RB, k.nb), dim3(KNT), 0, s, k.st, k.act, k.red, k.cnt, k.n3, k.RB, 0ull, 0ull);
  note_launch(s, 1);
}
template <typename R> void launch_norm(const KrylovLaunch& k, cudaStream_t s) {
  if (k.cond_reset)
    launch_pdl(k_norm<R, true>, dim3(k.RB, k.nb), dim3(KNT), 0, s, k.st, k.act, k.red, k.cnt, k.n3, k.RB, k.cond_reset);
  else
    launch_pdl(k_norm<R, false>, dim3(k.RB, k.nb), dim3(KNT), 0, s, k.st, k.act, k.red, k.cnt, k.n3, k.RB, 0ull);
  note_launch(s, 1);
}
template <typename R> void launch_fin(const KrylovLaunch& k, cudaStream_t s) {
  launch_pdl(k_fin<R>, dim3(k.RB, k.nb), dim3(KNT), 0, s, k.st, k.act, k.cnt, k.n3, k.RB);
  note_launch(s, 1);
}

#define DDA_INST(R)                                                   \
  template void launch_init<R>(const KrylovLaunch&, cudaStream_t);   \
  template void launch_alpha<R>(const KrylovLaunch&, cudaStream_t);  \
  template void launch_sy<R>(const KrylovLaunch&, cudaStream_t);     \
  template void launch_zeta<R>(const KrylovLaunch&, cudaStream_t);   \
  template void launch_uzrx<R>(const KrylovLaunch&, cudaStream_t);   \
  template void launch_norm<R>(const KrylovLaunch&, cudaStream_t);   \
  template void launch_fin<R>(const KrylovLaunch&, cudaStream_t);
DDA_INST(float)
DDA_INST(double)

}  // namespace dda
