"""Continuous-batching DDA solve server on one GPU.

Requests (a lattice: inverse polarizability + incident field, k, d) arrive
at any time.  Each is padded into a cubic size bucket -- zero polarizability
outside the scatterer is exactly what the reference's lattices carry in
their empty voxels, so padding changes no physics (the operator's rows and
columns of empty sites are zero and Krylov vectors stay zero there) -- and
admitted into a free slot of that bucket's :class:`SlotPool`.  A pool
iterates all its occupied slots together in one captured graph
(``dda_slots_run``); slots finish and are refilled independently
(``dda_slots_poll``), so a long solve never holds back short ones.

* Green cache: the FFT'd interaction tensor depends on the padded box, the
  FFT lengths, k and d only; it is built once per key on the device and
  shared by every request with that key (LRU under a byte budget).
* HBM admission: a bucket's pool is created with as many slots as fit the
  memory budget (``slots_per_bucket`` at most); requests wait in FIFO order
  while their bucket is full.
* Latency: per request, from submission to the poll that returned it;
  ``stats()`` gives p50 / p99 and throughput.

Every slot runs the reference's solve_gpbicgstab (Gpbicgstab.py:879-1201)
recurrence on its own state, so a request's result does not depend on what
else is in its pool (the GPU tests check this bit for bit).
"""
from __future__ import annotations

import ctypes as C
import math
import time
from collections import OrderedDict, deque
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L
from .engine import (SolveInfo, Preconditioner, _device, _info, as_device, fft_lengths, free_device_bytes,
                     green_octant_pair, stream_handle, _C64, _C128)

PRECISIONS = {"c64": L.DDA_PREC_C64, "c128": L.DDA_PREC_C128, "mixed": L.DDA_PREC_MIXED}
DEFAULT_BUCKETS = (8, 12, 16, 24, 32, 40, 48, 64, 80, 96, 128, 160, 192, 256)


def slot_bytes(box, L_, precision, precondition=False) -> int:
    """Device bytes one pool slot holds: 16 Krylov vectors (17 with the
    preconditioned vector) and the two FFT scratch volumes in the solver
    dtype, plus the FP64 right-hand side and residual of a mixed slot.  A
    preconditioner on the pool's FFT grid shares the scratch."""
    nx, ny, nz = box
    Lx, Ly, Lz = L_
    n3 = nx * ny * nz * 3
    esz = 16 if precision == "c128" else 8
    b = ((17 if precondition else 16) * n3 + nx * ny * Lz * 3 + nx * Ly * Lz * 3) * esz
    if precision == "mixed":
        b += 2 * n3 * 16
    return b


def precond_bytes(L_, precision="mixed") -> int:
    """One preconditioner octant in the precision a pool of ``precision``
    reads (complex64 for mixed and c64 pools)."""
    return 6 * (L_[0] // 2 + 1) * (L_[1] // 2 + 1) * (L_[2] // 2 + 1) * (16 if precision == "c128" else 8)


def request_bytes(box, precision, L_=None) -> int:
    """Per-request tensors: inv_alpha and E_inc / P in the solve precisions,
    plus the request's preconditioner octant (the solve precision) when L_
    (its grid) is given."""
    n = box[0] * box[1] * box[2]
    extra = precond_bytes(L_, precision) if L_ is not None else 0
    if precision == "mixed":
        return n * (8 + 16) + n * 3 * 16 * 2 + extra
    esz = 16 if precision == "c128" else 8
    return n * esz + n * 3 * esz * 2 + extra


def choose_bucket(shape, buckets=DEFAULT_BUCKETS) -> int:
    """Smallest cubic bucket edge that holds the lattice."""
    m = max(int(v) for v in shape)
    for b in sorted(buckets):
        if b >= m:
            return int(b)
    raise ValueError(f"lattice {tuple(shape)} exceeds the largest bucket {max(buckets)}")


def pool_slots(box, L_, precision, budget_bytes, cap, precondition=False) -> int:
    """Slots a pool may have under ``budget_bytes`` (HBM admission)."""
    per = slot_bytes(box, L_, precision, precondition) + request_bytes(box, precision,
                                                                       L_ if precondition else None)
    return int(max(0, min(int(cap), int(budget_bytes) // per)))


class SlotPool:
    """``dda_slots_*`` pool: ``nslots`` solver instances of one box / FFT size.
    ``precond_L``: make a preconditioned pool (the precon=True solve) whose
    requests bring a ``Preconditioner`` on that grid."""

    def __init__(self, box, L_, nslots, precision="mixed", gscale=1.0, device=None, precond_L=None):
        self.device = _device(device)
        self.box = tuple(int(v) for v in box)
        self.L = tuple(int(v) for v in L_)
        self.precision = precision
        self.nslots = int(nslots)
        self.precond_L = tuple(int(v) for v in precond_L) if precond_L is not None else None
        self._ctx = L.context(self.device.index)
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            if self.precond_L is None:
                L.check(L.lib().dda_slots_create(self._ctx.handle, PRECISIONS[precision], *self.box, *self.L,
                                                 float(gscale), self.nslots, C.byref(h)))
            else:
                P_ = self.precond_L
                L.check(L.lib().dda_slots_create_pre(self._ctx.handle, PRECISIONS[precision], *self.box, *self.L,
                                                     float(gscale), *P_, 1.0 / (P_[0] * P_[1] * P_[2]),
                                                     self.nslots, C.byref(h)))
        self._h = h
        self._fin = (C.c_int * self.nslots)()
        self._res = (L.dda_result * self.nslots)()
        self._keep = {}        # slot -> tensors the slot reads / writes

    def close(self):
        if getattr(self, "_h", None):
            L.lib().dda_slots_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def free_slot(self) -> int:
        return L.lib().dda_slots_free_slot(self._h)

    def admit(self, slot, ghat, inv_alpha, E_inc, tol=1e-5, inner_tol=1e-4, max_iter=2000, max_outer=12,
              ratio=100.0, preconditioner=None):
        """Start a solve in ``slot``.  ``ghat``: engine-layout octant, a
        (complex64, complex128) pair for mixed pools; inv_alpha / E_inc on the
        device in the pool's precision (complex128 for mixed pools);
        ``preconditioner`` (a ``Preconditioner`` on the pool's grid) for
        preconditioned pools.  Returns the output tensor, valid once the slot
        is reported finished."""
        if (self.precond_L is None) != (preconditioner is None):
            raise ValueError("a preconditioned pool needs a preconditioner per request, a plain one none")
        if preconditioner is not None and (preconditioner.L != self.precond_L or preconditioner.shape != self.box):
            raise ValueError("preconditioner grid / box differs from the pool's")
        lo, hi = L.dda_instance(), L.dda_instance()
        dev = self.device
        if self.precision == "mixed":
            g64, g128 = ghat
            ia128 = as_device(inv_alpha, _C128, dev)
            ia64 = ia128.to(_C64)
            E = as_device(E_inc, _C128, dev).reshape(*self.box, 3)
            P = torch.empty_like(E)
            lo.ghat, lo.inv_alpha = g64.data_ptr(), ia64.data_ptr()
            hi.ghat, hi.inv_alpha, hi.e_inc, hi.p_out = g128.data_ptr(), ia128.data_ptr(), E.data_ptr(), P.data_ptr()
            keep = (g64, g128, ia64, ia128, E, P)
        else:
            dt = _C64 if self.precision == "c64" else _C128
            g = ghat
            ia = as_device(inv_alpha, dt, dev)
            E = as_device(E_inc, dt, dev).reshape(*self.box, 3)
            P = torch.empty_like(E)
            inst = lo if self.precision == "c64" else hi
            inst.ghat, inst.inv_alpha, inst.e_inc, inst.p_out = g.data_ptr(), ia.data_ptr(), E.data_ptr(), P.data_ptr()
            keep = (g, ia, E, P)
        with torch.cuda.device(dev):
            if preconditioner is None:
                L.check(L.lib().dda_slots_admit(self._h, int(slot), C.byref(lo), C.byref(hi), float(tol),
                                                float(inner_tol), int(max_iter), int(max_outer), float(ratio),
                                                stream_handle(dev)))
            else:
                ph = preconditioner.octant(_C128 if self.precision == "c128" else _C64)
                keep = (preconditioner, ph) + keep
                L.check(L.lib().dda_slots_admit_pre(self._h, int(slot), C.byref(lo), C.byref(hi), ph.data_ptr(),
                                                    float(tol), float(inner_tol), int(max_iter), int(max_outer),
                                                    float(ratio), stream_handle(dev)))
        self._keep[int(slot)] = keep
        return P

    def run(self, niter):
        with torch.cuda.device(self.device):
            L.check(L.lib().dda_slots_run(self._h, int(niter)))

    def ready(self) -> bool:
        """Whether the pool's enqueued iterations have all finished (a poll
        would not wait)."""
        with torch.cuda.device(self.device):
            r = L.lib().dda_slots_ready(self._h)
        if r < 0:
            L.check(-r)
        return r == 1

    def poll(self):
        """[(slot, SolveInfo, P)] of the slots that finished; they become free."""
        nf, nr = C.c_int(0), C.c_int(0)
        with torch.cuda.device(self.device):
            L.check(L.lib().dda_slots_poll(self._h, self._fin, self._res, C.byref(nf), C.byref(nr)))
        self.running = nr.value
        out = []
        for q in range(nf.value):
            s = self._fin[q]
            keep = self._keep.pop(s)
            out.append((s, _info(self._res[q]), keep[-1]))
        return out

    def release(self, slot):
        L.check(L.lib().dda_slots_release(self._h, int(slot)))
        self._keep.pop(int(slot), None)


class GreenCache:
    """Device-resident FFT(-G) octants keyed by (box, L, k, d), LRU under a
    byte budget.  Entries are (complex64, complex128) engine-layout pairs
    from one FP64 build."""

    def __init__(self, budget_bytes=8 << 30, device=None):
        self.device = _device(device)
        self.budget = int(budget_bytes)
        self.bytes = 0
        self.hits = 0
        self.misses = 0
        self._d: OrderedDict = OrderedDict()

    @staticmethod
    def key(box, L_, k, d):
        return (tuple(int(v) for v in box), tuple(int(v) for v in L_), float(k), float(d))

    def get(self, box, L_, k, d):
        key = self.key(box, L_, k, d)
        if key in self._d:
            self._d.move_to_end(key)
            self.hits += 1
            return self._d[key]
        self.misses += 1
        g128, g64 = green_octant_pair(box, k, d, L_, 1.0 / (L_[0] * L_[1] * L_[2]), self.device)
        nbytes = g128.numel() * 16 + g64.numel() * 8
        while self._d and self.bytes + nbytes > self.budget:
            _, (a, b) = self._d.popitem(last=False)
            self.bytes -= a.numel() * 8 + b.numel() * 16
        self._d[key] = (g64, g128)
        self.bytes += nbytes
        return g64, g128

    def __len__(self):
        return len(self._d)


@dataclass
class Request:
    """One solve: inv_alpha (nx,ny,nz), E_inc (nx,ny,nz,3), k, d.

    Lazy form: inv_alpha = E_inc = None with ``shape`` set and ``build`` a
    callable returning (inv_alpha, E_inc); the arrays are then made only when
    the request is admitted into a slot, so a queue of waiting requests holds
    no device memory."""
    inv_alpha: object
    E_inc: object
    k: float
    d: float
    tol: float = 1e-5
    max_iter: int = 2000
    rid: int = -1
    t_submit: float = 0.0
    t_done: float = 0.0
    P: object = None
    info: SolveInfo | None = None
    bucket: int = 0
    shape: tuple = ()
    build: object = None
    pre_key: object = None     # requests with one key share one preconditioner (same lattice, k, d)


@dataclass
class _Bucket:
    n: int
    L: tuple
    pool: SlotPool
    queue: deque = field(default_factory=deque)
    active: dict = field(default_factory=dict)    # slot -> Request
    outstanding: bool = False                     # a chunk of iterations is enqueued and not yet polled
    nbytes: int = 0                               # HBM the pool holds, charged to the budget
    seq: int = 0                                  # order in which the outstanding chunk was enqueued


class DDAServer:
    """Continuous-batching server (one GPU, one pool per cubic size bucket).

    precision: 'mixed' (complex64 sweeps + FP64 refinement, the default),
    'c64' or 'c128'.  precondition: run every request as the reference's
    precon=True solve, with the engine's circulant preconditioner of its
    padded lattice on the bucket's FFT grid (built when the request is
    admitted).  hbm_budget: bytes the pools may hold (default: 60% of the
    free device memory at construction, after torch's cached blocks are
    released; the rest is left to Green builds, the Green cache and the
    requests' arrays).  A new bucket whose pool does not fit what is left
    closes idle buckets' pools, least recently used first; a request is
    refused (MemoryError) only when not one slot fits after that."""

    def __init__(self, precision="mixed", buckets=DEFAULT_BUCKETS, slots_per_bucket=16, chunk_iters=8,
                 hbm_budget=None, green_budget=8 << 30, inner_tol=1e-4, max_outer=12, ratio=100.0, device=None,
                 precondition=False, launch_tuner=None):
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        self.device = _device(device)
        self.precision = precision
        self.precondition = bool(precondition)
        self.buckets = tuple(sorted(int(b) for b in buckets))
        self.slots_per_bucket = int(slots_per_bucket)
        self.chunk = int(chunk_iters)
        if hbm_budget is None:
            # cached blocks (torch's, the engine's) are handed back first,
            # or they would count as used
            hbm_budget = int(0.6 * free_device_bytes(self.device))   # the rest: Green builds, caches, requests
        self.hbm_budget = int(hbm_budget)
        self.hbm_used = 0
        self.green = GreenCache(green_budget, self.device)
        self.inner_tol, self.max_outer, self.ratio = float(inner_tol), int(max_outer), float(ratio)
        self._b: dict[int, _Bucket] = {}
        self._next = 0
        self._seq = 0
        self.done: list[Request] = []
        self._pre: dict = {}       # pre_key -> [Preconditioner or None, requests not yet finished]
        # optional batch.LaunchTuner: each new bucket's matvec launch variant
        # is measured (complex64 sweeps, or the c128 solve) for its slot count
        self.launch_tuner = launch_tuner

    # -- buckets ------------------------------------------------------------
    def bucket_for(self, shape) -> int:
        return choose_bucket(shape, self.buckets)

    def _evict_idle(self, need):
        """Close the pools of idle buckets (nothing queued, running or
        enqueued), least recently used first, until ``need`` bytes of the
        budget are free or no idle bucket is left."""
        for n in list(self._b):
            if self.hbm_budget - self.hbm_used >= need:
                return
            b = self._b[n]
            if b.queue or b.active or b.outstanding:
                continue
            b.pool.close()
            self.hbm_used -= b.nbytes
            del self._b[n]

    def _bucket(self, n) -> _Bucket:
        if n in self._b:
            b = self._b.pop(n)       # most recently used last
            self._b[n] = b
            return b
        box = (n, n, n)
        L_ = fft_lengths(box, _C64 if self.precision == "c64" else _C128)
        pre = self.precondition
        per = slot_bytes(box, L_, self.precision, pre) + request_bytes(box, self.precision, L_ if pre else None)
        want = pool_slots(box, L_, self.precision, self.hbm_budget, self.slots_per_bucket, pre)
        if want >= 1 and self.hbm_budget - self.hbm_used < want * per:
            self._evict_idle(want * per)
        room = self.hbm_budget - self.hbm_used
        ns = pool_slots(box, L_, self.precision, room, self.slots_per_bucket, pre)
        if ns < 1:
            raise MemoryError(f"bucket {n}^3 needs {per / 2**20:.0f} MiB per slot; "
                              f"{room / 2**20:.0f} MiB of the HBM budget is left")
        if self.launch_tuner is not None:
            self.launch_tuner.tune(box, L_, _C128 if self.precision == "c128" else _C64, ns)
        pool = SlotPool(box, L_, ns, self.precision, 1.0, self.device, precond_L=L_ if pre else None)
        self.hbm_used += ns * per
        b = _Bucket(n, L_, pool, nbytes=ns * per)
        self._b[n] = b
        return b

    # -- requests -----------------------------------------------------------
    def submit(self, req: Request) -> Request:
        """Queue a request (arrays on the host or the device, or lazy)."""
        ia = req.inv_alpha
        if ia is None:
            if req.build is None or len(req.shape) != 3:
                raise ValueError("a lazy request needs build() and shape")
            shape = tuple(int(v) for v in req.shape)
        else:
            shape = tuple(int(v) for v in (ia.shape if hasattr(ia, "shape") else np.shape(ia)))
        if len(shape) != 3:
            raise ValueError("inv_alpha must have shape (nx, ny, nz)")
        req.shape = shape
        req.bucket = self.bucket_for(shape)
        # the bucket's pool first: a request its budget cannot hold is refused
        # (MemoryError) before anything is allocated or registered
        b = self._bucket(req.bucket)
        req.rid = self._next
        self._next += 1
        req.t_submit = time.perf_counter()
        if self.precondition and req.pre_key is not None:
            self._pre.setdefault(req.pre_key, [None, 0])[1] += 1
        b.queue.append(req)
        return req

    def _preconditioner(self, req, ia, L_):
        """The request's preconditioner (shared by requests with one pre_key)."""
        dts = (_C128,) if self.precision == "c128" else (_C64,)
        if req.pre_key is None:
            return Preconditioner(inv_alpha=ia, k=req.k, d=req.d, L_=L_, device=self.device, dtypes=dts)
        ent = self._pre[req.pre_key]
        if ent[0] is None:
            ent[0] = Preconditioner(inv_alpha=ia, k=req.k, d=req.d, L_=L_, device=self.device, dtypes=dts)
        return ent[0]

    def _release_pre(self, req):
        if self.precondition and req.pre_key is not None:
            ent = self._pre.get(req.pre_key)
            if ent is not None:
                ent[1] -= 1
                if ent[1] <= 0:
                    del self._pre[req.pre_key]

    def _pad(self, req, n):
        dt = _C64 if self.precision == "c64" else _C128
        ia = as_device(req.inv_alpha, dt, self.device)
        E = as_device(req.E_inc, dt, self.device).reshape(*req.shape, 3)
        if req.shape == (n, n, n):
            return ia, E
        nx, ny, nz = req.shape
        iap = torch.zeros((n, n, n), dtype=dt, device=self.device)
        Ep = torch.zeros((n, n, n, 3), dtype=dt, device=self.device)
        iap[:nx, :ny, :nz] = ia
        Ep[:nx, :ny, :nz] = E
        return iap, Ep

    def _fill(self, b: _Bucket):
        while b.queue:
            s = b.pool.free_slot()
            if s < 0:
                return
            req = b.queue.popleft()
            if req.inv_alpha is None:
                req.inv_alpha, req.E_inc = req.build()
            g64, g128 = self.green.get((b.n,) * 3, b.L, req.k, req.d)
            ghat = (g64, g128) if self.precision == "mixed" else (g64 if self.precision == "c64" else g128)
            ia, E = self._pad(req, b.n)
            pre = self._preconditioner(req, ia, b.L) if self.precondition else None
            b.pool.admit(s, ghat, ia, E, tol=req.tol, inner_tol=self.inner_tol, max_iter=req.max_iter,
                         max_outer=self.max_outer, ratio=self.ratio, preconditioner=pre)
            b.active[s] = req

    def pending(self) -> int:
        return sum(len(b.queue) + len(b.active) for b in self._b.values())

    def step(self) -> list:
        """For every bucket whose pool is idle: collect the requests its last
        chunk finished, admit waiting requests into the freed slots and
        enqueue the next ``chunk_iters`` iterations at once.  Pools still
        running their chunk are left alone, so a pool of short iterations is
        refilled as often as it finishes instead of once per chunk of the
        slowest pool; when no idle pool has work, the step waits for the
        chunk that was enqueued first.  Returns the finished requests."""
        out = []
        todo, busy = [], []
        for b in self._b.values():
            (busy if b.outstanding and not b.pool.ready() else todo).append(b)
        if busy and not any(b.outstanding or b.queue for b in todo):
            todo = [min(busy, key=lambda b: b.seq)]
        for b in todo:
            if b.outstanding:
                for s, info, P in b.pool.poll():
                    req = b.active.pop(s)
                    req.t_done = time.perf_counter()
                    nx, ny, nz = req.shape
                    req.P = P[:nx, :ny, :nz] if P.shape[:3] != req.shape else P
                    req.info = info
                    self._release_pre(req)
                    out.append(req)
                b.outstanding = False
            self._fill(b)
            if b.active:
                b.pool.run(self.chunk)
                b.outstanding = True
                self._seq += 1
                b.seq = self._seq
        self.done.extend(out)
        return out

    def drain(self, timeout_s=600.0) -> list:
        """Step until every submitted request has finished."""
        t0 = time.perf_counter()
        out = []
        while self.pending():
            out.extend(self.step())
            if time.perf_counter() - t0 > timeout_s:
                raise TimeoutError(f"{self.pending()} requests still running after {timeout_s} s")
        return out

    def serve(self, requests, arrivals_s=None, timeout_s=600.0) -> list:
        """Replay ``requests`` arriving at offsets ``arrivals_s`` (seconds
        from now; all at once when None) and run until all finish."""
        reqs = list(requests)
        arr = [0.0] * len(reqs) if arrivals_s is None else list(arrivals_s)
        order = sorted(range(len(reqs)), key=lambda j: arr[j])
        t0 = time.perf_counter()
        q = 0
        out = []
        while q < len(order) or self.pending():
            now = time.perf_counter() - t0
            while q < len(order) and arr[order[q]] <= now:
                r = self.submit(reqs[order[q]])
                r.t_submit = t0 + arr[order[q]]
                q += 1
            if self.pending():
                out.extend(self.step())
            elif q < len(order):
                time.sleep(max(0.0, min(1e-3, arr[order[q]] - now)))
            if now > timeout_s:
                raise TimeoutError("serve loop exceeded its time limit")
        return out

    def stats(self, reqs=None) -> dict:
        reqs = self.done if reqs is None else reqs
        if not reqs:
            return {"n": 0}
        lat = np.array([r.t_done - r.t_submit for r in reqs])
        span = max(r.t_done for r in reqs) - min(r.t_submit for r in reqs)
        return {"n": len(reqs), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3),
                "solves_per_s": len(reqs) / span if span > 0 else math.inf,
                "green_hits": self.green.hits, "green_misses": self.green.misses,
                "pools": {b.n: b.pool.nslots for b in self._b.values()}}

    def close(self):
        for b in self._b.values():
            b.pool.close()
        self._b.clear()
        self.hbm_used = 0
