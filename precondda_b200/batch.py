"""Many geometries of uneven size solved together on one GPU.

Each geometry (a lattice with its own k and d) carries several right-hand
sides (polarisations x incidence directions).  Geometries are padded into
size buckets -- zero inverse polarizability in the padding is exactly an
empty voxel, so the physics does not change -- and every bucket is a slot
pool (``serve.SlotPool``) holding all right-hand sides of its geometries.
The pools run on their own streams and are advanced round-robin, so buckets
of different size are in flight on the device at the same time, and each
pool retires converged right-hand sides while the rest continue (the
reference solves one right-hand side of one lattice at a time,
Gpbicgstab.py:879-1201).  The synthetic workloads live in workloads.py.

``PaddingTuner`` picks each geometry's padded box and FFT lengths: for every
candidate shape (per-axis padding to the next bucket edge, or the enclosing
cube, whose kernels are specialised at compile time) it times the batched
matvec on the device once and keeps the cheapest per right-hand side.
``LaunchTuner`` then picks, per bucket and batch width, the matvec launch
variant (x-pass kernel and CTAs per SM, fused or separate z/y passes) the
same way and records it in the engine's tuning table.
"""
from __future__ import annotations

import itertools
import json
import math
import os
import time
from collections import defaultdict
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L
from .engine import _C64, _C128, _device, fft_lengths, green_octant_pair, compiled_fft_lengths, free_device_bytes
from .engine import Preconditioner
from .serve import SlotPool, precond_bytes, request_bytes, slot_bytes

DEFAULT_EDGES = (8, 12, 16, 20, 24, 32, 40, 48, 64, 72, 80, 96, 128, 144, 160, 192, 256)


@dataclass
class Geometry:
    """One lattice: inverse polarizability (nx,ny,nz) and its right-hand sides."""
    inv_alpha: torch.Tensor
    k: float
    d: float
    E_incs: list
    tag: dict = field(default_factory=dict)

    @property
    def shape(self):
        return tuple(int(v) for v in self.inv_alpha.shape)


# --------------------------------------------------------------------------
# padding autotuner
# --------------------------------------------------------------------------
def _next_edge(n, edges):
    for e in sorted(edges):
        if e >= n:
            return int(e)
    raise ValueError(f"box edge {n} exceeds the largest bucket edge {max(edges)}")


class PaddingTuner:
    """Chooses (padded box, FFT lengths) per geometry by timing the
    batched matvec of each candidate shape once (results cached, optionally
    in a JSON file)."""

    def __init__(self, precision="mixed", edges=DEFAULT_EDGES, nb=16, device=None, cache_path=None, measure=True):
        self.device = _device(device)
        self.dtype = _C64 if precision in ("mixed", "c64") else _C128
        self.edges = tuple(edges)
        self.nb = int(nb)
        self.measure = measure
        self.cache_path = cache_path
        self.times: dict = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.times = {tuple(json.loads(k)): v for k, v in json.load(f).items()}

    def candidates(self, shape):
        pad = tuple(_next_edge(n, self.edges) for n in shape)
        c = _next_edge(max(shape), self.edges)
        out = {pad, (c, c, c)}
        return sorted(out)

    def lengths(self, box):
        sizes = compiled_fft_lengths(self.dtype)
        return tuple(2 * b if 2 * b in sizes else min(s for s in sizes if s >= 2 * b) for b in box)

    def cost(self, box):
        """Seconds per right-hand side per matvec for a padded box."""
        L_ = self.lengths(box)
        key = tuple(box) + tuple(L_) + (self.nb,)
        if key in self.times:
            return self.times[key]
        if not self.measure:
            n = np.prod(L_)
            t = 1e-12 * n * math.log2(n) * 3 + 1e-9 * np.prod(box)
        else:
            t = self._time(box, L_)
        self.times[key] = t
        if self.cache_path:
            with open(self.cache_path, "w") as f:
                json.dump({json.dumps(list(k)): v for k, v in self.times.items()}, f)
        return t

    def _time(self, box, L_):
        # one matvec of a filled box of this shape (the solver's cost per
        # iteration is two matvecs plus streaming updates over the box)
        from .engine import DDAOperator
        dev = self.device
        ia = torch.full(box, 1.0 / (0.02 + 0.002j), dtype=_C128, device=dev)
        op = DDAOperator(ia, 6.0, 0.05, dtype=self.dtype, L_=L_, device=dev)
        x = torch.randn(*box, 3, dtype=self.dtype, device=dev)
        for _ in range(2):
            op.matvec(x)
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        reps = 5
        e0.record()
        for _ in range(reps):
            op.matvec(x)
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    def plan(self, shapes):
        """[(box, L)] per geometry shape."""
        out = []
        for s in shapes:
            best = min(self.candidates(s), key=lambda b: self.cost(b))
            out.append((best, self.lengths(best)))
        return out


# --------------------------------------------------------------------------
# launch-variant autotuner
# --------------------------------------------------------------------------
def launch_candidates(box, L_, dtype, nb):
    """DDA_TUNE_* flag sets worth timing for one bucket.  Cubic boxes on the
    (2n)^3 grid of 64^3 and 128^3, where the variants are built: for
    complex64 the one-tile, staged or packed-pair x pass, plain or
    packed-pair y and z passes, and with and without the cluster-fused z/y
    passes (one-instance 64^3 launches, where they are the default, and any
    128^3 launch, where they are not).  Other buckets, and complex128, have
    the default only.  (The L2 prefetch of DDA_TUNE_PREFETCH measured slower
    at every size and precision and is not a candidate.)"""
    cube = box[0] == box[1] == box[2] and L_[0] == L_[1] == L_[2] == 2 * box[0]
    if not (cube and L_[0] in (128, 256)) or dtype != _C64:
        return [0]
    x_opts = [0, L.DDA_TUNE_P3PIPE, L.DDA_TUNE_P3PAIR]
    y_opts = [0, L.DDA_TUNE_YPAIR | L.DDA_TUNE_ZPAIR]
    pf_opts = [0]
    zy_opts = [0]
    if L_[0] == 128 and nb == 1:
        zy_opts = [0, L.DDA_TUNE_NO_FUSED_ZY | L.DDA_TUNE_NO_FUSED_INV]
    elif L_[0] == 256:
        zy_opts = [0, L.DDA_TUNE_FUSED]
    return [a | y | p | b for a in x_opts for y in y_opts for p in pf_opts for b in zy_opts]


class LaunchTuner:
    """Picks the matvec launch variant (block shapes: which x-pass kernel
    and how many of its CTAs per SM, fused or separate z/y passes) per
    (dtype, padded box, FFT lengths, batch-width class) by timing a batched
    matvec of each candidate on the device, L2 flushed between launches.
    A candidate replaces the default launch only when it is faster by more
    than ``margin`` (3 %: the isolated matvec of a filled box stands in for
    the solver's launches, so near-ties keep the default).  The winner goes
    into the engine's tuning table (dda_tuning_set), and
    into an optional JSON cache so later runs skip the timing.  ``timer``
    replaces the device timing (tests)."""

    def __init__(self, device=None, cache_path=None, reps=5, timer=None, margin=0.03):
        self.device = _device(device) if timer is None else None
        self.margin = float(margin)
        self.cache_path = cache_path
        self.reps = int(reps)
        self.timer = timer
        self.best: dict = {}
        self.times: dict = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.best = {tuple(json.loads(k)): v for k, v in json.load(f).items()}

    @staticmethod
    def key(box, L_, dtype, nb):
        return (0 if dtype == _C64 else 1,) + tuple(int(v) for v in box) + tuple(int(v) for v in L_) + \
            (int(nb),)

    def tune(self, box, L_, dtype, nb):
        """Flags chosen for this bucket (measured once, then cached)."""
        k = self.key(box, L_, dtype, nb)
        if k not in self.best:
            cands = launch_candidates(box, L_, dtype, nb)
            if len(cands) == 1:
                self.best[k] = cands[0]
            else:
                t = {f: self._time(box, L_, dtype, nb, f) for f in cands}
                self.times[k] = t
                best = min(t, key=t.get)
                # a variant replaces the default only when measurably faster
                if 0 in t and t[best] > (1.0 - self.margin) * t[0]:
                    best = 0
                self.best[k] = best
            if self.cache_path:
                with open(self.cache_path, "w") as f:
                    json.dump({json.dumps(list(kk)): v for kk, v in self.best.items()}, f)
        self.apply(box, L_, dtype, nb, self.best[k])
        return self.best[k]

    def apply(self, box, L_, dtype, nb, flags):
        if self.timer is not None:
            return
        code = L.DDA_C64 if dtype == _C64 else L.DDA_C128
        L.check(L.lib().dda_tuning_set(code, *[int(v) for v in box], *[int(v) for v in L_], int(nb), int(flags)))

    def _time(self, box, L_, dtype, nb, flags):
        if self.timer is not None:
            return self.timer(box, L_, dtype, nb, flags)
        from .engine import DDAOperator, matvec_batch
        dev = self.device
        self.apply(box, L_, dtype, nb, flags)
        ia = torch.full(box, 1.0 / (0.02 + 0.002j), dtype=_C128, device=dev)
        op = DDAOperator(ia, 6.0, 0.05, dtype=dtype, L_=L_, device=dev)
        xs = [torch.randn(*box, 3, dtype=dtype, device=dev) for _ in range(nb)]
        flush = torch.empty(48 << 20, dtype=torch.float32, device=dev)      # 192 MB > L2
        run = (lambda: matvec_batch([op] * nb, xs)) if nb > 1 else (lambda: op.matvec(xs[0]))
        for _ in range(2):
            run()
        ts = []
        for _ in range(self.reps):
            flush.add_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            run()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        return float(np.median(ts))


# --------------------------------------------------------------------------
# execution
# --------------------------------------------------------------------------
def _pad(t, box, extra=()):
    if tuple(t.shape[:3]) == tuple(box):
        return t.contiguous()
    out = torch.zeros(tuple(box) + tuple(extra), dtype=t.dtype, device=t.device)
    nx, ny, nz = t.shape[:3]
    out[:nx, :ny, :nz] = t
    return out


@dataclass
class BatchResult:
    P: list            # per geometry: list of P (cropped to the geometry's box), one per RHS
    info: list         # per geometry: list of SolveInfo
    plan: list         # per geometry: (box, L)
    seconds: float     # device-synchronised wall time of the solve phase
    solves: int


def green_bytes(L_):
    """Both precisions of one FFT'd interaction octant."""
    return 6 * (L_[0] // 2 + 1) * (L_[1] // 2 + 1) * (L_[2] // 2 + 1) * (16 + 8)


def item_bytes(box, L_, precision, nrhs, ngeom, precondition=False):
    """Device bytes a bucket item holds while it runs: its slot pool, the
    per-request tensors and padded copies, and one octant per geometry (two
    with a preconditioner)."""
    n = box[0] * box[1] * box[2]
    per_rhs = slot_bytes(box, L_, precision, precondition) + request_bytes(box, precision) + 3 * n * 16 + n * 8
    return nrhs * per_rhs + ngeom * (green_bytes(L_) + n * 16 + (precond_bytes(L_, precision) if precondition else 0))


def solve_geometries(geoms, tol=1e-5, precision="mixed", inner_tol=1e-4, max_iter=2000, max_outer=12,
                     ratio=100.0, chunk=8, tuner=None, hbm_budget=None, device=None, keep_results=True,
                     on_result=None, precondition=False):
    """Solve every right-hand side of every geometry.

    Buckets (geometries sharing a padded box and FFT lengths) become slot
    pools; pools are started while the HBM budget (default 75% of the free
    memory) allows, advanced round-robin on their own streams, and a new
    bucket starts as soon as a running one finishes.  ``precondition`` runs
    the reference's precon=True solve with one engine preconditioner per
    geometry (its padded lattice, the bucket's FFT grid).  ``on_result(g, j,
    P, info)`` is called for each finished right-hand side (P cropped to the
    geometry's box); P is also kept in the result unless ``keep_results`` is
    False."""
    from collections import deque
    dev = _device(device)
    tuner = tuner or PaddingTuner(precision, device=dev)
    plan = tuner.plan([g.shape for g in geoms])
    groups = defaultdict(list)
    for gi, (box, L_) in enumerate(plan):
        groups[(box, L_)].append(gi)
    free = free_device_bytes(dev)
    if hbm_budget is None:
        hbm_budget = int(0.75 * free)
    # items: buckets, largest first, split so that each fits the budget
    items = deque()
    for key in sorted(groups, key=lambda k: -np.prod(k[0])):
        box, L_ = key
        acc = []
        for g in groups[key]:
            trial = acc + [g]
            if acc and item_bytes(box, L_, precision, sum(len(geoms[x].E_incs) for x in trial),
                                  len(trial), precondition) > hbm_budget:
                items.append((key, acc))
                acc = [g]
            else:
                acc = trial
        if acc:
            items.append((key, acc))

    Ps = [[None] * len(g.E_incs) for g in geoms]
    infos = [[None] * len(g.E_incs) for g in geoms]

    def start(key, gl):
        box, L_ = key
        nrhs = sum(len(geoms[g].E_incs) for g in gl)
        pool = SlotPool(box, L_, nrhs, precision, 1.0, dev, precond_L=L_ if precondition else None)
        where, slot = {}, 0
        try:
            for g in gl:
                G = geoms[g]
                g128, g64 = green_octant_pair(box, G.k, G.d, L_, 1.0 / (L_[0] * L_[1] * L_[2]), dev)
                ia = _pad(G.inv_alpha.to(_C128), box)
                pre = (Preconditioner(inv_alpha=ia, k=G.k, d=G.d, L_=L_, device=dev,
                                      dtypes=(_C128,) if precision == "c128" else (_C64,))
                       if precondition else None)
                if precision == "c64":
                    ia = ia.to(_C64)
                gh = (g64, g128) if precision == "mixed" else (g64 if precision == "c64" else g128)
                for j, E in enumerate(G.E_incs):
                    Ep = _pad(E.to(_C64 if precision == "c64" else _C128), box, (3,))
                    pool.admit(slot, gh, ia, Ep, tol=tol, inner_tol=inner_tol, max_iter=max_iter,
                               max_outer=max_outer, ratio=ratio, preconditioner=pre)
                    where[slot] = (g, j)
                    slot += 1
        except BaseException:
            pool.close()
            raise
        return pool, where, item_bytes(box, L_, precision, nrhs, len(gl), precondition)

    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    active, fresh, used = [], [], 0
    seq, chunk_seq = itertools.count(), {}     # order in which each pool's current chunk was enqueued
    while items or active or fresh:
        while items:
            key, gl = items[0]
            est = item_bytes(key[0], key[1], precision, sum(len(geoms[g].E_incs) for g in gl), len(gl),
                             precondition)
            if (active or fresh) and used + est > hbm_budget:
                break
            try:
                entry = start(key, gl)
            except (MemoryError, torch.cuda.OutOfMemoryError):
                if not (active or fresh):
                    raise
                torch.cuda.empty_cache()
                break
            items.popleft()
            entry[0].run(chunk)             # a new pool starts iterating at once
            chunk_seq[id(entry[0])] = next(seq)
            fresh.append(entry)
            used += entry[2]
        # pools whose last chunk has finished are polled and given their next
        # chunk right away, so no pool waits for the slowest one; when none
        # has finished, the loop waits for the chunk enqueued first
        ready = [e[0].ready() for e in active]
        if active and not any(ready):
            ready[min(range(len(active)), key=lambda i: chunk_seq[id(active[i][0])])] = True
        still = []
        for (pool, where, est), rdy in zip(active, ready):
            if not rdy:
                still.append((pool, where, est))
                continue
            for s, info, P in pool.poll():
                g, j = where[s]
                nx, ny, nz = geoms[g].shape
                Pc = P[:nx, :ny, :nz]
                infos[g][j] = info
                if on_result is not None:
                    on_result(g, j, Pc, info)
                if keep_results:
                    Ps[g][j] = Pc
            if pool.running:
                pool.run(chunk)
                chunk_seq[id(pool)] = next(seq)
                still.append((pool, where, est))
            else:
                pool.close()
                used -= est
        active = still + fresh
        fresh = []
    torch.cuda.synchronize(dev)
    secs = time.perf_counter() - t0
    n = sum(len(g.E_incs) for g in geoms)
    return BatchResult(Ps, infos, plan, secs, n)
