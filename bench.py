#!/usr/bin/env python
"""DDA benchmark: solves/s of the mixed-precision GPBiCGSTAB solve on the
64^3 sphere precision workload (137,376 dipoles, m = 1.7+0.1i, |m|kd = 0.5,
x- and y-polarised plane waves along +z, complex64 sweeps to 1e-4 inside FP64
refinement to a true relative residual of 1e-6), plus the matvec roofline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line is printed by rank 0.  Under torchrun each rank solves its own
replica of the workload on its GPU (the solve does not shard); value is the
solves of all ranks over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import gc
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DDA solves/s, p99 latency, matvec GB/s; mixed vs FP64 at C_ext err≤1e-4"
WORKLOAD = "sphere64_precision: 64^3 box, 137376 dipoles, m=1.7+0.1i, |m|kd=0.5, lambda=0.5um, RR alpha, " \
           "x+y polarisations along +z, true relative residual 1e-6"
SOLVER = "c64 GPBiCGSTAB sweeps (tol 1e-4, right-preconditioned: precon=True with the engine's circulant) in FP64 " \
         "iterative refinement to 1e-6"
N_BOX, M_REF, KD_M, WAVELENGTH = 64, 1.7 + 0.1j, 0.5, 0.5
TOL, INNER_TOL, MAX_ITER, RATIO = 1e-6, 1e-4, 2000, 100.0
# Iterations the reference's complex128 GPBiCGSTAB (ratio 100, tol 1e-6) takes
# on this problem, x polarisation, measured with the CPU oracle; it scales the
# CPU per-iteration time to a whole solve for the CPU arms (oracle run: 123
# iterations, relative residual 7.0e-7).
REF_ITERS_64 = 123
# DRAM bytes (read + write) of the complex64 64^3 two-RHS matvec (five
# passes, both right-hand sides in one launch), from an ncu capture of that
# launch (bench.py --profile-matvec 64 --profile-rhs 2); the passes'
# intermediates stay in L2, so this is below the algorithmic bytes.
MATVEC64_C64_RHS2_DRAM_BYTES = 181.9e6


def problem(n=N_BOX, m=M_REF):
    from precondda_b200 import calculate_alpha, sphere_occupancy, incident_field
    k = 2 * math.pi / WAVELENGTH
    d = KD_M / (abs(m) * k)
    occ = sphere_occupancy(n, n / 2.0)
    alpha = np.where(occ, calculate_alpha(m, d, k, method="RR"), 0).astype(np.complex128)
    inv_alpha = np.where(occ, 1.0 / np.where(occ, alpha, 1), 0).astype(np.complex128)
    Ex = incident_field((n, n, n), d, k, (0, 0, 1), (1, 0, 0))
    Ey = incident_field((n, n, n), d, k, (0, 0, 1), (0, 1, 0))
    return k, d, inv_alpha, [Ex, Ey], int(occ.sum())


def matvec_bytes(shape, esz):
    """Algorithmic bytes of one pruned 5-pass matvec: c*[82 N + 6 (nx+1)(ny+1)(nz+1)]."""
    nx, ny, nz = shape
    return esz * (82 * nx * ny * nz + 6 * (nx + 1) * (ny + 1) * (nz + 1))


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region
    (every 50 ms, so that the default 0.2 s region gets several samples)."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        return self.start()

    def start(self, wait_s=5.0):
        """Start sampling and wait (bounded) for the first sample."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < wait_s and self.proc.poll() is None:
                time.sleep(0.05)
            self.lines.clear()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0])); mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init():
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v):
    """Largest value over the ranks (the slowest rank's time)."""
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(ws, units_per_rank, seconds):
    """Whole-job throughput of independent replicas: all ranks' units over
    the slowest rank's time."""
    return units_per_rank * ws / max_over_ranks(ws, seconds)


# --------------------------------------------------------------------------
# CPU arms (oracle port of the reference algorithm, complex128, all cores)
# --------------------------------------------------------------------------
REF_SOLVER = ("oracle port of the reference's solve_gpbicgstab (Gpbicgstab.py:879-1201), complex128, precon=False "
              "(the reference's runnable path: its preconditioner builder is missing), scipy.fft on all host cores")


class CpuSolve:
    """The CPU baseline: the oracle's complex128 restatement of the
    reference's GPBiCGSTAB on the workload, with its Green octant built once
    (timed) and iterations timed in real multi-iteration runs of the
    recurrence."""

    def __init__(self):
        from oracle import dda_oracle as O
        self.O = O
        self.k, self.d, self.ia, self.Es, _ = problem()
        self.mask = self.ia != 0
        t0 = time.perf_counter()
        self.G = O.generate_interaction_row(N_BOX, N_BOX, N_BOX, self.k, self.d)
        self.t_green = time.perf_counter() - t0

    def iteration_time(self, n_iter):
        """Seconds per iteration over one run of n_iter iterations."""
        t0 = time.perf_counter()
        self.O.solve_gpbicgstab((N_BOX,) * 3, self.ia, self.G, self.Es[0], self.mask, RATIO, n_iter, target=TOL)
        return (time.perf_counter() - t0) / n_iter

    def solves_per_s(self, t_it):
        return 1.0 / (self.t_green + t_it * REF_ITERS_64)


def run_reference(args, ws, rank):
    if rank != 0:
        return
    n_it = 3
    cpu = CpuSolve()
    for _ in range(args.warmup):
        cpu.iteration_time(1)
    samples = [cpu.iteration_time(n_it) for _ in range(args.steps)]
    t_it = statistics.median(samples)
    value = cpu.solves_per_s(t_it)
    cores = os.cpu_count()
    sample = (f"{n_it} iterations of the complex128 GPBiCGSTAB recurrence per step at 64^3 (FFT 128^3), x "
              f"polarisation; solves/s = 1 / (Green build {cpu.t_green:.2f} s + {REF_ITERS_64} iterations x the "
              f"median per-iteration time); {REF_ITERS_64} is the iteration count of the full solve to 1e-6")
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_it * n_it, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded sphere lattice)",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "solver": REF_SOLVER, "global_batch": 2, "parallelism": "replicas"},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------
def time_matvec(op, reps, flush):
    import torch
    x = torch.randn(*op.shape, 3, dtype=op.dtype, device=op.device)
    for _ in range(3):
        op.matvec(x)
    torch.cuda.synchronize()
    ts = []
    s = torch.cuda.current_stream()
    for _ in range(reps):
        flush.add_(1.0)          # evict L2 between launches
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        op.matvec(x)
        e1.record(s)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1) / 1e3)
    return statistics.median(ts)


def time_matvec_batch(ops, reps, flush):
    """Median time of one batched matvec launch sequence over len(ops)
    right-hand sides (the form the solver launches), L2 flushed before each."""
    import torch
    import precondda_b200 as P
    xs = [torch.randn(*op.shape, 3, dtype=op.dtype, device=op.device) for op in ops]
    for _ in range(3):
        P.engine.matvec_batch(ops, xs)
    torch.cuda.synchronize()
    ts = []
    s = torch.cuda.current_stream()
    for _ in range(reps):
        flush.add_(1.0)
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        P.engine.matvec_batch(ops, xs)
        e1.record(s)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1) / 1e3)
    return statistics.median(ts)


def ellipsoid128_16rhs(dev, seed=3):
    """The 128^3 mixed-over-plain measurement: the seeded rotated ellipsoid
    (semi-axes (64, 48, 40) d, |m|kd = 0.6) with 2 polarisations x 8
    incidence directions (16 right-hand sides), all solved in one batched
    mixed-precision launch (complex64 sweeps to 1e-4, FP64 refinement to
    1e-6, precon=True), against the plain complex128 GPU solve of one
    right-hand side at a time and the same 16 in one complex128 batch.
    C_ext / C_abs errors are taken against complex128 solves to 1e-10."""
    import torch
    import precondda_b200 as P
    from precondda_b200.workloads import ellipsoid128_spec, build_geometry, sphere_directions
    spec = ellipsoid128_spec(seed=seed)
    spec.pop("fixed_pols")
    spec["dirs"] = sphere_directions(8, np.random.default_rng(seed + 100))
    spec["pols"] = 2
    ia, k, d, Es = build_geometry(spec, dev)
    op = P.DDAOperator(ia, k, d, dtype=torch.complex128, device=dev, with_twin=True)
    pre = op.preconditioner()
    n = len(Es)
    stream = torch.cuda.current_stream(dev)

    def timed(fn):
        fn()                                   # warm-up: same batch size (workspace, graph capture)
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True); a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        out = fn()
        a1.record(stream)
        torch.cuda.synchronize()
        return a0.elapsed_time(a1) / 1e3, out

    t_mix, (Pm, im) = timed(lambda: P.solve_many([op] * n, Es, tol=TOL, max_iter=4000, ratio=RATIO,
                                                  precision="mixed", inner_tol=INNER_TOL, preconditioner=pre))
    t_one, (_, i1) = timed(lambda: P.solve_many([op], Es[:1], tol=TOL, max_iter=4000, ratio=RATIO,
                                                 precision="c128", preconditioner=pre))
    t_pb, (Pp, ip) = timed(lambda: P.solve_many([op] * n, Es, tol=TOL, max_iter=4000, ratio=RATIO,
                                                 precision="c128", preconditioner=pre))
    nerr = 2
    Pf, _ = P.solve_many([op] * nerr, Es[:nerr], tol=1e-10, max_iter=4000, ratio=RATIO, precision="c128",
                         preconditioner=pre)
    err = lambda a, b: abs(a - b) / abs(b)
    acc = []
    for j in range(nerr):
        cm, cp_, cf = (op.cross_sections(Pm[j], Es[j]), op.cross_sections(Pp[j], Es[j]),
                       op.cross_sections(Pf[j], Es[j]))
        acc.append({"mixed_C_ext_rel_err": err(cm[0], cf[0]), "mixed_C_abs_rel_err": err(cm[1], cf[1]),
                    "plain_C_ext_rel_err": err(cp_[0], cf[0]), "C_ext": cf[0], "C_abs": cf[1]})
    mixed = n / t_mix
    plain_one = 1.0 / t_one
    plain_batch = n / t_pb
    return {"workload": f"128^3 box, {int((ia != 0).sum().item())} dipoles, rotated ellipsoid (64,48,40)d, "
                        f"m={spec['m']:.4f}, |m|kd=0.6, 2 pols x 8 directions = {n} right-hand sides, tol 1e-6, "
                        f"precon=True",
            "mixed_batched_solves_per_s": mixed, "plain_c128_one_rhs_solves_per_s": plain_one,
            "plain_c128_batched_solves_per_s": plain_batch,
            "mixed_batched_over_plain_c128": mixed / plain_one,
            "mixed_batched_over_plain_c128_batched": mixed / plain_batch,
            "iterations": {"mixed_inner": [i.iters for i in im], "outer": [i.outer for i in im],
                           "plain_c128_one": i1[0].iters, "plain_c128_batched": [i.iters for i in ip]},
            "true_relres_max": max(i.true_relres for i in im),
            "accuracy_vs_fp64": acc,
            "seconds": {"mixed_batch": t_mix, "plain_one": t_one, "plain_batch": t_pb}}


def _extra(fn, *a):
    """One of the default line's extra workloads; a failure of one (an HBM
    budget refusal, an out-of-memory error, a time limit) is reported in its
    key and leaves the headline measurement standing."""
    import traceback
    try:
        return fn(*a)
    except (MemoryError, TimeoutError, ValueError, RuntimeError) as e:
        traceback.print_exc(file=sys.stderr)
        return {"error": f"{type(e).__name__}: {e}"}


def batch64_block(args, ws, rank, local):
    """The batching configuration (64 geometries x 16 right-hand sides)
    measured inside the default run, summarised (single GPU only)."""
    if ws != 1:
        return None
    a = argparse.Namespace(**vars(args))
    a.geometries, a.warmup, a.steps = 64, 1, 1
    gc.collect()
    ln = run_batch64(a, ws, rank, local, emit=False)
    return {"workload": ln["config"]["workload"], "solves_per_s": ln["value"], "e2e_solves_per_s": ln["e2e"]["value"],
            "converged": ln["converged"], "rhs": ln["config"]["global_batch"], "iterations": ln["iterations"],
            "solve_seconds": ln["solve_seconds"]}


def serve_block(args, ws, rank, local, rate=3.0, duration=20.0):
    """The serving configuration's request mix at a rate one GPU sustains
    (3 requests/s for 20 s), measured inside the default run: request and
    right-hand-side p50/p99 latency and solves/s (single GPU only)."""
    if ws != 1:
        return None
    a = argparse.Namespace(**vars(args))
    a.rates, a.duration = str(rate), duration
    gc.collect()            # the earlier blocks' operators, before the server sizes its budget
    ln = run_serve(a, ws, rank, local, emit=False)
    c = ln["curve"][-1]
    return {"workload": ln["config"]["workload"], "offered_requests_per_s": rate, "seconds": duration,
            "hbm_budget_GiB": ln["config"]["hbm_budget_GiB"], "pools": ln["config"]["pools"],
            "rhs_per_s": c["rhs_per_s"], "requests_per_s": c["requests_per_s"],
            "request_p50_ms": c["request_p50_ms"], "request_p99_ms": c["request_p99_ms"],
            "rhs_p50_ms": c["rhs_p50_ms"], "rhs_p99_ms": c["rhs_p99_ms"], "converged": c["converged"],
            "rhs": c["rhs"], "green_hits": c["green_hits"], "green_misses": c["green_misses"]}


def sphere32_plain(dev):
    """The plain-method configuration on the GPU: 32^3 sphere (17,256
    dipoles, m = 1.5+0.01i, |m|kd = 0.5), complex128 GPBiCGSTAB from P0 = 0,
    tol 1e-6, maxiter 2000, ratio 100, precon=False, x polarisation."""
    import torch
    import precondda_b200 as P
    k, d, ia, Es, ndip = problem(32, 1.5 + 0.01j)
    op = P.DDAOperator(ia, k, d, dtype=torch.complex128, device=dev)
    E = torch.as_tensor(Es[0], device=dev)
    op.solve(E, tol=TOL, max_iter=MAX_ITER, ratio=RATIO)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    a0 = torch.cuda.Event(enable_timing=True); a1 = torch.cuda.Event(enable_timing=True)
    reps = 5
    a0.record(stream)
    for _ in range(reps):
        Pg, info = op.solve(E, tol=TOL, max_iter=MAX_ITER, ratio=RATIO)
    a1.record(stream)
    torch.cuda.synchronize()
    t = a0.elapsed_time(a1) / 1e3 / reps
    cext, cabs, csca = op.cross_sections(Pg, E)
    return {"workload": f"32^3 sphere, {ndip} dipoles, m=1.5+0.01i, complex128 plain (precon=False), tol 1e-6",
            "solves_per_s": 1.0 / t, "iterations": info.iters, "C_ext": cext, "C_abs": cabs, "C_sca": csca}


def run_ours(args, ws, rank, local):
    import torch
    import precondda_b200 as P
    from precondda_b200 import _lib as L

    dev = torch.device("cuda", local)
    k, d, ia, Es, ndip = problem()
    op = P.DDAOperator(ia, k, d, dtype=torch.complex128, device=dev, with_twin=True)
    op64 = op.twin(torch.complex64)
    # the reference's precon=True solve with the engine's circulant
    # preconditioner on the operator's grid, built once per geometry like the
    # Green octant (inside the e2e step below)
    pre = op.preconditioner()
    # launch variants of the buckets the timed work runs, measured before it
    from precondda_b200.batch import LaunchTuner
    tuner = LaunchTuner(device=dev)
    if not args.no_tune:
        tuner.tune(op.shape, op.L, torch.complex64, 2)
        tuner.tune((128,) * 3, (256,) * 3, torch.complex64, 16)

    def step(precision="mixed", preconditioner=pre, tol=TOL):
        return P.solve_many([op, op], Es_dev, tol=tol, max_iter=MAX_ITER, ratio=RATIO, precision=precision,
                            inner_tol=INNER_TOL, preconditioner=preconditioner)

    def time_steps(n, **kw):
        """(solves/s, infos) of n steps timed on the stream."""
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True); a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(n):
            _, inf = step(**kw)
        a1.record(stream)
        torch.cuda.synchronize()
        return 2 * n / (a0.elapsed_time(a1) / 1e3), inf

    Es_dev = [torch.as_tensor(E, device=dev) for E in Es]
    stream = torch.cuda.current_stream(dev)
    for _ in range(max(args.warmup, 1)):
        Ps, infos = step()
    torch.cuda.synchronize()
    # --- timed region: device-resident inputs -------------------------------
    lc0 = L.lib().dda_kernel_launches()
    with ClockSampler(dev.index) as clk:
        barrier(ws)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lat = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            Ps, infos = step()
            lat.append(time.perf_counter() - t0)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(ws)
    launches = L.lib().dda_kernel_launches() - lc0
    t = e0.elapsed_time(e1) / 1e3
    t = max_over_ranks(ws, t)
    solves = 2 * args.steps * ws
    value = solves / t
    # --- end to end through the public API with host buffers ---------------
    ia_h = torch.from_numpy(ia).pin_memory()
    Es_h = [torch.from_numpy(E).pin_memory() for E in Es]
    h2d = ia_h.numel() * 16 + sum(E.numel() * 16 for E in Es_h)
    d2h = 0
    # pinned host buffers for the results (the D2H of P is part of the step)
    P_h = [torch.empty(E.shape, dtype=torch.complex128, pin_memory=True) for E in Es_h]
    copy_stream = torch.cuda.Stream(dev)

    def e2e_step():
        ia_d = ia_h.to(dev, non_blocking=True)
        # the incident fields cross on a second stream while the Green and
        # preconditioner builds (which need only inv_alpha) run
        copy_stream.wait_stream(stream)
        with torch.cuda.stream(copy_stream):
            Ed = [E.to(dev, non_blocking=True) for E in Es_h]
        op_e = P.DDAOperator(ia_d, k, d, dtype=torch.complex128, L_=op.L, device=dev, with_twin=True)
        pre_e = op_e.preconditioner()
        stream.wait_stream(copy_stream)
        for e_ in Ed:
            e_.record_stream(stream)
        Pe, inf_e = P.solve_many([op_e, op_e], Ed, tol=TOL, max_iter=MAX_ITER, ratio=RATIO, precision="mixed",
                                 inner_tol=INNER_TOL, preconditioner=pre_e)
        xs_ = [op_e.cross_sections(Pe[j], Ed[j]) for j in range(2)]
        for j in range(2):
            P_h[j].copy_(Pe[j], non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        return xs_

    # untimed warm-up of the end-to-end step, like the device-resident leg
    for _ in range(max(args.warmup, 1)):
        e2e_step()
    barrier(ws)
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True); f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    xs = None
    e2e_steps = []
    for _ in range(args.steps):
        ts0 = time.perf_counter()
        xs = e2e_step()
        e2e_steps.append(time.perf_counter() - ts0)
    d2h = sum(p.numel() * 16 for p in P_h)
    f1.record(stream)
    torch.cuda.synchronize()
    te = max_over_ranks(ws, f0.elapsed_time(f1) / 1e3)
    e2e = solves / te
    out = {}
    if rank == 0 and not args.no_extra:
        # --- accuracy: mixed vs all-FP64 solve -------------------------------
        Pf, inf_f = P.solve_many([op, op], Es_dev, tol=1e-10, max_iter=4000, ratio=RATIO, precision="c128")
        cerr = []
        for j in range(2):
            cm = op.cross_sections(Ps[j], Es_dev[j])
            cf = op.cross_sections(Pf[j], Es_dev[j])
            cerr.append({"C_ext_rel_err": abs(cm[0] - cf[0]) / abs(cf[0]),
                         "C_abs_rel_err": abs(cm[1] - cf[1]) / abs(cf[1]),
                         "P_rel_err": float(torch.linalg.vector_norm(Ps[j] - Pf[j]) /
                                            torch.linalg.vector_norm(Pf[j])),
                         "C_ext": cm[0], "C_abs": cm[1], "C_sca": cm[2]})
        # --- plain complex128 solves (denominator of the 3x target) and the
        # unpreconditioned solves (the reference's precon=False), same problem
        nplain = max(1, min(args.steps, 3))
        step(precision="c128")
        plain, inf_p = time_steps(nplain, precision="c128")
        step(preconditioner=None)
        mixed_np, inf_mnp = time_steps(nplain, preconditioner=None)
        step(precision="c128", preconditioner=None)
        plain_np, inf_pnp = time_steps(nplain, precision="c128", preconditioner=None)
        # --- roofline of the matvec (complex64, the inner solve's) -----------
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MB > L2
        # the dominant kernel as the timed solve launches it: one complex64
        # matvec over both right-hand sides (gridDim.y = 2)
        t_mv = time_matvec_batch([op64, op64], 20, flush)
        t_mv1 = time_matvec(op64, 20, flush)
        peak, peak_kind = measured_peak()
        B = matvec_bytes(op.shape, 8)
        ach = 2 * B / t_mv / 1e9
        roof = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "traffic": MATVEC64_C64_RHS2_DRAM_BYTES, "traffic_from": "ncu capture of this launch (profile)",
                "kernel": "5-pass matvec, complex64, 64^3 box (FFT 128^3), both right-hand sides in one launch",
                "algorithmic_bytes": 2 * B, "ms": t_mv * 1e3, "peak_kind": peak_kind,
                "single_rhs": {"ms": t_mv1 * 1e3, "GBps": B / t_mv1 / 1e9, "frac": B / t_mv1 / 1e9 / peak}}
        # 128^3 box (the large-solve size) for both precisions
        ia128 = np.zeros((128, 128, 128), np.complex128)
        ia128[16:112, 20:108, 24:104] = 1.0 / (0.01 + 0.001j)
        big = {}
        for dt, esz, name in ((torch.complex64, 8, "c64"), (torch.complex128, 16, "c128")):
            opb = P.DDAOperator(ia128, k, d, dtype=dt, device=dev)
            tb = time_matvec(opb, 10, flush)
            Bb = matvec_bytes(opb.shape, esz)
            big[name] = {"ms": tb * 1e3, "GBps": Bb / tb / 1e9, "frac": Bb / tb / 1e9 / peak,
                         "algorithmic_bytes": Bb}
            del opb
        del flush
        out = {"ellipsoid128_16rhs": _extra(ellipsoid128_16rhs, dev), "sphere32_plain_c128": _extra(sphere32_plain, dev),
               "batch64": _extra(batch64_block, args, ws, rank, local),
               "serve": _extra(serve_block, args, ws, rank, local),
               "launch_tuning": {json.dumps(list(k)): {"flags": v, "seconds": tuner.times.get(k)}
                                 for k, v in tuner.best.items()}}
        out.update({"roofline": roof, "matvec_128": big, "plain_c128_solves_per_s": plain,
               "mixed_over_plain": value / ws / plain,
               "unpreconditioned": {"mixed_solves_per_s": mixed_np, "plain_c128_solves_per_s": plain_np,
                                    "mixed_over_plain": mixed_np / plain_np,
                                    "mixed_inner_total": [i.iters for i in inf_mnp],
                                    "plain_c128": [i.iters for i in inf_pnp],
                                    "preconditioned_over_unpreconditioned": value / ws / mixed_np},
               "accuracy_vs_fp64": cerr,
               "iterations": {"mixed_inner_total": [i.iters for i in infos], "outer": [i.outer for i in infos],
                              "true_relres": [i.true_relres for i in infos],
                              "plain_c128": [i.iters for i in inf_p]},
               "step_latency_ms": {"p50": 1e3 * statistics.median(lat), "max": 1e3 * max(lat),
                                   "samples": len(lat),
                                   "what": "host wall time of one timed solve step (both polarisations); serving "
                                           "request latency p50/p99 is the serve block's"}})
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c64+fp64",
                "data": "synthetic (seeded sphere lattice; no dataset)",
                "config": {"workload": WORKLOAD, "solver": SOLVER, "global_batch": 2 * ws, "dipoles": ndip,
                           "box": [N_BOX] * 3,
                           "fft": list(op.L), "parallelism": "replicas" if ws > 1 else "single",
                           "preconditioner": f"precon=True: occupancy-weighted circulant on the {pre.L[0]}^3 grid "
                                             "(complex64 sweeps; FP64 refinement residual unpreconditioned)",
                           "l2": "working set > L2 (c64 + c128 workspaces ~0.4 GB); roofline launches flush L2"},
                "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "step_ms_p50": 1e3 * statistics.median(e2e_steps), "step_ms_max": 1e3 * max(e2e_steps),
                        "includes": "H2D of inv_alpha and E_inc, Green build, preconditioner build, mixed solve, "
                                    "cross sections, D2H of P"},
                "gpu_launches": int(launches)}
        line.update(out)
        if ws == 1 and not args.no_cpu:
            cpu = CpuSolve()
            n_it = 3
            t_it = cpu.iteration_time(n_it)
            v = cpu.solves_per_s(t_it)
            line["cpu_baseline"] = {"value": v, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
                                    "solver": REF_SOLVER,
                                    "sample": f"Green build ({cpu.t_green:.2f} s) + {n_it} iterations of the "
                                              f"complex128 recurrence at 64^3, scaled to the {REF_ITERS_64} "
                                              f"iterations of the full solve to 1e-6"}
            # like-for-like algorithm: the GPU's unpreconditioned (precon=False)
            # solves against the same CPU baseline
            if "unpreconditioned" in line:
                line["unpreconditioned"]["mixed_vs_cpu"] = line["unpreconditioned"]["mixed_solves_per_s"] / v
                line["unpreconditioned"]["plain_c128_vs_cpu"] = line["unpreconditioned"]["plain_c128_solves_per_s"] / v
        line["clocks"] = clk.summary()
        print(json.dumps(line), flush=True)


def run_profile_matvec(args, local):
    """Matvecs only, for ncu: box n^3 (sphere-like fill), given dtype."""
    import torch
    import precondda_b200 as P
    dev = torch.device("cuda", local)
    n = args.profile_matvec
    dt = torch.complex64 if args.dtype == "c64" else torch.complex128
    k = 2 * math.pi / WAVELENGTH
    d = KD_M / (abs(M_REF) * k)
    from precondda_b200 import sphere_occupancy
    occ = sphere_occupancy(n, n / 2.0)
    ia = np.where(occ, 1.0 / (0.01 + 0.001j), 0).astype(np.complex128)
    op = P.DDAOperator(ia, k, d, dtype=dt, device=dev)
    x = torch.randn(n, n, n, 3, dtype=dt, device=dev)
    nr = max(1, args.profile_rhs)
    for _ in range(args.reps):
        y = op.matvec(x) if nr == 1 else P.engine.matvec_batch([op] * nr, [x] * nr)[0]
    torch.cuda.synchronize()
    out = {"profile_matvec": n, "dtype": args.dtype, "reps": args.reps, "L": op.L, "rhs": nr,
           "p3_variant": os.environ.get("DDA_P3_VARIANT", "default"), "checksum": float(y.abs().sum())}
    if args.time:
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
        t = time_matvec(op, 20, flush) if nr == 1 else time_matvec_batch([op] * nr, 20, flush)
        B = nr * matvec_bytes(op.shape, 8 if dt == torch.complex64 else 16)
        peak, _ = measured_peak()
        out.update({"ms": t * 1e3, "GBps": B / t / 1e9, "frac": B / t / 1e9 / peak})
    print(json.dumps(out))


# --------------------------------------------------------------------------
# other workloads (one JSON line each; the default run is the sphere64 line)
# --------------------------------------------------------------------------
def _line(metric, value, unit, args, ws, t, config, dtype="c64+fp64", **extra):
    out = {"metric": metric, "value": value, "unit": unit, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": 1e3 * t / max(args.steps, 1), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded lattices; no dataset)", "config": config}
    out.update(extra)
    return out


def run_large128(args, ws, rank, local):
    """Large single solve: 128^3 box, rotated ellipsoid with semi-axes
    (64, 48, 40) d, m from the seed, |m|kd = 0.6; mixed precision vs plain
    complex128 at tol 1e-6 and the C_ext / C_abs error of each against a
    complex128 solve to 1e-10."""
    import torch
    import precondda_b200 as P
    from precondda_b200 import _lib as L
    from precondda_b200.workloads import ellipsoid128_spec, build_geometry
    dev = torch.device("cuda", local)
    spec = ellipsoid128_spec(seed=3 + rank)
    ia, k, d, Es = build_geometry(spec, dev)
    op = P.DDAOperator(ia, k, d, dtype=torch.complex128, device=dev, with_twin=True)
    E = Es[0]
    pre = op.preconditioner()

    def solve(prec, tol=TOL, preconditioner=pre):
        return P.solve_many([op], [E], tol=tol, max_iter=4000, ratio=RATIO, precision=prec, inner_tol=INNER_TOL,
                            preconditioner=preconditioner)

    def timed(prec, preconditioner):
        solve(prec, preconditioner=preconditioner)
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True); a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        Px, ix = solve(prec, preconditioner=preconditioner)
        a1.record(stream)
        torch.cuda.synchronize()
        return 1.0 / (a0.elapsed_time(a1) / 1e3), Px, ix

    for _ in range(max(args.warmup, 1)):
        solve("mixed")
    torch.cuda.synchronize()
    lc0 = L.lib().dda_kernel_launches()
    stream = torch.cuda.current_stream(dev)
    with ClockSampler(dev.index) as clk:
        barrier(ws)
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            Pm, im = solve("mixed")
        e1.record(stream)
        torch.cuda.synchronize()
    launches = L.lib().dda_kernel_launches() - lc0
    t = max_over_ranks(ws, e0.elapsed_time(e1) / 1e3)
    value = args.steps * ws / t
    if rank != 0:
        return
    plain, Pp, ip = timed("c128", pre)
    mixed_np, _, imn = timed("mixed", None)
    plain_np, _, ipn = timed("c128", None)
    Pf, iff = solve("c128", tol=1e-10, preconditioner=None)
    cm, cp, cf = (op.cross_sections(Pm[0], E), op.cross_sections(Pp[0], E), op.cross_sections(Pf[0], E))
    err = lambda a, b: abs(a - b) / abs(b)
    nocc = int((ia != 0).sum().item())
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    t_mv = time_matvec(op.twin(torch.complex64), 10, flush)
    peak, pk = measured_peak()
    B = matvec_bytes(op.shape, 8)
    line = _line(METRIC, value, "solves/s", args, ws, t,
                 {"workload": f"large128: 128^3 box ({nocc} dipoles), ellipsoid semi-axes (64,48,40)d, seeded Euler "
                              f"angles, m={spec['m']:.4f}, |m|kd=0.6, mixed c64 (1e-4) + FP64 refinement to 1e-6",
                  "box": [128] * 3, "fft": list(op.L), "parallelism": "replicas" if ws > 1 else "single",
                  "preconditioner": f"precon=True: occupancy-weighted circulant on the {pre.L[0]}^3 grid"},
                 gpu_launches=int(launches),
                 plain_c128_solves_per_s=plain, mixed_over_plain=value / ws / plain,
                 unpreconditioned={"mixed_solves_per_s": mixed_np, "plain_c128_solves_per_s": plain_np,
                                   "mixed_over_plain": mixed_np / plain_np, "mixed_inner": imn[0].iters,
                                   "plain_c128": ipn[0].iters,
                                   "preconditioned_over_unpreconditioned": value / ws / mixed_np},
                 iterations={"mixed_inner": im[0].iters, "outer": im[0].outer, "plain_c128": ip[0].iters,
                             "true_relres_mixed": im[0].true_relres},
                 accuracy_vs_fp64={"mixed": {"C_ext_rel_err": err(cm[0], cf[0]), "C_abs_rel_err": err(cm[1], cf[1])},
                                   "plain_c128": {"C_ext_rel_err": err(cp[0], cf[0]),
                                                  "C_abs_rel_err": err(cp[1], cf[1])},
                                   "C_ext": cf[0], "C_abs": cf[1]},
                 roofline={"bound": "hbm", "achieved": B / t_mv / 1e9, "peak": peak, "unit": "GB/s",
                           "frac": B / t_mv / 1e9 / peak, "traffic": None, "peak_kind": pk,
                           "kernel": "5-pass matvec, complex64, 128^3 box (FFT 256^3)", "ms": t_mv * 1e3,
                           "algorithmic_bytes": B},
                 clocks=clk.summary())
    print(json.dumps(line), flush=True)


def run_batch64(args, ws, rank, local, emit=True):
    """64 rotated ellipsoids with box edges 16-96, 2 polarisations x 8
    incidence directions each (1024 right-hand sides), mixed precision to
    1e-5, autotuned padding per size bucket, buckets as concurrent slot pools."""
    import torch
    from precondda_b200 import _lib as L
    from precondda_b200.batch import Geometry, PaddingTuner, solve_geometries
    from precondda_b200.workloads import random_ellipsoid_spec, build_geometry
    from precondda_b200.engine import cross_sections
    dev = torch.device("cuda", local)
    rng = np.random.default_rng(40 + rank)
    specs = [random_ellipsoid_spec(rng) for _ in range(args.geometries)]
    tuner = PaddingTuner("mixed", device=dev)
    plan = tuner.plan([tuple(s["box"]) for s in specs])   # autotune outside the timed region
    from precondda_b200.batch import LaunchTuner
    ltun = LaunchTuner(device=dev)
    per_bucket = {}
    for s_, (box, L_) in zip(specs, plan):
        per_bucket[(box, L_)] = per_bucket.get((box, L_), 0) + len(s_["dirs"]) * s_.get("pols", 2)
    if not args.no_tune:
        for (box, L_), nrhs in per_bucket.items():
            ltun.tune(box, L_, torch.complex64, nrhs)
    # untimed warm-up: every geometry's bucket with one right-hand side, so the
    # timed pass does not pay first launches of its kernel sizes, pool graph
    # captures or the memory pool's first growth
    if args.warmup > 0:
        warm = []
        for sp in specs:
            ia, k, d, Es = build_geometry(sp, dev)
            warm.append(Geometry(ia, k, d, Es[:1]))
        solve_geometries(warm, tol=1e-5, precision="mixed", inner_tol=1e-4, tuner=tuner, device=dev,
                         keep_results=False, precondition=not args.no_precondition)
        del warm
    torch.cuda.synchronize()
    lc0 = L.lib().dda_kernel_launches()
    with ClockSampler(dev.index) as clk:
        barrier(ws)
        t_all = time.perf_counter()
        geoms = []
        for sp in specs:
            ia, k, d, Es = build_geometry(sp, dev)
            geoms.append(Geometry(ia, k, d, Es))
        torch.cuda.synchronize()
        t_build = time.perf_counter() - t_all
        xs = {}

        def on_result(g, j, Pv, info):
            G = geoms[g]
            xs[(g, j)] = cross_sections(Pv.contiguous(), G.E_incs[j], G.inv_alpha, G.k)

        res = solve_geometries(geoms, tol=1e-5, precision="mixed", inner_tol=1e-4, tuner=tuner, device=dev,
                               keep_results=False, on_result=on_result, precondition=not args.no_precondition,
                               chunk=args.chunk)
        torch.cuda.synchronize()
        t_all = time.perf_counter() - t_all
    launches = L.lib().dda_kernel_launches() - lc0
    t = max_over_ranks(ws, res.seconds)
    te = max_over_ranks(ws, t_all)
    n = res.solves
    if rank != 0:
        return
    infos = [i for gi in res.info for i in gi]
    its = [i.iters for i in infos]
    buckets = {}
    for (box, L_) in res.plan:
        key = "x".join(map(str, box))
        buckets[key] = buckets.get(key, 0) + 1
    line = _line(METRIC, n * ws / t, "solves/s", args, ws, t,
                 {"workload": f"batch64: {len(specs)} rotated ellipsoids, box edges U{{16..96}}, semi-axes 0.3-0.5 x "
                              f"edge, m Re U[1.3,2], Im U[0,0.3], lambda U[0.4,0.8] um, |m|kd=0.5, 2 pols x 8 "
                              f"directions ({n} RHS), mixed c64 (1e-4) + FP64 refinement to 1e-5",
                  "global_batch": n * ws, "parallelism": "replicas" if ws > 1 else "single",
                  "preconditioner": "none (precon=False)" if args.no_precondition else
                                    "precon=True: occupancy-weighted circulant per geometry on its bucket's grid",
                  "buckets": buckets},
                 e2e={"value": n * ws / te, "unit": "solves/s", "h2d_bytes_per_step": 0,
                      "d2h_bytes_per_step": 3 * 8 * n,
                      "includes": "device voxelisation and incident fields from seeded specs, Green builds, padded "
                                  "batched solves, cross sections of every RHS to the host"},
                 gpu_launches=int(launches),
                 solve_seconds=res.seconds, build_seconds=t_build,
                 converged=sum(i.status == "converged" for i in infos),
                 iterations={"mean_inner": float(np.mean(its)), "max_inner": int(max(its)),
                             "mean_outer": float(np.mean([i.outer for i in infos]))},
                 clocks=clk.summary())
    if emit:
        print(json.dumps(line), flush=True)
    return line


def serve_stream(srv, stream, dev, tol=1e-5):
    """Replay one Poisson stream through the server: each request's
    right-hand sides are submitted at its arrival time as lazy requests (the
    lattice and incident fields are built on the device when a request
    enters a slot, once per request group), steps run until all finish.
    Returns (groups {q: (arrival, [Request])}, wall seconds)."""
    import torch
    from precondda_b200.serve import Request
    from precondda_b200.workloads import build_geometry
    groups = {}
    t0 = time.perf_counter()
    q = 0
    while q < len(stream) or srv.pending():
        now = time.perf_counter() - t0
        while q < len(stream) and stream[q][0] <= now:
            arr, sp = stream[q]
            cache = {}

            def make(j, sp=sp, cache=cache):
                def build():
                    if "geo" not in cache:
                        cache["geo"] = build_geometry(sp, dev)
                    ia, k_, d_, Es = cache["geo"]
                    E = Es[j]
                    cache["left"] = cache.get("left", len(Es)) - 1
                    if cache["left"] == 0:
                        cache.clear()
                    return ia, E
                return build

            lam, m = sp["wavelength"], sp["m"]
            k = 2 * math.pi / lam
            d = sp["mkd"] / (abs(m) * k)
            reqs = []
            n_rhs = len(sp["dirs"]) * (len(sp["fixed_pols"]) if "fixed_pols" in sp else sp.get("pols", 2))
            for j in range(n_rhs):
                r = srv.submit(Request(inv_alpha=None, E_inc=None, k=k, d=d, tol=tol, shape=tuple(sp["box"]),
                                       build=make(j), pre_key=("group", q)))
                r.t_submit = t0 + arr
                reqs.append(r)
            groups[q] = (t0 + arr, reqs)
            q += 1
        if srv.pending():
            for r in srv.step():
                r.P = r.inv_alpha = r.E_inc = None          # results are not kept
        elif q < len(stream):
            time.sleep(min(1e-3, max(0.0, stream[q][0] - now)))
    torch.cuda.synchronize()
    return groups, time.perf_counter() - t0


def serve_summary(groups, span):
    lat_req = np.array([max(r.t_done for r in reqs) - ta for ta, reqs in groups.values()])
    rhs = [r for _, reqs in groups.values() for r in reqs]
    lat_rhs = np.array([r.t_done - r.t_submit for r in rhs])
    return {"requests": len(groups), "rhs": len(rhs), "seconds": span, "rhs_per_s": len(rhs) / span,
            "requests_per_s": len(groups) / span,
            "request_p50_ms": float(np.percentile(lat_req, 50) * 1e3),
            "request_p99_ms": float(np.percentile(lat_req, 99) * 1e3),
            "rhs_p50_ms": float(np.percentile(lat_rhs, 50) * 1e3),
            "rhs_p99_ms": float(np.percentile(lat_rhs, 99) * 1e3),
            "converged": sum(r.info.status == "converged" for r in rhs)}, rhs


def run_serve(args, ws, rank, local, emit=True):
    """Poisson request streams, 40% spheres, 40% ellipsoids, 20% random-walk
    aggregates, boxes 16^3-128^3, 1-16 incidences each, served by continuous
    batching with HBM admission and Green-tensor reuse.  One stream per
    offered rate in --rates (the value and latency keys are the last rate's;
    every rate's solves/s and p50/p99 go in the "curve" key)."""
    import torch
    from precondda_b200 import _lib as L
    from precondda_b200.serve import DDAServer, Request
    from precondda_b200.workloads import serving_stream, build_geometry
    dev = torch.device("cuda", local)
    rates = [float(v) for v in str(args.rates).split(",")] if args.rates else [args.rate]
    from precondda_b200.batch import LaunchTuner
    srv = DDAServer(precision="mixed", slots_per_bucket=args.slots, chunk_iters=args.chunk, device=dev,
                    precondition=not args.no_precondition,
                    launch_tuner=None if args.no_tune else LaunchTuner(device=dev))
    # warm the kernels of every bucket outside the timed region
    warm = sorted({srv.bucket_for(sp["box"]) for r in rates
                   for _, sp in serving_stream(50 + rank, rate=r, duration=args.duration)})
    for b in warm:
        ia, k, d, Es = build_geometry({"kind": "sphere", "box": (b, b, b), "radius_d": b / 2.0, "m": 1.5 + 0.01j,
                                       "wavelength": 0.5, "mkd": 0.5, "dirs": np.array([[0.0, 0.0, 1.0]]),
                                       "pols": 1}, dev)
        srv.submit(Request(inv_alpha=ia, E_inc=Es[0], k=k, d=d, tol=1e-5))
    srv.drain()
    curve = []
    lc0 = L.lib().dda_kernel_launches()
    with ClockSampler(dev.index) as clk:
        for rate in rates:
            srv.done.clear()
            srv.green.hits = srv.green.misses = 0
            stream = serving_stream(50 + rank, rate=rate, duration=args.duration)
            torch.cuda.synchronize()
            barrier(ws)
            groups, span = serve_stream(srv, stream, dev)
            summ, rhs = serve_summary(groups, span)
            summ.update({"offered_requests_per_s": rate, "green_hits": srv.green.hits,
                         "green_misses": srv.green.misses})
            curve.append(summ)
    launches = L.lib().dda_kernel_launches() - lc0
    if rank != 0:
        return
    last = curve[-1]
    st = srv.stats(rhs)
    line = _line(METRIC, last["rhs_per_s"], "solves/s", args, ws, last["seconds"],
                 {"workload": f"serve: Poisson {rates[-1]}/s over {args.duration} s ({last['requests']} requests, "
                              f"{last['rhs']} RHS), 40% spheres / 40% ellipsoids / 20% aggregates (K 4-32, r 6-12 d), "
                              f"boxes 16^3-128^3, m Re U[1.3,2] Im U[0,0.5], lambda U[0.4,0.8] um, 1-16 incidences, "
                              f"mixed precision to 1e-5, continuous batching",
                  "parallelism": "replicas" if ws > 1 else "single", "slots_per_bucket": args.slots,
                  "hbm_budget_GiB": round(srv.hbm_budget / 2**30, 2),
                  "preconditioner": "none (precon=False)" if args.no_precondition else
                                    "precon=True: occupancy-weighted circulant per request group on its bucket's grid",
                  "pools": {str(k): v for k, v in st.get("pools", {}).items()}},
                 latency_ms={"request_p50": last["request_p50_ms"], "request_p99": last["request_p99_ms"],
                             "rhs_p50": last["rhs_p50_ms"], "rhs_p99": last["rhs_p99_ms"]},
                 requests_per_s=last["requests_per_s"], curve=curve,
                 green_cache={"hits": last["green_hits"], "misses": last["green_misses"]},
                 converged=last["converged"], gpu_launches=int(launches), clocks=clk.summary())
    srv.close()
    if emit:
        print(json.dumps(line), flush=True)
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-tune", action="store_true",
                    help="no launch-variant tuning, the defaults (for profiler captures, whose serialised "
                         "timing would mislead the tuner, and A/B runs)")
    ap.add_argument("--no-extra", action="store_true",
                    help="default workload: only the timed solves and e2e (no extra blocks; for launch-list captures)")
    ap.add_argument("--profile-matvec", type=int, default=0, help="only run matvecs on an n^3 box (for ncu)")
    ap.add_argument("--profile-rhs", type=int, default=1,
                    help="with --profile-matvec: right-hand sides per launch (gridDim.y)")
    ap.add_argument("--dtype", default="c64", choices=["c64", "c128"])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--time", action="store_true", help="with --profile-matvec: time 20 launches (L2 flushed)")
    ap.add_argument("--workload", default="sphere64", choices=["sphere64", "large128", "batch64", "serve"],
                    help="sphere64 (default): the precision configuration; large128: 128^3 ellipsoid; "
                         "batch64: 64 geometries x 16 RHS; serve: Poisson request stream")
    ap.add_argument("--geometries", type=int, default=64, help="batch64: number of geometries")
    ap.add_argument("--rate", type=float, default=20.0, help="serve: arrivals per second")
    ap.add_argument("--duration", type=float, default=60.0, help="serve: seconds of arrivals per rate")
    ap.add_argument("--rates", default="", help="serve: comma-separated offered rates (requests/s), one stream each")
    ap.add_argument("--slots", type=int, default=16, help="serve: slots per size bucket")
    ap.add_argument("--chunk", type=int, default=8, help="batch64 / serve: iterations per pool chunk between polls")
    ap.add_argument("--no-precondition", action="store_true",
                    help="batch64 / serve: the reference's precon=False solve instead of the preconditioned one")
    args = ap.parse_args()
    ws, rank, local = dist_init()
    if args.profile_matvec:
        run_profile_matvec(args, local)
        return
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        elif args.workload == "large128":
            run_large128(args, ws, rank, local)
        elif args.workload == "batch64":
            run_batch64(args, ws, rank, local)
        elif args.workload == "serve":
            run_serve(args, ws, rank, local)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
