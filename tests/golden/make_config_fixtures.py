"""Golden fixtures at the benchmark configurations' full sizes.

Run from the repository root (takes about half an hour on 8 cores):

    python oracle/build_ref.py                           # the reference's kernels, for --with-ref
    python tests/golden/make_config_fixtures.py [--ref <reference checkout>]

It writes ``tests/golden/config_fixtures.npz`` (+ ``.json`` notes):

* ``c1_*``   the 32^3 sphere of the plain complex128 configuration (radius
  16 d, m = 1.5+0.01i, |m|kd = 0.5, RR alpha, +z incidence, x polarised,
  tol 1e-6, maxiter 2000, ratio 100).  Solved twice: by the reference's own
  ``solve_gpbicgstab`` (complex64, precon=False, run unchanged through
  ``oracle/ref_loader.py``) and by the oracle's complex128 restatement.
  Stored per solve: the iteration count, lowest/first residuals, C_ext /
  C_abs / C_sca (FP64 sums over the solve's P), ||P|| and P at a seeded
  sample of sites.
* ``c2_*``   the 64^3 sphere of the precision configuration (radius 32 d,
  m = 1.7+0.1i, |m|kd = 0.5, x and y polarisations): the oracle's complex128
  solve to a relative residual of 1e-8, the FP64 truth the mixed-precision
  solve is held to.  Same stored quantities.
* ``mv128_*`` one matvec on a 128^3 box: y = oracle.interaction_mult(x) for a
  seeded x on a seeded occupancy (random 40 % fill inside an ellipsoid),
  stored as ||y|| and y at a seeded sample of sites.

The sample sites and every seeded input are regenerated by the tests from
the seeds recorded here (numpy's default_rng is platform independent).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import dda_oracle as O  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "config_fixtures.npz")
NSAMPLE = 4096


def sphere_problem(n, m, pol):
    """The configurations' sphere: box n^3, radius n/2 in lattice units,
    |m|kd = 0.5 at lambda = 0.5 um, RR polarizability, +z incidence."""
    k = 2 * math.pi / 0.5
    d = 0.5 / (abs(m) * k)
    occ = O.sphere_lattice(n, n / 2.0)
    alpha = np.where(occ, O.calculate_alpha(m, d, k, method="RR"), 0).astype(np.complex128)
    E = O.incident_field((n, n, n), d, k, (0, 0, 1), pol)
    return k, d, alpha, E


def sample_sites(shape, seed, count=NSAMPLE):
    """Flat site indices of a seeded sample (sorted, without repeats)."""
    n = int(np.prod(shape))
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n, size=min(count, n), replace=False))


def mv128_problem(seed=128):
    """Seeded 128^3 matvec input: occupancy = 40 % random fill inside an
    ellipsoid of semi-axes (60, 50, 40), x = complex normal per component."""
    n = 128
    rng = np.random.default_rng(seed)
    k = 2 * math.pi / 0.5
    m = 1.6 + 0.1j
    d = 0.6 / (abs(m) * k)
    c = n / 2.0
    ax = np.arange(n) + 0.5 - c
    X, Y, Z = np.meshgrid(ax, ax, ax, indexing="ij")
    inside = (X / 60) ** 2 + (Y / 50) ** 2 + (Z / 40) ** 2 <= 1.0
    occ = inside & (rng.random((n, n, n)) < 0.4)
    a = O.calculate_alpha(m, d, k, method="RR")
    ia = np.where(occ, 1.0 / a, 0).astype(np.complex128)
    x = rng.standard_normal((n, n, n, 3)) + 1j * rng.standard_normal((n, n, n, 3))
    return k, d, ia, x


def main(ref, with_ref):
    fx, notes = {}, {}

    def put(name, val, note):
        fx[name] = np.asarray(val)
        notes[name] = note

    def put_solve(tag, P, E, ia, k, iters, low, first, seed, what):
        cext, cabs, csca = O.cross_sections(np.asarray(P, np.complex128), E, ia, k)
        sites = sample_sites(P.shape[:3], seed)
        put(f"{tag}_iters", np.array(int(iters)), f"{what}: iterations")
        put(f"{tag}_lowfirst", np.array([float(low), float(first)]), f"{what}: lowest/initial, first/initial")
        put(f"{tag}_xsec", np.array([cext, cabs, csca]), f"{what}: C_ext, C_abs, C_sca (FP64 sums over its P)")
        put(f"{tag}_Pnorm", np.array(float(np.linalg.norm(P))), f"{what}: ||P||")
        put(f"{tag}_Psample", np.asarray(P).reshape(-1, 3)[sites].astype(np.complex128),
            f"{what}: P at the sample sites (seed {seed})")

    # ---- configuration 1: 32^3 sphere, complex128 plain
    n, m = 32, 1.5 + 0.01j
    k, d, alpha, E = sphere_problem(n, m, (1, 0, 0))
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    put("c1_kd", np.array([k, d]), "k, d of the 32^3 sphere")
    put("c1_nocc", np.array(int(mask.sum())), "occupied sites")
    t0 = time.time()
    it, P, low, first = O.solve_gpbicgstab((n,) * 3, ia, G, E, mask, 100, 2000, target=1e-6)
    print(f"c1 oracle: {it} iterations, {time.time() - t0:.1f} s", flush=True)
    put_solve("c1_oracle", P, E, ia, k, it, low, first, 1, "oracle complex128 solve (tol 1e-6, ratio 100)")
    if with_ref:
        from oracle import ref_loader
        R = ref_loader.load(ref)
        cp = ref_loader.cupy_shim
        t0 = time.time()
        with ref_loader.quiet():
            a = cp.asarray(alpha, dtype=np.complex64)
            inv_alpha = cp.where(a != 0, 1.0 / a, 0)
            rmask = a != 0
            Gm = R.ddaforgit.generate_interaction_row(n, n, n, k, d, True, False)
            pre = np.zeros((n + 1, n + 1, n + 1, 6), np.complex64)
            rit, rP, rlow, rfirst = R.Gpbicgstab.solve_gpbicgstab((n, n, n), inv_alpha, Gm, pre, E, rmask, 100,
                                                                  2000, target=1e-6, precon=False)
        print(f"c1 reference: {int(rit)} iterations, {time.time() - t0:.1f} s", flush=True)
        put_solve("c1_ref", np.asarray(rP), E, ia, k, rit, rlow, rfirst, 1,
                  "the reference's solve_gpbicgstab (complex64, precon=False, tol 1e-6, ratio 100)")

    # ---- configuration 2: 64^3 sphere, FP64 truth for both polarisations
    n, m = 64, 1.7 + 0.1j
    for j, pol in enumerate(((1, 0, 0), (0, 1, 0))):
        k, d, alpha, E = sphere_problem(n, m, pol)
        ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
        t0 = time.time()
        it, P, low, first = O.solve_gpbicgstab((n,) * 3, ia, G, E, mask, 100, 4000, target=1e-8)
        rr = O.true_relative_residual(P, E, G, ia, mask)
        print(f"c2 pol {j}: {it} iterations, true relres {rr:.2e}, {time.time() - t0:.1f} s", flush=True)
        put_solve(f"c2_p{j}", P, E, ia, k, it, low, first, 2 + j,
                  f"oracle complex128 solve to 1e-8, polarisation {'xy'[j]}")
        put(f"c2_p{j}_relres", np.array(rr), "true relative residual of that solve")
    put("c2_kd", np.array([k, d]), "k, d of the 64^3 sphere")

    # ---- 128^3 matvec
    k, d, ia, x = mv128_problem()
    mask = ia != 0
    t0 = time.time()
    G = O.generate_interaction_row(128, 128, 128, k, d)
    y = O.interaction_mult(x, G, ia, mask)
    print(f"mv128: {time.time() - t0:.1f} s", flush=True)
    sites = sample_sites((128,) * 3, 128)
    put("mv128_kd", np.array([k, d]), "k, d of the 128^3 matvec problem (seed 128)")
    put("mv128_ynorm", np.array(float(np.linalg.norm(y))), "||interaction_mult(x)||")
    put("mv128_ysample", y.reshape(-1, 3)[sites], "interaction_mult(x) at the sample sites (seed 128)")
    np.savez_compressed(OUT, **fx)
    with open(OUT.replace(".npz", ".json"), "w") as f:
        json.dump({"generator": "tests/golden/make_config_fixtures.py", "entries": notes}, f, indent=1)
    print(f"wrote {OUT} ({os.path.getsize(OUT) / 1024:.0f} KiB)")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    ap.add_argument("--no-ref", action="store_true", help="skip the reference's own 32^3 solve")
    a = ap.parse_args()
    ref = a.ref
    if ref is None and not a.no_ref:
        from oracle import build_ref
        ref = build_ref.reference_dir()
    main(ref, not a.no_ref)
