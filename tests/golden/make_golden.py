"""Generate golden fixtures by running the reference's own code on the CPU.

Run from the repository root in a checkout that has the reference:

    python oracle/build_ref.py                 # compile its kernel strings
    python tests/golden/make_golden.py [--ref <reference checkout>]

The reference (Toastlovesjam/preconDDA) is executed unchanged through
``oracle/ref_loader.py``: ``Gpbicgstab.solve_gpbicgstab``,
``Gpbicgstab.interaction_mult`` / ``inner_product`` /
``calculate_zeta_eta_twostep`` / ``fft_matvec3`` (with precon=True, given a
preconditioner octant), ``ExcitedField.E_field_solver`` and, from
``ddaforgit.py``, ``calculate_alpha``, ``build_problem_from_shapes`` and
``generate_interaction_row``.  Its device kernels run as CPU builds of their
CUDA-C source; everything else is its own Python.  The outputs are written to
``tests/golden/ref_fixtures.npz`` (inputs included), which the tests read
without needing the reference.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import build_ref, ref_loader  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "ref_fixtures.npz")


def main(ref):
    R = ref_loader.load(ref)
    cp = ref_loader.cupy_shim
    G, E_ = R.Gpbicgstab, R.ExcitedField
    D = R.ddaforgit
    fx = {}
    meta = {"reference": "Toastlovesjam/preconDDA", "entries": {}}

    def put(name, val, note):
        fx[name] = np.asarray(val)
        meta["entries"][name] = note

    # ---- polarizability (ddaforgit.py:403-437)
    cases = [(1.5 + 0.01j, 0.02, 2 * np.pi / 0.5), (1.7 + 0.1j, 0.023365, 2 * np.pi / 0.5),
             (2.0 + 0.5j, 0.01, 2 * np.pi / 0.8), (1.33 + 0j, 0.05, 2 * np.pi / 0.6)]
    al = []
    for n, d, k in cases:
        al.append([D.calculate_alpha(n, d, k, method="CM"), D.calculate_alpha(n, d, k, method="RR"),
                   D.calculate_alpha(n, d, k, (0, 0, 1), (1, 0, 0), method="LDR"),
                   D.calculate_alpha(n, d, k, (0, 0, 1), (0, 0, 1), method="LDR")])
    put("alpha_cases", np.array([[c[0], c[1], c[2]] for c in cases], dtype=np.complex128), "(n, d, k) per row")
    put("alpha_values", np.array(al), "CM, RR, LDR(a=z,e=x), LDR(a=z,e=z) per case")

    # ---- lattice setup (ddaforgit.py:1591-1651, reference default LDR)
    with ref_loader.quiet():
        pr = D.build_problem_from_shapes([{"type": "sphere", "center": [0.1, 0.1, 0.1], "radius": 0.08, "n": 1.5}],
                                         np.array([0.0, 0.0, 1.0]), [1.0, 0.0, 0.0], 0.5, 0.02)
    put("sphere_alpha", pr["alpha_array"], "build_problem_from_shapes sphere c=0.1 r=0.08 n=1.5 lambda=0.5 d=0.02")
    put("sphere_E", pr["E_inc"], "E_inc of that problem (k along z, x-polarised)")
    with ref_loader.quiet():
        pe = D.build_problem_from_shapes([{"type": "ellipsoid", "center": [0.12, 0.1, 0.08], "semi_axes":
                                           [0.11, 0.07, 0.05], "n": 1.6 + 0.05j}],
                                         np.array([1.0, 0.0, 0.0]), [0.0, 0.0, 1.0], 0.6, 0.02)
    put("ellipsoid_alpha", pe["alpha_array"], "ellipsoid c=(.12,.1,.08) a=(.11,.07,.05) n=1.6+0.05i lambda=0.6 d=.02")
    put("ellipsoid_E", pe["E_inc"], "E_inc, k along x, z-polarised")

    # ---- Green's tensor FFT octant (ddaforgit.py:1046-1080)
    k, d = 2 * np.pi / 0.5, 0.04
    with ref_loader.quiet():
        put("green_468_c64", np.asarray(D.generate_interaction_row(4, 6, 8, k, d, True, False)),
            "generate_interaction_row(4,6,8,k=4pi,d=0.04) complex64")
        put("green_468_c128", np.asarray(D.generate_interaction_row(4, 6, 8, k, d, True, True)),
            "same, complex128")
    put("green_468_kd", np.array([k, d]), "k, d of the Green fixtures")

    # ---- solver problems: spheres with RR alpha, plus the ellipsoid (LDR)
    def sphere_case(n, m, kd_m, seed):
        k = 2 * np.pi / 0.5
        d = kd_m / (abs(m) * k)
        c = n / 2.0
        ax = np.arange(n) + 0.5 - c
        X, Y, Z = np.meshgrid(ax, ax, ax, indexing="ij")
        dist = np.sqrt(X * X + Y * Y + Z * Z)
        occ = (dist < n / 2.0) | (np.abs(dist - n / 2.0) < 1e-7)
        alpha = np.where(occ, D.calculate_alpha(m, d, k, method="RR"), 0)
        axd = [np.arange(n) * d] * 3
        XX, YY, ZZ = np.meshgrid(*axd, indexing="ij")
        ph = np.exp(1j * k * ZZ)
        E = np.zeros((n, n, n, 3), np.complex128)
        E[..., 0] = ph
        return k, d, alpha, E

    probs = {"s8": sphere_case(8, 1.5 + 0.01j, 0.5, 1), "s10": sphere_case(10, 1.7 + 0.1j, 0.5, 2)}
    kk = 2 * np.pi / 0.6
    probs["ell"] = (kk, 0.02, pe["alpha_array"], pe["E_inc"])
    for name, (k, d, alpha, E) in probs.items():
        nx, ny, nz = alpha.shape
        with ref_loader.quiet():
            # prepare_interaction_matrices' alpha handling (ddaforgit.py:1099-1108), then the Green row
            a = cp.asarray(alpha, dtype=np.complex64)
            inv_alpha = cp.where(a != 0, 1.0 / a, 0)
            mask = a != 0
            Gm = D.generate_interaction_row(nx, ny, nz, k, d, True, False)
            pre = np.zeros((nx + 1, ny + 1, nz + 1, 6), np.complex64)
            it, P, low, first = G.solve_gpbicgstab((nx, ny, nz), inv_alpha, Gm, pre, E, mask, 100, 500,
                                                   target=1e-5, precon=False)
            Ef = E_.E_field_solver(np.asarray(P), Gm, (nx, ny, nz))
        put(f"{name}_kd", np.array([k, d]), "k, d")
        put(f"{name}_alpha", alpha, "polarizability array")
        put(f"{name}_E", E, "incident field")
        put(f"{name}_G", np.asarray(Gm), "generate_interaction_row complex64 octant")
        put(f"{name}_iters", np.array(int(it)), "solve_gpbicgstab iterations (ratio 100, target 1e-5)")
        put(f"{name}_lowfirst", np.array([float(low), float(first)]), "lowest/initial, first/initial")
        put(f"{name}_P", np.asarray(P), "solution P (nx,ny,nz,3) complex64")
        put(f"{name}_Efield", np.asarray(Ef), "E_field_solver(P)")

    # ---- preconditioned path (precon=True): the reference's fft_matvec3 and
    # solve_gpbicgstab given the engine's preconditioner octant (restated by
    # the oracle's circulant_preconditioner; the reference's own builders are
    # missing), on a grid just above the box (L = 12 >= n = 10; the engine
    # compiles L = 12, not 10) and on the doubled grid (L = 2n)
    from oracle import dda_oracle as O
    k, d, alpha, E = probs["s10"]
    n = alpha.shape[0]
    ia_o = np.where(alpha != 0, 1.0 / np.where(alpha != 0, alpha, 1), 0)
    for Lp in (12, 2 * n):
        pre = O.circulant_preconditioner(ia_o, k, d, L=(Lp,) * 3).astype(np.complex64)
        rng = np.random.default_rng(9)
        x = (rng.standard_normal((n, n, n, 3)) + 1j * rng.standard_normal((n, n, n, 3))).astype(np.complex64)
        with ref_loader.quiet():
            a = cp.asarray(alpha, dtype=np.complex64)
            inv_alpha = cp.where(a != 0, 1.0 / a, 0)
            mask = a != 0
            maskf = cp.asarray(mask, dtype=np.float32)[..., None]
            chunks = G.setup_chunked_values(Lp // 2, Lp // 2, Lp // 2)
            y = G.fft_matvec3(cp.asarray(x).ravel(), None, cp.asarray(pre), maskf, chunks, n, n, n, True)
            it, P, low, first = G.solve_gpbicgstab((n, n, n), inv_alpha, fx["s10_G"], pre, E, mask, 100, 500,
                                                   target=1e-5, precon=True)
        tag = f"pre{Lp}"
        put(f"{tag}_octant", pre, f"s10 preconditioner octant on the {Lp}^3 grid, complex64 (hx,hy,hz,6)")
        put(f"{tag}_x", x, "seeded input of fft_matvec3")
        put(f"{tag}_Mx", np.asarray(y).reshape(n, n, n, 3), "fft_matvec3(x, octant, precon=True)")
        put(f"{tag}_iters", np.array(int(it)), "solve_gpbicgstab(s10, precon=True) iterations (ratio 100, 1e-5)")
        put(f"{tag}_lowfirst", np.array([float(low), float(first)]), "lowest/initial, first/initial")
        put(f"{tag}_P", np.asarray(P), "solution P = M p_current (nx,ny,nz,3) complex64")

    # ---- matvec and reductions on seeded vectors
    k, d, alpha, E = probs["s8"]
    rng = np.random.default_rng(123)
    x = (rng.standard_normal((8, 8, 8, 3)) + 1j * rng.standard_normal((8, 8, 8, 3))).astype(np.complex64)
    with ref_loader.quiet():
        a = cp.asarray(alpha, dtype=np.complex64)
        ia = cp.where(a != 0, 1.0 / a, 0)
        chunks = G.setup_chunked_values(8, 8, 8)
        ia3 = cp.repeat(ia, 3)
        maskf = cp.asarray(a != 0, dtype=np.float32)[..., None]
        y = G.interaction_mult(cp.asarray(x).ravel(), None, cp.asarray(fx["s8_G"]), ia3, maskf, chunks, 8, 8, 8)
        v = [cp.asarray((rng.standard_normal(3000) + 1j * rng.standard_normal(3000)).astype(np.complex64))
             for _ in range(3)]
        ip = G.inner_product(v[0], v[1])
        ze = G.calculate_zeta_eta_twostep(v[0], v[1], v[2])
    put("mv_x", x, "matvec input (s8 problem)")
    put("mv_y", np.asarray(y), "interaction_mult(x) flattened 3N")
    put("red_v", np.stack([np.asarray(t) for t in v]), "three seeded complex64 vectors (y, t, s)")
    put("red_inner", np.array(complex(ip)), "inner_product(v0, v1) = sum conj(v0) v1")
    put("red_zeta_eta", np.array([complex(ze[0]), complex(ze[1])]), "calculate_zeta_eta_twostep(y=v0, t=v1, s=v2)")
    np.savez_compressed(OUT, **fx)
    with open(OUT.replace(".npz", ".json"), "w") as f:
        json.dump(meta, f, indent=1)
    print(f"wrote {OUT} ({os.path.getsize(OUT) / 1024:.0f} KiB, {len(fx)} arrays)")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="reference checkout (default: oracle.build_ref.reference_dir())")
    main(ap.parse_args().ref or build_ref.reference_dir())
