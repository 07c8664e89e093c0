"""The CPU oracle against golden vectors produced by the reference's own code
(tests/golden/make_golden.py).  The reference computes in complex64, the
oracle in complex128, so tolerances are complex64-sized."""
import os

import numpy as np
import pytest

from oracle import dda_oracle as O

FX = os.path.join(os.path.dirname(__file__), "golden", "ref_fixtures.npz")


@pytest.fixture(scope="module")
def fx():
    return np.load(FX)


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def test_alpha_matches_reference(fx):
    for (n, d, k), vals in zip(fx["alpha_cases"], fx["alpha_values"]):
        got = [O.calculate_alpha(n, d.real, k.real, method="CM"), O.calculate_alpha(n, d.real, k.real, method="RR"),
               O.calculate_alpha(n, d.real, k.real, (0, 0, 1), (1, 0, 0), method="LDR"),
               O.calculate_alpha(n, d.real, k.real, (0, 0, 1), (0, 0, 1), method="LDR")]
        assert np.allclose(got, vals, rtol=1e-14, atol=0)


def test_lattice_setup_matches_reference(fx):
    from precondda_b200 import build_problem_from_shapes
    pr = build_problem_from_shapes([{"type": "sphere", "center": [0.1, 0.1, 0.1], "radius": 0.08, "n": 1.5}],
                                   np.array([0.0, 0.0, 1.0]), [1.0, 0.0, 0.0], 0.5, 0.02)
    assert np.array_equal(pr["alpha_array"], fx["sphere_alpha"])
    assert np.allclose(pr["E_inc"], fx["sphere_E"], rtol=0, atol=1e-15)
    pe = build_problem_from_shapes([{"type": "ellipsoid", "center": [0.12, 0.1, 0.08],
                                     "semi_axes": [0.11, 0.07, 0.05], "n": 1.6 + 0.05j}],
                                   np.array([1.0, 0.0, 0.0]), [0.0, 0.0, 1.0], 0.6, 0.02)
    assert np.array_equal(pe["alpha_array"], fx["ellipsoid_alpha"])
    assert np.allclose(pe["E_inc"], fx["ellipsoid_E"], rtol=0, atol=1e-15)


def test_green_octant_matches_reference(fx):
    k, d = fx["green_468_kd"]
    G = O.generate_interaction_row(4, 6, 8, k, d)
    assert _rel(G, fx["green_468_c128"]) < 1e-13
    assert _rel(G, fx["green_468_c64"]) < 1e-6


def test_matvec_matches_reference(fx):
    k, d = fx["s8_kd"]
    ia, mask, G, _ = O.prepare_interaction_matrices(fx["s8_alpha"], k, d)
    y = O.interaction_mult(fx["mv_x"].astype(np.complex128), G, ia, mask).ravel()
    assert _rel(y, fx["mv_y"]) < 2e-6


def test_reductions_match_reference(fx):
    v0, v1, v2 = [x.astype(np.complex128) for x in fx["red_v"]]
    assert abs(np.vdot(v0, v1) - fx["red_inner"]) / abs(fx["red_inner"]) < 1e-5
    yy, tt, yt, ty, ys, ts = (np.vdot(v0, v0), np.vdot(v1, v1), np.vdot(v0, v1), np.vdot(v1, v0),
                              np.vdot(v0, v2), np.vdot(v1, v2))
    den = tt * yy - yt * ty
    zeta, eta = (yy * ts - ys * ty) / den, (tt * ys - yt * ts) / den
    ref = fx["red_zeta_eta"]
    assert abs(zeta - ref[0]) / abs(ref[0]) < 1e-4 and abs(eta - ref[1]) / abs(ref[1]) < 1e-4


@pytest.mark.parametrize("name", ["s8", "s10", "ell"])
def test_solver_matches_reference(fx, name):
    k, d = fx[f"{name}_kd"]
    alpha = fx[f"{name}_alpha"]
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    it, P, low, first = O.solve_gpbicgstab(alpha.shape, ia, G, fx[f"{name}_E"], mask, 100, 500, target=1e-5)
    assert it == int(fx[f"{name}_iters"])
    Pr = fx[f"{name}_P"]
    assert np.linalg.norm(P - Pr) / np.linalg.norm(Pr) < 1e-4
    lo, fi = fx[f"{name}_lowfirst"]
    assert abs(first - fi) / fi < 1e-4
    assert abs(low - lo) / lo < 5e-2          # complex64 recursion near the target
    Ef = O.E_field_solver(Pr.astype(np.complex128), G, alpha.shape)
    assert _rel(Ef, fx[f"{name}_Efield"]) < 1e-5
