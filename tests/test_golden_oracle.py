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


@pytest.mark.parametrize("Lp", [12, 20])
def test_preconditioned_path_matches_reference(fx, Lp):
    """precon=True: the oracle's preconditioner application and
    right-preconditioned GPBiCGSTAB against the reference's own fft_matvec3
    and solve_gpbicgstab(precon=True), given the same preconditioner octant
    (which the oracle's builder restates to complex64 rounding)."""
    k, d = fx["s10_kd"]
    alpha = fx["s10_alpha"]
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    pre = fx[f"pre{Lp}_octant"]
    assert pre.shape == (Lp // 2 + 1,) * 3 + (6,)
    built = O.circulant_preconditioner(ia, k, d, L=(Lp,) * 3)
    assert _rel(built, pre) < 1e-6
    Mx = O.precondition_apply(fx[f"pre{Lp}_x"], pre.astype(np.complex128), mask)
    assert _rel(Mx, fx[f"pre{Lp}_Mx"]) < 1e-5
    it, P, low, first = O.solve_gpbicgstab(alpha.shape, ia, G, fx["s10_E"], mask, 100, 500, target=1e-5,
                                           preconditioner=pre.astype(np.complex128))
    assert it == int(fx[f"pre{Lp}_iters"]) and it < int(fx["s10_iters"])
    Pr = fx[f"pre{Lp}_P"]
    assert np.linalg.norm(P - Pr) / np.linalg.norm(Pr) < 1e-4
    assert abs(first - fx[f"pre{Lp}_lowfirst"][1]) / fx[f"pre{Lp}_lowfirst"][1] < 1e-4


def test_occupancy_weights_of_a_full_box_are_chan_weights():
    """For a filled box the weights are T. Chan's per-axis factors
    prod (1 - |j_i|/n_i) of the optimal circulant of a Toeplitz matrix."""
    shape = (4, 6, 5)
    W = O.occupancy_weights(np.ones(shape, bool))
    for j in [(0, 0, 0), (1, 2, 3), (-3, 5, -4), (2, -1, 0)]:
        idx = tuple(jj % (2 * n) for jj, n in zip(j, shape))
        want = np.prod([1 - abs(jj) / n for jj, n in zip(j, shape)])
        assert abs(W[idx] - want) < 1e-12


def test_precondition_apply_is_the_dense_circulant_inverse():
    """M x with the engine's octant equals mask * inv(C) x for the dense
    circulant C = abar I + sum_j w(j) G(j) shift_j on the L-periodic grid
    (folded), the matrix the builder inverts."""
    shape, L = (3, 4, 3), (4, 4, 4)
    rng = np.random.default_rng(4)
    k, d = 2 * np.pi / 0.5, 0.03
    ia = np.where(rng.random(shape) < 0.7, 20.0 + 3.0j + rng.random(shape), 0)
    pre = O.circulant_preconditioner(ia, k, d, L=L)
    occ = ia != 0
    abar = ia[occ].mean()
    La = tuple(2 * n for n in shape)
    Gw = O.green_embedded(*shape, k, d, La) * O.occupancy_weights(occ)[..., None]
    npt = int(np.prod(L))
    Cm = np.zeros((npt, 3, npt, 3), complex)
    pts = [np.unravel_index(p, L) for p in range(npt)]
    for p, P_ in enumerate(pts):
        Cm[p, :, p, :] += abar * np.eye(3)
        for q, Q_ in enumerate(pts):
            t = tuple((a - b) % Ln for a, b, Ln in zip(P_, Q_, L))
            for i_ in np.ndindex(*La):
                off = [ii if ii < n else ii - Lan for ii, n, Lan in zip(i_, shape, La)]
                if all(o % Ln == tt for o, Ln, tt in zip(off, L, t)) and any(o != 0 for o in off):
                    g = Gw[i_]
                    Cm[p, :, q, :] += np.array([[g[0], g[1], g[2]], [g[1], g[3], g[4]], [g[2], g[4], g[5]]])
    Ci = np.linalg.inv(Cm.reshape(3 * npt, 3 * npt))
    x = rng.standard_normal(shape + (3,)) + 1j * rng.standard_normal(shape + (3,))
    xp = np.zeros(L + (3,), complex)
    xp[:shape[0], :shape[1], :shape[2]] = x
    y = (Ci @ xp.reshape(-1)).reshape(L + (3,))[:shape[0], :shape[1], :shape[2]] * occ[..., None]
    assert _rel(O.precondition_apply(x, pre, occ), y) < 1e-10


SHAPES = os.path.join(os.path.dirname(__file__), "golden", "shape_fixtures.npz")


def _shape_cases():
    import json
    with open(SHAPES.replace(".npz", ".json")) as f:
        cases = json.load(f)["cases"]
    out = []
    for name, c in cases.items():
        shapes = []
        for s in c["shapes"]:
            s = dict(s)
            if isinstance(s["n"], str):
                s["n"] = complex(s["n"])
            shapes.append(s)
        out.append((name, shapes, c))
    return out


@pytest.mark.parametrize("name,shapes,case", _shape_cases(), ids=[c[0] for c in _shape_cases()])
def test_shape_lattices_match_reference(name, shapes, case):
    """Rectangle, cylinder (every axis, with the reference's own x/y-axis
    handling) and prism lattices, site for site, against the reference's
    build_problem_from_shapes (tests/golden/make_shape_fixtures.py)."""
    from precondda_b200 import build_problem_from_shapes
    ref = np.load(SHAPES)[f"{name}_alpha"]
    pr = build_problem_from_shapes(shapes, np.array(case["k_direction"]), case["polarization"],
                                   case["wavelength"], case["spacing"])
    assert pr["alpha_array"].shape == ref.shape
    assert np.array_equal(pr["alpha_array"], ref)


def test_geometric_cylinder_flag_differs_from_reference_axes():
    """geometric=True is the axis-true cylinder; the default reproduces the
    reference (which fills the window below c_z + h/2 for the x/y axes)."""
    from precondda_b200.lattice import Cylinder, inside_cylinder
    pts = np.stack(np.meshgrid(*[np.arange(-10, 10) + 0.5] * 3, indexing="ij"), -1).reshape(-1, 3)
    ref = inside_cylinder(pts, (0, 0, 0), 4.0, 6.0, "x")
    geo = inside_cylinder(pts, (0, 0, 0), 4.0, 6.0, "x", geometric=True)
    assert ref.sum() != geo.sum()
    # geometric x-axis cylinder: |x| <= 3 and y^2 + z^2 <= 16
    exp = (np.abs(pts[:, 0]) <= 3.0) & (pts[:, 1] ** 2 + pts[:, 2] ** 2 <= 16.0)
    assert np.array_equal(geo, exp)
    assert Cylinder("c", (0, 0, 0), 1, 1, "y").geometric is False
