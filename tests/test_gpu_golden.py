"""The engine against golden vectors produced by the reference's own code
(tests/golden/make_golden.py), through the reference-named API and the C ABI.
The engine's complex64 path is compared with the reference's complex64
results; its complex128 path with the FP64 Green fixture."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

FX = os.path.join(os.path.dirname(__file__), "golden", "ref_fixtures.npz")


@pytest.fixture(scope="module")
def fx():
    return np.load(FX)


def _rel(a, b):
    a = a.cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return float(np.abs(a - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def test_green_matches_reference(fx):
    import precondda_b200 as P
    k, d = fx["green_468_kd"]
    g128 = P.generate_interaction_row(4, 6, 8, k, d, double_precision=True)
    g64 = P.generate_interaction_row(4, 6, 8, k, d, double_precision=False)
    assert _rel(g128, fx["green_468_c128"]) < 1e-13
    assert _rel(g64, fx["green_468_c64"]) < 1e-6
    full = P.generate_interaction_row(4, 6, 8, k, d, reduced=False, double_precision=True)
    assert tuple(full.shape) == (8, 12, 16, 6)


def test_interaction_mult_matches_reference(fx):
    import precondda_b200 as P
    alpha = fx["s8_alpha"]
    ia = np.where(alpha != 0, 1.0 / np.where(alpha != 0, alpha, 1), 0)
    y = P.interaction_mult(fx["mv_x"], None, fx["s8_G"], np.repeat(ia, 3), alpha != 0, None, 8, 8, 8)
    assert _rel(y, fx["mv_y"]) < 2e-6


@pytest.mark.parametrize("name", ["s8", "s10", "ell"])
def test_solve_gpbicgstab_matches_reference(fx, name):
    import precondda_b200 as P
    alpha = fx[f"{name}_alpha"]
    ia = np.where(alpha != 0, 1.0 / np.where(alpha != 0, alpha, 1), 0)
    it, Pg, low, first = P.solve_gpbicgstab(alpha.shape, ia, fx[f"{name}_G"], None, fx[f"{name}_E"], alpha != 0,
                                            100, 500, target=1e-5, precon=False)
    assert it == int(fx[f"{name}_iters"])
    Pr = fx[f"{name}_P"]
    assert np.linalg.norm(Pg.cpu().numpy() - Pr) / np.linalg.norm(Pr) < 1e-4
    lo, fi = fx[f"{name}_lowfirst"]
    assert abs(first - fi) / fi < 1e-4
    Ef = P.E_field_solver(Pr, fx[f"{name}_G"], alpha.shape)
    assert _rel(Ef, fx[f"{name}_Efield"]) < 1e-5
