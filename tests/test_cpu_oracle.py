"""CPU checks of the oracle restatement itself (no GPU)."""
import numpy as np
import pytest

from oracle import dda_oracle as O


def _prob(shape, seed, fill=0.6):
    rng = np.random.default_rng(seed)
    k = 2 * np.pi / 0.5
    d = 0.4 / k
    a = O.calculate_alpha(1.6 + 0.05j, d, k, method="RR")
    alpha = np.where(rng.random(shape) < fill, a, 0)
    x = rng.standard_normal(shape + (3,)) + 1j * rng.standard_normal(shape + (3,))
    return k, d, alpha, x


@pytest.mark.parametrize("shape", [(4, 4, 4), (3, 5, 4), (2, 6, 3)])
def test_fft_matvec_equals_dense(shape):
    k, d, alpha, x = _prob(shape, 1)
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    y = O.interaction_mult(x, G, ia, mask)
    yd = O.dense_interaction_mult(x, ia, k, d, mask)
    assert np.abs(y - yd).max() / np.abs(yd).max() < 1e-12


@pytest.mark.parametrize("L", [(10, 12, 16), (12, 16, 20)])
def test_larger_embedding_gives_same_product(L):
    shape = (4, 5, 6)
    k, d, alpha, x = _prob(shape, 2)
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    ia2, mask2, G2, _ = O.prepare_interaction_matrices(alpha, k, d, L=L)
    y1 = O.interaction_mult(x, G, ia, mask)
    y2 = O.interaction_mult(x, G2, ia2, mask2, L=L)
    assert np.abs(y1 - y2).max() / np.abs(y1).max() < 1e-12


def test_octant_mirror_reproduces_full_spectrum():
    shape = (4, 6, 8)
    k, d = 2 * np.pi / 0.5, 0.03
    full = O.generate_interaction_row(*shape, k, d, reduced=False)
    oct_ = O.generate_interaction_row(*shape, k, d, reduced=True)
    T = O.expand_octant(oct_, full.shape[:3])
    comp = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    for c, (a, b) in enumerate(comp):
        assert np.abs(T[..., a, b] - full[..., c]).max() < 1e-10 * np.abs(full).max()


def test_nyquist_planes_and_origin_zero():
    G = O.green_embedded(4, 4, 4, 10.0, 0.05)
    assert np.all(G[0, 0, 0] == 0)
    assert np.all(G[4] == 0) and np.all(G[:, 4] == 0) and np.all(G[:, :, 4] == 0)


def test_sphere_site_counts():
    assert O.sphere_lattice(32, 16.0).sum() == 17256
    assert O.sphere_lattice(64, 32.0).sum() == 137376


def test_alpha_variants():
    n, d, k = 1.5 + 0.01j, 0.02, 2 * np.pi / 0.5
    cm = O.calculate_alpha(n, d, k, method="CM")
    rr = O.calculate_alpha(n, d, k, method="RR")
    assert np.isclose(1 / rr, 1 / cm - 2j / 3 * k ** 3)
    ldr = O.calculate_alpha(n, d, k, (0, 0, 1), (1, 0, 0), method="LDR")
    b1, b2 = -1.891531, 0.1648469
    assert np.isclose(1 / ldr, 1 / cm + (b1 + n ** 2 * b2) * k ** 2 / d - 2j / 3 * k ** 3)
    with pytest.raises(ValueError):
        O.calculate_alpha(n, d, k, method="LDR")
    with pytest.raises(ValueError):
        O.calculate_alpha(n, d, k, method="XX")


def test_mie_small_sphere_rayleigh_limit():
    # Rayleigh limit: Qsca = 8/3 x^4 |(m^2-1)/(m^2+2)|^2
    m, x = 1.5 + 0.0j, 0.01
    qe, qs = O.mie_qext_qsca(m, x)
    ray = 8 / 3 * x ** 4 * abs((m * m - 1) / (m * m + 2)) ** 2
    assert abs(qs - ray) / ray < 1e-3
    assert abs(qe - qs) / qs < 1e-6          # non-absorbing


def test_mie_optical_theorem_limits():
    qe, qs = O.mie_qext_qsca(1.33 + 0.0j, 50.0)
    assert 1.9 < qe < 2.3 and abs(qe - qs) < 1e-8   # extinction paradox regime


def test_oracle_solver_converges_and_cross_sections_positive():
    n, m = 8, 1.5 + 0.01j
    k = 2 * np.pi / 0.5
    d = 0.5 / (abs(m) * k)
    occ = O.sphere_lattice(n, n / 2)
    alpha = np.where(occ, O.calculate_alpha(m, d, k, method="RR"), 0)
    E = O.incident_field((n, n, n), d, k, (0, 0, 1), (1, 0, 0))
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    it, P, low, first = O.solve_gpbicgstab((n, n, n), ia, G, E, mask, 100, 300, target=1e-8)
    assert it > 0
    assert O.true_relative_residual(P, E, G, ia, mask) < 1e-7
    ce, ca, cs = O.cross_sections(P, E, ia, k)
    assert ce > 0 and ca > 0 and cs > 0


def test_oracle_solver_reports_max_iter_and_nan():
    n = 6
    k = 2 * np.pi / 0.5
    d = 0.05
    alpha = np.full((n, n, n), O.calculate_alpha(2.0 + 0.5j, d, k, method="RR"))
    E = O.incident_field((n, n, n), d, k, (0, 0, 1), (1, 0, 0))
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    it, P, low, first = O.solve_gpbicgstab((n, n, n), ia, G, E, mask, 100, 3, target=1e-14)
    assert it == 3
    Enan = E.copy()
    Enan[0, 0, 0, 0] = np.nan
    it, P, low, first = O.solve_gpbicgstab((n, n, n), ia, G, Enan, mask, 100, 10, target=1e-6)
    assert it < 0
