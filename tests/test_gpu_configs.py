"""Parity at the benchmark configurations' full sizes.

* The 32^3 plain complex128 sphere (radius 16 d, m = 1.5+0.01i, tol 1e-6,
  maxiter 2000): the engine's solve against the oracle's, run here in full
  (same iteration count, P and the cross sections to 1e-8), and against the
  reference's own complex64 solve_gpbicgstab (tests/golden/config_fixtures.npz,
  made by tests/golden/make_config_fixtures.py: same iteration count, cross
  sections and sampled P to the reference's complex64 rounding).
* The 64^3 precision sphere (m = 1.7+0.1i, x and y polarisations): the mixed
  complex64 + FP64-refinement solves (preconditioned and not) and the plain
  complex128 solve against the oracle's complex128 solve to 1e-8 (fixture):
  C_ext, C_abs, C_sca and sampled P within 1e-4.
* One 128^3 matvec in both precisions against oracle.interaction_mult on a
  seeded input (fixture: sampled y and ||y||).
"""
import math
import os

import numpy as np
import pytest
import torch

from oracle import dda_oracle as O

pytestmark = pytest.mark.gpu

FX = os.path.join(os.path.dirname(__file__), "golden", "config_fixtures.npz")
C64, C128 = torch.complex64, torch.complex128


@pytest.fixture(scope="module")
def fx():
    return np.load(FX)


def _sample_sites(shape, seed, count=4096):
    n = int(np.prod(shape))
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n, size=min(count, n), replace=False))


def _sphere(n, m, pol):
    k = 2 * math.pi / 0.5
    d = 0.5 / (abs(m) * k)
    occ = O.sphere_lattice(n, n / 2.0)
    alpha = np.where(occ, O.calculate_alpha(m, d, k, method="RR"), 0).astype(np.complex128)
    E = O.incident_field((n, n, n), d, k, (0, 0, 1), pol)
    return k, d, alpha, E


def _rel_sample(P, sample, seed):
    Ps = np.asarray(P).reshape(-1, 3)[_sample_sites(np.asarray(P).shape[:3], seed)]
    return float(np.abs(Ps - sample).max() / np.abs(sample).max())


def _xsec_err(got, ref):
    return max(abs(g - r) / abs(r) for g, r in zip(got, ref))


def test_sphere32_plain_c128_solve_matches_oracle_and_reference(fx):
    import precondda_b200 as P
    n, m = 32, 1.5 + 0.01j
    k, d, alpha, E = _sphere(n, m, (1, 0, 0))
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    assert int(mask.sum()) == int(fx["c1_nocc"]) == 17256
    it_o, P_o, low_o, first_o = O.solve_gpbicgstab((n,) * 3, ia, G, E, mask, 100, 2000, target=1e-6)
    op = P.DDAOperator(ia, k, d, dtype=C128)
    Pg, info = op.solve(E, tol=1e-6, max_iter=2000, ratio=100)
    Pn = Pg.cpu().numpy()
    # against the oracle, run here
    assert info.iters == it_o == int(fx["c1_oracle_iters"])
    assert np.abs(Pn - P_o).max() / np.abs(P_o).max() < 1e-8
    assert abs(info.lowest_rel - low_o) <= 1e-8 * low_o
    xs = op.cross_sections(Pg, E)
    assert _xsec_err(xs, O.cross_sections(P_o, E, ia, k)) < 1e-8
    assert O.true_relative_residual(Pn, E, G, ia, mask) < 1e-6 * 5
    # against the reference's own complex64 solve of the same problem
    assert info.iters == int(fx["c1_ref_iters"])
    assert _xsec_err(xs, fx["c1_ref_xsec"]) < 1e-4
    assert _rel_sample(Pn, fx["c1_ref_Psample"], 1) < 1e-4
    assert abs(np.linalg.norm(Pn) - float(fx["c1_ref_Pnorm"])) / float(fx["c1_ref_Pnorm"]) < 1e-5


def test_sphere32_reference_api_solve_matches_reference(fx):
    """The drop-in solve_gpbicgstab (complex64 like the reference's) on the
    32^3 sphere: the reference's iteration count and outputs."""
    import precondda_b200 as P
    n, m = 32, 1.5 + 0.01j
    k, d, alpha, E = _sphere(n, m, (1, 0, 0))
    a = alpha.astype(np.complex64)
    inv_alpha = np.where(a != 0, 1.0 / np.where(a != 0, a, 1), 0).astype(np.complex64)
    G = P.generate_interaction_row(n, n, n, k, d, True, False)
    it, Pr, low, first = P.solve_gpbicgstab((n, n, n), inv_alpha, G, None, E, a != 0, 100, 2000, target=1e-6,
                                            precon=False)
    Pn = Pr.cpu().numpy() if hasattr(Pr, "cpu") else np.asarray(Pr)
    assert abs(int(it) - int(fx["c1_ref_iters"])) <= 1
    ia = np.where(alpha != 0, 1.0 / np.where(alpha != 0, alpha, 1), 0)
    assert _xsec_err(O.cross_sections(Pn.astype(np.complex128), E, ia, k), fx["c1_ref_xsec"]) < 1e-4
    assert _rel_sample(Pn, fx["c1_ref_Psample"], 1) < 1e-4


@pytest.mark.parametrize("precond", [False, True])
def test_config2_mixed_solves_match_fp64_oracle(fx, precond):
    import precondda_b200 as P
    n, m = 64, 1.7 + 0.1j
    pols = [(1, 0, 0), (0, 1, 0)]
    k, d, alpha, _ = _sphere(n, m, pols[0])
    Es = [_sphere(n, m, p)[3] for p in pols]
    ia = np.where(alpha != 0, 1.0 / np.where(alpha != 0, alpha, 1), 0)
    op = P.DDAOperator(ia, k, d, dtype=C128, with_twin=True)
    pre = op.preconditioner() if precond else None
    Ed = [torch.as_tensor(E, device="cuda") for E in Es]
    Pm, infos = P.solve_many([op, op], Ed, tol=1e-6, max_iter=2000, ratio=100, precision="mixed",
                             inner_tol=1e-4, preconditioner=pre)
    Pc, infc = P.solve_many([op, op], Ed, tol=1e-6, max_iter=2000, ratio=100, precision="c128",
                            preconditioner=pre)
    for j in range(2):
        truth = fx[f"c2_p{j}_xsec"]
        for Pj, inf in ((Pm[j], infos[j]), (Pc[j], infc[j])):
            assert inf.status == "converged", inf
            xs = op.cross_sections(Pj, Ed[j])
            assert _xsec_err(xs, truth) < 1e-4, (j, xs, truth)
            Pn = Pj.cpu().numpy()
            assert _rel_sample(Pn, fx[f"c2_p{j}_Psample"], 2 + j) < 1e-4
            assert abs(np.linalg.norm(Pn) - float(fx[f"c2_p{j}_Pnorm"])) / float(fx[f"c2_p{j}_Pnorm"]) < 1e-5
        assert infos[j].true_relres <= 1e-6
    # one instance alone: the single-instance launch path (cluster-fused z/y
    # passes of the 64^3 complex64 kernels) gives the batched result's physics
    P1, i1 = op.solve(Es[0], tol=1e-6, max_iter=2000, ratio=100, precision="mixed", inner_tol=1e-4,
                      preconditioner=pre)
    assert i1.status == "converged"
    assert _xsec_err(op.cross_sections(P1, Ed[0]), fx["c2_p0_xsec"]) < 1e-4


def test_matvec_128_matches_oracle_fixture(fx):
    import precondda_b200 as P
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "mcf", os.path.join(os.path.dirname(__file__), "golden", "make_config_fixtures.py"))
    mcf = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mcf)
    k, d, ia, x = mcf.mv128_problem()
    assert np.allclose(fx["mv128_kd"], [k, d], rtol=0, atol=0)
    sample = fx["mv128_ysample"]
    ynorm = float(fx["mv128_ynorm"])
    for dt, tol in ((C128, 1e-11), (C64, 2e-5)):
        op = P.DDAOperator(ia, k, d, dtype=dt)
        assert tuple(op.L) == (256, 256, 256)
        y = op.matvec(torch.as_tensor(x, device="cuda").to(dt)).cpu().numpy()
        assert _rel_sample(y, sample, 128) < tol, dt
        assert abs(np.linalg.norm(y) - ynorm) / ynorm < tol
        del op
