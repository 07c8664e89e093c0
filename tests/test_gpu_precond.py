"""The preconditioned path (the reference's precon=True) on the GPU: the
engine's preconditioner builder against the oracle's restatement, the
preconditioner application and the right-preconditioned GPBiCGSTAB against
the reference's own outputs (tests/golden) and the oracle."""
import os

import numpy as np
import pytest
import torch

from oracle import dda_oracle as O

pytestmark = pytest.mark.gpu

C64, C128 = torch.complex64, torch.complex128
FX = os.path.join(os.path.dirname(__file__), "golden", "ref_fixtures.npz")


@pytest.fixture(scope="module")
def fx():
    return np.load(FX)


def _rel(a, b):
    a = np.asarray(a); b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _sphere(n, m, wavelength=0.5, kd=0.5, pol=(1, 0, 0)):
    k = 2 * np.pi / wavelength
    d = kd / (abs(m) * k)
    occ = O.sphere_lattice(n, n / 2.0)
    a = O.calculate_alpha(m, d, k, method="RR")
    ia = np.where(occ, 1.0 / a, 0).astype(np.complex128)
    E = O.incident_field((n, n, n), d, k, (0, 0, 1), pol)
    return k, d, ia, E


def _blob(shape, seed, m=2.0 + 0.1j):
    """An irregular scatterer (no axis-reflection symmetry)."""
    rng = np.random.default_rng(seed)
    k = 2 * np.pi / 0.6
    d = 0.5 / (abs(m) * k)
    g = np.stack(np.meshgrid(*[np.arange(n) + 0.5 for n in shape], indexing="ij"), -1)
    occ = np.zeros(shape, bool)
    for _ in range(4):
        c = rng.random(3) * np.array(shape)
        r = 0.25 * min(shape) * (1 + rng.random())
        occ |= ((g - c) ** 2).sum(-1) <= r * r
    a = O.calculate_alpha(m, d, k, method="RR")
    ia = np.where(occ, 1.0 / a, 0).astype(np.complex128)
    E = O.incident_field(shape, d, k, (0, 0, 1), (1, 0, 0))
    return k, d, ia, E


@pytest.mark.parametrize("shape,L", [((10, 10, 10), (12, 12, 12)), ((10, 10, 10), (20, 20, 20)),
                                     ((8, 12, 16), (8, 12, 16)), ((8, 12, 16), (16, 24, 32)),
                                     ((7, 9, 11), (8, 12, 12))])
def test_builder_matches_oracle(shape, L):
    import precondda_b200 as P
    k, d, ia, _ = _blob(shape, seed=sum(shape))
    pre = P.Preconditioner(inv_alpha=ia, k=k, d=d, L_=L)
    assert pre.L == L and abs(pre.scale * np.prod(L) - 1) < 1e-15
    got = pre.reference_octant(C128).cpu().numpy()
    want = O.circulant_preconditioner(ia, k, d, L=L)
    assert got.shape == want.shape
    assert _rel(got, want) < 1e-10
    assert _rel(pre.reference_octant(C64).cpu().numpy(), want) < 1e-6


@pytest.mark.parametrize("Lp", [12, 20])
def test_apply_and_solve_match_reference(fx, Lp):
    """fft_matvec3 and solve_gpbicgstab(precon=True) through the engine's
    reference API, given the octant the reference was run with."""
    import precondda_b200 as P
    alpha = fx["s10_alpha"]
    ia = np.where(alpha != 0, 1.0 / np.where(alpha != 0, alpha, 1), 0)
    pre = fx[f"pre{Lp}_octant"]
    n = alpha.shape[0]
    y = P.fft_matvec3(fx[f"pre{Lp}_x"], None, pre, alpha != 0, None, n, n, n, True)
    assert _rel(y.reshape(n, n, n, 3).cpu().numpy(), fx[f"pre{Lp}_Mx"]) < 2e-6
    x = torch.as_tensor(fx[f"pre{Lp}_x"]).reshape(-1)
    assert P.fft_matvec3(x, None, pre, alpha != 0, None, n, n, n, False) is not None
    it, Pg, low, first = P.solve_gpbicgstab(alpha.shape, ia, fx["s10_G"], pre, fx["s10_E"], alpha != 0, 100, 500,
                                            target=1e-5, precon=True)
    assert it == int(fx[f"pre{Lp}_iters"])
    Pr = fx[f"pre{Lp}_P"]
    assert np.linalg.norm(Pg.cpu().numpy() - Pr) / np.linalg.norm(Pr) < 1e-4
    assert abs(first - fx[f"pre{Lp}_lowfirst"][1]) / fx[f"pre{Lp}_lowfirst"][1] < 1e-4


@pytest.mark.parametrize("n,m,L", [(10, 2.5 + 0.1j, None), (16, 1.7 + 0.1j, (32, 32, 32)),
                                   (12, 2.0 + 0.1j, (12, 12, 12))])
def test_c128_preconditioned_solve_matches_oracle(n, m, L):
    import precondda_b200 as P
    k, d, ia, E = _sphere(n, m)
    op = P.DDAOperator(ia, k, d, dtype=C128)
    pre = op.preconditioner(L)
    Pg, info = op.solve(E, tol=1e-6, max_iter=500, preconditioner=pre)
    G = O.generate_interaction_row(n, n, n, k, d, L=op.L)
    mask = ia != 0
    it, Pr, low, first = O.solve_gpbicgstab((n, n, n), ia, G, E, mask, 100, 500, target=1e-6,
                                            preconditioner=pre.reference_octant(C128).cpu().numpy())
    assert info.status == "converged" and info.iters == it
    assert _rel(Pg.cpu().numpy(), Pr) < 1e-8
    assert abs(info.first_rel - first) < 1e-9
    it0, _, _, _ = O.solve_gpbicgstab((n, n, n), ia, G, E, mask, 100, 500, target=1e-6)
    assert it < it0
    assert O.true_relative_residual(Pg.cpu().numpy(), E, G, ia, mask, L=op.L) < 2e-6


def test_mixed_and_c64_preconditioned_solves():
    """Mixed precision with preconditioned complex64 sweeps reaches the FP64
    target in fewer inner iterations; c64 agrees with the FP64 solution."""
    import precondda_b200 as P
    n, m = 24, 2.5 + 0.1j
    k, d, ia, E = _sphere(n, m)
    op = P.DDAOperator(ia, k, d, dtype=C128, with_twin=True)
    P0, i0 = op.solve(E, tol=1e-7, max_iter=2000, precision="mixed")
    P1, i1 = op.solve(E, tol=1e-7, max_iter=2000, precision="mixed", preconditioner=True)
    assert i0.status == "converged" and i1.status == "converged" and i1.true_relres <= 1e-7
    assert i1.iters < i0.iters
    assert np.linalg.norm((P1 - P0).cpu().numpy()) / np.linalg.norm(P0.cpu().numpy()) < 1e-6
    P2, i2 = op.solve(E, tol=1e-5, max_iter=2000, precision="c64", preconditioner=True)
    assert i2.status == "converged"
    assert np.linalg.norm(P2.cpu().numpy() - P0.cpu().numpy()) / np.linalg.norm(P0.cpu().numpy()) < 1e-4


def test_batched_preconditioned_solve_equals_single():
    """Two geometries of one box, each with its own preconditioner, solved in
    one batch: the same iterations and solutions as alone."""
    import precondda_b200 as P
    shape = (12, 12, 12)
    ops, Es, pres = [], [], []
    for seed, m in ((1, 1.8 + 0.05j), (2, 2.6 + 0.2j)):
        k, d, ia, E = _blob(shape, seed, m)
        op = P.DDAOperator(ia, k, d, dtype=C128)
        ops.append(op); Es.append(E); pres.append(op.preconditioner())
    Pb, ib = P.solve_many(ops, Es, tol=1e-7, max_iter=500, preconditioner=pres)
    for op, E, pre, Pj, ij in zip(ops, Es, pres, Pb, ib):
        Ps, is_ = op.solve(E, tol=1e-7, max_iter=500, preconditioner=pre)
        assert ij.iters == is_.iters and ij.status == "converged"
        assert np.abs((Pj - Ps).cpu().numpy()).max() / np.abs(Ps.cpu().numpy()).max() < 1e-10


def test_run_solver_default_precon_and_errors():
    """run_solver's default precon=True now runs (prepare_interaction_matrices
    returns the engine's preconditioner); precon=True without one is an
    error."""
    import precondda_b200 as P
    n, m = 10, 1.7 + 0.1j
    k = 2 * np.pi / 0.5
    d = 0.5 / (abs(m) * k)
    occ = O.sphere_lattice(n, n / 2.0)
    alpha = np.where(occ, O.calculate_alpha(m, d, k, method="RR"), 0)
    E = O.incident_field((n, n, n), d, k, (0, 0, 1), (1, 0, 0))
    ia, mask, G, pre = P.prepare_interaction_matrices((n, n, n), k, None, 3 * n, 3 * n, 3 * n, alpha, d)
    assert tuple(pre.shape) == tuple(G.shape) == (n + 1, n + 1, n + 1, 6) and pre.dtype == C64   # grid 2n
    it, Pg, low = P.run_solver((n, n, n), k, alpha, d, 3 * n, 3 * n, 3 * n, None, E, max_iter=500)
    it0, _, _ = P.run_solver((n, n, n), k, alpha, d, 3 * n, 3 * n, 3 * n, None, E, precon=False, max_iter=500)
    assert 0 < it < it0
    G_o = O.generate_interaction_row(n, n, n, k, d)
    ia_o = np.where(occ, 1.0 / np.where(occ, alpha, 1), 0)
    assert O.true_relative_residual(Pg.cpu().numpy(), E, G_o, ia_o, occ) < 1e-4
    with pytest.raises(ValueError):
        P.solve_gpbicgstab((n, n, n), ia, G, None, E, mask, 100, 10, precon=True)
    with pytest.raises(NotImplementedError):
        P.solve_gpbicgstab((n, n, n), ia, G, pre, E, mask, 100, 10, precon=True, is_2d=True)


def test_precond_edge_cases_and_errors():
    """Zero right-hand side, an empty lattice and bad C-ABI arguments."""
    import ctypes as C
    import precondda_b200 as P
    from precondda_b200 import _lib as L
    n, m = 8, 2.0 + 0.1j
    k, d, ia, E = _sphere(n, m)
    op = P.DDAOperator(ia, k, d, dtype=C128)
    pre = op.preconditioner()
    Pz, iz = op.solve(np.zeros_like(E), tol=1e-6, max_iter=50, preconditioner=pre)
    assert float(Pz.abs().max()) == 0.0
    # a batch where one instance has no right-hand side: the other is unaffected
    Pb, ib = P.solve_many([op, op], [E, np.zeros_like(E)], tol=1e-6, max_iter=200, preconditioner=pre)
    Ps, is_ = op.solve(E, tol=1e-6, max_iter=200, preconditioner=pre)
    assert ib[0].iters == is_.iters and float(Pb[1].abs().max()) == 0.0
    # an empty lattice: prepare_interaction_matrices returns no preconditioner
    alpha0 = np.zeros((n, n, n), np.complex128)
    _, _, _, pre0 = P.prepare_interaction_matrices((n, n, n), k, None, 0, 0, 0, alpha0, d)
    assert pre0 is None
    # C ABI argument checks
    ctx = L.context(0)
    lib = L.lib()
    out = torch.empty((6, 9, 9, 9), dtype=C128, device="cuda")
    iac = torch.as_tensor(ia, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert lib.dda_precond_build(ctx.handle, n, n, n, 6, 16, 16, k, d, iac.data_ptr(), L.GHAT_ENGINE,
                                 out.data_ptr(), None, s) == L.DDA_ERR_BAD_SHAPE          # grid < box
    assert lib.dda_precond_build(ctx.handle, n, n, n, 16, 16, 16, k, d, None, L.GHAT_ENGINE,
                                 out.data_ptr(), None, s) == L.DDA_ERR_ARG                # no inv_alpha
    assert lib.dda_precond_build(ctx.handle, n, n, n, 16, 16, 16, k, d, iac.data_ptr(), 7,
                                 out.data_ptr(), None, s) == L.DDA_ERR_ARG                # bad layout
    h = C.c_void_p()
    assert lib.dda_precond_op_create(ctx.handle, L.DDA_C128, n, n, n, 14, 16, 16, out.data_ptr(), 1.0,
                                      iac.data_ptr(), C.byref(h)) == L.DDA_ERR_BAD_SHAPE  # 14: not compiled
    with pytest.raises(ValueError):
        P.Preconditioner(inv_alpha=ia, k=k, d=d, L_=(4, 16, 16))                          # grid < box


@pytest.mark.parametrize("case", ["cube64", "blob"])
def test_fused_preconditioner_handoff_equals_separate_passes(monkeypatch, case):
    """A M with M's last pass and A's first in one kernel (the M vector
    handed over in shared memory, never in HBM) gives the separate passes'
    iterates bit for bit: c64, c128 and mixed preconditioned solves, on a
    cubic box (compile-time kernels) and an irregular scatterer in a ragged
    box (runtime-size kernels), two right-hand sides in one batch."""
    import precondda_b200 as P
    if case == "cube64":
        k, d, ia, E = _sphere(64, 1.7 + 0.1j)
        E2 = O.incident_field((64,) * 3, d, k, (0, 0, 1), (0, 1, 0))
    else:
        k, d, ia, E = _blob((20, 24, 28), 5, 2.2 + 0.1j)
        E2 = O.incident_field((20, 24, 28), d, k, (0, 1, 0), (1, 0, 0))
    op = P.DDAOperator(ia, k, d, dtype=C128, with_twin=True)
    pre = op.preconditioner()

    def run():
        op._ctx.trim()                      # cached iteration graphs hold the kernels of their capture
        out = []
        for prec, tol in (("c64", 1e-5), ("c128", 1e-7), ("mixed", 1e-7)):
            Ps, infos = P.solve_many([op, op], [E, E2], tol=tol, max_iter=400, precision=prec, preconditioner=pre)
            out.append(([p.clone() for p in Ps], [(i.iters, i.outer, i.status) for i in infos]))
        return out

    fused = run()
    monkeypatch.setenv("DDA_NO_MA_FUSE", "1")
    separate = run()
    for (Pf, inf), (Ps, ins) in zip(fused, separate):
        assert inf == ins
        assert all(st == "converged" for _, _, st in inf)
        for a, b in zip(Pf, Ps):
            assert torch.equal(a, b)
