"""GPU parity of the engine against the CPU oracle (complex128 restatement of
the reference's algorithm).  Every call goes through libdda_b200.so."""
import numpy as np
import pytest
import torch

from oracle import dda_oracle as O

pytestmark = pytest.mark.gpu

C64, C128 = torch.complex64, torch.complex128


def _pkg():
    import precondda_b200 as P
    return P


def _rand_problem(shape, seed, m=1.5 + 0.1j, fill=0.7, wavelength=0.5, kd=0.4):
    rng = np.random.default_rng(seed)
    k = 2 * np.pi / wavelength
    d = kd / k
    a = O.calculate_alpha(m, d, k, method="RR")
    alpha = np.where(rng.random(shape) < fill, a, 0).astype(np.complex128)
    x = rng.standard_normal(shape + (3,)) + 1j * rng.standard_normal(shape + (3,))
    return k, d, alpha, x


def _rel(a, b):
    a = np.asarray(a); b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("shape,L", [((4, 6, 8), None), ((6, 10, 12), None), ((5, 7, 9), None),
                                     ((4, 4, 4), (16, 12, 8))])
def test_green_octant_matches_oracle(shape, L):
    P = _pkg()
    k, d = 2 * np.pi / 0.5, 0.02
    Ls = L or P.fft_lengths(shape)
    g = P.green_octant(shape, k, d, Ls, 1.0, C128).cpu().numpy()
    ref = O.generate_interaction_row(*shape, k, d, L=Ls)
    assert g.shape == ref.shape
    assert _rel(g, ref) < 1e-12
    g64 = P.green_octant(shape, k, d, Ls, 1.0, C64).cpu().numpy()
    assert _rel(g64, ref) < 1e-6


@pytest.mark.parametrize("shape", [(8, 8, 8), (6, 10, 12), (5, 7, 9), (12, 4, 6), (16, 16, 16)])
@pytest.mark.parametrize("dtype,tol", [(C128, 1e-12), (C64, 2e-5)])
def test_matvec_matches_oracle(shape, dtype, tol):
    P = _pkg()
    k, d, alpha, x = _rand_problem(shape, seed=sum(shape))
    ia, mask, _, _ = O.prepare_interaction_matrices(alpha, k, d)
    op = P.DDAOperator(ia, k, d, dtype=dtype)
    Gref = O.generate_interaction_row(*shape, k, d, L=op.L)
    ref = O.interaction_mult(x, Gref, ia, mask, L=op.L)
    y = op.matvec(x).cpu().numpy()
    assert _rel(y, ref) < tol
    # the other pass-5 modes
    conv = O.fft_convolve(x, Gref, op.L)
    assert _rel(op.conv(x).cpu().numpy(), conv) < tol
    assert _rel(op.conv_masked(x).cpu().numpy(), conv * mask[..., None]) < tol
    b = x[::-1].copy()
    r = op.residual(b, x).cpu().numpy()
    assert _rel(r, b * mask[..., None] - ref) < tol


@pytest.mark.parametrize("variant", ["0", "1", "2"])
@pytest.mark.parametrize("shape", [(8, 8, 8), (6, 10, 12), (16, 12, 32), (32, 32, 32)])
@pytest.mark.parametrize("dtype,tol", [(C128, 1e-12), (C64, 2e-5)])
def test_matvec_pass3_variants(variant, shape, dtype, tol, monkeypatch):
    P = _pkg()
    monkeypatch.setenv("DDA_P3_VARIANT", variant)
    k, d, alpha, x = _rand_problem(shape, seed=7)
    ia, mask, _, _ = O.prepare_interaction_matrices(alpha, k, d)
    op = P.DDAOperator(ia, k, d, dtype=dtype)
    Gref = O.generate_interaction_row(*shape, k, d, L=op.L)
    ref = O.interaction_mult(x, Gref, ia, mask, L=op.L)
    assert _rel(op.matvec(x).cpu().numpy(), ref) < tol


@pytest.mark.parametrize("n", [4, 6, 10, 12, 16, 20, 24, 32, 36, 40, 48, 64, 72, 80, 96, 128, 144, 160])
@pytest.mark.parametrize("dtype,tol", [(C128, 1e-12), (C64, 2e-5)])
def test_cubic_kernels_launch_and_match_general(n, dtype, tol, monkeypatch):
    """Every compiled cubic FFT length up to 320 (box n^3 on (2n)^3) launches
    and equals the runtime-size kernels on the same operator.  Above 170
    registers per thread a 384-thread CTA cannot launch, so this catches
    launch-bound mistakes at lengths no other test reaches."""
    P = _pkg()
    k, d, alpha, x = _rand_problem((n,) * 3, seed=n)
    ia, _, _, _ = O.prepare_interaction_matrices(alpha, k, d)
    op = P.DDAOperator(ia, k, d, dtype=dtype)
    assert tuple(op.L) == (2 * n,) * 3
    monkeypatch.delenv("DDA_NO_CUBE", raising=False)
    cube = op.matvec(x).cpu().numpy()
    monkeypatch.setenv("DDA_NO_CUBE", "1")
    general = op.matvec(x).cpu().numpy()
    assert np.isfinite(cube).all()
    assert _rel(cube, general) < tol


@pytest.mark.parametrize("dtype", [C64, C128])
@pytest.mark.parametrize("n,nb", [(64, 1), (64, 3), (128, 1), (128, 2)])
def test_staged_x_pass_equals_one_tile_kernel(n, nb, dtype, monkeypatch):
    """The staged persistent x pass (bulk-copied input tiles, one tile
    ahead) does the arithmetic of the one-tile-per-CTA kernel: equal to
    rounding (the compiler may contract a complex product's multiply-add
    differently in the two kernels), alone and in batched launches (several
    instances per launch), in the interaction and preconditioner
    products."""
    P = _pkg()
    ops, xs = [], []
    for j in range(nb):
        k, d, alpha, x = _rand_problem((n,) * 3, seed=n + j, fill=0.5)
        ia, _, _, _ = O.prepare_interaction_matrices(alpha, k, d)
        ops.append(P.DDAOperator(ia, k, d, dtype=dtype))
        xs.append(torch.as_tensor(x, device="cuda").to(dtype))
    monkeypatch.setenv("DDA_P3PIPE", "1")
    a = P.engine.matvec_batch(ops, xs) if nb > 1 else [ops[0].matvec(xs[0])]
    monkeypatch.delenv("DDA_P3PIPE", raising=False)
    b = P.engine.matvec_batch(ops, xs) if nb > 1 else [ops[0].matvec(xs[0])]
    tol = 2e-6 if dtype == C64 else 1e-13
    for u, v in zip(a, b):
        assert _rel(u.cpu().numpy(), v.cpu().numpy()) < tol
    if nb == 1 and n == 64:
        pre = ops[0].preconditioner()
        monkeypatch.setenv("DDA_P3PIPE", "1")
        pa = pre.apply(xs[0], dtype)
        monkeypatch.delenv("DDA_P3PIPE", raising=False)
        pb = pre.apply(xs[0], dtype)
        assert _rel(pa.cpu().numpy(), pb.cpu().numpy()) < tol


@pytest.mark.parametrize("n,nb", [(64, 1), (64, 3), (128, 1), (128, 2)])
def test_pair_x_pass_matches_one_tile_kernel(n, nb, monkeypatch):
    """The packed-pair x, y and z passes (two transforms per thread in
    FP32x2 lanes) against the one-component kernels and the oracle:
    complex64 rounding only, alone and batched, in the interaction and
    preconditioner products (a single-instance 64^3 matvec uses the
    cluster-fused z/y kernels, so there only the x pass changes; the
    preconditioner check turns them off)."""
    P = _pkg()
    ops, xs, xn = [], [], []
    for j in range(nb):
        k, d, alpha, x = _rand_problem((n,) * 3, seed=2 * n + j, fill=0.5)
        ia, _, _, _ = O.prepare_interaction_matrices(alpha, k, d)
        ops.append(P.DDAOperator(ia, k, d, dtype=C64))
        xs.append(torch.as_tensor(x, device="cuda").to(C64))
        xn.append((ia, k, d, x))
    monkeypatch.setenv("DDA_P3PAIR", "1")
    monkeypatch.setenv("DDA_YPAIR", "1")
    monkeypatch.setenv("DDA_ZPAIR", "1")
    a = P.engine.matvec_batch(ops, xs) if nb > 1 else [ops[0].matvec(xs[0])]
    monkeypatch.delenv("DDA_P3PAIR", raising=False)
    c = P.engine.matvec_batch(ops, xs) if nb > 1 else [ops[0].matvec(xs[0])]     # y and z pairs alone
    monkeypatch.delenv("DDA_YPAIR", raising=False)
    monkeypatch.delenv("DDA_ZPAIR", raising=False)
    b = P.engine.matvec_batch(ops, xs) if nb > 1 else [ops[0].matvec(xs[0])]
    for u, w, v in zip(a, c, b):
        assert _rel(u.cpu().numpy(), v.cpu().numpy()) < 2e-6
        assert _rel(w.cpu().numpy(), v.cpu().numpy()) < 2e-6
    if n == 64:
        ia, k, d, x = xn[0]
        mask = ia != 0
        ref = O.interaction_mult(x, O.generate_interaction_row(n, n, n, k, d), ia, mask)
        assert _rel(a[0].cpu().numpy(), ref) < 2e-5
        if nb == 1:
            pre = ops[0].preconditioner()
            monkeypatch.setenv("DDA_P3PAIR", "1")
            monkeypatch.setenv("DDA_YPAIR", "1")
            monkeypatch.setenv("DDA_ZPAIR", "1")
            monkeypatch.setenv("DDA_NO_FUSED_ZY", "1")
            pa = pre.apply(xs[0], C64)
            for v in ("DDA_P3PAIR", "DDA_YPAIR", "DDA_ZPAIR"):
                monkeypatch.delenv(v, raising=False)
            pb = pre.apply(xs[0], C64)
            monkeypatch.delenv("DDA_NO_FUSED_ZY", raising=False)
            assert _rel(pa.cpu().numpy(), pb.cpu().numpy()) < 2e-6


@pytest.mark.parametrize("dtype", [C64, C128])
@pytest.mark.parametrize("n,nb", [(64, 2), (128, 1)])
def test_prefetch_changes_no_result(n, nb, dtype, monkeypatch):
    """The L2 prefetch of the x and y passes' input (DDA_PREFETCH=1) adds
    prefetch instructions to the same kernels: results equal bit for bit."""
    P = _pkg()
    ops, xs = [], []
    for j in range(nb):
        k, d, alpha, x = _rand_problem((n,) * 3, seed=3 * n + j, fill=0.5)
        ia, _, _, _ = O.prepare_interaction_matrices(alpha, k, d)
        ops.append(P.DDAOperator(ia, k, d, dtype=dtype))
        xs.append(torch.as_tensor(x, device="cuda").to(dtype))
    mv = lambda: P.engine.matvec_batch(ops, xs) if nb > 1 else [ops[0].matvec(xs[0])]
    monkeypatch.setenv("DDA_PREFETCH", "1")
    a = mv()
    monkeypatch.delenv("DDA_PREFETCH", raising=False)
    b = mv()
    for u, v in zip(a, b):
        assert torch.equal(u, v)


def test_matvec_dense_tiny():
    P = _pkg()
    k, d, alpha, x = _rand_problem((4, 4, 4), seed=3)
    ia, mask, _, _ = O.prepare_interaction_matrices(alpha, k, d)
    op = P.DDAOperator(ia, k, d, dtype=C128)
    dense = O.dense_interaction_mult(x, ia, k, d, mask)
    assert _rel(op.matvec(x).cpu().numpy(), dense) < 1e-12


def _sphere_problem(n, m, kd=0.5, wavelength=0.5, pol=(1, 0, 0), kdir=(0, 0, 1)):
    k = 2 * np.pi / wavelength
    d = kd / (abs(m) * k)
    occ = O.sphere_lattice(n, n / 2.0)
    a = O.calculate_alpha(m, d, k, method="RR")
    alpha = np.where(occ, a, 0).astype(np.complex128)
    E = O.incident_field((n, n, n), d, k, kdir, pol)
    return k, d, alpha, E


@pytest.mark.parametrize("n,m", [(8, 1.5 + 0.01j), (12, 1.7 + 0.1j)])
def test_solver_c128_matches_oracle(n, m):
    P = _pkg()
    k, d, alpha, E = _sphere_problem(n, m)
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    it_ref, P_ref, low_ref, first_ref = O.solve_gpbicgstab((n, n, n), ia, G, E, mask, 100, 500, target=1e-6)
    op = P.DDAOperator(ia, k, d, dtype=C128, L_=(2 * n,) * 3)
    Pg, info = op.solve(E, tol=1e-6, max_iter=500, ratio=100)
    assert info.iters == it_ref > 0
    assert _rel(Pg.cpu().numpy(), P_ref) < 1e-8
    assert abs(info.lowest_rel - low_ref) <= 1e-8 * max(low_ref, 1e-12) + 1e-14
    assert abs(info.first_rel - first_ref) <= 1e-9
    rr = O.true_relative_residual(Pg.cpu().numpy(), E, G, ia, mask)
    assert rr < 5e-6


def test_solver_c64_close_to_oracle():
    P = _pkg()
    n, m = 12, 1.5 + 0.01j
    k, d, alpha, E = _sphere_problem(n, m)
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    _, P_ref, _, _ = O.solve_gpbicgstab((n, n, n), ia, G, E, mask, 100, 500, target=1e-8)
    op = P.DDAOperator(ia, k, d, dtype=C64)
    Pg, info = op.solve(E, tol=1e-5, max_iter=500, ratio=100)
    assert info.status == "converged"
    err = np.linalg.norm(Pg.cpu().numpy() - P_ref) / np.linalg.norm(P_ref)
    assert err < 1e-4


def test_mixed_precision_reaches_fp64_tolerance():
    P = _pkg()
    n, m = 12, 1.7 + 0.1j
    k, d, alpha, E = _sphere_problem(n, m)
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    _, P_ref, _, _ = O.solve_gpbicgstab((n, n, n), ia, G, E, mask, 100, 1000, target=1e-10)
    op = P.DDAOperator(ia, k, d, dtype=C128)
    Pg, info = op.solve(E, tol=1e-6, max_iter=500, ratio=100, precision="mixed", inner_tol=1e-4)
    assert info.status == "converged", info
    assert info.true_relres <= 1e-6
    Pn = Pg.cpu().numpy()
    assert O.true_relative_residual(Pn, E, G, ia, mask) <= 1.05e-6
    assert np.linalg.norm(Pn - P_ref) / np.linalg.norm(P_ref) < 1e-5
    ce, ca, cs = O.cross_sections(P_ref, E, ia, k)
    ge, ga, gs = op.cross_sections(Pg, E)
    assert abs(ge - ce) / abs(ce) < 1e-5 and abs(ga - ca) / abs(ca) < 1e-5


def test_cross_sections_match_oracle():
    P = _pkg()
    rng = np.random.default_rng(5)
    shape = (6, 7, 8)
    ia = np.where(rng.random(shape) < 0.6, rng.standard_normal(shape) + 1j * rng.standard_normal(shape), 0)
    Pv = rng.standard_normal(shape + (3,)) + 1j * rng.standard_normal(shape + (3,))
    E = rng.standard_normal(shape + (3,)) + 1j * rng.standard_normal(shape + (3,))
    k = 3.7
    ref = O.cross_sections(Pv, E, ia, k, E0=1.3)
    got = P.cross_sections(torch.tensor(Pv, device="cuda"), E, ia, k, E0=1.3)
    for a, b in zip(got, ref):
        assert abs(a - b) <= 1e-11 * max(abs(b), 1.0)


def test_batch_matches_single():
    P = _pkg()
    n, m = 10, 1.5 + 0.05j
    k, d, alpha, _ = _sphere_problem(n, m)
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    op = P.DDAOperator(ia, k, d, dtype=C128)
    dirs = [((0, 0, 1), (1, 0, 0)), ((0, 0, 1), (0, 1, 0)), ((1, 0, 0), (0, 0, 1)), ((0, 1, 0), (1, 0, 0))]
    Es = [O.incident_field((n, n, n), d, k, kd_, pol) for kd_, pol in dirs]
    Pb, infos = P.solve_many([op] * len(Es), Es, tol=1e-6, max_iter=400, ratio=100)
    for E, Pj, inf in zip(Es, Pb, infos):
        Ps, inf1 = op.solve(E, tol=1e-6, max_iter=400, ratio=100)
        assert inf.iters == inf1.iters
        assert _rel(Pj.cpu().numpy(), Ps.cpu().numpy()) < 1e-9


def test_reference_api_solve_and_near_field():
    P = _pkg()
    n, m = 8, 1.5 + 0.01j
    k, d, alpha, E = _sphere_problem(n, m)
    ia, mask, G, _ = P.prepare_interaction_matrices((n, n, n), k, None, 0, 0, 0, alpha, d, double_precision=True)
    iters, Pg, low, first = P.solve_gpbicgstab((n, n, n), ia, G, None, E, mask, 100, 300, target=1e-6,
                                               precon=False, dtype=C128)
    ia_o, mask_o, G_o, _ = O.prepare_interaction_matrices(alpha, k, d)
    assert np.abs(G.cpu().numpy() - G_o).max() / np.abs(G_o).max() < 1e-12
    it_ref, P_ref, _, _ = O.solve_gpbicgstab((n, n, n), ia_o, G_o, E, mask_o, 100, 300, target=1e-6)
    assert iters == it_ref
    assert _rel(Pg.cpu().numpy(), P_ref) < 1e-8
    Ef = P.E_field_solver(Pg, G, (n, n, n), dtype=C128).cpu().numpy()
    assert _rel(Ef, O.E_field_solver(P_ref, G_o, (n, n, n))) < 1e-8
    with pytest.raises(ValueError):
        P.E_field_solver(Pg.reshape(-1)[:-3], G, (n, n, n))
    with pytest.raises(ValueError):          # precon=True needs a preconditioner
        P.solve_gpbicgstab((n, n, n), ia, G, None, E, mask, 100, 10, precon=True)


def test_device_voxelizer_matches_host_membership():
    from precondda_b200.lattice import (Sphere, Ellipsoid, Rectangle, Cylinder, Prism, shape_membership,
                                        voxelize_device, euler_rotation)
    d = 0.05
    box = (30, 26, 22)
    R = euler_rotation(0.4, 1.0, -0.3)
    shapes = [Rectangle("r", (0.7, 0.6, 0.5), (0.6, 0.5, 0.4), 1.5),
              Ellipsoid("e", (0.75, 0.65, 0.55), (0.5, 0.35, 0.25), 1.7, rotation=R),
              Cylinder("c", (0.5, 0.7, 0.5), 0.2, 0.5, "y", 1.4),
              Cylinder("g", (0.6, 0.5, 0.6), 0.15, 0.45, "x", 1.45, geometric=True),
              Prism("p", (1.0, 0.6, 0.6), 0.2, 6, 0.4, 1.3, axis="x"),
              Sphere("s", (0.4, 0.4, 0.4), 0.23, 1.6)]
    vals = [1.0 + 0.5j, 2.0 - 1.0j, 3.0 + 0.25j, 3.5 + 1j, 4.0, 5.0 - 0.125j]
    # whole-box membership (no mark_shapes window)
    got = voxelize_device(shapes, vals, box, d, window=False).cpu().numpy()
    pts = O.voxel_centres(box, d).reshape(-1, 3)
    ref = np.zeros(box, np.complex128).reshape(-1)
    for s, v in zip(shapes, vals):
        ref[shape_membership(s, pts)] = v
    assert np.array_equal(got.reshape(-1), ref)


def test_device_incident_field_matches_host():
    from precondda_b200.lattice import incident_field_device
    k = 2 * np.pi / 0.6
    kdir = np.array([0.3, -0.5, 0.8]); kdir /= np.linalg.norm(kdir)
    pol = np.array([1.0, 0.2 + 0.1j, 0.0])
    got = incident_field_device((9, 7, 5), 0.03, k * kdir, pol).cpu().numpy()
    ref = O.incident_field((9, 7, 5), 0.03, k, kdir, pol)
    assert np.abs(got - ref).max() < 1e-13


@pytest.mark.parametrize("n", [11, 20])
def test_fused_krylov_steps_match_oracle(n, monkeypatch):
    """alpha, s/y and zeta/eta carried by the matvec passes (DDA_FUSE_KRYLOV=1)
    follow the reference's recurrence like the separate kernels do."""
    P = _pkg()
    monkeypatch.setenv("DDA_FUSE_KRYLOV", "1")
    k, d, alpha, E = _sphere_problem(n, 1.6 + 0.05j)
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    it_ref, P_ref, low_ref, _ = O.solve_gpbicgstab((n, n, n), ia, G, E, mask, 100, 500, target=1e-6)
    op = P.DDAOperator(ia, k, d, dtype=C128, L_=(2 * n,) * 3 if n == 20 else None)
    Pg, info = op.solve(E, tol=1e-6, max_iter=500, ratio=100)
    assert info.iters == it_ref
    assert _rel(Pg.cpu().numpy(), P_ref) < 1e-8
    Pm, im = op.solve(E, tol=1e-6, max_iter=500, ratio=100, precision="mixed")
    assert im.status == "converged" and im.true_relres <= 1e-6
    # preconditioned: s and y formed by M's first pass
    op._ctx.trim()
    pre = op.preconditioner()
    it_p, P_p, _, _ = O.solve_gpbicgstab((n, n, n), ia, G, E, mask, 100, 500, target=1e-6,
                                         preconditioner=pre.reference_octant(C128).cpu().numpy())
    Pq, iq = op.solve(E, tol=1e-6, max_iter=500, ratio=100, preconditioner=pre)
    assert iq.iters == it_p and _rel(Pq.cpu().numpy(), P_p) < 1e-8


@pytest.mark.parametrize("dtype,tol", [(C128, 1e-11), (C64, 2e-5)])
def test_far_field_matches_oracle(dtype, tol):
    P = _pkg()
    rng = np.random.default_rng(11)
    shape = (5, 7, 6)
    Pv = rng.standard_normal(shape + (3,)) + 1j * rng.standard_normal(shape + (3,))
    dirs = rng.standard_normal((17, 3))
    k, d = 9.0, 0.07
    ref = O.far_field(Pv, d, k, dirs)
    got = P.far_field(torch.tensor(Pv, device="cuda").to(dtype), d, k, dirs)
    assert np.abs(got - ref).max() / np.abs(ref).max() < tol


def test_far_field_optical_theorem_and_energy():
    """F at the incidence direction gives C_ext (optical theorem), and the
    integral of |F|^2 over the sphere equals C_ext - C_abs (energy balance of
    the dipole system with the radiative-reaction polarizability)."""
    P = _pkg()
    n, m = 10, 1.5 + 0.02j
    k, d, alpha, E = _sphere_problem(n, m)
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    op = P.DDAOperator(ia, k, d, dtype=C128)
    Pg, info = op.solve(E, tol=1e-11, max_iter=800, ratio=100)
    ce, ca, cs = op.cross_sections(Pg, E)
    E0 = np.array([1.0, 0.0, 0.0])
    Ff = P.far_field(Pg, d, k, [[0.0, 0.0, 1.0]])[0]
    c_ext_ot = 4 * np.pi / k * np.imag(np.conj(E0) @ Ff)
    assert abs(c_ext_ot - ce) / abs(ce) < 1e-10
    # Gauss-Legendre in cos(theta) x uniform phi
    xg, wg = np.polynomial.legendre.leggauss(24)
    nphi = 48
    phi = 2 * np.pi * np.arange(nphi) / nphi
    ct = np.repeat(xg, nphi)
    st = np.sqrt(1 - ct ** 2)
    ph = np.tile(phi, len(xg))
    dirs = np.stack([st * np.cos(ph), st * np.sin(ph), ct], -1)
    w = np.repeat(wg, nphi) * (2 * np.pi / nphi)
    dcs = P.differential_cross_section(Pg, d, k, dirs)
    c_sca_int = float((dcs * w).sum())
    assert abs(c_sca_int - cs) / cs < 1e-6


def test_matvec_batch_equals_single_launches():
    P = _pkg()
    from precondda_b200 import _lib as L
    shape = (12, 12, 12)
    ops, xs = [], []
    for seed in (1, 2, 3):
        k, d, alpha, x = _rand_problem(shape, seed=seed)
        ia, _, _, _ = O.prepare_interaction_matrices(alpha, k / (1 + 0 * seed), d)
        ops.append(P.DDAOperator(ia, k, d, dtype=C64, L_=(24, 24, 24)))
        xs.append(x)
    ys = P.engine.matvec_batch(ops, xs)
    for op, x, y in zip(ops, xs, ys):
        assert torch.equal(y, op.matvec(x))
    bs = [x[::-1].copy() for x in xs]
    rs = P.engine.matvec_batch(ops, xs, L.MV_RESIDUAL, bs)
    for op, x, b, r in zip(ops, xs, bs, rs):
        assert torch.equal(r, op._mv(L.MV_RESIDUAL, x, b))


def test_cluster_fused_zy_passes_equal_separate(monkeypatch):
    """At 64^3 in complex64 the matvec runs passes 1+2 and 4+5 as
    thread-block-cluster kernels (the z/y intermediate stays in distributed
    shared memory).  They give the separate passes' results bit for bit --
    dense vectors in every combine mode, occupied-site vectors inside c64 and
    mixed solves -- and the product matches the oracle."""
    P = _pkg()
    from precondda_b200 import _lib as L
    shape = (64, 64, 64)
    k, d, alpha, x = _rand_problem(shape, seed=11)
    ia = np.where(alpha != 0, 1.0 / np.where(alpha != 0, alpha, 1), 0)
    op = P.DDAOperator(ia, k, d, dtype=C64)
    assert tuple(op.L) == (128, 128, 128)
    b = x[::-1].copy()
    modes = [(L.MV_AX, None), (L.MV_RESIDUAL, b), (L.MV_CONV, None), (L.MV_CONV_MASKED, None)]
    k2, d2, alpha2, E = _sphere_problem(64, 1.7 + 0.1j)
    ia2 = np.where(alpha2 != 0, 1.0 / np.where(alpha2 != 0, alpha2, 1), 0)
    op2 = P.DDAOperator(ia2, k2, d2, dtype=C128)

    def run():
        op._ctx.trim()                      # cached iteration graphs hold the kernels of their capture
        mv = [op._mv(m, x, bb).clone() for m, bb in modes]
        Pc, ic = op2.solve(E, tol=1e-4, max_iter=400, precision="c64")
        Pm, im = op2.solve(E, tol=1e-6, max_iter=400, precision="mixed")
        return mv, (Pc.clone(), ic), (Pm.clone(), im)

    fused = run()
    for env in ("DDA_NO_FUSED_INV", "DDA_NO_FUSED_ZY"):
        monkeypatch.setenv(env, "1")
        other = run()
        for f, s in zip(fused[0], other[0]):
            assert torch.equal(f, s)
        for (Pf, inf), (Ps, ins) in zip(fused[1:], other[1:]):
            assert inf.iters == ins.iters and inf.outer == ins.outer
            assert torch.equal(Pf, Ps)
    assert fused[2][1].status == "converged" and fused[2][1].true_relres <= 1e-6
    mask = ia != 0
    Gref = O.generate_interaction_row(*shape, k, d, L=op.L)
    ref = O.interaction_mult(x, Gref, ia, mask, L=op.L)
    assert _rel(fused[0][0].cpu().numpy(), ref) < 2e-5


@pytest.mark.parametrize("nb", [1, 2])
def test_fused_zy_passes_128_match_separate(nb, monkeypatch):
    """The 128^3 cluster-fused z/y kernels (clusters of eight, one CTA per
    SM, T1 kept on chip; for launches of any width, where the tuning table
    selects them) against the separate passes in every product mode, and
    the first mode against the oracle."""
    P = _pkg()
    from precondda_b200 import _lib as L
    shape = (128, 128, 128)
    ops, xs = [], []
    for j in range(nb):
        k, d, alpha, x = _rand_problem(shape, seed=128 + j, fill=0.4)
        ia = np.where(alpha != 0, 1.0 / np.where(alpha != 0, alpha, 1), 0)
        ops.append(P.DDAOperator(ia, k, d, dtype=C64))
        xs.append(torch.as_tensor(x, device="cuda").to(C64))
    assert tuple(ops[0].L) == (256, 256, 256)
    bs = [x.flip(0).contiguous() for x in xs]

    def run():
        out = []
        for m in (L.MV_AX, L.MV_RESIDUAL, L.MV_CONV, L.MV_CONV_MASKED):
            b = bs if m == L.MV_RESIDUAL else None
            out.append(P.engine.matvec_batch(ops, xs, mode=m, bs=b) if nb > 1 else
                       [ops[0]._mv(m, xs[0], b[0] if b else None)])
        return out

    sep = run()
    from precondda_b200 import _lib as LL
    code = LL.DDA_C64
    for nbk in (1, nb):
        LL.check(LL.lib().dda_tuning_set(code, *shape, 256, 256, 256, nbk, LL.DDA_TUNE_FUSED))
    try:
        fused = run()
    finally:
        for nbk in (1, nb):
            LL.lib().dda_tuning_set(code, *shape, 256, 256, 256, nbk, -1)
    for fm, sm in zip(fused, sep):
        for f, s in zip(fm, sm):
            assert _rel(f.cpu().numpy(), s.cpu().numpy()) < 2e-6
    if nb == 1:
        k, d, alpha, x = _rand_problem(shape, seed=128, fill=0.4)
        ia = np.where(alpha != 0, 1.0 / np.where(alpha != 0, alpha, 1), 0)
        ref = O.interaction_mult(x, O.generate_interaction_row(*shape, k, d), ia, ia != 0)
        assert _rel(fused[0][0].cpu().numpy(), ref) < 2e-5
