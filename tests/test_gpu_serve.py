"""Continuous batching (slot pools and the request server) on the GPU: each
request's result equals the oracle's / a lone solve's, and is the same bit
for bit whether it runs alone or mixed with other requests."""
import numpy as np
import pytest
import torch

from oracle import dda_oracle as O

pytestmark = pytest.mark.gpu

C64, C128 = torch.complex64, torch.complex128


def _sphere(n, m, radius=None, kd=0.5, wavelength=0.5, kdir=(0, 0, 1), pol=(1, 0, 0), box=None):
    k = 2 * np.pi / wavelength
    d = kd / (abs(m) * k)
    box = box or (n, n, n)
    occ = O.sphere_lattice(n, (radius or n / 2.0))
    a = O.calculate_alpha(m, d, k, method="RR")
    alpha = np.zeros(box, np.complex128)
    alpha[:n, :n, :n] = np.where(occ, a, 0)
    E = O.incident_field(box, d, k, kdir, pol)
    return k, d, alpha, E


def _run_pool(pool, limit=400):
    out = {}
    for _ in range(limit):
        pool.run(4)
        for s, info, P in pool.poll():
            out[s] = (info, P)
        if pool.running == 0:
            return out
    raise AssertionError("pool did not finish")


def test_slot_pool_c128_matches_oracle():
    import precondda_b200 as P
    from precondda_b200.serve import SlotPool
    n, m = 8, 1.5 + 0.01j
    k, d, alpha, E = _sphere(n, m)
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    it_ref, P_ref, low_ref, first_ref = O.solve_gpbicgstab((n, n, n), ia, G, E, mask, 100, 500, target=1e-6)
    L = (2 * n,) * 3
    ghat = P.green_octant((n, n, n), k, d, L, 1.0 / (L[0] * L[1] * L[2]), C128, layout="engine")
    pool = SlotPool((n, n, n), L, 3, "c128")
    Pd = pool.admit(1, ghat, torch.tensor(ia, device="cuda"), torch.tensor(E, device="cuda"), tol=1e-6,
                    max_iter=500)
    res = _run_pool(pool)
    assert list(res) == [1]
    info, Pout = res[1]
    assert Pout.data_ptr() == Pd.data_ptr()
    assert info.status == "converged" and info.iters == it_ref
    assert np.abs(Pout.cpu().numpy() - P_ref).max() / np.abs(P_ref).max() < 1e-8
    assert abs(info.lowest_rel - low_ref) <= 1e-8 * max(low_ref, 1e-12) + 1e-14
    assert abs(info.first_rel - first_ref) <= 1e-9
    pool.close()


def test_slot_pool_ready_reports_idle_stream():
    """dda_slots_ready: idle after the stream drains, and a pool that was
    reported ready polls without waiting (the result is the same as a
    blocking poll's)."""
    import precondda_b200 as P
    from precondda_b200.serve import SlotPool
    n = 8
    k, d, alpha, E = _sphere(n, 1.5 + 0.01j)
    ia, mask, G, _ = O.prepare_interaction_matrices(alpha, k, d)
    L = (2 * n,) * 3
    ghat = P.green_octant((n, n, n), k, d, L, 1.0 / (L[0] * L[1] * L[2]), C128, layout="engine")
    pool = SlotPool((n, n, n), L, 2, "c128")
    assert pool.ready()
    pool.admit(0, ghat, torch.tensor(ia, device="cuda"), torch.tensor(E, device="cuda"), tol=1e-6, max_iter=500)
    done = {}
    for _ in range(500):
        pool.run(4)
        torch.cuda.synchronize()
        assert pool.ready()
        for s, info, Pout in pool.poll():
            done[s] = info
        if pool.running == 0:
            break
    assert done[0].status == "converged"
    assert pool.ready()
    pool.close()


def _requests(P, specs):
    reqs = []
    for (n, m, kdir, pol, tol) in specs:
        k, d, alpha, E = _sphere(n, m, kdir=kdir, pol=pol)
        ia = np.where(alpha != 0, 1.0 / np.where(alpha != 0, alpha, 1), 0)
        reqs.append(P.serve.Request(inv_alpha=ia, E_inc=E, k=k, d=d, tol=tol, max_iter=600))
    return reqs


SPECS = [
    (12, 1.7 + 0.1j, (0, 0, 1), (1, 0, 0), 1e-6),     # the request followed alone and in the mix
    (10, 1.5 + 0.01j, (0, 0, 1), (0, 1, 0), 1e-6),
    (16, 1.33 + 0.0j, (1, 0, 0), (0, 0, 1), 1e-7),
    (14, 2.0 + 0.3j, (0, 1, 0), (1, 0, 0), 1e-5),
    (9, 1.6 + 0.02j, (0, 0, 1), (1, 0, 0), 1e-6),
    (16, 1.5 + 0.1j, (0, 0, 1), (0, 1, 0), 1e-6),
]


@pytest.mark.parametrize("precision", ["mixed", "c128", "c64"])
def test_result_same_alone_and_in_the_mix(precision):
    import precondda_b200 as P
    from precondda_b200.serve import DDAServer
    cfg = dict(precision=precision, buckets=(16,), slots_per_bucket=3, chunk_iters=3)
    srv = DDAServer(**cfg)
    alone = srv.submit(_requests(P, SPECS[:1])[0])
    srv.drain()
    P_alone, info_alone = alone.P.cpu().numpy().copy(), alone.info
    srv.close()

    srv = DDAServer(**cfg)
    reqs = _requests(P, SPECS)
    first = [srv.submit(r) for r in reqs[1:3]]
    srv.step()
    srv.step()                               # the target enters while others are mid-solve
    tgt = srv.submit(reqs[0])
    for r in reqs[3:]:
        srv.submit(r)                        # more requests than slots: some wait in the queue
    srv.drain()
    assert all(r.info is not None for r in reqs)
    assert tgt.info.iters == info_alone.iters and tgt.info.outer == info_alone.outer
    assert tgt.info.status == info_alone.status
    if precision != "c64":
        assert tgt.info.status == "converged"
    assert np.array_equal(tgt.P.cpu().numpy(), P_alone)
    st = srv.stats()
    assert st["n"] == len(reqs) and st["p99_ms"] >= st["p50_ms"] > 0
    assert st["green_misses"] == len({(r.k, r.d) for r in reqs})
    srv.close()
    del first


def test_release_frees_slot_for_a_clean_restart():
    import precondda_b200 as P
    from precondda_b200.serve import SlotPool
    n = 10
    L = P.fft_lengths((n, n, n), C64)
    reqs = []
    for m in (1.5 + 0.01j, 1.8 + 0.2j):
        k, d, alpha, E = _sphere(n, m)
        ia, _, _, _ = O.prepare_interaction_matrices(alpha, k, d)
        g = P.green_octant((n, n, n), k, d, L, 1.0 / (L[0] * L[1] * L[2]), C64, layout="engine")
        reqs.append((g, torch.tensor(ia, device="cuda"), torch.tensor(E, device="cuda")))
    fresh = SlotPool((n, n, n), L, 2, "c64")
    fresh.admit(0, *reqs[1], tol=1e-5, max_iter=400)
    ref = _run_pool(fresh)[0]
    fresh.close()
    pool = SlotPool((n, n, n), L, 2, "c64")
    pool.admit(0, *reqs[0], tol=1e-5, max_iter=400)
    pool.run(3)
    pool.release(0)                         # cancelled mid-solve
    assert pool.free_slot() == 0
    pool.admit(0, *reqs[1], tol=1e-5, max_iter=400)
    got = _run_pool(pool)[0]
    assert got[0].iters == ref[0].iters
    assert np.array_equal(got[1].cpu().numpy(), ref[1].cpu().numpy())
    pool.close()


def test_padded_request_solves_its_own_lattice():
    import precondda_b200 as P
    from precondda_b200.serve import DDAServer
    k = 2 * np.pi / 0.5
    d = 0.5 / (1.6 * k)
    rng = np.random.default_rng(3)
    shape = (10, 12, 14)
    a = O.calculate_alpha(1.6 + 0.05j, d, k, method="RR")
    occ = rng.random(shape) < 0.6
    ia = np.where(occ, 1.0 / a, 0).astype(np.complex128)
    E = O.incident_field(shape, d, k, (0, 0, 1), (1, 0, 0))
    srv = DDAServer(precision="mixed", buckets=(16, 32), slots_per_bucket=2)
    r = srv.submit(P.serve.Request(inv_alpha=ia, E_inc=E, k=k, d=d, tol=1e-7))
    srv.drain()
    assert r.bucket == 16 and r.P.shape == shape + (3,)
    assert r.info.status == "converged" and r.info.true_relres <= 1e-7
    op = P.DDAOperator(ia, k, d, dtype=C128)
    res = op.residual(E, r.P.contiguous()).cpu().numpy()
    b = E * (ia != 0)[..., None]
    assert np.linalg.norm(res) / np.linalg.norm(b) < 2e-7
    srv.close()


def test_mixed_pool_matches_batched_mixed_solve():
    import precondda_b200 as P
    from precondda_b200.serve import DDAServer
    n, m = 12, 1.7 + 0.1j
    k, d, alpha, E = _sphere(n, m)
    ia, _, _, _ = O.prepare_interaction_matrices(alpha, k, d)
    op = P.DDAOperator(ia, k, d, dtype=C128)
    Pb, info_b = op.solve(E, tol=1e-6, max_iter=500, precision="mixed")
    srv = DDAServer(precision="mixed", buckets=(12,), slots_per_bucket=2, chunk_iters=5)
    r = srv.submit(P.serve.Request(inv_alpha=ia, E_inc=E, k=k, d=d, tol=1e-6, max_iter=500))
    srv.drain()
    assert r.info.status == "converged" and r.info.true_relres <= 1e-6
    assert r.info.outer == info_b.outer
    assert abs(r.info.iters - info_b.iters) <= 2
    Pn = r.P.cpu().numpy()
    assert np.linalg.norm(Pn - Pb.cpu().numpy()) / np.linalg.norm(Pn) < 1e-5
    srv.close()


def test_slot_pool_argument_errors():
    import precondda_b200 as P
    from precondda_b200.serve import SlotPool
    from precondda_b200._lib import DDAError
    n = 8
    k, d, alpha, E = _sphere(n, 1.5 + 0.01j)
    ia, _, _, _ = O.prepare_interaction_matrices(alpha, k, d)
    L = (16, 16, 16)
    g = P.green_octant((n, n, n), k, d, L, 1.0 / 4096, C128, layout="engine")
    pool = SlotPool((n, n, n), L, 2, "c128")
    assert pool.poll() == [] and pool.running == 0
    pool.admit(0, g, torch.tensor(ia, device="cuda"), torch.tensor(E, device="cuda"), tol=1e-6)
    with pytest.raises(DDAError):
        pool.admit(0, g, torch.tensor(ia, device="cuda"), torch.tensor(E, device="cuda"))   # occupied
    with pytest.raises(DDAError):
        pool.admit(5, g, torch.tensor(ia, device="cuda"), torch.tensor(E, device="cuda"))   # no such slot
    assert pool.free_slot() == 1
    res = _run_pool(pool)
    assert res[0][0].status == "converged"
    pool.close()
    with pytest.raises(Exception):
        SlotPool((n, n, n), (14, 16, 16), 1, "c128")       # FFT length < 2n


def test_preconditioned_pool_matches_batched_solve():
    """A preconditioned slot runs the same precon=True solve as the batched
    solver: same iterations and solution."""
    import precondda_b200 as P
    from precondda_b200.serve import SlotPool
    n, m = 12, 2.2 + 0.1j
    k, d, alpha, E = _sphere(n, m)
    ia, _, _, _ = O.prepare_interaction_matrices(alpha, k, d)
    op = P.DDAOperator(ia, k, d, dtype=C128)
    pre = op.preconditioner()
    Pb, ib = op.solve(E, tol=1e-7, max_iter=500, preconditioner=pre)
    pool = SlotPool((n, n, n), op.L, 2, "c128", precond_L=op.L)
    with pytest.raises(ValueError):
        pool.admit(0, op.ghat, op.inv_alpha, torch.tensor(E, device="cuda"), tol=1e-7)       # no preconditioner
    Pd = pool.admit(0, op.ghat, op.inv_alpha, torch.tensor(E, device="cuda"), tol=1e-7, max_iter=500,
                    preconditioner=pre)
    res = _run_pool(pool)
    info, Pout = res[0]
    assert Pout.data_ptr() == Pd.data_ptr()
    assert info.status == "converged" and info.iters == ib.iters
    assert np.abs((Pout - Pb).cpu().numpy()).max() / np.abs(Pb.cpu().numpy()).max() < 1e-10
    pool.close()
    plain = SlotPool((n, n, n), op.L, 1, "c128")
    with pytest.raises(ValueError):
        plain.admit(0, op.ghat, op.inv_alpha, torch.tensor(E, device="cuda"), preconditioner=pre)
    plain.close()


@pytest.mark.parametrize("precision", ["mixed", "c64"])
def test_preconditioned_server_same_alone_and_in_the_mix(precision):
    import precondda_b200 as P
    from precondda_b200.serve import DDAServer
    cfg = dict(precision=precision, buckets=(16,), slots_per_bucket=3, chunk_iters=3, precondition=True)
    srv = DDAServer(**cfg)
    alone = srv.submit(_requests(P, SPECS[:1])[0])
    srv.drain()
    P_alone, info_alone = alone.P.cpu().numpy().copy(), alone.info
    srv.close()
    srv = DDAServer(**cfg)
    reqs = _requests(P, SPECS)
    for r in reqs[1:3]:
        srv.submit(r)
    srv.step()
    tgt = srv.submit(reqs[0])
    for r in reqs[3:]:
        srv.submit(r)
    srv.drain()
    assert tgt.info.iters == info_alone.iters and np.array_equal(tgt.P.cpu().numpy(), P_alone)
    if precision == "mixed":
        assert all(r.info.status == "converged" and r.info.true_relres <= r.tol for r in reqs)
    srv.close()
    # fewer iterations than the unpreconditioned server on the same request
    srv = DDAServer(**dict(cfg, precondition=False))
    r0 = srv.submit(_requests(P, SPECS[:1])[0])
    srv.drain()
    assert info_alone.iters < r0.info.iters
    srv.close()
