"""Failure statuses on the GPU, made on the host (no device fault involved).

The reference's return codes (Gpbicgstab.py:1099-1115, :1162-1201): i+1
when converged, max_iter when the loop ran out, -(i+1) on NaN or stagnation.
Each case runs through the engine's solve, the reference API, a batched
solve next to healthy instances, a slot pool and the request server, and
is checked against the oracle's code for the same input.  The server's HBM
admission refuses a request its budget cannot hold before allocating, and
queues requests beyond its slots.
"""
import numpy as np
import pytest
import torch

from oracle import dda_oracle as O

pytestmark = pytest.mark.gpu

C64, C128 = torch.complex64, torch.complex128


def _sphere(n=8, m=1.5 + 0.01j, pol=(1, 0, 0)):
    k = 2 * np.pi / 0.5
    d = 0.5 / (abs(m) * k)
    occ = O.sphere_lattice(n, n / 2.0)
    alpha = np.where(occ, O.calculate_alpha(m, d, k, method="RR"), 0).astype(np.complex128)
    E = O.incident_field((n, n, n), d, k, (0, 0, 1), pol)
    ia = np.where(occ, 1.0 / np.where(occ, alpha, 1), 0)
    return k, d, alpha, ia, E


def _poisoned(E, ia, value):
    """E_inc with one occupied site's x component set to ``value``."""
    Eb = E.copy()
    site = tuple(np.argwhere(ia != 0)[len(np.argwhere(ia != 0)) // 2])
    Eb[site + (0,)] = value
    return Eb


@pytest.mark.parametrize("value", [np.nan, np.inf])
def test_nonfinite_incident_field_returns_reference_code(value):
    import precondda_b200 as P
    n = 8
    k, d, alpha, ia, E = _sphere(n)
    Eb = _poisoned(E, ia, value)
    mask = ia != 0
    G = O.generate_interaction_row(n, n, n, k, d)
    with np.errstate(all="ignore"):
        it_o, _, _, _ = O.solve_gpbicgstab((n,) * 3, ia, G, Eb, mask, 100, 200, target=1e-6)
    assert it_o < 0
    op = P.DDAOperator(ia, k, d, dtype=C128)
    for prec in ("c128", "c64"):
        opp = op if prec == "c128" else op.twin(C64)
        _, info = opp.solve(Eb, tol=1e-6, max_iter=200, ratio=100)
        assert info.iters == it_o and info.status == "nan_or_stagnation", (prec, info)
    _, info = P.DDAOperator(ia, k, d, dtype=C128, with_twin=True).solve(Eb, tol=1e-6, max_iter=200, ratio=100,
                                                                           precision="mixed")
    assert info.iters < 0 and info.status == "nan_or_stagnation", info
    # the reference API (complex128 form) returns the code itself
    Gr = P.generate_interaction_row(n, n, n, k, d, True, True)
    it, _, _, _ = P.solve_gpbicgstab((n,) * 3, ia, Gr, None, Eb, mask, 100, 200, target=1e-6, precon=False,
                                     dtype=C128)
    assert it == it_o


def test_max_iter_returns_max_iter_and_best_iterate():
    import precondda_b200 as P
    n = 8
    k, d, alpha, ia, E = _sphere(n, m=1.7 + 0.1j)
    mask = ia != 0
    G = O.generate_interaction_row(n, n, n, k, d)
    it_o, P_o, low_o, _ = O.solve_gpbicgstab((n,) * 3, ia, G, E, mask, 100, 3, target=1e-12)
    assert it_o == 3
    op = P.DDAOperator(ia, k, d, dtype=C128)
    Pg, info = op.solve(E, tol=1e-12, max_iter=3, ratio=100)
    assert info.iters == 3 and info.status == "max_iter"
    assert np.abs(Pg.cpu().numpy() - P_o).max() / np.abs(P_o).max() < 1e-8
    assert abs(info.lowest_rel - low_o) <= 1e-8 * low_o
    Gr = P.generate_interaction_row(n, n, n, k, d, True, True)
    it, _, _, _ = P.solve_gpbicgstab((n,) * 3, ia, Gr, None, E, mask, 100, 3, target=1e-12, precon=False,
                                     dtype=C128)
    assert it == 3


def test_batched_failures_leave_healthy_instances_alone():
    """One batch: a healthy solve, a NaN right-hand side and a healthy solve
    that runs out of iterations; each instance ends as it does alone."""
    import precondda_b200 as P
    n = 8
    k, d, alpha, ia, E = _sphere(n)
    Eb = _poisoned(E, ia, np.nan)
    op = P.DDAOperator(ia, k, d, dtype=C128)
    alone = op.solve(E, tol=1e-6, max_iter=200, ratio=100)
    Ps, infos = P.solve_many([op, op], [E, Eb], tol=1e-6, max_iter=200, ratio=100, precision="c128")
    assert infos[0].iters == alone[1].iters and infos[0].status == "converged"
    assert torch.equal(Ps[0], alone[0])
    assert infos[1].iters == -1 and infos[1].status == "nan_or_stagnation"
    _, inf3 = P.solve_many([op, op], [E, E], tol=1e-6, max_iter=2, ratio=100, precision="c128")
    assert all(i.iters == 2 and i.status == "max_iter" for i in inf3)


@pytest.mark.parametrize("precision", ["c128", "mixed"])
def test_slot_pool_reports_nan_request(precision):
    import precondda_b200 as P
    from precondda_b200.serve import SlotPool
    n = 8
    k, d, alpha, ia, E = _sphere(n)
    Eb = _poisoned(E, ia, np.nan)
    L = (2 * n,) * 3
    g128 = P.green_octant((n,) * 3, k, d, L, 1.0 / (L[0] * L[1] * L[2]), C128, layout="engine")
    g64 = P.green_octant((n,) * 3, k, d, L, 1.0 / (L[0] * L[1] * L[2]), C64, layout="engine")
    ghat = (g64, g128) if precision == "mixed" else g128
    pool = SlotPool((n,) * 3, L, 2, precision)
    ia_d = torch.tensor(ia, device="cuda")
    pool.admit(0, ghat, ia_d, torch.tensor(E, device="cuda"), tol=1e-6, max_iter=200)
    pool.admit(1, ghat, ia_d, torch.tensor(Eb, device="cuda"), tol=1e-6, max_iter=200)
    out = {}
    for _ in range(200):
        pool.run(4)
        for s, info, Pout in pool.poll():
            out[s] = info
        if pool.running == 0:
            break
    pool.close()
    assert out[0].status == "converged"
    assert out[1].status == "nan_or_stagnation" and out[1].iters < 0


def test_server_reports_statuses_and_refuses_over_budget():
    import precondda_b200 as P
    from precondda_b200.serve import DDAServer, Request
    n = 8
    k, d, alpha, ia, E = _sphere(n)
    Eb = _poisoned(E, ia, np.nan)
    srv = DDAServer(precision="c128", buckets=(8, 16), slots_per_bucket=4)
    reqs = [srv.submit(Request(ia, E, k, d, tol=1e-6, max_iter=200)),
            srv.submit(Request(ia, Eb, k, d, tol=1e-6, max_iter=200)),
            srv.submit(Request(ia, E, k, d, tol=1e-12, max_iter=3))]
    srv.drain(timeout_s=120)
    assert reqs[0].info.status == "converged"
    assert reqs[1].info.status == "nan_or_stagnation" and reqs[1].info.iters == -1
    assert reqs[2].info.status == "max_iter" and reqs[2].info.iters == 3
    srv.close()
    # a budget that holds no slot: the request is refused before any allocation
    torch.cuda.synchronize()
    before = torch.cuda.memory_allocated()
    tiny = DDAServer(precision="c128", buckets=(8,), slots_per_bucket=4, hbm_budget=1 << 10)
    with pytest.raises(MemoryError):
        tiny.submit(Request(ia, E, k, d, tol=1e-6))
    assert tiny.pending() == 0 and not tiny._b
    torch.cuda.synchronize()
    assert torch.cuda.memory_allocated() == before
    tiny.close()


def test_server_budget_of_one_slot_queues_the_rest():
    import precondda_b200 as P
    from precondda_b200.serve import DDAServer, Request, slot_bytes, request_bytes
    n = 8
    k, d, alpha, ia, E = _sphere(n)
    L = P.fft_lengths((n,) * 3)
    per = slot_bytes((n,) * 3, L, "c128") + request_bytes((n,) * 3, "c128")
    srv = DDAServer(precision="c128", buckets=(8,), slots_per_bucket=4, hbm_budget=per + per // 2)
    reqs = [srv.submit(Request(ia, E, k, d, tol=1e-6, max_iter=200)) for _ in range(3)]
    assert srv.stats()["n"] == 0 and srv._b[8].pool.nslots == 1
    srv.drain(timeout_s=120)
    assert all(r.info.status == "converged" for r in reqs)
    assert len({r.info.iters for r in reqs}) == 1
    srv.close()


def test_server_evicts_idle_bucket_for_a_new_one():
    """A budget that holds one bucket's pool: a request of another bucket
    closes the idle pool (its memory returns) instead of being refused; a
    bucket with work in flight is never closed."""
    import precondda_b200 as P
    from precondda_b200.serve import DDAServer, Request, slot_bytes, request_bytes
    k, d, alpha, ia8, E8 = _sphere(8)
    _, _, _, ia12, E12 = _sphere(12)
    per12 = slot_bytes((12,) * 3, P.fft_lengths((12,) * 3), "c128") + request_bytes((12,) * 3, "c128")
    srv = DDAServer(precision="c128", buckets=(8, 12), slots_per_bucket=1, hbm_budget=per12 + per12 // 4)
    r8 = srv.submit(Request(ia8, E8, k, d, tol=1e-6, max_iter=200))
    # bucket 8 holds a queued request: bucket 12 does not fit beside it
    with pytest.raises(MemoryError):
        srv.submit(Request(ia12, E12, k, d, tol=1e-6, max_iter=200))
    srv.drain(timeout_s=120)
    assert r8.info.status == "converged" and list(srv._b) == [8]
    r12 = srv.submit(Request(ia12, E12, k, d, tol=1e-6, max_iter=200))
    assert list(srv._b) == [12] and srv.hbm_used == srv._b[12].nbytes
    srv.drain(timeout_s=120)
    assert r12.info.status == "converged"
    # the 12^3 result matches a solve of its own
    alone = P.DDAOperator(ia12, k, d, dtype=C128).solve(E12, tol=1e-6, max_iter=200, ratio=100)
    assert r12.info.iters == alone[1].iters
    srv.close()
    assert srv.hbm_used == 0
