"""Many geometries of uneven size solved together (size buckets, padding
autotuner, concurrent slot pools): every right-hand side matches its own
solve on the unpadded lattice."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

C128 = torch.complex128


def test_solve_geometries_matches_single_solves():
    import precondda_b200 as P
    from precondda_b200.batch import Geometry, PaddingTuner, solve_geometries
    from precondda_b200.workloads import random_ellipsoid_spec, build_geometry
    rng = np.random.default_rng(7)
    specs = [random_ellipsoid_spec(rng, edge=(9, 20), n_dirs=1) for _ in range(4)]
    geoms = [Geometry(*build_geometry(sp)) for sp in specs]
    tuner = PaddingTuner("mixed", edges=(8, 12, 16, 20, 24))
    res = solve_geometries(geoms, tol=1e-6, precision="mixed", tuner=tuner, chunk=4)
    assert res.solves == sum(len(g.E_incs) for g in geoms) == 8
    for g, (box, L), Ps, infos in zip(geoms, res.plan, res.P, res.info):
        assert all(b >= n for b, n in zip(box, g.shape))
        op = P.DDAOperator(g.inv_alpha, g.k, g.d, dtype=C128)
        for E, Pb, info in zip(g.E_incs, Ps, infos):
            assert info.status == "converged" and info.true_relres <= 1e-6
            assert tuple(Pb.shape) == g.shape + (3,)
            r = op.residual(E, Pb.contiguous())
            b = E * (g.inv_alpha != 0)[..., None]
            assert float(torch.linalg.vector_norm(r) / torch.linalg.vector_norm(b)) < 3e-6
            Ps_, _ = op.solve(E, tol=1e-9, precision="c128")
            err = float(torch.linalg.vector_norm(Pb - Ps_) / torch.linalg.vector_norm(Ps_))
            assert err < 1e-4


def test_padding_tuner_prefers_measured_cheaper_shape():
    from precondda_b200.batch import PaddingTuner
    t = PaddingTuner("mixed", edges=(16, 32, 64))
    cands = t.candidates((30, 17, 9))
    assert (32, 32, 16) in cands and (32, 32, 32) in cands
    box, L = t.plan([(30, 17, 9)])[0]
    assert box in cands and L == tuple(2 * b for b in box)
    assert t.cost(box) <= min(t.cost(c) for c in cands) + 1e-12


def test_preconditioned_geometries_converge_in_fewer_iterations():
    """solve_geometries(precondition=True): one engine preconditioner per
    geometry on its bucket's grid; every RHS reaches the FP64 target with
    fewer inner iterations than without, and the solutions agree."""
    import precondda_b200 as P
    from precondda_b200.batch import Geometry, PaddingTuner, solve_geometries
    from precondda_b200.workloads import random_ellipsoid_spec, build_geometry
    rng = np.random.default_rng(11)
    specs = [random_ellipsoid_spec(rng, edge=(10, 24), n_dirs=1) for _ in range(3)]
    geoms = [Geometry(*build_geometry(sp)) for sp in specs]
    tuner = PaddingTuner("mixed", edges=(12, 16, 24), measure=False)
    r0 = solve_geometries(geoms, tol=1e-6, precision="mixed", tuner=tuner, chunk=4)
    r1 = solve_geometries(geoms, tol=1e-6, precision="mixed", tuner=tuner, chunk=4, precondition=True)
    it0 = sum(i.iters for gi in r0.info for i in gi)
    it1 = sum(i.iters for gi in r1.info for i in gi)
    assert it1 < it0
    for g, P0s, P1s, infos in zip(geoms, r0.P, r1.P, r1.info):
        for P0, P1, info in zip(P0s, P1s, infos):
            assert info.status == "converged" and info.true_relres <= 1e-6
            assert float(torch.linalg.vector_norm(P1 - P0) / torch.linalg.vector_norm(P0)) < 1e-5
