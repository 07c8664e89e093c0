"""CPU checks of the host-side product code and of the C-ABI library (no
compute calls: there is no GPU here)."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import dda_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    txt = open(os.path.join(ROOT, "include", "dda_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(dda_[a-z0-9_]+)\s*\(", txt)))


def _lib():
    from precondda_b200 import _lib as L
    if not os.path.exists(L.LIB_PATH):
        pytest.skip("engine library not built")
    return L


def test_library_exports_every_declared_symbol():
    L = _lib()
    lib = L.lib()
    decl = _declared_symbols()
    assert len(decl) >= 10
    for name in decl:
        assert hasattr(lib, name), name
    assert set(decl) == set(L.EXPORTS)


def test_library_host_only_entry_points():
    L = _lib()
    lib = L.lib()
    assert lib.dda_version() >= 100
    ok = [n for n in range(2, 600, 2) if lib.dda_fft_length_ok(n, L.DDA_C128)]
    assert 16 in ok and 64 in ok and 128 in ok and 256 in ok and 512 in ok
    assert not lib.dda_fft_length_ok(22, L.DDA_C128)      # 11 is not a compiled factor
    assert not lib.dda_fft_length_ok(7, L.DDA_C128)       # odd
    for n in ok:
        m = n
        for p in (2, 3, 5, 7):
            while m % p == 0:
                m //= p
        assert m == 1


def test_fft_lengths_choice():
    _lib()
    from precondda_b200 import fft_lengths
    assert fft_lengths((32, 32, 32)) == (64, 64, 64)
    assert fft_lengths((64, 48, 128)) == (128, 96, 256)
    Lx, Ly, Lz = fft_lengths((33, 50, 7))
    assert Lx >= 66 and Ly >= 100 and Lz >= 14
    with pytest.raises(ValueError):
        fft_lengths((11, 4, 4), exact=True)


def test_alpha_matches_oracle():
    from precondda_b200 import calculate_alpha
    for meth in ("CM", "RR"):
        assert calculate_alpha(1.7 + 0.1j, 0.02, 12.0, method=meth) == O.calculate_alpha(1.7 + 0.1j, 0.02, 12.0,
                                                                                         method=meth)
    a = calculate_alpha(1.7 + 0.1j, 0.02, 12.0, (0, 0, 1), (1, 0, 0))
    assert a == O.calculate_alpha(1.7 + 0.1j, 0.02, 12.0, (0, 0, 1), (1, 0, 0))


def test_sphere_and_ellipsoid_occupancy():
    from precondda_b200 import sphere_occupancy, ellipsoid_occupancy, euler_rotation
    assert sphere_occupancy(32, 16.0).sum() == 17256
    assert np.array_equal(sphere_occupancy(20, 9.3), O.sphere_lattice(20, 9.3))
    R = euler_rotation(0.3, 1.1, -0.7)
    assert np.allclose(R @ R.T, np.eye(3))
    occ = ellipsoid_occupancy((24, 20, 16), (10, 8, 6), R)
    pts = O.voxel_centres((24, 20, 16), 1.0) - np.array([12.0, 10.0, 8.0])
    ref = O.ellipsoid_mask(pts.reshape(-1, 3), (0, 0, 0), (10, 8, 6), rotation=R).reshape(24, 20, 16)
    assert np.array_equal(occ, ref)


def test_build_problem_from_shapes_sphere():
    from precondda_b200 import build_problem_from_shapes
    d = 0.02
    prob = build_problem_from_shapes([{"type": "sphere", "center": [0.16, 0.16, 0.16], "radius": 0.16, "n": 1.5}],
                                     np.array([0.0, 0.0, 1.0]), [1.0, 0.0, 0.0], 0.5, d, method="RR")
    a = prob["alpha_array"]
    assert a.shape[0] % 2 == 0 and a.shape[1] % 2 == 0 and a.shape[2] % 2 == 0
    assert np.count_nonzero(a) > 0
    assert np.all(a[a != 0] == O.calculate_alpha(1.5, d, 2 * np.pi / 0.5, method="RR"))
    E = prob["E_inc"]
    assert E.shape == a.shape + (3,)
    assert np.allclose(E, O.incident_field(a.shape, d, 2 * np.pi / 0.5, (0, 0, 1), (1, 0, 0)))


def test_trim_zero_faces_pads_to_even():
    from precondda_b200 import trim_zero_faces
    a = np.zeros((9, 9, 9), complex)
    a[2:5, 1:8, 3:4] = 1
    t = trim_zero_faces(a)
    assert t.shape == (4, 8, 2)
    assert np.array_equal(t, O.trim_zero_faces(a))


def test_shape_membership_zoo():
    from precondda_b200.lattice import inside_rectangle, inside_cylinder, inside_prism
    g = O.voxel_centres((12, 12, 12), 1.0).reshape(-1, 3)
    r = inside_rectangle(g, (6, 6, 6), (4, 6, 8))
    assert r.sum() == 4 * 6 * 8
    c = inside_cylinder(g, (6, 6, 6), 3.0, 4.0, "z")
    assert c.sum() > 0 and c.sum() < np.pi * 9 * 4 * 1.3
    p = inside_prism(g, (6, 6, 6), 4.0, 6.0, 4, "z")
    assert p.sum() > 0
    # a square prism (4 sides, vertices on the axes) has area 2 r^2
    assert abs(p.sum() / 6 - 2 * 16) < 12


def test_serve_buckets_and_hbm_admission():
    from precondda_b200.serve import choose_bucket, pool_slots, slot_bytes, request_bytes
    assert choose_bucket((10, 12, 14), (8, 16, 32)) == 16
    assert choose_bucket((16, 3, 3), (8, 16, 32)) == 16
    assert choose_bucket((17, 3, 3), (8, 16, 32)) == 32
    with pytest.raises(ValueError):
        choose_bucket((33, 1, 1), (8, 16, 32))
    box, L = (64, 64, 64), (128, 128, 128)
    n3 = 64 ** 3 * 3
    scratch = 64 * 64 * 128 * 3 + 64 * 128 * 128 * 3
    assert slot_bytes(box, L, "c64") == (16 * n3 + scratch) * 8
    assert slot_bytes(box, L, "c128") == (16 * n3 + scratch) * 16
    assert slot_bytes(box, L, "mixed") == (16 * n3 + scratch) * 8 + 2 * n3 * 16
    per = slot_bytes(box, L, "mixed") + request_bytes(box, "mixed")
    assert pool_slots(box, L, "mixed", 10 * per + per // 2, 64) == 10
    assert pool_slots(box, L, "mixed", 10 * per, 4) == 4
    assert pool_slots(box, L, "mixed", per - 1, 4) == 0
    # preconditioned pools: one more vector per slot, the request's octant in
    # the precision the pool reads
    from precondda_b200.serve import precond_bytes
    assert slot_bytes(box, L, "mixed", True) == slot_bytes(box, L, "mixed") + n3 * 8
    assert slot_bytes(box, L, "c128", True) == slot_bytes(box, L, "c128") + n3 * 16
    assert precond_bytes(L, "mixed") == 6 * 65 ** 3 * 8 and precond_bytes(L, "c128") == 6 * 65 ** 3 * 16
    assert request_bytes(box, "mixed", L) == request_bytes(box, "mixed") + precond_bytes(L, "mixed")
    perp = slot_bytes(box, L, "mixed", True) + request_bytes(box, "mixed", L)
    assert pool_slots(box, L, "mixed", 3 * perp, 64, precondition=True) == 3
    from precondda_b200.batch import item_bytes
    assert item_bytes(box, L, "mixed", 4, 1, True) > item_bytes(box, L, "mixed", 4, 1)


def test_workload_generators_are_seeded_and_valid():
    from precondda_b200 import workloads as W
    a = W.serving_stream(3, rate=20, duration=5)
    b = W.serving_stream(3, rate=20, duration=5)
    assert [x[0] for x in a] == [x[0] for x in b] and len(a) > 50
    kinds = {sp["kind"] for _, sp in a}
    assert kinds <= {"sphere", "ellipsoid", "aggregate"} and len(kinds) == 3
    assert all(16 <= max(sp["box"]) <= 128 for _, sp in a)
    assert all(1 <= len(sp["dirs"]) <= 16 for _, sp in a)
    rng = np.random.default_rng(0)
    c, r = W.random_walk_aggregate(12, (6, 12), rng)
    assert len(c) == 12
    for i in range(12):
        for j in range(i):
            assert np.linalg.norm(c[i] - c[j]) >= r[i] + r[j] - 1e-6
    # every sphere after the first touches an earlier one
    for i in range(1, 12):
        assert min(abs(np.linalg.norm(c[i] - c[j]) - r[i] - r[j]) for j in range(i)) < 1e-6
    e = W.random_ellipsoid_spec(np.random.default_rng(1))
    assert all(16 <= b <= 96 for b in e["box"]) and len(e["dirs"]) == 8
    k1, k2 = W.transverse_pair(np.array([0.3, -0.5, 0.81]) / np.linalg.norm([0.3, -0.5, 0.81]))
    assert abs(k1 @ k2) < 1e-12


def test_results_file_layout(tmp_path):
    from precondda_b200.results import save_results_to_file
    P = (np.arange(2 * 3 * 4 * 3) + 1j).reshape(2, 3, 4, 3).astype(np.complex64)
    problem = {"grid_size": (2, 3, 4), "lattice_spacing": 0.02, "wavelength": 0.5, "k_direction": [0, 0, 1],
               "E_polarization": [1, 0, 0], "k": 12.566370614359172}
    shapes = [{"type": "sphere", "center": [0.1, 0.1, 0.1], "n": 1.5, "radius": 0.08},
              {"type": "prism", "center": [0, 0, 0], "n": 2.0, "radius": 0.05, "height": 0.1, "sides": 6,
               "axis": "z"}]
    fn = str(tmp_path / "run.txt")
    files = save_results_to_file(fn, problem, [np.nan, np.nan], shapes, (17, P, 3.2e-7), (1.0, 0.25, 0.75))
    assert files == [fn, fn.replace(".txt", "_polarization.npy")]
    txt = open(fn).read().splitlines()
    assert txt[0] == "DDA Problem Analysis Results" and txt[1] == "=" * 50
    assert "Grid size: (2, 3, 4)" in txt and "Lattice spacing: 0.020000" in txt
    assert "Shape 1: sphere" in txt and "  Radius: 0.08" in txt and "  Sides: 6" in txt
    assert "AI PREDICTION: Failed" in txt
    assert "Iterations: 17" in txt and "Final norm: 3.200000e-07" in txt and "Status: Converged" in txt
    assert "Polarization array shape: (2, 3, 4, 3)" in txt and "C_sca: 7.500000000e-01" in txt
    assert np.array_equal(np.load(files[1]), P)


def test_result_files_match_reference(tmp_path):
    """save_results_to_file against the reference's own writer
    (tests/golden/make_results_fixture.py): every line but the time stamp,
    and the polarisation arrays exactly."""
    import json
    import sys as _sys
    from precondda_b200 import build_problem_from_shapes
    from precondda_b200.results import save_results_to_file
    gold = os.path.join(os.path.dirname(__file__), "golden", "ref_results")
    _sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_results_fixture as M
    with open(os.path.join(gold, "cases.json")) as f:
        meta = json.load(f)
    pr = build_problem_from_shapes(M.SHAPES, np.array(meta["k_direction"]), meta["polarization"],
                                   meta["wavelength"], meta["spacing"])
    assert list(pr["grid_size"]) == meta["grid_size"]
    P = M.polarization(tuple(pr["grid_size"]))
    for name, c in M.CASES.items():
        fn = str(tmp_path / f"{name}.txt")
        save_results_to_file(fn, pr, np.array(c["prediction"]), M.SHAPES, (c["iterations"], P, c["final_norm"]))
        got = open(fn).read().splitlines()
        ref = open(os.path.join(gold, f"{name}.txt")).read().splitlines()
        assert len(got) == len(ref), name
        for g, r in zip(got, ref):
            if r.startswith("Results saved on:"):
                continue
            if r.startswith("Full polarization array saved to:"):
                assert os.path.basename(g.split(": ", 1)[1]) == os.path.basename(r.split(": ", 1)[1])
                continue
            assert g == r, (name, g, r)
        assert np.array_equal(np.load(fn.replace(".txt", "_polarization.npy")),
                              np.load(os.path.join(gold, f"{name}_polarization.npy")))


def test_launch_tuner_picks_fastest_candidate_and_caches(tmp_path):
    """LaunchTuner's selection logic with a fake device timer: the candidate
    set per bucket, the fastest flags chosen (the default kept within the
    margin), cached (also in JSON) and not timed twice."""
    import torch
    from precondda_b200 import _lib as L
    from precondda_b200.batch import LaunchTuner, launch_candidates
    c64, c128 = torch.complex64, torch.complex128
    xs = [0, L.DDA_TUNE_P3PIPE, L.DDA_TUNE_P3PAIR]
    ys = [0, L.DDA_TUNE_YPAIR | L.DDA_TUNE_ZPAIR]
    ps = [0]
    nofused = L.DDA_TUNE_NO_FUSED_ZY | L.DDA_TUNE_NO_FUSED_INV
    assert launch_candidates((64,) * 3, (128,) * 3, c64, 1) == [
        x | y | p | z for x in xs for y in ys for p in ps for z in (0, nofused)]
    c128k = [x | y | p | z for x in xs for y in ys for p in ps for z in (0, L.DDA_TUNE_FUSED)]
    assert launch_candidates((128,) * 3, (256,) * 3, c64, 16) == c128k
    assert launch_candidates((64,) * 3, (128,) * 3, c64, 4) == [x | y | p for x in xs for y in ys for p in ps]
    assert launch_candidates((40, 30, 20), (80, 64, 40), c64, 4) == [0]
    assert launch_candidates((64,) * 3, (128,) * 3, c128, 1) == [0]
    calls = []

    def timer(box, L_, dtype, nb, flags):
        calls.append(flags)
        return 3.0 - (0.5 if flags == L.DDA_TUNE_P3PAIR | L.DDA_TUNE_FUSED else 0.0) - \
            (0.3 if flags == L.DDA_TUNE_P3PAIR else 0.0)

    path = str(tmp_path / "launch.json")
    t = LaunchTuner(cache_path=path, timer=timer)
    best = L.DDA_TUNE_P3PAIR | L.DDA_TUNE_FUSED
    assert t.tune((128,) * 3, (256,) * 3, c64, 16) == best
    assert sorted(calls) == sorted(c128k)
    assert t.tune((128,) * 3, (256,) * 3, c64, 16) == best
    assert len(calls) == len(c128k)                  # cached
    assert t.tune((40, 30, 20), (80, 64, 40), c64, 4) == 0 and len(calls) == len(c128k)   # single candidate
    t2 = LaunchTuner(cache_path=path, timer=lambda *a: 1 / 0)
    assert t2.tune((128,) * 3, (256,) * 3, c64, 16) == best                        # from the JSON cache
    # within the margin of the default: the default stays
    t3 = LaunchTuner(timer=lambda box, L_, dt, nb, f: 1.0 - 0.01 * (f == L.DDA_TUNE_P3PAIR))
    assert t3.tune((128,) * 3, (256,) * 3, c64, 16) == 0
