"""The reference's result files for one problem, as a golden fixture.

Run from the repository root in a checkout that has the reference:

    python oracle/build_ref.py
    python tests/golden/make_results_fixture.py [--ref <reference checkout>]

The reference's ``save_results_to_file`` (ddaforgit.py:1653-1749) runs
unchanged through ``oracle/ref_loader.py`` on a problem from its own
``build_problem_from_shapes`` (two shapes), a fixed predictor output and a
solver result (iterations, a seeded polarisation array, final norm), for a
converged, a not-converged and a failed solve and for a failed prediction.
It writes ``tests/golden/ref_results/<case>.txt`` and
``<case>_polarization.npy`` plus ``cases.json`` with the inputs; the tests
regenerate the same files with ``precondda_b200.results`` and compare them
(every line but the time stamp; the arrays exactly).
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import build_ref, ref_loader  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "ref_results")

SHAPES = [{"type": "sphere", "center": [0.1, 0.1, 0.1], "radius": 0.05, "n": 1.5},
          {"type": "cylinder", "center": [0.1, 0.12, 0.1], "radius": 0.03, "height": 0.08, "axis": "z",
           "n": 1.7 + 0.1j}]
CASES = {
    "converged": {"prediction": [0.8, -0.3], "iterations": 42, "final_norm": 3.25e-6},
    "maxiter": {"prediction": [1.25, 0.5], "iterations": 10000, "final_norm": 1.5e-3},
    "failed": {"prediction": [float("nan"), float("nan")], "iterations": -7, "final_norm": float("nan")},
}


def polarization(shape, seed=5):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(shape + (3,)) + 1j * rng.standard_normal(shape + (3,))).astype(np.complex64)


def main(ref):
    R = ref_loader.load(ref)
    D = R.ddaforgit
    os.makedirs(OUT, exist_ok=True)
    with ref_loader.quiet():
        pr = D.build_problem_from_shapes(SHAPES, np.array([0.0, 0.0, 1.0]), [1.0, 0.0, 0.0], 0.5, 0.01)
    P = polarization(tuple(pr["grid_size"]))
    os.chdir(ROOT)             # relative names: the files record the .npy path as given
    for name, c in CASES.items():
        fn = os.path.relpath(os.path.join(OUT, f"{name}.txt"), ROOT)
        with ref_loader.quiet():
            D.save_results_to_file(fn, pr, np.array(c["prediction"]), SHAPES, (c["iterations"], P, c["final_norm"]))
        print(name, os.path.getsize(fn), flush=True)
    meta = {"generator": "tests/golden/make_results_fixture.py",
            "shapes": [{k: (str(v) if isinstance(v, complex) else v) for k, v in s.items()} for s in SHAPES],
            "k_direction": [0.0, 0.0, 1.0], "polarization": [1.0, 0.0, 0.0], "wavelength": 0.5, "spacing": 0.01,
            "grid_size": [int(v) for v in pr["grid_size"]], "cases": CASES}
    with open(os.path.join(OUT, "cases.json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    main(ap.parse_args().ref or build_ref.reference_dir())
