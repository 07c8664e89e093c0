"""Golden lattices of the reference's rectangle, cylinder and prism shapes.

Run from the repository root in a checkout that has the reference:

    python oracle/build_ref.py
    python tests/golden/make_shape_fixtures.py [--ref <reference checkout>]

The reference's ``build_problem_from_shapes`` (ddaforgit.py:1591-1651) runs
unchanged through ``oracle/ref_loader.py``: ShapeManager, process_shapes (LDR
polarizability, centre snapping), calculate_grid_extents, mark_shapes with
its per-shape index window (:615-661), the Numba membership functions
(:461-572) and trim_zero_faces.  The cases cover the three cylinder axes
(the x- and y-axis cylinders show the reference's own axis handling: radius
always in the (x, y) plane, signed z offset in the height test, bounded by
the mark_shapes window), the rectangle, prisms along every axis and an
overlapping multi-shape case.  Output: ``tests/golden/shape_fixtures.npz``
(+ ``.json`` with the case descriptions).
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

OUT = os.path.join(ROOT, "tests", "golden", "shape_fixtures.npz")

# (name, shapes, k_direction, polarisation, wavelength, spacing)
CASES = [
    ("cyl_z", [{"type": "cylinder", "center": [0.1, 0.1, 0.1], "radius": 0.05, "height": 0.12, "axis": "z",
                "n": 1.5}], [0.0, 0.0, 1.0], [1.0, 0.0, 0.0], 0.5, 0.005),
    ("cyl_y", [{"type": "cylinder", "center": [0.1, 0.1, 0.1], "radius": 0.05, "height": 0.12, "axis": "y",
                "n": 1.5}], [0.0, 0.0, 1.0], [1.0, 0.0, 0.0], 0.5, 0.005),
    ("cyl_x", [{"type": "cylinder", "center": [0.12, 0.1, 0.09], "radius": 0.04, "height": 0.16, "axis": "x",
                "n": 1.6 + 0.05j}], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0], 0.6, 0.005),
    ("rect", [{"type": "rectangle", "center": [0.1, 0.12, 0.08], "dimensions": [0.1, 0.14, 0.06],
               "n": 1.4 + 0.02j}], [0.0, 0.0, 1.0], [0.0, 1.0, 0.0], 0.5, 0.005),
    ("prism_z6", [{"type": "prism", "center": [0.1, 0.1, 0.1], "radius": 0.06, "height": 0.1, "sides": 6,
                   "axis": "z", "n": 1.5}], [0.0, 0.0, 1.0], [1.0, 0.0, 0.0], 0.5, 0.005),
    ("prism_y5", [{"type": "prism", "center": [0.1, 0.1, 0.1], "radius": 0.07, "height": 0.08, "sides": 5,
                   "axis": "y", "n": 1.7 + 0.1j}], [0.0, 1.0, 0.0], [1.0, 0.0, 0.0], 0.5, 0.005),
    ("prism_x4", [{"type": "prism", "center": [0.11, 0.1, 0.1], "radius": 0.06, "height": 0.1, "sides": 4,
                   "axis": "x", "n": 1.5}], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], 0.5, 0.005),
    ("mix", [{"type": "rectangle", "center": [0.1, 0.1, 0.1], "dimensions": [0.12, 0.08, 0.1], "n": 1.4},
             {"type": "cylinder", "center": [0.1, 0.1, 0.12], "radius": 0.03, "height": 0.14, "axis": "x",
              "n": 1.8 + 0.02j},
             {"type": "sphere", "center": [0.1, 0.08, 0.1], "radius": 0.035, "n": 2.0 + 0.1j}],
     [0.0, 0.0, 1.0], [1.0, 0.0, 0.0], 0.5, 0.005),
]


def main(ref):
    R = ref_loader.load(ref)
    D = R.ddaforgit
    fx, notes = {}, {}
    for name, shapes, kdir, pol, wl, d in CASES:
        with ref_loader.quiet():
            pr = D.build_problem_from_shapes(shapes, np.array(kdir), pol, wl, d)
        fx[f"{name}_alpha"] = np.asarray(pr["alpha_array"])
        notes[name] = {"shapes": [{k: (str(v) if isinstance(v, complex) else v) for k, v in s.items()}
                                  for s in shapes],
                       "k_direction": kdir, "polarization": pol, "wavelength": wl, "spacing": d,
                       "grid": list(np.asarray(pr["alpha_array"]).shape),
                       "occupied": int((np.asarray(pr["alpha_array"]) != 0).sum())}
        print(name, notes[name]["grid"], notes[name]["occupied"], flush=True)
    np.savez_compressed(OUT, **fx)
    with open(OUT.replace(".npz", ".json"), "w") as f:
        json.dump({"generator": "tests/golden/make_shape_fixtures.py", "cases": notes}, f, indent=1)
    print(f"wrote {OUT} ({os.path.getsize(OUT) / 1024:.0f} KiB)")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    main(ap.parse_args().ref or build_ref.reference_dir())
