"""The device voxeliser against the reference's own lattices.

tests/golden/shape_fixtures.npz holds alpha arrays made by the reference's
build_problem_from_shapes (ddaforgit.py:1591-1651) for rectangles, cylinders
along every axis (with the reference's own x/y-axis handling), prisms along
every axis and an overlapping mix.  Here the shapes are processed on the host
(centre snapping, grid extents), voxelised by the engine's k_voxelize with the
mark_shapes windows, trimmed, and compared site for site."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = os.path.join(os.path.dirname(__file__), "golden", "shape_fixtures.npz")


def _cases():
    with open(SHAPES.replace(".npz", ".json")) as f:
        cases = json.load(f)["cases"]
    out = []
    for name, c in cases.items():
        shapes = [dict(s, n=complex(s["n"]) if isinstance(s["n"], str) else s["n"]) for s in c["shapes"]]
        out.append((name, shapes, c))
    return out


@pytest.mark.parametrize("name,shapes,case", _cases(), ids=[c[0] for c in _cases()])
def test_device_voxelizer_matches_reference_lattice(name, shapes, case):
    from precondda_b200.lattice import ShapeManager, mark_shapes_device, trim_zero_faces
    ref = np.load(SHAPES)[f"{name}_alpha"]
    sm = ShapeManager()
    for s in shapes:
        sm.add_shape(s["type"], **{k: v for k, v in s.items() if k != "type"})
    d = case["spacing"]
    k = 2 * np.pi / case["wavelength"]
    sm.process_shapes(k, np.array(case["k_direction"], dtype=np.float64), case["polarization"], d)
    grid = sm.calculate_grid_extents(d)
    got = mark_shapes_device(grid, d, list(sm.shapes.values())).cpu().numpy()
    got = trim_zero_faces(got)
    assert got.shape == ref.shape
    assert np.array_equal(got, ref)
