"""Result files in the reference's format.

``save_results_to_file`` writes the text summary the reference writes
(ddaforgit.py:1653-1749) -- problem parameters, shapes, the predictor
section, solver results -- and the polarisation array next to it as
``<name>_polarization.npy``, so tools that read the reference's output read
these files unchanged.  A cross-section block (which the reference does not
compute) is appended after the solver results when given.
"""
from __future__ import annotations

import numpy as np


def _as_host(a):
    if a is None:
        return None
    if hasattr(a, "detach"):            # torch
        return a.detach().cpu().numpy()
    if hasattr(a, "get"):               # CuPy
        return a.get()
    return np.asarray(a)


def _shape_lines(shape):
    t = shape["type"]
    out = [f"Shape: {t}", f"  Center: {shape['center']}", f"  Refractive index: {shape['n']}"]
    if t in ("sphere", "cylinder", "prism"):
        out.append(f"  Radius: {shape['radius']}")
    if t in ("cylinder", "prism"):
        out.append(f"  Height: {shape['height']}")
    if t == "prism":
        out.append(f"  Sides: {shape['sides']}")
    if t in ("cylinder", "prism"):
        out.append(f"  Axis: {shape['axis']}")
    if t == "rectangle":
        out.append(f"  Dimensions: {shape['dimensions']}")
    if t == "ellipsoid":
        out.append(f"  Semi-axes: {shape['semi_axes']}")
    return out


def save_results_to_file(filename, problem, prediction, shapes, solver_result=None, cross_sections=None,
                         max_iter=10000):
    """Write the reference's DDA result summary.

    problem: dict with grid_size, lattice_spacing, wavelength, k_direction,
    E_polarization, k (build_problem_from_shapes' keys); prediction: the
    predictor output (two floats, NaN when absent); shapes: list of shape
    dicts; solver_result: run_solver's (iterations, P, final_norm);
    cross_sections: optional (C_ext, C_abs, C_sca).  Returns the names of the
    files written."""
    written = [filename]
    lines = ["DDA Problem Analysis Results", "=" * 50, "", "PROBLEM PARAMETERS:",
             f"Grid size: {problem['grid_size']}",
             f"Lattice spacing: {problem['lattice_spacing']:.6f}",
             f"Wavelength: {problem['wavelength']:.6f}",
             f"Wave direction: {problem['k_direction']}",
             f"Polarization: {problem['E_polarization']}",
             f"k (wave number): {problem['k']:.6f}", "", "SHAPES:"]
    for i, sh in enumerate(shapes, 1):
        body = _shape_lines(sh)
        lines.append(f"Shape {i}: {sh['type']}")
        lines.extend(body[1:])
        lines.append("")
    pred = np.asarray(prediction, dtype=float) if prediction is not None else np.array([np.nan])
    if pred.size >= 2 and not np.any(np.isnan(pred)):
        mult = complex(pred[0], pred[1])
        lines += ["AI PREDICTION:", f"Optimal multiplier: {mult.real:.6f} + {mult.imag:.6f}j",
                  f"Magnitude: {abs(mult):.6f}",
                  f"Phase: {np.angle(mult):.6f} radians ({np.degrees(np.angle(mult)):.2f} degrees)", ""]
    else:
        lines += ["AI PREDICTION: Failed", ""]
    if solver_result is not None:
        iterations, pol, final_norm = solver_result
        lines += ["SOLVER RESULTS:", f"Iterations: {iterations}", f"Final norm: {final_norm:.6e}",
                  "First norm: Not available from run_solver"]
        if iterations is not None:
            if 0 < iterations < max_iter:
                lines.append("Status: Converged")
            elif iterations == max_iter:
                lines.append("Status: Did not converge (max iterations reached)")
            elif iterations < 0:
                lines.append("Status: Failed (NaN or error condition)")
            else:
                lines.append("Status: Unknown")
        pol = _as_host(pol)
        if pol is not None:
            lines += [f"Polarization array shape: {pol.shape}", f"Polarization array dtype: {pol.dtype}"]
            pol_name = filename.replace(".txt", "_polarization.npy")
            np.save(pol_name, pol)
            written.append(pol_name)
            lines.append(f"Full polarization array saved to: {pol_name}")
        else:
            lines.append("Polarization array: Not available")
        if cross_sections is not None:
            ce, ca, cs = (float(v) for v in cross_sections)
            lines += ["", "CROSS SECTIONS (Draine & Flatau 1994):", f"C_ext: {ce:.9e}", f"C_abs: {ca:.9e}",
                      f"C_sca: {cs:.9e}"]
    else:
        lines.append("SOLVER RESULTS: Not run")
    lines += ["", f"Results saved on: {np.datetime64('now')}"]
    with open(filename, "w") as f:
        f.write("\n".join(lines) + "\n")
    return written
