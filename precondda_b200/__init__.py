"""B200-native discrete-dipole-approximation engine.

Drop-in for the reference's (Toastlovesjam/preconDDA) DDA hot path:
lattice setup -> Green's-tensor FFT -> A.P matvec -> GPBiCGSTAB -> cross
sections / near field, computed by hand-written sm_100a CUDA kernels in
``libdda_b200.so`` (C ABI in include/dda_b200.h).
"""
from .lattice import (Shape, Sphere, Cylinder, Ellipsoid, Rectangle, Prism, ShapeManager, calculate_alpha,
                      mark_shapes, trim_zero_faces, create_alpha_and_n_arrays, incident_field,
                      build_problem_from_shapes, sphere_occupancy, ellipsoid_occupancy, euler_rotation)
from .engine import (DDAOperator, SolveInfo, solve_many, cross_sections, green_octant, fft_lengths,
                     compiled_fft_lengths, far_field, differential_cross_section, Preconditioner, precond_lengths)
from .reference_api import (generate_interaction_row, prepare_interaction_matrices, interaction_mult, fft_matvec,
                            fft_matvec3, E_field_solver, solve_gpbicgstab, Gpbicgstab, run_solver, expand_octant)

__all__ = [
    "Shape", "Sphere", "Cylinder", "Ellipsoid", "Rectangle", "Prism", "ShapeManager", "calculate_alpha",
    "mark_shapes", "trim_zero_faces", "create_alpha_and_n_arrays", "incident_field", "build_problem_from_shapes",
    "sphere_occupancy", "ellipsoid_occupancy", "euler_rotation",
    "DDAOperator", "SolveInfo", "solve_many", "cross_sections", "green_octant", "fft_lengths",
    "compiled_fft_lengths", "far_field", "differential_cross_section", "Preconditioner", "precond_lengths",
    "generate_interaction_row", "prepare_interaction_matrices", "interaction_mult", "fft_matvec", "fft_matvec3",
    "E_field_solver", "solve_gpbicgstab", "Gpbicgstab", "run_solver", "expand_octant",
]
