"""Load the reference's own DDA code on the CPU -- TEST INFRASTRUCTURE ONLY.

``load(ref_dir)`` returns a namespace with the reference's functions running
against ``oracle.cupy_shim`` (NumPy + the reference's kernels compiled for the
CPU) and a CPU proxy for ``torch``:

* ``Gpbicgstab`` and ``ExcitedField`` are imported unchanged from the
  reference checkout;
* from ``ddaforgit.py`` (which cannot be imported: it needs missing modules
  and a display) the definitions on the DDA path are extracted with ``ast``
  and executed: the shapes and ``ShapeManager``, ``calculate_alpha``, the
  membership tests (their Numba decorator replaced by a no-op), voxelisation,
  ``trim_zero_faces``, the Green's kernels, ``generate_interaction_row`` and
  ``build_problem_from_shapes``.

Used only by ``tests/golden/make_golden.py`` in a checkout that has the
reference; nothing on the GPU box or in the product imports it.
"""
from __future__ import annotations

import ast
import contextlib
import gc
import importlib.util
import io
import math
import os
import sys
import types

import numpy as np

from . import cupy_shim

DDAFORGIT_DEFS = (
    "free_gpu_memory", "Shape", "Sphere", "Cylinder", "Ellipsoid", "Rectangle", "Prism", "ShapeManager",
    "calculate_alpha", "sphere", "ellipsoid", "rectangle", "cylinder", "prism", "create_shape_data",
    "shape_calculators", "mark_shapes", "mark_shapes_n", "create_alpha_and_n_arrays", "trim_zero_faces",
    "greens_kernel_single", "greens_kernel_double", "generate_interaction_row", "build_problem_from_shapes",
    "save_results_to_file",
)


class _TorchCPU:
    """The ``torch`` the reference sees: real torch on the CPU, device
    arguments ignored, cuda.synchronize a no-op."""

    def __init__(self):
        import torch
        self._t = torch
        self.cuda = types.SimpleNamespace(synchronize=lambda *a, **k: None, empty_cache=lambda: None)

    def zeros(self, *a, device=None, **k):
        return self._t.zeros(*a, **k)

    def __getattr__(self, name):
        return getattr(self._t, name)


def _kernel_sources(path, module):
    out = {}
    tree = ast.parse(open(path).read())
    for node in ast.walk(tree):
        if isinstance(node, ast.Assign) and isinstance(node.value, ast.Call):
            f = node.value.func
            if isinstance(f, ast.Attribute) and f.attr in ("RawKernel", "ElementwiseKernel") and node.targets \
                    and isinstance(node.targets[0], ast.Name):
                strs = [a.value for a in node.value.args if isinstance(a, ast.Constant)]
                if f.attr == "RawKernel" and strs:
                    out[(module, node.targets[0].id)] = strs[0]
                elif f.attr == "ElementwiseKernel" and len(strs) >= 3:
                    out[(module, node.targets[0].id)] = strs[2]
    return out


def _import_file(path, name, torch_proxy):
    sys.modules["cupy"] = cupy_shim
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    with contextlib.redirect_stdout(io.StringIO()):
        spec.loader.exec_module(mod)
    mod.torch = torch_proxy
    mod.cp = cupy_shim
    return mod


def load(ref_dir):
    torch_proxy = _TorchCPU()
    srcs = {}
    for fn in ("Gpbicgstab.py", "ExcitedField.py", "ddaforgit.py"):
        srcs.update(_kernel_sources(os.path.join(ref_dir, fn), fn[:-3]))
    cupy_shim.register_sources(srcs)
    saved = sys.modules.get("cupy")
    try:
        gp = _import_file(os.path.join(ref_dir, "Gpbicgstab.py"), "ref_Gpbicgstab", torch_proxy)
        ef = _import_file(os.path.join(ref_dir, "ExcitedField.py"), "ref_ExcitedField", torch_proxy)
    finally:
        if saved is None:
            sys.modules.pop("cupy", None)
        else:
            sys.modules["cupy"] = saved
    # ddaforgit.py: selected top-level definitions only
    tree = ast.parse(open(os.path.join(ref_dir, "ddaforgit.py")).read())
    keep = []
    for node in tree.body:
        name = None
        if isinstance(node, (ast.FunctionDef, ast.ClassDef)):
            name = node.name
        elif isinstance(node, ast.Assign) and node.targets and isinstance(node.targets[0], ast.Name):
            name = node.targets[0].id
        if name in DDAFORGIT_DEFS:
            keep.append(node)
    nb = types.SimpleNamespace(jit=lambda *a, **k: (lambda f: f))
    ns = {"np": np, "cp": cupy_shim, "torch": torch_proxy, "nb": nb, "gc": gc, "math": math, "os": os,
          "__name__": "ref_ddaforgit"}
    code = compile(ast.Module(body=keep, type_ignores=[]), os.path.join(ref_dir, "ddaforgit.py"), "exec")
    exec(code, ns)
    dda = types.SimpleNamespace(**{k: ns[k] for k in DDAFORGIT_DEFS if k in ns})
    return types.SimpleNamespace(Gpbicgstab=gp, ExcitedField=ef, ddaforgit=dda)


@contextlib.contextmanager
def quiet():
    with contextlib.redirect_stdout(io.StringIO()):
        yield
