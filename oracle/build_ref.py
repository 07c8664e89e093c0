"""Compile the reference's own CUDA-C kernel strings for the CPU -- TEST
INFRASTRUCTURE ONLY (builds the checker, never the product).

The reference keeps its device code as CuPy ``RawKernel`` / ``ElementwiseKernel``
strings inside ``Gpbicgstab.py``, ``ExcitedField.py`` and ``ddaforgit.py``.  This
recipe reads those files from the reference checkout, extracts the strings with
``ast`` (the files are not imported), wraps each kernel with a launcher for the
CPU emulation in ``oracle/refshim`` and compiles everything with g++ into
``oracle/_ref/librefkernels.so`` plus a JSON manifest of the kernel signatures.
The generated C++ is written to a temporary directory and deleted; only the
shared library and the manifest stay (``oracle/_ref`` is not committed).

Kernels that are not on the DDA path (the preconditioner's template kernels and
the cuComplex gather/scatter helpers) are skipped.

Usage:  python oracle/build_ref.py [--ref <reference checkout>]

The checkout is found by ``reference_dir()``: ``$DDA_REFERENCE_DIR`` if set,
else the checkout path of the build container.
"""
from __future__ import annotations

import argparse
import ast
import json
import os
import re
import shutil
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
SHIM = os.path.join(HERE, "refshim")
DEFAULT_REF = "/root/reference"


def reference_dir():
    """Where this recipe reads the reference checkout: $DDA_REFERENCE_DIR, else
    the build container's checkout path.  It is the one place that names it."""
    return os.environ.get("DDA_REFERENCE_DIR", DEFAULT_REF)
FILES = ("Gpbicgstab.py", "ExcitedField.py", "ddaforgit.py")

_EW_TYPES = {"int32": "int", "int64": "long long", "float32": "float", "float64": "double",
             "complex64": "complex<float>", "complex128": "complex<double>", "bool": "bool"}


def _kernel_calls(path):
    """(python variable, kind, string args) for every kernel constructor."""
    tree = ast.parse(open(path).read())
    out = []
    for node in ast.walk(tree):
        if not isinstance(node, ast.Assign) or not isinstance(node.value, ast.Call):
            continue
        f = node.value.func
        if not (isinstance(f, ast.Attribute) and isinstance(f.value, ast.Name) and f.value.id == "cp"):
            continue
        if f.attr not in ("RawKernel", "ElementwiseKernel"):
            continue
        if not (node.targets and isinstance(node.targets[0], ast.Name)):
            continue
        args = [a.value for a in node.value.args if isinstance(a, ast.Constant)]
        out.append((node.targets[0].id, f.attr, args))
    return out


def _split_params(sig):
    params = []
    for p in sig.split(","):
        p = " ".join(p.split())
        if not p:
            continue
        m = re.match(r"(.*?)(\w+)$", p)
        ctype, name = m.group(1).strip(), m.group(2)
        params.append((ctype, name))
    return params


def _raw_kernel(mod, var, src, fname):
    if "cuFloatComplex" in src or "cuComplex" in src:
        return None
    src = "\n".join(ln for ln in src.splitlines() if not ln.strip().startswith("#include"))
    m = re.search(r'extern\s+"C"\s+__global__\s+void\s+(\w+)\s*\(([^)]*)\)', src)
    if not m:
        return None
    cname = f"{mod}__{var}"
    params = _split_params(m.group(2))
    src = src[:m.start(1)] + cname + src[m.end(1):]
    src = src.replace('extern "C"', "", 1)
    barriers = "__syncthreads" in src
    names = ", ".join(n for _, n in params)
    plist = ", ".join(f"{t} {n}" for t, n in params)
    wrapper = (f'extern "C" void launch__{cname}(unsigned gx_, unsigned bx_, {plist}) {{\n'
               f"  refshim::run_grid(gx_, bx_, {'true' if barriers else 'false'}, [&]() {{ {cname}({names}); }});\n}}\n")
    code = f"// {mod}.{var} ({fname})\n{src}\n{wrapper}"
    man = {"module": mod, "var": var, "kind": "raw", "symbol": f"launch__{cname}",
           "params": [{"ctype": t, "name": n, "pointer": "*" in t} for t, n in params], "barriers": barriers}
    return code, man


def _ew_kernel(mod, var, in_params, out_params, body, name):
    ins, outs = [], []
    for spec, dst in ((in_params, ins), (out_params, outs)):
        for p in spec.split(","):
            toks = p.split()
            if not toks:
                continue
            raw = toks[0] == "raw"
            if raw:
                toks = toks[1:]
            ty, nm = toks[0], toks[1]
            if ty not in _EW_TYPES:
                return None              # generic-type kernels are not on the path
            dst.append((_EW_TYPES[ty], nm, raw))
    if any(not raw for _, _, raw in outs):
        return None
    cname = f"{mod}__{var}"
    plist = ", ".join([f"{t} {n}" for t, n, _ in ins] + [f"{t}* {n}" for t, n, _ in outs])
    code = (f"// {mod}.{var} ({name})\n"
            f'extern "C" void ew__{cname}(long long size_, {plist}) {{\n'
            f"  for (long long i_ = 0; i_ < size_; ++i_) {{\n"
            f"    const long long i = i_;\n"
            f"    [&]() {{\n{body}\n    }}();\n  }}\n}}\n")
    man = {"module": mod, "var": var, "kind": "elementwise", "symbol": f"ew__{cname}",
           "params": [{"ctype": t, "name": n, "pointer": False} for t, n, _ in ins] +
                     [{"ctype": t + "*", "name": n, "pointer": True} for t, n, _ in outs]}
    return code, man


def build(ref=None, verbose=False):
    ref = ref or reference_dir()
    os.makedirs(OUT, exist_ok=True)
    units, manifest = [], []
    for fn in FILES:
        path = os.path.join(ref, fn)
        mod = fn[:-3]
        for var, kind, args in _kernel_calls(path):
            if kind == "RawKernel" and len(args) >= 2:
                r = _raw_kernel(mod, var, args[0], args[1])
            elif kind == "ElementwiseKernel" and len(args) >= 4:
                r = _ew_kernel(mod, var, *args[:4])
            else:
                r = None
            if r:
                units.append(r[0])
                manifest.append(r[1])
    tmp = tempfile.mkdtemp(prefix="refk_")
    try:
        gen = os.path.join(tmp, "refkernels.cpp")
        with open(gen, "w") as f:
            f.write('#include "prelude.h"\n#include <functional>\n')
            f.write("namespace refshim { void run_grid(unsigned, unsigned, bool, const std::function<void()>&); }\n")
            f.write("\n".join(units))
        lib = os.path.join(OUT, "librefkernels.so")
        cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-w", "-I", SHIM, gen,
               os.path.join(SHIM, "fibers.cpp"), "-o", lib]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"g++ failed:\n{r.stderr[-4000:]}")
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    with open(os.path.join(OUT, "kernels.json"), "w") as f:
        json.dump(manifest, f, indent=1)
    return lib, manifest


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    a = ap.parse_args()
    lib, man = build(a.ref, verbose=True)
    print(lib)
    for m in man:
        print(f"  {m['module']}.{m['var']:40s} {m['kind']:12s} barriers={m.get('barriers', False)}")
