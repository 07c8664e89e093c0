"""Build libdda_b200.so (the engine's C-ABI shared library) for sm_100a.

Each CUDA source is compiled to an object in parallel with nvcc, then linked
into ``precondda_b200/libdda_b200.so``.  Run as a script or call ``build()``.
Objects go to ``precondda_b200/_build`` and are rebuilt when a source or
header is newer than the object.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdda_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
_DEFINES: list = []
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I", CSRC, "-I", INCLUDE]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers_mtime() -> float:
    hs = [h for pat in ("*.cuh", "*.inc", "*.h") for h in glob.glob(os.path.join(CSRC, pat))] + \
        glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, nvcc: str, hdr_t: float, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_t):
        return obj
    cmd = [nvcc, "-c", src, "-o", obj] + ARCH + FLAGS + [f"-D{d}" for d in _DEFINES]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False, jobs: int | None = None, defines=(), out: str | None = None,
          build_dir: str | None = None) -> str:
    """Compile all csrc/*.cu and link libdda_b200.so (or ``out``); returns its
    path.  ``defines`` are extra -D macros (tuning variants)."""
    global BUILD
    if build_dir:
        BUILD = build_dir
    lib_path = out or LIB
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr_t = _headers_mtime()
    global _DEFINES
    _DEFINES = list(defines)
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, nvcc, hdr_t, verbose), srcs))
    if os.path.exists(lib_path) and os.path.getmtime(lib_path) >= max(os.path.getmtime(o) for o in objs):
        return lib_path
    tmp = lib_path + ".tmp"
    cmd = [nvcc, "-shared", "-o", tmp] + objs + ARCH + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, lib_path)
    return lib_path


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
