"""NumPy-backed stand-in for the parts of CuPy the reference uses -- TEST
INFRASTRUCTURE ONLY.

With this module installed as ``cupy`` (and a CPU proxy for ``torch``), the
reference's own ``Gpbicgstab.py`` / ``ExcitedField.py`` and its Green /
polarizability / lattice functions run unchanged on the CPU.  Arrays are a
NumPy subclass with CuPy's ``.get()``; ``RawKernel`` and ``ElementwiseKernel``
dispatch to the reference's CUDA-C strings compiled for the CPU by
``oracle/build_ref.py`` (``oracle/_ref/librefkernels.so``).  ``fuse`` runs the
fused function directly and keeps complex64 results complex64, matching CuPy's
scalar-casting rules for 0-d operands.
"""
from __future__ import annotations

import builtins
import ctypes
import json
import os
import types

import numpy as np
import scipy.fft as _sfft

_HERE = os.path.dirname(os.path.abspath(__file__))
_REF = os.path.join(_HERE, "_ref")

complex64 = np.complex64
complex128 = np.complex128
float32 = np.float32
float64 = np.float64
int32 = np.int32
bool_ = np.bool_
newaxis = None


class ndarray(np.ndarray):
    """NumPy array with CuPy's device-to-host accessor."""

    def get(self):
        return np.array(self)


def _w(a):
    if isinstance(a, np.ndarray):
        return a.view(ndarray)
    return np.asarray(a).view(ndarray)


def asarray(a, dtype=None):
    return _w(np.asarray(a, dtype=dtype))


def array(a, dtype=None):
    return _w(np.array(a, dtype=dtype))


def zeros(shape, dtype=float):
    return _w(np.zeros(shape, dtype=dtype))


def zeros_like(a, dtype=None):
    return _w(np.zeros_like(np.asarray(a), dtype=dtype))


def empty_like(a, dtype=None):
    return _w(np.empty_like(np.asarray(a), dtype=dtype))


def arange(*a, **k):
    return _w(np.arange(*a, **k))


def repeat(a, r, axis=None):
    return _w(np.repeat(np.asarray(a), r, axis=axis))


def where(c, a, b):
    return _w(np.where(np.asarray(c), a, b))


def unique(a):
    return _w(np.unique(np.asarray(a)))


def sqrt(a):
    return _w(np.sqrt(a))


def sum(a, axis=None):  # noqa: A001 - CuPy's name
    return _w(np.sum(np.asarray(a), axis=axis))


def abs(a):  # noqa: A001
    return _w(np.abs(a))


def mean(a):
    return _w(np.mean(np.asarray(a)))


def conj(a):
    return _w(np.conj(a))


def pad(a, w, mode="constant"):
    return _w(np.pad(np.asarray(a), w, mode=mode))


def transpose(a, axes):
    return _w(np.transpose(np.asarray(a), axes))


def reshape(a, s):
    return _w(np.reshape(np.asarray(a), s))


def matmul(a, b):
    return _w(np.matmul(a, b))


def stack(a, axis=0):
    return _w(np.stack([np.asarray(x) for x in a], axis=axis))


def meshgrid(*a, **k):
    return [_w(x) for x in np.meshgrid(*[np.asarray(x) for x in a], **k)]


def all(a, axis=None):  # noqa: A001
    return _w(np.all(np.asarray(a), axis=axis))


def asnumpy(a):
    return np.array(a)


def from_dlpack(t):
    return _w(np.from_dlpack(t))


class _linalg:
    @staticmethod
    def norm(a):
        return _w(np.linalg.norm(np.asarray(a)))


linalg = _linalg()


class _fft:
    @staticmethod
    def fftn(a, axes=None):
        # single-precision input stays single precision, as with cuFFT
        return _w(_sfft.fftn(np.asarray(a), axes=axes))


fft = _fft()


class _Pool:
    def free_all_blocks(self):
        pass


_default_memory_pool = _Pool()


def get_default_memory_pool():
    return _default_memory_pool


class _Stream:
    def synchronize(self):
        pass


class _Event:
    def record(self):
        pass

    def synchronize(self):
        pass


cuda = types.SimpleNamespace(Stream=types.SimpleNamespace(null=_Stream()), Event=_Event,
                             get_elapsed_time=lambda a, b: 0.0)


def fuse(*dargs, **dkw):
    """cp.fuse: run the function; complex64 stays complex64 (CuPy casts 0-d
    operands like scalars)."""
    def deco(f):
        def run(*args):
            out = f(*args)
            if builtins.any(isinstance(a, np.ndarray) and a.ndim > 0 and a.dtype == np.complex64 for a in args):
                out = np.asarray(out).astype(np.complex64, copy=False)
            return _w(out)
        run.__name__ = getattr(f, "__name__", "fused")
        return run
    if dargs and callable(dargs[0]) and not dkw:
        return deco(dargs[0])
    return deco


# --------------------------------------------------------------------------
# kernels: the reference's CUDA-C strings compiled for the CPU
# --------------------------------------------------------------------------
_lib = None
_manifest = None


def _load():
    global _lib, _manifest
    if _lib is None:
        so = os.path.join(_REF, "librefkernels.so")
        if not os.path.exists(so):
            raise RuntimeError("reference kernels not built: run python oracle/build_ref.py")
        _lib = ctypes.CDLL(so)
        _manifest = json.load(open(os.path.join(_REF, "kernels.json")))
    return _lib, _manifest


_CT = {"int": ctypes.c_int, "long long": ctypes.c_longlong, "float": ctypes.c_float, "double": ctypes.c_double,
       "bool": ctypes.c_bool}


def _find(src, name):
    lib, man = _load()
    cands = [m for m in man if m["kind"] == "raw" and (m["var"] == name or m["symbol"].endswith("__" + name))]
    for m in cands:
        return m
    raise KeyError(name)


def _ptr(a):
    a = np.asarray(a)
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("kernel argument must be contiguous")
    return ctypes.c_void_p(a.ctypes.data)


class RawKernel:
    """cp.RawKernel(src, name): launches the compiled reference kernel."""

    _by_src: dict = {}

    def __init__(self, src, name, **kw):
        lib, man = _load()
        self.name = name
        # the same source may be registered by several modules; match on the
        # (whitespace-normalised) source text via the manifest order
        key = " ".join(src.split())
        self.meta = RawKernel._by_src.get(key)
        if self.meta is None:
            try:
                self.meta = _match_source(src, name)
            except KeyError:            # off the DDA path: constructible, not callable
                self.fn = None
                return
            RawKernel._by_src[key] = self.meta
        self.fn = getattr(lib, self.meta["symbol"])

    def __call__(self, grid, block, args):
        if self.fn is None:
            raise NotImplementedError(f"kernel {self.name} is not part of the emulated path")
        ps = self.meta["params"]
        if len(ps) != len(args):
            raise TypeError(f"{self.name}: expected {len(ps)} arguments")
        cargs = [ctypes.c_uint(int(grid[0])), ctypes.c_uint(int(block[0]))]
        keep = []
        for p, a in zip(ps, args):
            if p["pointer"]:
                arr = np.asarray(a)
                keep.append(arr)
                cargs.append(_ptr(arr))
            else:
                base = p["ctype"].replace("const", "").strip()
                cargs.append(_CT[base](a.item() if isinstance(a, np.ndarray) else a))
        self.fn(*cargs)


_SOURCES: dict = {}


def register_sources(mapping):
    """(module, var) -> source text, from the reference files (for matching)."""
    _SOURCES.update(mapping)


def _match_source(src, name):
    lib, man = _load()
    key = " ".join(src.split())
    for m in man:
        s = _SOURCES.get((m["module"], m["var"]))
        if s is not None and " ".join(s.split()) == key:
            return m
    return _find(src, name)


class ElementwiseKernel:
    """cp.ElementwiseKernel(in, out, body, name): element loop compiled from
    the reference's body; raw outputs are filled through a contiguous buffer."""

    def __init__(self, in_params, out_params, body, name, **kw):
        lib, man = _load()
        key = " ".join(body.split())
        self.meta = None
        for m in man:
            s = _SOURCES.get((m["module"], m["var"]))
            if m["kind"] == "elementwise" and s is not None and " ".join(s.split()) == key:
                self.meta = m
        self.name = name
        if self.meta is None:           # off the DDA path: constructible, not callable
            self.fn = None
            return
        self.fn = getattr(lib, self.meta["symbol"])
        self.n_in = builtins.sum(1 for p in self.meta["params"] if not p["pointer"])

    def __call__(self, *args, size=None):
        if self.fn is None:
            raise NotImplementedError(f"kernel {self.name} is not part of the emulated path")
        ps = self.meta["params"]
        ins, outs = args[:self.n_in], args[self.n_in:]
        cargs = [ctypes.c_longlong(int(size))]
        for p, a in zip(ps[:self.n_in], ins):
            cargs.append(_CT[p["ctype"]](a))
        bufs = []
        for p, o in zip(ps[self.n_in:], outs):
            dt = np.complex64 if "float>" in p["ctype"] else (np.complex128 if "double>" in p["ctype"] else None)
            buf = np.zeros(int(size), dtype=dt)
            bufs.append((buf, o))
            cargs.append(ctypes.c_void_p(buf.ctypes.data))
        self.fn(*cargs)
        for buf, o in bufs:
            np.asarray(o)[...] = buf.reshape(np.asarray(o).shape)
