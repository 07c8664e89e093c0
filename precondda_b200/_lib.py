"""ctypes binding of libdda_b200.so (declared in include/dda_b200.h).

The shared library is the engine; this module only loads it, declares the
prototypes and turns status codes into Python exceptions.  There is no
fallback: if the library is missing or the device cannot be used, every entry
point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
# DDA_LIB_PATH selects an alternative build of the same library (A/B tuning).
LIB_PATH = os.environ.get("DDA_LIB_PATH") or os.path.join(_HERE, "libdda_b200.so")

DDA_C64 = 0
DDA_C128 = 1
DDA_PREC_C64, DDA_PREC_C128, DDA_PREC_MIXED = 0, 1, 2

DDA_OK = 0
DDA_ERR_BAD_SHAPE = 1
DDA_ERR_OOM = 2
DDA_NOT_CONVERGED = 3
DDA_ERR_NAN = 4
DDA_ERR_TIMEOUT = 5
DDA_ERR_CUDA = 6
DDA_ERR_ARG = 7

GHAT_REFERENCE = 0
GHAT_ENGINE = 1

MV_AX = 0
MV_RESIDUAL = 1
MV_CONV = 2
MV_CONV_MASKED = 3

# every symbol include/dda_b200.h declares
EXPORTS = (
    "dda_version", "dda_last_error", "dda_kernel_launches", "dda_ctx_create", "dda_ctx_destroy", "dda_ctx_trim",
    "dda_fft_length_ok", "dda_green_build", "dda_ghat_to_engine", "dda_op_create", "dda_op_destroy", "dda_matvec",
    "dda_matvec_noalloc", "dda_gpbicgstab", "dda_solve_batch", "dda_solve_mixed_batch", "dda_cross_sections",
    "dda_voxelize", "dda_incident_field", "dda_slots_create", "dda_slots_destroy", "dda_slots_capacity",
    "dda_slots_free_slot", "dda_slots_admit", "dda_slots_run", "dda_slots_ready", "dda_slots_poll",
    "dda_slots_release",
    "dda_far_field", "dda_matvec_batch", "dda_precond_build", "dda_precond_op_create", "dda_gpbicgstab_pre",
    "dda_solve_batch_pre", "dda_solve_mixed_batch_pre", "dda_slots_create_pre", "dda_slots_admit_pre",
    "dda_tuning_set", "dda_tuning_get",
)

DDA_TUNE_P3PIPE, DDA_TUNE_P3PIPE_1SM, DDA_TUNE_NO_FUSED_ZY, DDA_TUNE_NO_FUSED_INV, DDA_TUNE_P3PAIR = 1, 2, 4, 8, 16
DDA_TUNE_YPAIR, DDA_TUNE_ZPAIR, DDA_TUNE_FUSED, DDA_TUNE_PREFETCH = 32, 64, 128, 256


class DDAError(RuntimeError):
    """Failure reported by the engine's C ABI."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[dda status {code}] {msg}")
        self.code = code


class dda_instance(C.Structure):
    _fields_ = [("ghat", C.c_void_p), ("inv_alpha", C.c_void_p), ("e_inc", C.c_void_p), ("p_out", C.c_void_p)]


SHAPE_SPHERE, SHAPE_ELLIPSOID, SHAPE_RECTANGLE, SHAPE_CYLINDER, SHAPE_PRISM = range(5)
SHAPE_WINDOW, SHAPE_GEOMETRIC_AXES = 1, 2


class dda_shape(C.Structure):
    _fields_ = [("type", C.c_int), ("axis", C.c_int), ("sides", C.c_int), ("flags", C.c_int),
                ("center", C.c_double * 3), ("p", C.c_double * 4), ("rot", C.c_double * 9),
                ("inv_alpha", C.c_double * 2), ("win", C.c_int * 6), ("reserved", C.c_int * 2)]


class dda_result(C.Structure):
    _fields_ = [("iters", C.c_int), ("status", C.c_int), ("lowest_rel", C.c_double), ("first_rel", C.c_double),
                ("true_relres", C.c_double), ("outer", C.c_int), ("resets", C.c_int)]


_lib = None
_lock = threading.Lock()


def _declare(lib):
    vp, i, d, ll = C.c_void_p, C.c_int, C.c_double, C.c_longlong
    lib.dda_version.restype = i
    lib.dda_last_error.restype = C.c_char_p
    lib.dda_kernel_launches.restype = ll
    lib.dda_ctx_create.argtypes = [i, C.POINTER(vp)]
    lib.dda_ctx_destroy.argtypes = [vp]
    lib.dda_ctx_destroy.restype = None
    lib.dda_ctx_trim.argtypes = [vp]
    lib.dda_fft_length_ok.argtypes = [i, i]
    lib.dda_green_build.argtypes = [vp, i, i, i, i, i, i, d, d, d, i, vp, vp, vp]
    lib.dda_ghat_to_engine.argtypes = [vp, i, i, i, i, vp, vp, vp]
    lib.dda_op_create.argtypes = [vp, i, i, i, i, i, i, i, vp, d, vp, C.POINTER(vp)]
    lib.dda_op_destroy.argtypes = [vp]
    lib.dda_op_destroy.restype = None
    lib.dda_matvec.argtypes = [vp, i, vp, vp, vp, vp]
    lib.dda_matvec_noalloc.argtypes = [i, i, i, i, i, i, i, vp, d, vp, i, vp, vp, vp, vp]
    lib.dda_tuning_set.argtypes = [i, i, i, i, i, i, i, i, i]
    lib.dda_tuning_get.argtypes = [i, i, i, i, i, i, i, i, C.POINTER(C.c_int)]
    lib.dda_gpbicgstab.argtypes = [vp, vp, d, i, d, vp, C.POINTER(dda_result), vp]
    lib.dda_solve_batch.argtypes = [vp, i, i, i, i, i, i, i, d, C.POINTER(dda_instance), i, d, i, d,
                                    C.POINTER(dda_result), vp]
    lib.dda_solve_mixed_batch.argtypes = [vp, i, i, i, i, i, i, d, C.POINTER(dda_instance),
                                          C.POINTER(dda_instance), i, d, d, i, i, d, C.POINTER(dda_result), vp]
    lib.dda_cross_sections.argtypes = [vp, i, ll, vp, vp, vp, d, d, C.POINTER(d), vp]
    lib.dda_voxelize.argtypes = [vp, i, C.POINTER(dda_shape), i, i, i, i, d, C.POINTER(d), vp, vp]
    lib.dda_incident_field.argtypes = [vp, i, i, i, i, d, C.POINTER(d), C.POINTER(d), vp, vp]
    lib.dda_slots_create.argtypes = [vp, i, i, i, i, i, i, i, d, i, C.POINTER(vp)]
    lib.dda_slots_destroy.argtypes = [vp]
    lib.dda_slots_destroy.restype = None
    lib.dda_slots_capacity.argtypes = [vp]
    lib.dda_slots_free_slot.argtypes = [vp]
    lib.dda_slots_admit.argtypes = [vp, i, C.POINTER(dda_instance), C.POINTER(dda_instance), d, d, i, i, d, vp]
    lib.dda_slots_run.argtypes = [vp, i]
    lib.dda_slots_ready.argtypes = [vp]
    lib.dda_slots_poll.argtypes = [vp, C.POINTER(i), C.POINTER(dda_result), C.POINTER(i), C.POINTER(i)]
    lib.dda_slots_release.argtypes = [vp, i]
    lib.dda_slots_create_pre.argtypes = [vp, i, i, i, i, i, i, i, d, i, i, i, d, i, C.POINTER(vp)]
    lib.dda_slots_admit_pre.argtypes = [vp, i, C.POINTER(dda_instance), C.POINTER(dda_instance), vp, d, d, i, i,
                                        d, vp]
    lib.dda_far_field.argtypes = [vp, i, i, i, i, d, d, vp, i, C.POINTER(d), C.POINTER(d), vp]
    lib.dda_matvec_batch.argtypes = [C.POINTER(vp), i, i, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), vp]
    lib.dda_precond_build.argtypes = [vp, i, i, i, i, i, i, d, d, vp, i, vp, vp, vp]
    lib.dda_precond_op_create.argtypes = [vp, i, i, i, i, i, i, i, vp, d, vp, C.POINTER(vp)]
    lib.dda_gpbicgstab_pre.argtypes = [vp, vp, vp, d, i, d, vp, C.POINTER(dda_result), vp]
    lib.dda_solve_batch_pre.argtypes = [vp, i, i, i, i, i, i, i, d, i, i, i, d, C.POINTER(vp),
                                        C.POINTER(dda_instance), i, d, i, d, C.POINTER(dda_result), vp]
    lib.dda_solve_mixed_batch_pre.argtypes = [vp, i, i, i, i, i, i, d, i, i, i, d, C.POINTER(vp),
                                              C.POINTER(dda_instance), C.POINTER(dda_instance), i, d, d, i, i, d,
                                              C.POINTER(dda_result), vp]
    return lib


def lib():
    """The loaded engine library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise ImportError(f"libdda_b200.so not found at {LIB_PATH}; build it with "
                                      f"`python -m precondda_b200.build_lib` (or __graft_entry__.build())")
                _lib = _declare(C.CDLL(LIB_PATH))
    return _lib


def check(rc: int) -> int:
    """Raise DDAError for any status other than OK / NOT_CONVERGED / NAN."""
    if rc in (DDA_OK, DDA_NOT_CONVERGED, DDA_ERR_NAN):
        return rc
    msg = lib().dda_last_error()
    msg = msg.decode() if msg else ""
    if rc == DDA_ERR_BAD_SHAPE:
        raise ValueError(msg)
    if rc == DDA_ERR_OOM:
        raise MemoryError(msg)
    raise DDAError(rc, msg)


class Context:
    """Engine context bound to one CUDA device (twiddles, workspaces)."""

    def __init__(self, device: int):
        self.device = device
        h = C.c_void_p()
        check(lib().dda_ctx_create(device, C.byref(h)))
        self.handle = h

    def trim(self):
        check(lib().dda_ctx_trim(self.handle))

    def __del__(self):
        try:
            if self.handle:
                lib().dda_ctx_destroy(self.handle)
        except Exception:
            pass


_ctxs: dict[int, Context] = {}


def context(device: int) -> Context:
    with _lock:
        c = _ctxs.get(device)
    if c is None:
        c = Context(device)
        with _lock:
            _ctxs[device] = c
    return c
