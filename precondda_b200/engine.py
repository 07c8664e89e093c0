"""Device-resident DDA operator and solvers on top of the C ABI.

``DDAOperator`` holds, for one geometry on one GPU, the FFT'd interaction
tensor (built once per (grid, kd) by the engine's Green kernels), the inverse
polarizability and the transform scratch.  Its methods call the engine's
sm_100a kernels through ``libdda_b200.so``; PyTorch only provides device
memory and the current stream.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib as L

_C64, _C128 = torch.complex64, torch.complex128


def _dt_code(dtype) -> int:
    if dtype == _C64:
        return L.DDA_C64
    if dtype == _C128:
        return L.DDA_C128
    raise TypeError(f"dtype must be complex64 or complex128, got {dtype}")


def _device(device=None) -> torch.device:
    if device is None:
        if not torch.cuda.is_available():
            raise RuntimeError("the DDA engine needs a CUDA device; none is available")
        return torch.device("cuda", torch.cuda.current_device())
    d = torch.device(device)
    if d.type != "cuda":
        raise RuntimeError("the DDA engine runs on CUDA devices only")
    return torch.device("cuda", d.index if d.index is not None else torch.cuda.current_device())


def as_device(x, dtype, device) -> torch.Tensor:
    """Contiguous device tensor of ``dtype`` from a torch tensor, any
    DLPack-capable array (CuPy, JAX, ...) or anything NumPy accepts."""
    if not isinstance(x, torch.Tensor):
        if hasattr(x, "__dlpack__") and not isinstance(x, np.ndarray):
            x = torch.from_dlpack(x)
        else:
            x = torch.from_numpy(np.ascontiguousarray(np.asarray(x)))
    return x.to(device=device, dtype=dtype).contiguous()


def stream_handle(device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def free_device_bytes(device=None) -> int:
    """Device memory that new pools and workspaces can have: torch's cached
    blocks, the engine context's cached solver workspaces and the freed
    blocks the engine keeps in the device's stream-ordered pool (the context
    sets that pool's release threshold to keep them) are handed back first,
    so none of them counts as used."""
    dev = _device(device)
    torch.cuda.synchronize(dev)
    torch.cuda.empty_cache()
    L.context(dev.index).trim()
    free, _ = torch.cuda.mem_get_info(dev)
    return int(free)


_compiled_cache: dict[int, list] = {}


def compiled_fft_lengths(dtype=_C128) -> list:
    code = _dt_code(dtype)
    if code not in _compiled_cache:
        lib = L.lib()
        _compiled_cache[code] = [n for n in range(2, 1025, 2) if lib.dda_fft_length_ok(n, code)]
    return _compiled_cache[code]


def fft_lengths(shape, dtype=_C128, exact=False):
    """FFT lengths (Lx,Ly,Lz): the smallest compiled length >= 2n per axis
    (exactly 2n when ``exact``, as the reference's octant layout needs)."""
    sizes = compiled_fft_lengths(dtype)
    out = []
    for n in shape:
        if exact:
            if 2 * n not in sizes:
                raise ValueError(f"no compiled FFT length 2*{n}={2 * n}; compiled lengths: {sizes}")
            out.append(2 * n)
        else:
            cand = [s for s in sizes if s >= 2 * n]
            if not cand:
                raise ValueError(f"box axis {n} too large (largest FFT length {sizes[-1]})")
            out.append(cand[0])
    return tuple(out)


def green_octant(shape, k, d, L_=None, scale=1.0, dtype=_C128, device=None, layout="reference") -> torch.Tensor:
    """scale * FFT(-G) on the octant (Lx/2+1, Ly/2+1, Lz/2+1), computed in
    FP64 by the engine (generate_interaction_row, ddaforgit.py:1046-1080).
    layout "reference": (hx,hy,hz,6) as the reference stores it;
    "engine": (6,hx,hy,hz) as the engine's kernels read it."""
    dev = _device(device)
    nx, ny, nz = (int(v) for v in shape)
    Lx, Ly, Lz = L_ if L_ is not None else fft_lengths(shape, _C128, exact=False)
    h = (Lx // 2 + 1, Ly // 2 + 1, Lz // 2 + 1)
    eng = layout == "engine"
    out = torch.empty((6,) + h if eng else h + (6,), dtype=dtype, device=dev)
    ctx = L.context(dev.index)
    with torch.cuda.device(dev):
        p128 = out.data_ptr() if dtype == _C128 else None
        p64 = out.data_ptr() if dtype == _C64 else None
        L.check(L.lib().dda_green_build(ctx.handle, nx, ny, nz, Lx, Ly, Lz, float(k), float(d), float(scale),
                                        L.GHAT_ENGINE if eng else L.GHAT_REFERENCE, p128, p64,
                                        stream_handle(dev)))
    return out


def green_octant_pair(shape, k, d, L_, scale, device=None):
    """Engine-layout octant in complex128 and complex64 from one FP64 build."""
    dev = _device(device)
    nx, ny, nz = (int(v) for v in shape)
    Lx, Ly, Lz = L_
    h = (Lx // 2 + 1, Ly // 2 + 1, Lz // 2 + 1)
    g128 = torch.empty((6,) + h, dtype=_C128, device=dev)
    g64 = torch.empty((6,) + h, dtype=_C64, device=dev)
    ctx = L.context(dev.index)
    with torch.cuda.device(dev):
        L.check(L.lib().dda_green_build(ctx.handle, nx, ny, nz, Lx, Ly, Lz, float(k), float(d), float(scale),
                                        L.GHAT_ENGINE, g128.data_ptr(), g64.data_ptr(), stream_handle(dev)))
    return g128, g64


def ghat_to_engine(ghat_ref: torch.Tensor) -> torch.Tensor:
    """(hx,hy,hz,6) reference-layout octant -> (6,hx,hy,hz) engine layout."""
    dev = ghat_ref.device
    hx, hy, hz, six = ghat_ref.shape
    out = torch.empty((6, hx, hy, hz), dtype=ghat_ref.dtype, device=dev)
    ctx = L.context(dev.index)
    with torch.cuda.device(dev):
        L.check(L.lib().dda_ghat_to_engine(ctx.handle, _dt_code(ghat_ref.dtype), hx, hy, hz,
                                           ghat_ref.contiguous().data_ptr(), out.data_ptr(), stream_handle(dev)))
    return out


def precond_lengths(shape, dtype=_C128):
    """The cheapest preconditioner grid: the smallest compiled FFT length >= n
    per axis (the circulant folded onto the box's own period, about a third
    of a matvec to apply).  It works well at moderate contrast; at |m| >~ 3
    the unfolded grid (the operator's, >= 2n, the default) is far more
    robust (64^3 sphere, m = 3.5+0.05i: 3.0k -> 3.1k iterations folded,
    -> 0.64k unfolded)."""
    sizes = compiled_fft_lengths(dtype)
    out = []
    for n in shape:
        cand = [s for s in sizes if s >= n]
        if not cand:
            raise ValueError(f"box axis {n} too large for a preconditioner grid (largest {sizes[-1]})")
        out.append(cand[0])
    return tuple(out)


class Preconditioner:
    """Right preconditioner M of the reference's precon=True GPBiCGSTAB
    (Gpbicgstab.py:1002-1199):

        M x = mask * IFFT[ P . FFT(pad x) ]  on the grid L >= n, cropped

    applied like fft_matvec3 (Gpbicgstab.py:633-668).  Built by the engine
    (``dda_precond_build``) as the inverse of the occupancy-weighted
    circulant approximation of ``op`` on the grid ``L_`` (default: the
    operator's FFT grid; ``precond_lengths`` gives the cheaper folded one) --
    the reference's own builders are not part of it
    (ddaforgit.py:1118-1136) -- or wrapped around a given octant in
    the reference's (L/2+1, L/2+1, L/2+1, 6) layout (``octant=``; its grid is
    2 (extent - 1) per axis, as fft_matvec3 reads it).
    """

    def __init__(self, op=None, L_=None, *, inv_alpha=None, k=None, d=None, octant=None, device=None,
                 dtypes=(_C128, _C64)):
        if op is not None:
            dev = op.device
            ia = op.twin(_C128).inv_alpha if op.dtype != _C128 else op.inv_alpha
            k, d = op.k, op.d
        else:
            dev = _device(device)
            ia = as_device(inv_alpha, _C128, dev)
        if ia.dim() != 3:
            raise ValueError("inv_alpha must have shape (nx, ny, nz)")
        self.device = dev
        self.shape = tuple(int(v) for v in ia.shape)
        self._ia = {_C128: ia}
        self._ctx = L.context(dev.index)
        if octant is not None:
            o = as_device(octant, octant.dtype if isinstance(octant, torch.Tensor) and octant.is_complex()
                          else _C128, dev)
            if o.dim() != 4 or o.shape[3] != 6:
                raise ValueError("preconditioner octant must have shape (hx, hy, hz, 6)")
            self.L = tuple(2 * (int(h) - 1) for h in o.shape[:3])
            for n, Ln in zip(self.shape, self.L):
                if Ln < n:
                    raise ValueError(f"preconditioner grid {self.L} smaller than the box {self.shape}")
            self._eng = {o.dtype: ghat_to_engine(o)}
        else:
            if k is None or d is None:
                raise ValueError("building a preconditioner needs k and d (or an operator)")
            if L_ is None:
                L_ = op.L if op is not None else fft_lengths(self.shape, _C128)
            self.L = tuple(int(v) for v in L_)
            # the octant in the precisions asked for (both from one FP64 build)
            h = tuple(v // 2 + 1 for v in self.L)
            e128 = torch.empty((6,) + h, dtype=_C128, device=dev) if _C128 in dtypes else None
            e64 = torch.empty((6,) + h, dtype=_C64, device=dev) if _C64 in dtypes else None
            if e128 is None and e64 is None:
                raise ValueError("dtypes must contain complex64 and/or complex128")
            with torch.cuda.device(dev):
                L.check(L.lib().dda_precond_build(self._ctx.handle, *self.shape, *self.L, float(k), float(d),
                                                  ia.data_ptr(), L.GHAT_ENGINE,
                                                  e128.data_ptr() if e128 is not None else None,
                                                  e64.data_ptr() if e64 is not None else None,
                                                  stream_handle(dev)))
            self._eng = {t: e for t, e in ((_C128, e128), (_C64, e64)) if e is not None}
        self.scale = 1.0 / (self.L[0] * self.L[1] * self.L[2])
        self._ops = {}

    def octant(self, dtype=_C128) -> torch.Tensor:
        """Engine-layout (6,hx,hy,hz) octant in ``dtype`` (converted from the
        other precision when only that one was built)."""
        if dtype not in self._eng:
            src = self._eng[_C128] if _C128 in self._eng else next(iter(self._eng.values()))
            self._eng[dtype] = src.to(dtype)
        return self._eng[dtype]

    def reference_octant(self, dtype=_C64) -> torch.Tensor:
        """(hx,hy,hz,6) octant, the layout the reference's solver takes."""
        return self.octant(dtype).permute(1, 2, 3, 0).contiguous()

    def _op(self, dtype):
        if dtype not in self._ops:
            if dtype not in self._ia:
                self._ia[dtype] = self._ia[_C128].to(dtype)
            h = C.c_void_p()
            with torch.cuda.device(self.device):
                L.check(L.lib().dda_precond_op_create(self._ctx.handle, _dt_code(dtype), *self.shape, *self.L,
                                                      self.octant(dtype).data_ptr(), self.scale,
                                                      self._ia[dtype].data_ptr(), C.byref(h)))
            self._ops[dtype] = h
        return self._ops[dtype]

    def apply(self, x, dtype=None) -> torch.Tensor:
        """M x (fft_matvec3 with precon=True), (nx,ny,nz,3)."""
        if dtype is None:
            dtype = x.dtype if isinstance(x, torch.Tensor) and x.is_complex() else _C128
        xv = as_device(x, dtype, self.device)
        if xv.numel() != int(np.prod(self.shape)) * 3:
            raise ValueError(f"vector size {xv.numel()} doesn't match the box {self.shape}")
        xv = xv.reshape(*self.shape, 3)
        y = torch.empty_like(xv)
        with torch.cuda.device(self.device):
            L.check(L.lib().dda_matvec(self._op(dtype), L.MV_CONV_MASKED, xv.data_ptr(), y.data_ptr(), None,
                                       stream_handle(self.device)))
        return y

    def __del__(self):
        try:
            for h in getattr(self, "_ops", {}).values():
                L.lib().dda_op_destroy(h)
        except Exception:
            pass


@dataclass
class SolveInfo:
    """Outcome of one solve (mirrors the reference's return tuple)."""
    iters: int
    status: str
    lowest_rel: float
    first_rel: float
    true_relres: float = float("nan")
    outer: int = 0
    resets: int = 0
    extra: dict = field(default_factory=dict)


_STATUS = {L.DDA_OK: "converged", L.DDA_NOT_CONVERGED: "max_iter", L.DDA_ERR_NAN: "nan_or_stagnation"}


def _info(r: L.dda_result) -> SolveInfo:
    return SolveInfo(int(r.iters), _STATUS.get(r.status, str(r.status)), float(r.lowest_rel), float(r.first_rel),
                     float(r.true_relres), int(r.outer), int(r.resets))


class DDAOperator:
    """A = diag(1/alpha) + off-diagonal dipole interactions of one lattice.

    Parameters
    ----------
    inv_alpha : (nx,ny,nz) complex, 0 outside the scatterer
    k, d      : wave number and lattice spacing (same length unit)
    dtype     : complex64 or complex128 for vectors and the tensor
    L         : FFT lengths (default: smallest compiled >= 2n)
    ghat      : optional precomputed octant (e.g. the reference's
                (nx+1,ny+1,nz+1,6) array); ``ghat_scale`` multiplies it inside
                the kernels (default 1/(Lx Ly Lz) for an unscaled FFT(-G)).
    """

    def __init__(self, inv_alpha, k, d, dtype=_C128, L_=None, ghat=None, ghat_scale=None, device=None,
                 with_twin=False):
        self.device = _device(device)
        self.dtype = dtype
        self.k = float(k)
        self.d = float(d)
        self.inv_alpha = as_device(inv_alpha, dtype, self.device)
        if self.inv_alpha.dim() != 3:
            raise ValueError("inv_alpha must have shape (nx, ny, nz)")
        self.shape = tuple(int(s) for s in self.inv_alpha.shape)
        self.nsite = int(np.prod(self.shape))
        if ghat is not None:
            if L_ is None:
                L_ = tuple(2 * n for n in self.shape)
            g_ref = as_device(ghat, dtype, self.device)
            want = (L_[0] // 2 + 1, L_[1] // 2 + 1, L_[2] // 2 + 1, 6)
            if tuple(g_ref.shape) != want:
                raise ValueError(f"interaction matrix shape {tuple(g_ref.shape)} != {want}")
            self.ghat = ghat_to_engine(g_ref)
            self.gscale = (1.0 / (L_[0] * L_[1] * L_[2])) if ghat_scale is None else float(ghat_scale)
        else:
            if L_ is None:
                L_ = fft_lengths(self.shape, dtype)
            if with_twin:
                # both precisions from one FP64 Green build
                g128, g64 = green_octant_pair(self.shape, self.k, self.d, L_, 1.0 / (L_[0] * L_[1] * L_[2]),
                                              self.device)
                self.ghat = g128 if dtype == _C128 else g64
                twin_ghat = g64 if dtype == _C128 else g128
            else:
                self.ghat = green_octant(self.shape, self.k, self.d, L_, 1.0 / (L_[0] * L_[1] * L_[2]), dtype,
                                         self.device, layout="engine")
            self.gscale = 1.0
        self.L = tuple(int(v) for v in L_)
        self._ctx = L.context(self.device.index)
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            L.check(L.lib().dda_op_create(self._ctx.handle, _dt_code(dtype), *self.shape, *self.L,
                                          self.ghat.data_ptr(), self.gscale, self.inv_alpha.data_ptr(),
                                          C.byref(h)))
        self._op = h
        self._twin = None
        if ghat is None and with_twin:
            tw = DDAOperator.__new__(DDAOperator)
            tw._init_from_engine_ghat(self, _C64 if dtype == _C128 else _C128, twin_ghat)
            self._twin = tw

    def _init_from_engine_ghat(self, other, dtype, ghat=None):
        """Precision twin of ``other`` sharing its scale; the tensor is
        ``ghat`` when given (already in ``dtype``), else ``other``'s converted."""
        self.device, self.dtype, self.k, self.d = other.device, dtype, other.k, other.d
        self.inv_alpha = other.inv_alpha.to(dtype)
        self.shape, self.nsite, self.L = other.shape, other.nsite, other.L
        self.ghat = ghat if ghat is not None else other.ghat.to(dtype)
        self.gscale = other.gscale
        self._ctx = other._ctx
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            L.check(L.lib().dda_op_create(self._ctx.handle, _dt_code(dtype), *self.shape, *self.L,
                                          self.ghat.data_ptr(), self.gscale, self.inv_alpha.data_ptr(),
                                          C.byref(h)))
        self._op = h
        self._twin = None

    def __del__(self):
        try:
            if getattr(self, "_op", None):
                L.lib().dda_op_destroy(self._op)
        except Exception:
            pass

    # -- helpers ---------------------------------------------------------
    @property
    def mask(self) -> torch.Tensor:
        return self.inv_alpha != 0

    def _vec(self, x) -> torch.Tensor:
        t = as_device(x, self.dtype, self.device)
        if t.numel() != self.nsite * 3:
            raise ValueError(f"vector size {t.numel()} doesn't match expected size {self.nsite * 3}")
        return t.reshape(*self.shape, 3)

    def _mv(self, mode, x, b=None) -> torch.Tensor:
        x = self._vec(x)
        y = torch.empty_like(x)
        bp = self._vec(b).data_ptr() if b is not None else None
        with torch.cuda.device(self.device):
            L.check(L.lib().dda_matvec(self._op, mode, x.data_ptr(), y.data_ptr(), bp, stream_handle(self.device)))
        return y

    # -- products --------------------------------------------------------
    def matvec(self, x) -> torch.Tensor:
        """A.x = inv_alpha x - mask * conv(x) (interaction_mult)."""
        return self._mv(L.MV_AX, x)

    def residual(self, b, x) -> torch.Tensor:
        """mask*b - A.x."""
        bm = self._vec(b) * self.mask[..., None]
        return self._mv(L.MV_RESIDUAL, x, bm)

    def conv(self, x) -> torch.Tensor:
        """IFFT[FFT(-G) FFT(x)] on the box, no mask (E_field_solver)."""
        return self._mv(L.MV_CONV, x)

    def conv_masked(self, x) -> torch.Tensor:
        """mask * conv(x) (fft_matvec)."""
        return self._mv(L.MV_CONV_MASKED, x)

    # -- precision twin (for mixed precision) ------------------------------
    def twin(self, dtype) -> "DDAOperator":
        """The same operator in another precision (tensor rebuilt in FP64
        and rounded, not down-converted from this one's)."""
        if dtype == self.dtype:
            return self
        if self._twin is None or self._twin.dtype != dtype:
            if self.gscale == 1.0:
                self._twin = DDAOperator(self.inv_alpha, self.k, self.d, dtype, self.L, device=self.device)
            else:
                self._twin = DDAOperator.__new__(DDAOperator)
                self._twin._init_from_engine_ghat(self, dtype)
        return self._twin

    # -- preconditioner ----------------------------------------------------
    def preconditioner(self, L_=None) -> Preconditioner:
        """The engine's circulant preconditioner of this operator on the grid
        L_ (default: this operator's FFT grid), built once."""
        want = tuple(L_) if L_ is not None else self.L
        pre = getattr(self, "_pre", None)
        if pre is None or pre.L != want:
            pre = Preconditioner(self, want)
            self._pre = pre
        return pre

    # -- solves ------------------------------------------------------------
    def solve(self, E_inc, tol=1e-5, max_iter=2000, ratio=100.0, precision=None, inner_tol=1e-4,
              max_outer=12, preconditioner=None):
        """Solve A.P = mask*E_inc from P0 = 0.

        precision: None/'native' (this operator's dtype, reference GPBiCGSTAB),
        'c64', 'c128', or 'mixed' (complex64 sweeps + FP64 refinement; P is
        complex128).  preconditioner: None, True (this operator's
        ``preconditioner()``) or a ``Preconditioner`` -- the reference's
        precon=True solve.  Returns (P, SolveInfo)."""
        P, infos = solve_many([self], [E_inc], tol=tol, max_iter=max_iter, ratio=ratio, precision=precision,
                              inner_tol=inner_tol, max_outer=max_outer, preconditioner=preconditioner)
        return P[0], infos[0]

    def cross_sections(self, P, E_inc, E0=1.0):
        return cross_sections(P, E_inc, self.inv_alpha, self.k, E0)


def matvec_batch(ops, xs, mode=L.MV_AX, bs=None):
    """[A_j x_j] for operators sharing box, FFT lengths, dtype and scale, in
    one batched launch sequence (mode: L.MV_AX, MV_RESIDUAL with bs,
    MV_CONV, MV_CONV_MASKED)."""
    ops = list(ops)
    if len(ops) != len(xs):
        raise ValueError("one vector per operator")
    _same_bucket(ops)
    o0 = ops[0]
    X = [o._vec(x) for o, x in zip(ops, xs)]
    Y = [torch.empty_like(x) for x in X]
    B = [o._vec(b) for o, b in zip(ops, bs)] if bs is not None else None
    nb = len(ops)
    arr = lambda v: (C.c_void_p * nb)(*v)
    with torch.cuda.device(o0.device):
        L.check(L.lib().dda_matvec_batch(arr([o._op.value for o in ops]), nb, int(mode),
                                         arr([x.data_ptr() for x in X]), arr([y.data_ptr() for y in Y]),
                                         arr([b.data_ptr() for b in B]) if B is not None else None,
                                         stream_handle(o0.device)))
    return Y


def _same_bucket(ops):
    o0 = ops[0]
    for o in ops[1:]:
        if o.shape != o0.shape or o.L != o0.L or o.dtype != o0.dtype or o.gscale != o0.gscale \
                or o.device != o0.device:
            raise ValueError("batched instances must share box, FFT lengths, dtype, tensor scale and device")


def _pre_list(ops, preconditioner):
    """Per-instance Preconditioner objects (sharing one grid) or None."""
    if preconditioner is None or preconditioner is False:
        return None
    if preconditioner is True:
        pres = [o.preconditioner() for o in ops]
    elif isinstance(preconditioner, Preconditioner):
        pres = [preconditioner] * len(ops)
    else:
        pres = list(preconditioner)
        if len(pres) != len(ops):
            raise ValueError("one preconditioner per operator instance")
    for p, o in zip(pres, ops):
        if not isinstance(p, Preconditioner) or p.shape != o.shape or p.L != pres[0].L:
            raise ValueError("preconditioners must be Preconditioner objects of the operators' box on one grid")
    return pres


def solve_many(ops, E_incs, tol=1e-5, max_iter=2000, ratio=100.0, precision=None, inner_tol=1e-4, max_outer=12,
               preconditioner=None):
    """Batched solve: instance j is (ops[j], E_incs[j]).  Instances may share
    an operator (many incidences) or not (many geometries of one box size).
    ``preconditioner`` (None, True, a Preconditioner or one per instance)
    selects the reference's precon=True solve; mixed precision
    preconditions its complex64 sweeps.  Returns ([P_j], [SolveInfo_j])."""
    ops = list(ops)
    if len(ops) != len(E_incs):
        raise ValueError("one incident field per operator instance")
    if not ops:
        return [], []
    _same_bucket(ops)
    o0 = ops[0]
    dev = o0.device
    nb = len(ops)
    res = (L.dda_result * nb)()
    ctx = L.context(dev.index)
    pres = _pre_list(ops, preconditioner)
    if precision in (None, "native"):
        precision = "c128" if o0.dtype == _C128 else "c64"
    if precision in ("c64", "c128"):
        dt = _C64 if precision == "c64" else _C128
        tops = [o.twin(dt) for o in ops]
        Es = [tops[j]._vec(E_incs[j]) for j in range(nb)]
        Ps = [torch.empty_like(e) for e in Es]
        inst = (L.dda_instance * nb)()
        for j in range(nb):
            inst[j].ghat = tops[j].ghat.data_ptr()
            inst[j].inv_alpha = tops[j].inv_alpha.data_ptr()
            inst[j].e_inc = Es[j].data_ptr()
            inst[j].p_out = Ps[j].data_ptr()
        t0 = tops[0]
        with torch.cuda.device(dev):
            if pres is None:
                L.check(L.lib().dda_solve_batch(ctx.handle, _dt_code(dt), *t0.shape, *t0.L, t0.gscale, inst, nb,
                                                float(tol), int(max_iter), float(ratio), res, stream_handle(dev)))
            else:
                ph = (C.c_void_p * nb)(*[p.octant(dt).data_ptr() for p in pres])
                L.check(L.lib().dda_solve_batch_pre(ctx.handle, _dt_code(dt), *t0.shape, *t0.L, t0.gscale,
                                                    *pres[0].L, pres[0].scale, ph, inst, nb, float(tol),
                                                    int(max_iter), float(ratio), res, stream_handle(dev)))
        return Ps, [_info(res[j]) for j in range(nb)]
    if precision != "mixed":
        raise ValueError("precision must be None, 'native', 'c64', 'c128' or 'mixed'")
    o64 = [o.twin(_C64) for o in ops]
    o128 = [o.twin(_C128) for o in ops]
    E128 = [o128[j]._vec(E_incs[j]) for j in range(nb)]
    P128 = [torch.empty_like(e) for e in E128]
    i64 = (L.dda_instance * nb)()
    i128 = (L.dda_instance * nb)()
    for j in range(nb):
        i64[j].ghat = o64[j].ghat.data_ptr()
        i64[j].inv_alpha = o64[j].inv_alpha.data_ptr()
        i128[j].ghat = o128[j].ghat.data_ptr()
        i128[j].inv_alpha = o128[j].inv_alpha.data_ptr()
        i128[j].e_inc = E128[j].data_ptr()
        i128[j].p_out = P128[j].data_ptr()
    t0 = o128[0]
    if o64[0].gscale != t0.gscale:
        raise ValueError("precision twins disagree on tensor scale")
    with torch.cuda.device(dev):
        if pres is None:
            L.check(L.lib().dda_solve_mixed_batch(ctx.handle, *t0.shape, *t0.L, t0.gscale, i64, i128, nb,
                                                  float(tol), float(inner_tol), int(max_iter), int(max_outer),
                                                  float(ratio), res, stream_handle(dev)))
        else:
            ph = (C.c_void_p * nb)(*[p.octant(_C64).data_ptr() for p in pres])
            L.check(L.lib().dda_solve_mixed_batch_pre(ctx.handle, *t0.shape, *t0.L, t0.gscale, *pres[0].L,
                                                      pres[0].scale, ph, i64, i128, nb, float(tol),
                                                      float(inner_tol), int(max_iter), int(max_outer), float(ratio),
                                                      res, stream_handle(dev)))
    return P128, [_info(res[j]) for j in range(nb)]


def far_field(P, d, k, directions):
    """Far-field scattering amplitude F(n) (ndir, 3) complex128 of the
    polarisation P (nx,ny,nz,3) for unit directions n:
    F = k^2 sum_j [P_j - n (n.P_j)] exp(-i k n.r_j), r_j = (i,j,k) d.
    dC_sca/dOmega = |F|^2 / |E0|^2."""
    if not isinstance(P, torch.Tensor):
        P = as_device(P, _C128, _device())
    dev = _device(P.device)
    dt = P.dtype if P.dtype in (_C64, _C128) else _C128
    P = as_device(P, dt, dev)
    if P.dim() != 4 or P.shape[3] != 3:
        raise ValueError("P must have shape (nx, ny, nz, 3)")
    dirs = np.ascontiguousarray(np.asarray(directions, dtype=np.float64).reshape(-1, 3))
    nd = dirs.shape[0]
    out = np.empty(nd * 6, dtype=np.float64)
    ctx = L.context(dev.index)
    with torch.cuda.device(dev):
        L.check(L.lib().dda_far_field(ctx.handle, _dt_code(dt), *P.shape[:3], float(d), float(k), P.data_ptr(), nd,
                                      dirs.ctypes.data_as(C.POINTER(C.c_double)),
                                      out.ctypes.data_as(C.POINTER(C.c_double)), stream_handle(dev)))
    o = out.reshape(nd, 3, 2)
    return o[..., 0] + 1j * o[..., 1]


def differential_cross_section(P, d, k, directions, E0=1.0):
    """dC_sca/dOmega = |F(n)|^2 / |E0|^2 for each direction."""
    F = far_field(P, d, k, directions)
    return (np.abs(F) ** 2).sum(axis=1) / abs(E0) ** 2


def cross_sections(P, E_inc, inv_alpha, k, E0=1.0):
    """(C_ext, C_abs, C_sca) reduced in FP64 on the device (Draine & Flatau
    1994); arrays are brought to the precision of P."""
    if not isinstance(P, torch.Tensor):
        P = as_device(P, _C128, _device())
    dev = _device(P.device)
    dt = P.dtype if P.dtype in (_C64, _C128) else _C128
    P = as_device(P, dt, dev)
    E = as_device(E_inc, dt, dev)
    ia = as_device(inv_alpha, dt, dev)
    nsite = ia.numel()
    if P.numel() != 3 * nsite or E.numel() != 3 * nsite:
        raise ValueError("P, E_inc and inv_alpha sizes disagree")
    out = (C.c_double * 3)()
    ctx = L.context(dev.index)
    with torch.cuda.device(dev):
        L.check(L.lib().dda_cross_sections(ctx.handle, _dt_code(dt), nsite, P.data_ptr(), E.data_ptr(),
                                           ia.data_ptr(), float(k), float(E0), out, stream_handle(dev)))
    return float(out[0]), float(out[1]), float(out[2])
