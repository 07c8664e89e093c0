"""The reference's call surface, backed by the engine.

Same names, argument meanings, return tuples and errors as the reference's
Python functions (Gpbicgstab.py, ExcitedField.py, ddaforgit.py), so callers
of that path can switch imports.  Arrays may be NumPy, torch or any
DLPack-capable device array; results are new torch CUDA tensors owned by the
caller (the reference returns new CuPy arrays).
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import (DDAOperator, Preconditioner, as_device, _device, fft_lengths, green_octant, solve_many,
                     cross_sections, SolveInfo)

_C64, _C128 = torch.complex64, torch.complex128


def _reference_octant_dims(nx, ny, nz):
    return (nx + 1, ny + 1, nz + 1, 6)


def generate_interaction_row(nx, ny, nz, k, lattice_spacing, reduced=True, double_precision=False):
    """FFT(-G) of the 2n-embedded Green's tensor (ddaforgit.py:1046-1080).

    reduced=True returns the (nx+1,ny+1,nz+1,6) octant; reduced=False the full
    (2nx,2ny,2nz,6) spectrum expanded from it by the mirror rule."""
    dt = _C128 if double_precision else _C64
    Ls = fft_lengths((nx, ny, nz), _C128, exact=True)
    oct_ = green_octant((nx, ny, nz), k, lattice_spacing, Ls, 1.0, dt, layout="reference")
    if reduced:
        return oct_
    return expand_octant(oct_, Ls)


def expand_octant(oct_, Ls):
    """Full (Lx,Ly,Lz,6) spectrum from the octant: index i > L/2 reads L - i,
    xy/xz/yz flip sign when exactly one index of the pair is mirrored
    (Gpbicgstab.py:192-211)."""
    dev = oct_.device
    idx, flip = [], []
    for Ln in Ls:
        i = torch.arange(Ln, device=dev)
        f = i > Ln // 2
        idx.append(torch.where(f, Ln - i, i))
        flip.append(f)
    full = oct_[idx[0]][:, idx[1]][:, :, idx[2]].clone()
    fx, fy, fz = flip[0][:, None, None], flip[1][None, :, None], flip[2][None, None, :]
    for comp, (a, b) in ((1, (fx, fy)), (2, (fx, fz)), (4, (fy, fz))):
        s = torch.where(a != b, -1.0, 1.0).to(full.real.dtype)
        full[..., comp] = full[..., comp] * s
    return full


def prepare_interaction_matrices(grid_size, k, refract_mult, x_expansion, y_expansion, z_expansion, alpha_array,
                                 lattice_spacing, reduced=True, is_2d=False, cutoff=False, double_precision=False):
    """(inv_alpha, mask, interaction_matrix, preconditioner) as in
    ddaforgit.py:1085-1159.  The reference's preconditioner builders
    (pre_preconditioner / circulant_approximation, :1118-1136) are not part
    of it; the preconditioner returned here is the engine's
    (``engine.Preconditioner``: the inverse of the occupancy-weighted
    circulant approximation of A) as a (L/2+1, L/2+1, L/2+1, 6) octant in the
    reference's layout on the interaction grid L (2n where compiled, else the
    next compiled length), the shape of the interaction octant.
    ``refract_mult`` and the expansions size the reference's missing builder
    and are accepted and ignored; is_2d returns None."""
    dt = _C128 if double_precision else _C64
    dev = _device()
    a = as_device(alpha_array, dt, dev)
    if cutoff:
        a = torch.where(a.abs() < 1.0, torch.zeros_like(a), a)
    nz_ = a != 0
    inv_alpha = torch.where(nz_, 1.0 / torch.where(nz_, a, torch.ones_like(a)), torch.zeros_like(a))
    mask = nz_
    nx, ny, nz = grid_size
    G = generate_interaction_row(nx, ny, nz, k, lattice_spacing, reduced=reduced, double_precision=double_precision)
    pre = None
    if not is_2d and bool(mask.any()):
        pre = Preconditioner(inv_alpha=inv_alpha.to(_C128), k=k, d=lattice_spacing,
                             device=dev).reference_octant(dt)
    return inv_alpha, mask, G, pre


def _inv_alpha_box(alpha_inv, nx, ny, nz, dt, dev):
    t = as_device(alpha_inv, dt, dev)
    if t.numel() == 3 * nx * ny * nz:          # the reference's repeat(inv_alpha, 3) form
        t = t.reshape(-1)[::3].contiguous()
    if t.numel() != nx * ny * nz:
        raise ValueError(f"inverse polarizability size {t.numel()} doesn't match grid {(nx, ny, nz)}")
    return t.reshape(nx, ny, nz)


def _mask_tensor(mask, ia):
    if isinstance(mask, torch.Tensor):
        return mask.to(ia.device).reshape(ia.shape).bool()
    return as_device(mask, torch.bool, ia.device).reshape(ia.shape)


# Operators built from the reference's arrays, cached so that a caller who
# loops on interaction_mult / solve_gpbicgstab with the same device arrays
# (as the reference's callers do) pays the octant layout conversion, the
# scratch allocation and the mask check once.  Only arrays the engine reads
# in place (device arrays of the compute dtype) are cached, keyed by address,
# shape, dtype and torch's in-place version counter; an entry keeps those
# arrays alive, so an address cannot be reused while it is cached.  Arrays
# changed in place by a library other than torch between calls are not
# detected: pass new arrays, or call clear_operator_cache().
_OP_CACHE: "OrderedDict" = None
_OP_CACHE_SIZE = 4


def clear_operator_cache():
    """Drop every cached operator."""
    global _OP_CACHE
    _OP_CACHE = None


def _in_place(orig, t):
    """Whether the device tensor t reads orig's memory (no copy was made)."""
    if isinstance(orig, torch.Tensor):
        return orig.is_cuda and orig.data_ptr() == t.data_ptr()
    cai = getattr(orig, "__cuda_array_interface__", None)
    return cai is not None and cai["data"][0] == t.data_ptr()


def _key(t):
    return (t.data_ptr(), tuple(t.shape), t.dtype, t._version)


def _op_from_reference(interaction_matrix, alpha_inv, nx, ny, nz, dt, mask=None, ia_tag=None, hold=None):
    """Operator of the reference's arrays (cached, see above).  ia_tag, when
    given, identifies inv_alpha in the cache instead of its address (for
    arrays the wrapper derives itself from a mask or a constant); ``hold``
    is kept alive with the entry (the array the tag's address belongs to)."""
    global _OP_CACHE
    from collections import OrderedDict
    dev = _device()
    G = as_device(interaction_matrix, dt, dev)
    if tuple(G.shape) != _reference_octant_dims(nx, ny, nz):
        raise ValueError(f"interaction matrix shape {tuple(G.shape)} != {_reference_octant_dims(nx, ny, nz)}")
    if ia_tag is not None and _OP_CACHE is not None and _in_place(interaction_matrix, G):
        ent = _OP_CACHE.get((_key(G), ia_tag, (nx, ny, nz), dt))
        if ent is not None:
            return ent["op"]
    ia = _inv_alpha_box(alpha_inv() if callable(alpha_inv) else alpha_inv, nx, ny, nz, dt, dev)
    if ia_tag is not None:
        cacheable = _in_place(interaction_matrix, G)
        key = (_key(G), ia_tag, (nx, ny, nz), dt) if cacheable else None
    else:
        cacheable = _in_place(interaction_matrix, G) and _in_place(alpha_inv, ia)
        key = (_key(G), _key(ia), (nx, ny, nz), dt) if cacheable else None
    if _OP_CACHE is None:
        _OP_CACHE = OrderedDict()
    ent = _OP_CACHE.get(key) if key is not None else None
    if ent is None:
        op = DDAOperator(ia, 1.0, 1.0, dtype=dt, L_=(2 * nx, 2 * ny, 2 * nz), ghat=G, device=dev)
        ent = {"op": op, "arrays": (G, ia, hold), "mask": None}
        if key is not None:
            _OP_CACHE[key] = ent
            while len(_OP_CACHE) > _OP_CACHE_SIZE:
                _OP_CACHE.popitem(last=False)
    elif key is not None:
        _OP_CACHE.move_to_end(key)
    if mask is not None:
        m = _mask_tensor(mask, ent["op"].inv_alpha)
        mk = _key(m) if _in_place(mask, m) else None
        if mk is None or mk != ent["mask"]:
            if not torch.equal(m, ent["op"].inv_alpha != 0):
                raise ValueError("mask must equal (inv_alpha != 0), as prepare_interaction_matrices builds it")
            ent["mask"] = mk
            ent["mask_ref"] = m
    return ent["op"]


def interaction_mult(in_array, out_array, interaction_matrix, alpha_inv, mask, chunk_params, nx, ny, nz,
                     dtype=_C64):
    """A.x = alpha_inv*x - mask*conv(x) (Gpbicgstab.py:828-830), flattened
    to 3N like the reference.  out_array and chunk_params are accepted and
    ignored (the engine needs no chunking)."""
    op = _op_from_reference(interaction_matrix, alpha_inv, nx, ny, nz, dtype, mask)
    return op.matvec(in_array).reshape(-1)


def fft_matvec(in_array, out_array, matrix, mask, chunk_params, nx, ny, nz, dtype=_C64):
    """mask * IFFT[Ghat FFT(pad x)] cropped (Gpbicgstab.py:742-772), 3N flat."""
    dev = _device()
    m = as_device(mask, torch.bool, dev).reshape(nx, ny, nz)
    tag = ("mask",) + _key(m) if _in_place(mask, m) else None
    op = _op_from_reference(matrix, lambda: torch.where(m, torch.ones((), dtype=dtype, device=dev),
                                                        torch.zeros((), dtype=dtype, device=dev)),
                            nx, ny, nz, dtype, ia_tag=tag, hold=m)
    return op.conv_masked(in_array).reshape(-1)


def _pre_from_reference(preconditioner, ia):
    if isinstance(preconditioner, Preconditioner):
        return preconditioner
    if preconditioner is None:
        raise ValueError("precon=True needs a preconditioner (prepare_interaction_matrices returns one)")
    return Preconditioner(inv_alpha=ia, octant=preconditioner, device=ia.device)


def fft_matvec3(in_array, out_array, preconditioner, mask, chunk_params, nx, ny, nz, precon, dtype=_C64):
    """Preconditioner application M x = mask * IFFT[P FFT(pad x)] on the
    octant's grid 2 (extent - 1), cropped (Gpbicgstab.py:633-668); the input
    unchanged (flattened) when precon is False.  out_array and chunk_params
    are accepted and ignored."""
    if not precon:
        return in_array.reshape(-1) if hasattr(in_array, "reshape") else np.ravel(in_array)
    dev = _device()
    m = as_device(mask, torch.bool, dev).reshape(nx, ny, nz)
    ia = torch.where(m, torch.ones((), dtype=_C128, device=dev), torch.zeros((), dtype=_C128, device=dev))
    return _pre_from_reference(preconditioner, ia).apply(in_array, dtype).reshape(-1)


def E_field_solver(polarization, interaction_matrix, grid_size, dtype=_C64):
    """Excited field IFFT[FFT(-A) FFT(P)] on the lattice, (nx,ny,nz,3), no
    mask and no alpha term (ExcitedField.py:129-195).  Raises ValueError on a
    size mismatch like the reference (:143-152)."""
    nx, ny, nz = grid_size
    expected = nx * ny * nz * 3
    size = polarization.numel() if isinstance(polarization, torch.Tensor) else np.size(polarization)
    if size != expected:
        raise ValueError(f"Polarization size {size} doesn't match expected size {expected}")
    dev = _device()
    op = _op_from_reference(interaction_matrix, lambda: torch.ones((nx, ny, nz), dtype=dtype, device=dev),
                            nx, ny, nz, dtype, ia_tag=("ones",))
    return op.conv(polarization)


def solve_gpbicgstab(grid_size, inv_alpha, interaction_matrix, preconditioner, E_inc, mask, ratio, max_iter,
                     target=1e-5, initial_p=None, is_2d=False, precon=True, dtype=_C64):
    """GPBiCGSTAB solve of A.P = E_inc*mask (Gpbicgstab.py:879-1201).

    Returns (iters, P (nx,ny,nz,3), lowest_norm/initial, first_norm/initial)
    with the reference's codes: i+1 when converged, max_iter when not,
    -(i+1) on NaN or stagnation.  The reference computes in complex64; pass
    dtype=torch.complex128 for the FP64 solve it imports from a missing
    module.  precon=True runs the reference's right-preconditioned
    recurrence with ``preconditioner`` (an octant in the reference's
    (hx,hy,hz,6) layout read on the grid 2 (extent - 1), as fft_matvec3
    reads it, or an ``engine.Preconditioner``); is_2d raises
    NotImplementedError."""
    if is_2d:
        raise NotImplementedError("the 2D preconditioned path is not part of the engine")
    nx, ny, nz = grid_size
    op = _op_from_reference(interaction_matrix, inv_alpha, nx, ny, nz, dtype, mask)
    pre = _pre_from_reference(preconditioner, op.inv_alpha.to(_C128)) if precon else None
    P, info = op.solve(E_inc, tol=target, max_iter=max_iter, ratio=ratio, preconditioner=pre)
    return info.iters, P, info.lowest_rel, info.first_rel


def Gpbicgstab(A, E_inc, tol=1e-5, maxiter=2000, ratio=100.0, precision=None, preconditioner=None):
    """Short form: solve A.P = E_inc for a DDAOperator A; returns (P, iters).
    ``preconditioner`` (None, True or an ``engine.Preconditioner``) selects
    the precon=True recurrence."""
    P, info = A.solve(E_inc, tol=tol, max_iter=maxiter, ratio=ratio, precision=precision,
                      preconditioner=preconditioner)
    return P, info.iters


def run_solver(grid_size, k, alpha_array, lattice_spacing, x_expansion, y_expansion, z_expansion, refract_mult,
               E_inc, precon=True, max_iter=20000, double=False, ratio=0):
    """prepare_interaction_matrices + solve_gpbicgstab with ratio forced to
    100, returning (iters, P, lowest_rel) (ddaforgit.py:1174-1210); errors
    are re-raised as RuntimeError("Solver failed: ...")."""
    try:
        inv_alpha, mask, G, pre = prepare_interaction_matrices(grid_size, k, refract_mult, x_expansion,
                                                               y_expansion, z_expansion, alpha_array,
                                                               lattice_spacing, double_precision=double)
        ratio = 100
        r = solve_gpbicgstab(grid_size, inv_alpha, G, pre, E_inc, mask, ratio, max_iter, precon=precon,
                             dtype=_C128 if double else _C64)
        return r[0], r[1], r[2]
    except Exception as e:  # noqa: BLE001 - same contract as the reference wrapper
        raise RuntimeError(f"Solver failed: {str(e)}")
