"""CPU oracle for the DDA hot path -- TEST INFRASTRUCTURE ONLY.

This module restates, in complex128 NumPy/SciPy, the algorithm of the
reference DDA engine (Toastlovesjam/preconDDA) for the path

    lattice -> Green's tensor FFT -> A.P matvec -> GPBiCGSTAB
            -> cross sections / near field.

It is the checker used by ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``.  Nothing in the
product package imports it.  Every function cites the reference file:line it
follows.  Parity of this restatement is pinned by fixtures produced by running
the reference's own ``Gpbicgstab.py`` / ``ExcitedField.py`` and the Green and
polarizability code of ``ddaforgit.py`` on the CPU (``tests/golden``).

Conventions (same as the reference):
  * vectors are C-order (nx, ny, nz, 3) complex, component index fastest;
  * the FFT'd interaction tensor is stored as the reduced octant
    (nx+1, ny+1, nz+1, 6) with components (xx, xy, xz, yy, yz, zz);
  * A.x = inv_alpha * x - mask * IFFT[ FFT(-G) . FFT(pad x) ]  (cropped).
"""
from __future__ import annotations

import math
import os

import numpy as np
import scipy.fft as sfft

_WORKERS = os.cpu_count() or 1

# component order of the 6 unique entries of the symmetric 3x3 block
# (ddaforgit.py:962-968)
_PAIRS = ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))
_COMP = np.array([[0, 1, 2], [1, 3, 4], [2, 4, 5]])


# --------------------------------------------------------------------------
# polarizability  (ddaforgit.py:403-437)
# --------------------------------------------------------------------------
def calculate_alpha(refractive_index, lattice_spacing, wave_number,
                    incident_direction=None, polarization_direction=None,
                    method="LDR"):
    """Clausius-Mossotti polarizability with RR / LDR corrections.

    Follows ddaforgit.py:403-437, including the LDR quirk S = (a.e)^2
    (ddaforgit.py:432).
    """
    n = np.complex128(refractive_index)
    d = np.float64(lattice_spacing)
    k = np.float64(wave_number)
    eps = n ** 2
    alpha_cm = (3 * d ** 3 / (4 * np.pi)) * (eps - 1) / (eps + 2)
    if method == "CM":
        return alpha_cm
    rr_term = (2 / 3) * 1j * (k * d) ** 3
    if method == "RR":
        return alpha_cm / (1 + (alpha_cm / d ** 3) * (-rr_term))
    if method == "LDR":
        if incident_direction is None or polarization_direction is None:
            raise ValueError("incident_direction and polarization_direction "
                             "required for LDR method")
        a = np.asarray(incident_direction, dtype=np.float64)
        e = np.asarray(polarization_direction, dtype=np.float64)
        b1, b2, b3 = -1.891531, 0.1648469, -1.7700004
        S = np.sum(np.dot(a, e) ** 2)
        ldr = (b1 + n ** 2 * b2 + n ** 2 * b3 * S) * (k * d) ** 2
        return alpha_cm / (1 + (alpha_cm / d ** 3) * (ldr - rr_term))
    raise ValueError("method must be 'CM', 'RR', or 'LDR'")


# --------------------------------------------------------------------------
# lattice  (ddaforgit.py:439-459, 615-661, 831-857, 1626-1632)
# --------------------------------------------------------------------------
def sphere_mask(points, center, radius, epsilon=1e-7):
    """Sphere membership, ddaforgit.py:439-448."""
    dist = np.sqrt(((points - np.asarray(center)) ** 2).sum(axis=-1))
    return (dist < radius) | (np.abs(dist - radius) < epsilon)


def ellipsoid_mask(points, center, semi_axes, epsilon=1e-7, rotation=None):
    """Ellipsoid membership, ddaforgit.py:450-459.

    ``rotation`` (3x3, body->lab) is an extension: the reference ellipsoid is
    axis aligned.  With a rotation the lab offset is mapped into the body frame
    by R^T before the quadric test.
    """
    off = points - np.asarray(center)
    if rotation is not None:
        off = off @ np.asarray(rotation)
    q = off / np.asarray(semi_axes)
    dist = np.sqrt((q ** 2).sum(axis=-1))
    return dist <= 1.0 + epsilon


def voxel_centres(shape, d, offset=0.5):
    """Voxel centre coordinates (i+0.5)d, ddaforgit.py:617, 643-647."""
    axes = [(np.arange(n) + offset) * d for n in shape]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    return np.stack([X, Y, Z], axis=-1)


def trim_zero_faces(array):
    """Crop to the non-zero bounding box, pad odd sizes to even.

    ddaforgit.py:831-857.
    """
    xm = np.any(np.any(array != 0, axis=2), axis=1)
    ym = np.any(np.any(array != 0, axis=2), axis=0)
    zm = np.any(np.any(array != 0, axis=1), axis=0)
    xs, xe = np.argmax(xm), len(xm) - np.argmax(xm[::-1])
    ys, ye = np.argmax(ym), len(ym) - np.argmax(ym[::-1])
    zs, ze = np.argmax(zm), len(zm) - np.argmax(zm[::-1])
    t = array[xs:xe, ys:ye, zs:ze]
    new = tuple(s + (s % 2) for s in t.shape)
    if new != t.shape:
        out = np.zeros(new, dtype=array.dtype)
        out[tuple(slice(0, s) for s in t.shape)] = t
        return out
    return t


def incident_field(grid_size, d, k, k_direction, e_polarization):
    """E_inc = e * exp(i k.r) with r = (i,j,k) d (no 0.5 offset).

    ddaforgit.py:1612-1632.
    """
    kvec = k * np.asarray(k_direction, dtype=np.float64)
    axes = [np.arange(0, n) * d for n in grid_size]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    phase = np.exp(1j * (kvec[0] * X + kvec[1] * Y + kvec[2] * Z))
    E = np.zeros((*grid_size, 3), dtype=np.complex128)
    for j in range(3):
        E[..., j] = e_polarization[j] * phase
    return E


def sphere_lattice(n_box, radius_d):
    """Boolean occupancy of a sphere of radius ``radius_d`` (units of d)
    centred in an ``n_box``^3 box with voxel centres at (i+0.5)d.  Same test
    as ddaforgit.py:439-448 in lattice units."""
    c = n_box / 2.0
    pts = voxel_centres((n_box,) * 3, 1.0)
    return sphere_mask(pts, (c, c, c), radius_d)


# --------------------------------------------------------------------------
# Green's tensor and its FFT  (ddaforgit.py:939-1080)
# --------------------------------------------------------------------------
def _axis_offsets(n, L):
    """Signed lattice offsets of the L-point circulant embedding of an
    n-site axis.  For L == 2n this is ddaforgit.py:951-953 with the plane
    i == n zeroed (ddaforgit.py:983); for L > 2n the unused middle indices
    n..L-n are zeroed the same way."""
    i = np.arange(L)
    off = np.where(i < n, i, i - L).astype(np.float64)
    valid = (i <= n - 1) | (i >= L - n + 1)
    return off, valid


def green_embedded(nx, ny, nz, k, d, L=None):
    """G on the (Lx,Ly,Lz) circulant grid, shape (Lx,Ly,Lz,6), complex128.

    G(r) = e^{ikr}/r [k^2 (rr - I) + (ikr - 1)/r^2 (3 rr - I)]
    ddaforgit.py:979-987; origin 0 (:955-958); Nyquist planes 0 (:983).
    """
    Lx, Ly, Lz = L if L is not None else (2 * nx, 2 * ny, 2 * nz)
    ox, vx = _axis_offsets(nx, Lx)
    oy, vy = _axis_offsets(ny, Ly)
    oz, vz = _axis_offsets(nz, Lz)
    X = ox[:, None, None] * d
    Y = oy[None, :, None] * d
    Z = oz[None, None, :] * d
    valid = vx[:, None, None] & vy[None, :, None] & vz[None, None, :]
    r2 = X * X + Y * Y + Z * Z
    origin = r2 == 0
    r2s = np.where(origin, 1.0, r2)
    r = np.sqrt(r2s)
    dirs = (X / r, Y / r, Z / r)
    ikr = 1j * k * r
    expt = np.exp(ikr) / r
    f2 = (ikr - 1.0) / r2s
    G = np.zeros((Lx, Ly, Lz, 6), dtype=np.complex128)
    for c, (a, b) in enumerate(_PAIRS):
        nc = dirs[a] * dirs[b]
        delta = 1.0 if a == b else 0.0
        val = expt * (k * k * (nc - delta) + (3.0 * nc - delta) * f2)
        val = np.where(valid & ~origin, val, 0.0)
        G[..., c] = val
    return G


def generate_interaction_row(nx, ny, nz, k, lattice_spacing, reduced=True,
                             L=None):
    """FFT(-G) per component, cropped to the (Lx/2+1, Ly/2+1, Lz/2+1, 6)
    octant when ``reduced``.  ddaforgit.py:1046-1080."""
    G = green_embedded(nx, ny, nz, k, lattice_spacing, L)
    Gh = sfft.fftn(-G, axes=(0, 1, 2), workers=_WORKERS)
    if not reduced:
        return Gh
    Lx, Ly, Lz = G.shape[:3]
    return np.ascontiguousarray(Gh[:Lx // 2 + 1, :Ly // 2 + 1, :Lz // 2 + 1])


def expand_octant(Ghat_oct, L):
    """Full (Lx,Ly,Lz,3,3) FFT-domain tensor from the reduced octant using the
    mirror index 2n-i for i > n and the sign flip of xy/xz/yz when exactly one
    index of the pair is mirrored.  Gpbicgstab.py:192-232."""
    Lx, Ly, Lz = L
    def mirror(Ln):
        i = np.arange(Ln)
        m = i > Ln // 2
        return np.where(m, Ln - i, i), m
    mx, fx = mirror(Lx)
    my, fy = mirror(Ly)
    mz, fz = mirror(Lz)
    Gfull = Ghat_oct[mx][:, my][:, :, mz]          # (Lx,Ly,Lz,6)
    FX = fx[:, None, None]
    FY = fy[None, :, None]
    FZ = fz[None, None, :]
    sxy = np.where(FX != FY, -1.0, 1.0)
    sxz = np.where(FX != FZ, -1.0, 1.0)
    syz = np.where(FY != FZ, -1.0, 1.0)
    T = np.empty((Lx, Ly, Lz, 3, 3), dtype=Ghat_oct.dtype)
    T[..., 0, 0] = Gfull[..., 0]
    T[..., 1, 1] = Gfull[..., 3]
    T[..., 2, 2] = Gfull[..., 5]
    T[..., 0, 1] = T[..., 1, 0] = sxy * Gfull[..., 1]
    T[..., 0, 2] = T[..., 2, 0] = sxz * Gfull[..., 2]
    T[..., 1, 2] = T[..., 2, 1] = syz * Gfull[..., 4]
    return T


def fft_convolve(x, Ghat_oct, L=None):
    """IFFT[ Ghat . FFT(pad x) ] cropped to the box (no mask).
    Gpbicgstab.py:742-772 / ExcitedField.py:159-195."""
    nx, ny, nz = x.shape[:3]
    if L is None:
        L = (2 * nx, 2 * ny, 2 * nz)
    Lx, Ly, Lz = L
    xp = np.zeros((Lx, Ly, Lz, 3), dtype=np.complex128)
    xp[:nx, :ny, :nz] = x
    X = sfft.fftn(xp, axes=(0, 1, 2), workers=_WORKERS)
    T = expand_octant(Ghat_oct, L)
    Y = np.einsum("...ij,...j->...i", T, X)
    y = sfft.ifftn(Y, axes=(0, 1, 2), workers=_WORKERS)
    return y[:nx, :ny, :nz]


def precondition_apply(x, P_oct, mask):
    """M.x = mask * IFFT[ P . FFT(pad x) ] on the preconditioner's own grid
    (2 (octant extent - 1) per axis; x placed at the origin, the result
    cropped to the box): fft_matvec3 with optimized_dot_product_reduced_kernel,
    Gpbicgstab.py:633-668 and :36-103 (same mirror rule as the interaction
    octant)."""
    x = np.asarray(x, dtype=np.complex128)
    L = tuple(2 * (int(s) - 1) for s in P_oct.shape[:3])
    y = fft_convolve(x, P_oct, L)
    return y * np.asarray(mask, dtype=bool)[..., None]


def occupancy_weights(occ):
    """w(j) for lattice offsets j in (-n, n)^3, on the (2nx,2ny,2nz) grid
    (offset j at index j mod 2n): the fraction of occupied sites whose
    neighbour at offset j is occupied, R(j)/R(0), R the autocorrelation of the
    occupancy, averaged over the 8 axis reflections of j so the weighted
    kernel keeps the per-axis parity of G (and its octant storage)."""
    occ = np.asarray(occ, dtype=bool)
    nx, ny, nz = occ.shape
    La = (2 * nx, 2 * ny, 2 * nz)
    m = np.zeros(La)
    m[:nx, :ny, :nz] = occ
    R = np.real(sfft.ifftn(np.abs(sfft.fftn(m)) ** 2))
    R = np.clip(R, 0.0, None) / max(R[0, 0, 0], 1e-300)
    idx = [np.arange(L_) for L_ in La]
    ref = [(-i) % L_ for i, L_ in zip(idx, La)]
    W = np.zeros(La)
    for sx in (idx[0], ref[0]):
        for sy in (idx[1], ref[1]):
            for sz in (idx[2], ref[2]):
                W += R[np.ix_(sx, sy, sz)]
    return W / 8.0


def circulant_preconditioner(inv_alpha, k, d, L=None):
    """Octant (hx,hy,hz,6) of the engine's preconditioner on the L grid
    (n <= L per axis; default L = n):

        P(q) = [abar I - FFT_L(-c)(q)]^-1,   c(t) = sum_{j = t mod L} w(j) G(j)

    abar = mean inverse polarizability of the occupied sites, G the lattice
    Green tensor at offsets j in (-n, n)^3 (zero at j = 0), w the occupancy
    weights (``occupancy_weights``).  c is T. Chan's optimal circulant of the
    masked interaction operator, folded onto the L-periodic grid; applied by
    ``precondition_apply`` (which scales by 1/(Lx Ly Lz) through its
    normalised inverse FFT) it is the inverse of that circulant.  The
    reference calls preconditioner builders it does not define
    (ddaforgit.py:1118-1136); this construction is the engine's own, written
    for the reference's application format (Gpbicgstab.py:36-103, :633-668).
    """
    ia = np.asarray(inv_alpha, dtype=np.complex128)
    nx, ny, nz = ia.shape
    occ = ia != 0
    abar = ia[occ].mean() if occ.any() else 1.0
    if L is None:
        L = (nx, ny, nz)
    La = (2 * nx, 2 * ny, 2 * nz)
    Gw = green_embedded(nx, ny, nz, k, d, La) * occupancy_weights(occ)[..., None]
    F = np.zeros(tuple(L) + (6,), dtype=np.complex128)
    tgt = []
    for n_, La_, L_ in zip((nx, ny, nz), La, L):
        i = np.arange(La_)
        tgt.append(np.where(i < n_, i, i - La_) % L_)
    np.add.at(F, np.ix_(*tgt), Gw)
    Gh = sfft.fftn(-F, axes=(0, 1, 2), workers=_WORKERS)
    Gh = Gh[:L[0] // 2 + 1, :L[1] // 2 + 1, :L[2] // 2 + 1]
    T = np.empty(Gh.shape[:3] + (3, 3), dtype=np.complex128)
    for a in range(3):
        for b in range(3):
            T[..., a, b] = -Gh[..., _COMP[a, b]]
        T[..., a, a] += abar
    Ti = np.linalg.inv(T)
    return np.ascontiguousarray(np.stack([Ti[..., a, b] for a, b in _PAIRS], axis=-1))


def prepare_interaction_matrices(alpha_array, k, d, cutoff=False, L=None):
    """(inv_alpha, mask, Ghat, None): ddaforgit.py:1085-1159 without the
    missing preconditioner builders."""
    a = np.asarray(alpha_array, dtype=np.complex128)
    if cutoff:
        a = np.where(np.abs(a) < 1.0, 0.0, a)
    inv_alpha = np.where(a != 0, 1.0 / np.where(a != 0, a, 1.0), 0)
    mask = a != 0
    nx, ny, nz = a.shape
    G = generate_interaction_row(nx, ny, nz, k, d, reduced=True, L=L)
    return inv_alpha, mask, G, None


def interaction_mult(x, Ghat_oct, inv_alpha, mask, L=None):
    """A.x = inv_alpha*x - mask*conv(x).  Gpbicgstab.py:473-475, 768-769,
    828-830."""
    x = np.asarray(x, dtype=np.complex128)
    nx, ny, nz = inv_alpha.shape
    x4 = x.reshape(nx, ny, nz, 3)
    conv = fft_convolve(x4, Ghat_oct, L) * mask[..., None]
    return inv_alpha[..., None] * x4 - conv


def E_field_solver(polarization, Ghat_oct, grid_size, L=None):
    """Excited field IFFT[FFT(-A) FFT(P)] cropped, no mask, no alpha term.
    ExcitedField.py:129-195 (size checks :139-152)."""
    nx, ny, nz = grid_size
    P = np.asarray(polarization, dtype=np.complex128)
    if P.size != nx * ny * nz * 3:
        raise ValueError(f"Polarization size {P.size} doesn't match expected "
                         f"size {nx * ny * nz * 3}")
    return fft_convolve(P.reshape(nx, ny, nz, 3), Ghat_oct, L)


def dense_interaction_mult(x, inv_alpha, k, d, mask):
    """O(N^2) direct A.x for tiny lattices, from the same Green formula
    (ddaforgit.py:979-987).  A_jk = G(r_j - r_k) for j != k, A_jj = 1/alpha."""
    inv = np.asarray(inv_alpha, dtype=np.complex128)
    nx, ny, nz = mask.shape
    idx = np.argwhere(np.ones((nx, ny, nz), bool)).astype(np.float64) * d
    x = np.asarray(x, dtype=np.complex128).reshape(-1, 3)
    R = idx[:, None, :] - idx[None, :, :]
    r2 = (R ** 2).sum(-1)
    diag = r2 == 0
    r2s = np.where(diag, 1.0, r2)
    r = np.sqrt(r2s)
    n = R / r[..., None]
    ikr = 1j * k * r
    expt = np.exp(ikr) / r
    f2 = (ikr - 1.0) / r2s
    I3 = np.eye(3)
    nn = n[..., :, None] * n[..., None, :]
    G = expt[..., None, None] * (k * k * (nn - I3) + f2[..., None, None]
                                 * (3 * nn - I3))
    G[diag] = 0
    conv = -np.einsum("jkab,kb->ja", G, x)     # conv with FFT(-G)
    m = mask.reshape(-1)
    out = inv.reshape(-1)[:, None] * x - m[:, None] * conv
    return out.reshape(nx, ny, nz, 3)


# --------------------------------------------------------------------------
# GPBiCGSTAB  (Gpbicgstab.py:879-1201), precon=False
# --------------------------------------------------------------------------
def _vdot(a, b):
    # inner_product: sum conj(a) * b  (Gpbicgstab.py:383-464)
    return np.vdot(a.ravel(), b.ravel())


def solve_gpbicgstab(grid_size, inv_alpha, Ghat_oct, E_inc, mask, ratio,
                     max_iter, target=1e-5, L=None, matvec=None, preconditioner=None):
    """GPBiCGSTAB with the reference's recurrence, resets, true-residual
    replacement at i==1, best-iterate tracking and return codes.

    Returns (iters, P (nx,ny,nz,3), lowest/initial, first/initial).
    Gpbicgstab.py:957-1201.  ``preconditioner`` (an octant for
    ``precondition_apply``) gives the reference's right-preconditioned form,
    precon=True: A is applied to M p and M s (:1008, :1026), the residual
    replacements use A M x (:1061-1064, :1143-1144) and the result is M x
    (:1171-1199); without it M = I (:634-635).
    """
    nx, ny, nz = grid_size
    mask = np.asarray(mask).astype(bool).reshape(nx, ny, nz)
    inv_alpha = np.asarray(inv_alpha, dtype=np.complex128).reshape(nx, ny, nz)
    if matvec is None:
        def matvec(v):
            return interaction_mult(v.reshape(nx, ny, nz, 3), Ghat_oct,
                                    inv_alpha, mask, L).ravel()
    if preconditioner is None:
        def msolve(v):
            return v
    else:
        def msolve(v):
            return precondition_apply(v.reshape(nx, ny, nz, 3), preconditioner, mask).ravel()
    amul = matvec

    def matvec(v):            # noqa: F811 -- A M
        return amul(msolve(v))
    b = (np.asarray(E_inc, dtype=np.complex128).reshape(nx, ny, nz, 3)
         * mask[..., None]).ravel()
    r = b.copy()
    r_hat = r.copy()
    p = r.copy()
    x = np.zeros_like(r)
    z = np.zeros_like(r)
    u = np.zeros_like(r)
    w = np.zeros_like(r)
    s = np.zeros_like(r)
    s_prev = np.zeros_like(r)
    initial_norm = float(np.linalg.norm(r))
    rho_1 = _vdot(r_hat, r)
    rho_0 = rho_1
    alpha = beta = zeta = eta = 0.0 + 0.0j
    lowest = initial_norm
    current = lowest
    previous_lowest = lowest
    first = 0.0
    best = np.zeros_like(r)
    last_change = 0
    was_reset = False
    i = 0
    for i in range(max_iter):
        v = matvec(p)
        alpha = rho_1 / _vdot(r_hat, v)
        s = r - alpha * v
        y = s_prev - s - alpha * w
        t = matvec(s)
        if i == 0 or was_reset:
            zeta = _vdot(t, s) / _vdot(t, t)
            eta = 0.0
            u = zeta * v
            z = zeta * s
            r = s - zeta * t
        else:
            # calculate_zeta_eta_twostep, Gpbicgstab.py:239-380
            yy = _vdot(y, y); tt = _vdot(t, t); yt = _vdot(y, t)
            ty = _vdot(t, y); ys = _vdot(y, s); ts = _vdot(t, s)
            den = tt * yy - yt * ty
            zeta = (yy * ts - ys * ty) / den
            eta = (tt * ys - yt * ts) / den
            u = zeta * v + eta * (s_prev - r + beta * u)
            z = zeta * r + eta * z - alpha * u
            r = s - eta * y - zeta * t
        x = x + alpha * p + z
        if i == 1:
            r = b - matvec(x)
        current = float(np.linalg.norm(r))
        if i == 0:
            first = current
        last_change += 1
        if (not np.isnan(current)) and (np.isnan(lowest) or current < lowest):
            last_change = 0
            lowest = current
            best = x.copy()
        if np.isnan(current) or last_change >= 5000:
            break
        elif current < target * initial_norm:
            break
        reset = False
        rho_0 = rho_1
        rho_1 = _vdot(r_hat, r)
        if ratio != 0:
            if i == 2 or (i > 2 and current < previous_lowest / ratio):
                reset = True
                previous_lowest = current
                last_change = 0
        was_reset = False
        if reset:
            if i % 100 != 0:
                r = b - matvec(x)
            r_hat = r.copy()
            beta = 0.0
            w = np.zeros_like(w)
            s_prev = s.copy()
            was_reset = True
            p = r.copy()
        else:
            beta = alpha / zeta * rho_1 / rho_0
            w = t + beta * v
            s_prev = s.copy()
            p = r + beta * (p - u)
    shp = (nx, ny, nz, 3)
    if np.isnan(current) or last_change >= 5000:
        return -(i + 1), msolve(best).reshape(shp), lowest / initial_norm, first / initial_norm
    if i < max_iter - 1 and current >= target * initial_norm:
        return -(i + 1), msolve(best).reshape(shp), lowest / initial_norm, first / initial_norm
    if current >= target * initial_norm:
        return max_iter, msolve(best).reshape(shp), lowest / initial_norm, first / initial_norm
    return i + 1, msolve(x).reshape(shp), lowest / initial_norm, first / initial_norm


def true_relative_residual(P, E_inc, Ghat_oct, inv_alpha, mask, L=None):
    """||E_inc*mask - A.P|| / ||E_inc*mask||."""
    b = np.asarray(E_inc) * np.asarray(mask)[..., None]
    r = b - interaction_mult(P, Ghat_oct, inv_alpha, np.asarray(mask), L)
    return float(np.linalg.norm(r) / np.linalg.norm(b))


# --------------------------------------------------------------------------
# cross sections (not in the reference; Draine & Flatau 1994, JOSA A 11:1491)
# --------------------------------------------------------------------------
def cross_sections(P, E_inc, inv_alpha, k, E0=1.0):
    """(C_ext, C_abs, C_sca) in the Gaussian units of the reference.

    C_ext = 4 pi k / |E0|^2 sum Im(E_inc* . P)
    C_abs = 4 pi k / |E0|^2 sum [ Im(P . conj(inv_alpha) P*) - 2/3 k^3 |P|^2 ]
    """
    P = np.asarray(P, dtype=np.complex128)
    E = np.asarray(E_inc, dtype=np.complex128)
    ia = np.asarray(inv_alpha, dtype=np.complex128)
    occ = ia != 0
    pref = 4 * np.pi * k / abs(E0) ** 2
    cext = pref * np.sum(np.imag(np.conj(E[occ]) * P[occ]))
    p2 = np.sum(np.abs(P) ** 2, axis=-1)
    cabs = pref * np.sum((np.imag(np.conj(ia)) * p2 - (2.0 / 3.0) * k ** 3 * p2)[occ])
    return float(cext), float(cabs), float(cext - cabs)


# --------------------------------------------------------------------------
# Mie theory (Bohren & Huffman 1983, appendix A: BHMIE recurrences)
# --------------------------------------------------------------------------
def far_field(P, d, k, directions):
    """Far-field amplitude F(n) = k^2 sum_j [P_j - n (n.P_j)] exp(-i k n.r_j),
    r_j = (i, j, k) d (the incident field's origin, ddaforgit.py:1626-1632);
    the standard DDA far field (Draine 1988), not present in the reference."""
    P = np.asarray(P)
    nx, ny, nz, _ = P.shape
    idx = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3) * d
    Pf = P.reshape(-1, 3)
    out = []
    for n in np.asarray(directions, float).reshape(-1, 3):
        n = n / np.linalg.norm(n)
        ph = np.exp(-1j * k * (idx @ n))
        S = (Pf * ph[:, None]).sum(0)
        out.append(k * k * (S - n * (n @ S)))
    return np.array(out)


def mie_qext_qsca(m, x):
    """Extinction and scattering efficiencies of a homogeneous sphere with
    relative index ``m`` and size parameter ``x`` (Bohren & Huffman BHMIE:
    downward logarithmic-derivative recurrence, upward Riccati-Bessel)."""
    m = complex(m)
    mx = m * x
    nstop = int(x + 4.0 * x ** (1.0 / 3.0) + 2.0)
    nmx = int(max(nstop, abs(mx))) + 16
    D = np.zeros(nmx + 1, dtype=np.complex128)
    for n in range(nmx, 0, -1):
        D[n - 1] = n / mx - 1.0 / (D[n] + n / mx)
    psi0, psi1 = math.cos(x), math.sin(x)
    chi0, chi1 = -math.sin(x), math.cos(x)
    xi1 = complex(psi1, -chi1)
    qext = qsca = 0.0
    for n in range(1, nstop + 1):
        psi = (2 * n - 1) / x * psi1 - psi0
        chi = (2 * n - 1) / x * chi1 - chi0
        xi = complex(psi, -chi)
        da = D[n] / m + n / x
        db = D[n] * m + n / x
        an = (da * psi - psi1) / (da * xi - xi1)
        bn = (db * psi - psi1) / (db * xi - xi1)
        qsca += (2 * n + 1) * (abs(an) ** 2 + abs(bn) ** 2)
        qext += (2 * n + 1) * (an + bn).real
        psi0, psi1 = psi1, psi
        chi0, chi1 = chi1, chi
        xi1 = complex(psi1, -chi1)
    return 2.0 * qext / x ** 2, 2.0 * qsca / x ** 2
