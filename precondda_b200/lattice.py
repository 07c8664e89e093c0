"""Dipole-lattice setup: shapes, polarizability, voxelisation, incident field.

Host-side problem setup, as in the reference (ddaforgit.py:53-857 and
build_problem_from_shapes, :1591-1651): shapes are described in physical
units, snapped to the lattice, voxelised at voxel centres (i+0.5)d, trimmed
to their bounding box (odd sizes padded to even) and turned into the
polarizability array alpha (nx,ny,nz) and the incident field E_inc
(nx,ny,nz,3).  ``voxelize_device`` and ``incident_field_device`` build the
same arrays with the engine's kernels, on the device, for large lattices and
the serving path.

Extensions over the reference: ellipsoids accept a rotation matrix (the
reference's ``axis`` field is unused), and sphere aggregates are a list of
spheres.
"""
from __future__ import annotations

import math

import numpy as np

EPS = 1e-7


# --------------------------------------------------------------------------
# shapes (ddaforgit.py:53-110)
# --------------------------------------------------------------------------
class Shape:
    def __init__(self, shape_id, n, group=None, priority=0):
        self.id = shape_id
        self.n = n
        self.group = group
        self.priority = priority
        self.value = None
        self.center = [0, 0, 0]


class Sphere(Shape):
    def __init__(self, shape_id, center, radius, n, group=None, priority=0):
        super().__init__(shape_id, n, group, priority)
        self.center = center
        self.radius = radius


class Cylinder(Shape):
    """Cylinder of the given axis.  ``geometric=False`` (the default) keeps
    the reference's membership test (ddaforgit.py:477-509) bit for bit: the
    radial distance is taken in the (x, y) plane whatever the axis, and for
    the x and y axes the height test compares the signed z offset with
    height/2, so such a cylinder fills its mark_shapes window below
    z = c_z + height/2.  ``geometric=True`` splits the axes as the axis
    names say."""

    def __init__(self, shape_id, center, radius, height, axis="z", n=1.5, group=None, priority=0, geometric=False):
        super().__init__(shape_id, n, group, priority)
        self.center = center
        self.radius = radius
        self.height = height
        self.axis = axis
        self.geometric = bool(geometric)


class Ellipsoid(Shape):
    def __init__(self, shape_id, center, semi_axes, n, axis="z", group=None, priority=0, rotation=None):
        super().__init__(shape_id, n, group, priority)
        self.center = center
        self.semi_axes = semi_axes
        self.axis = axis
        self.rotation = None if rotation is None else np.asarray(rotation, dtype=np.float64)


class Rectangle(Shape):
    def __init__(self, shape_id, center, dimensions, n, group=None, priority=0):
        super().__init__(shape_id, n, group, priority)
        self.center = center
        self.dimensions = dimensions


class Prism(Shape):
    def __init__(self, shape_id, center, radius, sides, height, n, axis="z", group=None, priority=0):
        super().__init__(shape_id, n, group, priority)
        self.center = center
        self.radius = radius
        self.sides = sides
        self.height = height
        self.axis = axis


_SHAPES = {"sphere": Sphere, "cylinder": Cylinder, "ellipsoid": Ellipsoid, "rectangle": Rectangle, "prism": Prism}


# --------------------------------------------------------------------------
# polarizability (ddaforgit.py:403-437)
# --------------------------------------------------------------------------
# lattice-dispersion-relation coefficients (Draine & Goodman 1993)
_LDR_B = (-1.891531, 0.1648469, -1.7700004)


def calculate_alpha(refractive_index, lattice_spacing, wave_number, incident_direction=None,
                    polarization_direction=None, method="LDR"):
    """Clausius-Mossotti polarizability with optional radiative-reaction (RR)
    or lattice-dispersion-relation (LDR) correction; LDR keeps the reference's
    S = (a.e)^2 (ddaforgit.py:432).  Each formula is evaluated in the
    reference's operation order (ddaforgit.py:403-437), so the values agree
    bit for bit."""
    m = np.complex128(refractive_index)
    d = np.float64(lattice_spacing)
    k = np.float64(wave_number)
    eps = m ** 2
    cm = (3 * d ** 3 / (4 * np.pi)) * (eps - 1) / (eps + 2)
    if method == "CM":
        return cm
    radiative = (2 / 3) * 1j * (k * d) ** 3
    if method == "RR":
        return cm / (1 + (cm / d ** 3) * (-radiative))
    if method == "LDR":
        if incident_direction is None or polarization_direction is None:
            raise ValueError("incident_direction and polarization_direction required for LDR method")
        a_hat = np.asarray(incident_direction, dtype=np.float64)
        e_hat = np.asarray(polarization_direction, dtype=np.float64)
        b1, b2, b3 = _LDR_B
        S = np.sum(np.dot(a_hat, e_hat) ** 2)
        dispersion = (b1 + m ** 2 * b2 + m ** 2 * b3 * S) * (k * d) ** 2
        return cm / (1 + (cm / d ** 3) * (dispersion - radiative))
    raise ValueError("method must be 'CM', 'RR', or 'LDR'")


# --------------------------------------------------------------------------
# membership tests (ddaforgit.py:439-613), vectorised over points (P,3)
# --------------------------------------------------------------------------
def inside_sphere(p, center, radius, eps=EPS):
    dist = np.sqrt(((p - np.asarray(center)) ** 2).sum(-1))
    return (dist < radius) | (np.abs(dist - radius) < eps)


def inside_ellipsoid(p, center, semi_axes, eps=EPS, rotation=None):
    off = p - np.asarray(center)
    if rotation is not None:
        off = off @ np.asarray(rotation)      # lab -> body frame (R^T applied to row vectors)
    q = off / np.asarray(semi_axes, dtype=np.float64)
    return np.sqrt((q ** 2).sum(-1)) <= 1.0 + eps


def inside_rectangle(p, center, dims, eps=EPS):
    h = np.asarray(dims, dtype=np.float64) / 2
    a = np.abs(p - np.asarray(center))
    dx, dy, dz = a[:, 0], a[:, 1], a[:, 2]
    inside = (dx <= h[0]) & (dy <= h[1]) & (dz <= h[2])
    edge = ((np.abs(dx - h[0]) < eps) & (dy <= h[1]) & (dz <= h[2])) | \
           ((np.abs(dy - h[1]) < eps) & (dx <= h[0]) & (dz <= h[2])) | \
           ((np.abs(dz - h[2]) < eps) & (dx <= h[0]) & (dy <= h[1]))
    return inside | edge


def _axis_split(p, center, axis):
    ax = {"x": 0, "y": 1, "z": 2}[axis]
    o = [i for i in range(3) if i != ax]
    return p[:, o], np.asarray(center)[o], p[:, ax], np.asarray(center)[ax]


def inside_cylinder(p, center, radius, height, axis="z", eps=EPS, geometric=False):
    if geometric:
        p2, c2, h, ch = _axis_split(p, center, axis)
        rd = np.sqrt(((p2 - c2) ** 2).sum(-1))
        dz = np.abs(h - ch)
    else:
        # the reference's form: radial distance in (x, y) for every axis;
        # signed z offset in the height test of the x and y axes
        off = p - np.asarray(center, dtype=np.float64)
        rd = np.sqrt(off[:, 0] * off[:, 0] + off[:, 1] * off[:, 1])
        dz = np.abs(off[:, 2]) if axis == "z" else off[:, 2]
    hh = height / 2
    inr = rd <= radius
    onr = np.abs(rd - radius) < eps
    inh = dz <= hh
    cap = np.abs(dz - hh) < eps
    return (inr & inh) | (onr & inh) | (inr & cap)


def inside_prism(p, center, radius, height, sides, axis="z", eps=EPS):
    p2, c2, h, ch = _axis_split(p, center, axis)
    ang = 2 * np.pi * np.arange(int(sides)) / sides
    vx = c2[0] + radius * np.cos(ang)
    vy = c2[1] + radius * np.sin(ang)
    px, py = p2[:, 0], p2[:, 1]
    inside = np.zeros(len(p), bool)
    edge = np.zeros(len(p), bool)
    nv = len(vx)
    for j in range(nv):
        j2 = (j + 1) % nv
        xi, yi, xj, yj = vx[j], vy[j], vx[j2], vy[j2]
        ex, ey = xj - xi, yj - yi
        ln = math.hypot(ex, ey)
        if ln > eps:
            ux, uy = ex / ln, ey / ln
            wx, wy = px - xi, py - yi
            proj = wx * ux + wy * uy
            dist = np.abs(wx * uy - wy * ux)
            edge |= (dist < eps) & (proj >= -eps) & (proj <= ln + eps) & ~edge
        with np.errstate(divide="ignore", invalid="ignore"):
            cross = ((yi > py) != (yj > py)) & (px < (xj - xi) * (py - yi) / (yj - yi) + xi)
        inside ^= cross & ~edge
    dz = np.abs(h - ch)
    hh = height / 2
    return (inside | edge) & ((dz <= hh) | (np.abs(dz - hh) < eps))


def shape_membership(shape, points):
    if isinstance(shape, Sphere):
        return inside_sphere(points, shape.center, shape.radius)
    if isinstance(shape, Ellipsoid):
        return inside_ellipsoid(points, shape.center, shape.semi_axes, rotation=shape.rotation)
    if isinstance(shape, Rectangle):
        return inside_rectangle(points, shape.center, shape.dimensions)
    if isinstance(shape, Cylinder):
        return inside_cylinder(points, shape.center, shape.radius, shape.height, shape.axis,
                               geometric=getattr(shape, "geometric", False))
    if isinstance(shape, Prism):
        return inside_prism(points, shape.center, shape.radius, shape.height, shape.sides, shape.axis)
    raise ValueError(f"Unsupported shape type: {type(shape)}")


def _max_dist(shape):
    return max(getattr(shape, "radius", 0), getattr(shape, "height", 0) / 2,
               max(getattr(shape, "semi_axes", [0, 0, 0])), max(getattr(shape, "dimensions", [0, 0, 0])) / 2)


# --------------------------------------------------------------------------
# shape manager (ddaforgit.py:112-400)
# --------------------------------------------------------------------------
class ShapeManager:
    def __init__(self):
        self.shapes = {}
        self.shape_counters = {}
        self.available_ids = set()
        self.available_groups = set()
        self.next_group = 1

    def get_next_id(self, shape_type):
        self.shape_counters[shape_type] = self.shape_counters.get(shape_type, 0) + 1
        return f"{shape_type}_{self.shape_counters[shape_type]}"

    def get_next_group(self):
        if self.available_groups:
            return f"group_{self.available_groups.pop()}"
        g = self.next_group
        self.next_group += 1
        return f"group_{g}"

    def add_shape(self, shape_type, **params):
        cls = _SHAPES.get(shape_type)
        if not cls:
            raise ValueError(f"Unknown shape type: {shape_type}")
        shape_id = params.pop("force_id", None) or self.get_next_id(shape_type)
        shape = cls(shape_id, **params)
        self.shapes[shape_id] = shape
        return shape_id

    def remove_shape(self, shape_id):
        if shape_id not in self.shapes:
            raise ValueError(f"Shape ID {shape_id} not found")
        del self.shapes[shape_id]
        self.available_ids.add(shape_id)

    def process_shapes(self, k, E_direction, E_polarization, lattice_spacing, adjust_all=True, method="LDR"):
        """Polarizability per refractive index and centre snapping to
        d*ceil(c/d) (ddaforgit.py:291-344)."""
        if not self.shapes:
            return
        srt = sorted(self.shapes.values(), key=lambda s: s.priority)
        amap = {n: calculate_alpha(n, lattice_spacing, k, E_direction, E_polarization, method=method)
                for n in set(s.n for s in srt)}
        for s in srt:
            s.value = amap[s.n]
        centers = np.array([s.center for s in srt], dtype=np.float64)
        if len(srt) == 1 or adjust_all:
            adj = lattice_spacing * np.ceil(centers / lattice_spacing)
        else:
            big = max(srt, key=_max_dist)
            bc = np.array(big.center, dtype=np.float64)
            adj = centers + (lattice_spacing * np.ceil(bc / lattice_spacing) - bc)
        for s, c in zip(srt, adj):
            s.center = c.tolist()

    def calculate_grid_extents(self, lattice_spacing, max_x=1e9, max_y=1e9, max_z=1e9):
        """Box size from the shapes' extents plus one spacing (ddaforgit.py:346-400)."""
        if not self.shapes:
            return 0, 0, 0
        mc = np.zeros(3)
        for s in self.shapes.values():
            c = np.array(s.center, dtype=np.float64)
            ext = _max_dist(s)
            if isinstance(s, Prism) and s.sides > 2:
                ext = max(ext, s.radius / np.cos(np.pi / s.sides))
            if isinstance(s, (Cylinder, Prism)):
                ai = {"x": 0, "y": 1, "z": 2}[s.axis]
                ev = np.full(3, ext)
                ev[ai] = s.height / 2
                smax = c + ev
            else:
                smax = c + ext
            mc = np.maximum(mc, smax)
        mc = np.minimum(mc, [max_x, max_y, max_z]) + lattice_spacing
        return tuple(min(int(np.ceil(mc[i] / lattice_spacing)), int(np.ceil(m / lattice_spacing)))
                     for i, m in enumerate((max_x, max_y, max_z)))


def mark_shapes(grid_shape, lattice_spacing, shapes, voxel_center=True, values="value"):
    """Voxelise shapes in insertion order, later shapes overwriting earlier
    ones (ddaforgit.py:615-709)."""
    nx, ny, nz = grid_shape
    off = 0.5 if voxel_center else 0.0
    out = np.zeros(grid_shape, dtype=np.complex128)
    for s in shapes:
        c = np.array(s.center, dtype=np.float64)
        mg = int(float(_max_dist(s) + EPS) / lattice_spacing) + 1
        ci = (c / lattice_spacing).astype(int)
        lo = np.maximum(0, ci - mg)
        hi = np.minimum([nx, ny, nz], ci + mg + 1)
        if np.any(hi <= lo):
            continue
        ax = [(np.arange(lo[i], hi[i]) + off) * lattice_spacing for i in range(3)]
        X, Y, Z = np.meshgrid(*ax, indexing="ij")
        pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
        ins = shape_membership(s, pts).reshape(X.shape)
        val = s.value if values == "value" else s.n
        sl = out[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]]
        if val != 0:
            sl[ins] = val
    return out


def trim_zero_faces(array):
    """Crop to the non-zero bounding box; odd sizes padded to even
    (ddaforgit.py:831-857)."""
    nz_ = array != 0
    if not nz_.any():
        return array[:0, :0, :0]
    xm = nz_.any(axis=(1, 2)); ym = nz_.any(axis=(0, 2)); zm = nz_.any(axis=(0, 1))
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


def create_alpha_and_n_arrays(shape_manager, lattice_spacing, voxel_center=True):
    """(alpha_array, n_array, shape) (ddaforgit.py:812-830)."""
    grid = shape_manager.calculate_grid_extents(lattice_spacing)
    shapes = list(shape_manager.shapes.values())
    a = trim_zero_faces(mark_shapes(grid, lattice_spacing, shapes, voxel_center))
    n = trim_zero_faces(mark_shapes(grid, lattice_spacing, shapes, voxel_center, values="n"))
    return a, n, a.shape


def incident_field(grid_size, lattice_spacing, k, k_direction, e_polarization):
    """E_inc = e exp(i k.r), r = (i,j,k) d with no half-voxel offset
    (ddaforgit.py:1626-1632)."""
    kv = k * np.asarray(k_direction, dtype=np.float64)
    ax = [np.arange(0, n) * lattice_spacing for n in grid_size]
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    ph = np.exp(1j * (kv[0] * X + kv[1] * Y + kv[2] * Z))
    E = np.empty((*grid_size, 3), dtype=np.complex128)
    for j in range(3):
        E[..., j] = e_polarization[j] * ph
    return E


def build_problem_from_shapes(shapes, k_direction, E_polarization, wavelength, lattice_spacing, method="LDR"):
    """Problem dictionary from shape descriptions (ddaforgit.py:1591-1651)."""
    sm = ShapeManager()
    for s in shapes:
        t = s["type"]
        kw = {k: v for k, v in s.items() if k != "type"}
        sm.add_shape(t, **kw)
    k = 2 * np.pi / wavelength
    kd = np.asarray(k_direction, dtype=np.float64)
    sm.process_shapes(k, kd, E_polarization, lattice_spacing, method=method)
    alpha, n_arr, grid = create_alpha_and_n_arrays(sm, lattice_spacing)
    grid = tuple(int(g) for g in grid)
    E = incident_field(grid, lattice_spacing, k, kd, E_polarization)
    return {"alpha_array": alpha, "n_array": n_arr, "grid_size": grid, "E_inc": E, "k": k,
            "lattice_spacing": lattice_spacing, "k_vec": k * kd, "k_direction": kd,
            "E_polarization": E_polarization, "wavelength": wavelength}


# --------------------------------------------------------------------------
# lattice-unit builders used by the benchmark workloads
# --------------------------------------------------------------------------
def sphere_occupancy(n_box, radius_d):
    """Sphere of radius ``radius_d`` (units of d) centred in an n_box^3 box,
    voxel centres at (i+0.5)d, same test as ddaforgit.py:439-448."""
    c = n_box / 2.0
    ax = np.arange(n_box) + 0.5 - c
    X, Y, Z = np.meshgrid(ax, ax, ax, indexing="ij")
    dist = np.sqrt(X * X + Y * Y + Z * Z)
    return (dist < radius_d) | (np.abs(dist - radius_d) < EPS)


def euler_rotation(a, b, g):
    """Z-Y-Z Euler rotation matrix (body -> lab)."""
    ca, sa, cb, sb, cg, sg = math.cos(a), math.sin(a), math.cos(b), math.sin(b), math.cos(g), math.sin(g)
    Rz1 = np.array([[ca, -sa, 0], [sa, ca, 0], [0, 0, 1]])
    Ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    Rz2 = np.array([[cg, -sg, 0], [sg, cg, 0], [0, 0, 1]])
    return Rz1 @ Ry @ Rz2


def ellipsoid_occupancy(box, semi_axes_d, rotation=None):
    """Ellipsoid centred in a box (units of d), optional rotation."""
    box = tuple(int(b) for b in box)
    c = np.array(box, dtype=np.float64) / 2.0
    ax = [np.arange(n) + 0.5 - c[i] for i, n in enumerate(box)]
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    pts = np.stack([X, Y, Z], -1).reshape(-1, 3)
    return inside_ellipsoid(pts, (0, 0, 0), semi_axes_d, rotation=rotation).reshape(box)


# --------------------------------------------------------------------------
# device builders: the same lattice built by the engine's kernels
# --------------------------------------------------------------------------
def _reference_window(s, d, box, shift=(0, 0, 0)):
    """mark_shapes' index window of shape s (ddaforgit.py:626-649) in the
    site indices of a box whose site 0 is the reference grid's site ``shift``."""
    c = np.array(s.center, dtype=np.float64)
    mg = int(float(_max_dist(s) + EPS) / d) + 1
    ci = (c / d).astype(int)
    lo = [max(0, int(ci[a]) - mg - shift[a]) for a in range(3)]
    hi = [min(int(box[a]), int(ci[a]) + mg + 1 - shift[a]) for a in range(3)]
    return lo, hi


def _shape_struct(s, inv_alpha, window=None):
    from . import _lib as L
    st = L.dda_shape()
    if window is not None:
        lo, hi = window
        st.flags |= L.SHAPE_WINDOW
        for a in range(3):
            st.win[2 * a], st.win[2 * a + 1] = int(lo[a]), int(hi[a])
    st.inv_alpha[0], st.inv_alpha[1] = float(np.real(inv_alpha)), float(np.imag(inv_alpha))
    for i in range(9):
        st.rot[i] = 1.0 if i in (0, 4, 8) else 0.0
    c = np.asarray(s.center, dtype=np.float64)
    st.center[0], st.center[1], st.center[2] = c
    ax = {"x": 0, "y": 1, "z": 2}
    if isinstance(s, Sphere):
        st.type, st.p[0] = L.SHAPE_SPHERE, float(s.radius)
    elif isinstance(s, Ellipsoid):
        st.type = L.SHAPE_ELLIPSOID
        for i in range(3):
            st.p[i] = float(s.semi_axes[i])
        if s.rotation is not None:
            R = np.asarray(s.rotation, dtype=np.float64).reshape(9)
            for i in range(9):
                st.rot[i] = R[i]
    elif isinstance(s, Rectangle):
        st.type = L.SHAPE_RECTANGLE
        for i in range(3):
            st.p[i] = float(s.dimensions[i])
    elif isinstance(s, Cylinder):
        st.type, st.p[0], st.p[1], st.axis = L.SHAPE_CYLINDER, float(s.radius), float(s.height), ax[s.axis]
        if getattr(s, "geometric", False):
            st.flags |= L.SHAPE_GEOMETRIC_AXES
    elif isinstance(s, Prism):
        st.type, st.p[0], st.p[1] = L.SHAPE_PRISM, float(s.radius), float(s.height)
        st.axis, st.sides = ax[s.axis], int(s.sides)
    else:
        raise ValueError(f"Unsupported shape type: {type(s)}")
    return st


def voxelize_device(shapes, inv_alphas, box, d, origin=(0.0, 0.0, 0.0), dtype=None, device=None, window=True):
    """inv_alpha (nx,ny,nz) on the device: voxel centres origin + (i+0.5) d,
    each site takes the inverse polarizability of the last shape containing
    it (the reference's mark_shapes order), 0 elsewhere.  ``window`` limits
    each shape to the index window mark_shapes evaluates it on (origin taken
    as a whole number of spacings); it bounds the reference's x- and y-axis
    cylinders and changes no other shape."""
    import ctypes as C
    import torch
    from . import _lib as L
    from .engine import _device, _dt_code, stream_handle
    dtype = dtype or torch.complex128
    dev = _device(device)
    n = len(shapes)
    shift = [int(round(float(o) / d)) for o in origin]
    wins = [_reference_window(s, d, box, shift) if window else None for s in shapes]
    arr = (L.dda_shape * n)(*[_shape_struct(s, a, w) for s, a, w in zip(shapes, inv_alphas, wins)])
    out = torch.empty(tuple(int(b) for b in box), dtype=dtype, device=dev)
    org = (C.c_double * 3)(*[float(v) for v in origin])
    ctx = L.context(dev.index)
    with torch.cuda.device(dev):
        L.check(L.lib().dda_voxelize(ctx.handle, _dt_code(dtype), arr, n, *out.shape, float(d), org,
                                     out.data_ptr(), stream_handle(dev)))
    return out


def mark_shapes_device(grid_shape, lattice_spacing, shapes, values="value", device=None):
    """mark_shapes (ddaforgit.py:615-661) on the device: the value (or the
    refractive index, values="n") of the last shape containing each voxel
    centre, within each shape's index window; complex128 (nx,ny,nz)."""
    vals = [s.value if values == "value" else s.n for s in shapes]
    return voxelize_device(shapes, vals, grid_shape, lattice_spacing, device=device)


def incident_field_device(box, d, k_vec, polarization, dtype=None, device=None):
    """Plane wave e exp(i k.r), r = (i,j,k) d, on the device (nx,ny,nz,3)."""
    import ctypes as C
    import torch
    from . import _lib as L
    from .engine import _device, _dt_code, stream_handle
    dtype = dtype or torch.complex128
    dev = _device(device)
    out = torch.empty(tuple(int(b) for b in box) + (3,), dtype=dtype, device=dev)
    kv = (C.c_double * 3)(*[float(v) for v in k_vec])
    e = np.asarray(polarization, dtype=np.complex128)
    pol = (C.c_double * 6)(e[0].real, e[0].imag, e[1].real, e[1].imag, e[2].real, e[2].imag)
    ctx = L.context(dev.index)
    with torch.cuda.device(dev):
        L.check(L.lib().dda_incident_field(ctx.handle, _dt_code(dtype), *out.shape[:3], float(d), kv, pol,
                                           out.data_ptr(), stream_handle(dev)))
    return out
