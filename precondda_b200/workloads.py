"""Seeded synthetic workloads of the benchmark configurations.

No dataset is involved: every lattice, refractive index, wavelength and
incidence is drawn from a seeded generator.  Specs are plain dicts; the
device lattices are built from them by ``build_geometry``.
"""
from __future__ import annotations

import math

import numpy as np

from .engine import _C128, _device
from .lattice import (Ellipsoid, Sphere, calculate_alpha, euler_rotation, incident_field_device, voxelize_device)


def sphere_directions(n, rng):
    """n unit vectors uniform on the sphere."""
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def transverse_pair(kdir):
    """Two orthonormal polarisations perpendicular to kdir."""
    kdir = np.asarray(kdir, float)
    a = np.array([1.0, 0.0, 0.0]) if abs(kdir[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    e1 = a - kdir * (a @ kdir)
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(kdir, e1)
    return e1, e2


def random_ellipsoid_spec(rng, edge=(16, 96), axis_frac=(0.3, 0.5), m_re=(1.3, 2.0), m_im=(0.0, 0.3),
                          wavelength=(0.4, 0.8), mkd=0.5, n_dirs=8, cubic=False):
    """Ellipsoid in a box with integer edges uniform in ``edge`` (one edge
    for all axes when ``cubic``), semi-axes ``axis_frac`` x the edge, random
    rotation, m and wavelength; d from |m| k d = ``mkd``; ``n_dirs``
    incidence directions uniform on the sphere, two polarisations each."""
    if cubic:
        box = (int(rng.integers(edge[0], edge[1] + 1)),) * 3
    else:
        box = tuple(int(v) for v in rng.integers(edge[0], edge[1] + 1, size=3))
    semi = tuple(float(rng.uniform(*axis_frac) * b) for b in box)
    rot = euler_rotation(*rng.uniform(0, 2 * np.pi, size=3))
    return {"kind": "ellipsoid", "box": box, "semi_axes_d": semi, "rotation": rot,
            "m": complex(rng.uniform(*m_re), rng.uniform(*m_im)), "wavelength": float(rng.uniform(*wavelength)),
            "mkd": mkd, "dirs": sphere_directions(n_dirs, rng), "pols": 2}


def random_sphere_spec(rng, edge=(16, 128), m_re=(1.3, 2.0), m_im=(0.0, 0.5), wavelength=(0.4, 0.8), mkd=0.5,
                       n_dirs=1):
    n = int(rng.integers(edge[0], edge[1] + 1))
    return {"kind": "sphere", "box": (n, n, n), "radius_d": n / 2.0,
            "m": complex(rng.uniform(*m_re), rng.uniform(*m_im)), "wavelength": float(rng.uniform(*wavelength)),
            "mkd": mkd, "dirs": sphere_directions(n_dirs, rng), "pols": 1}


def random_walk_aggregate(K, r_range, rng, max_tries=20000):
    """K touching spheres (radii in ``r_range``, units of d) placed by seeded
    random-walk attachment: each new sphere touches a randomly chosen earlier
    one in a random direction and overlaps none of the others."""
    centers, radii = [np.zeros(3)], [float(rng.uniform(*r_range))]
    tries = 0
    while len(centers) < K and tries < max_tries:
        tries += 1
        r = float(rng.uniform(*r_range))
        j = int(rng.integers(len(centers)))
        u = sphere_directions(1, rng)[0]
        c = centers[j] + u * (radii[j] + r)
        if all(np.linalg.norm(c - cc) >= rr + r - 1e-9 for cc, rr in zip(centers, radii)):
            centers.append(c)
            radii.append(r)
    return np.array(centers), np.array(radii)


def random_aggregate_spec(rng, K=(4, 32), r=(6, 12), max_edge=128, m_re=(1.3, 2.0), m_im=(0.0, 0.5),
                          wavelength=(0.4, 0.8), mkd=0.5, n_dirs=1):
    """Random-walk aggregate of K touching spheres in the smallest box that
    holds it (redrawn until the box fits ``max_edge``)."""
    while True:
        k = int(rng.integers(K[0], K[1] + 1))
        c, rad = random_walk_aggregate(k, r, rng)
        lo = (c - rad[:, None]).min(0)
        hi = (c + rad[:, None]).max(0)
        box = tuple(int(math.ceil(v)) + 2 for v in hi - lo)
        if max(box) <= max_edge:
            break
    return {"kind": "aggregate", "box": box, "centers_d": c, "radii_d": rad, "offset_d": 1.0 - lo,
            "m": complex(rng.uniform(*m_re), rng.uniform(*m_im)), "wavelength": float(rng.uniform(*wavelength)),
            "mkd": mkd, "dirs": sphere_directions(n_dirs, rng), "pols": 1}


def sphere_box_spec(n, m, wavelength=0.5, mkd=0.5, pols=((1, 0, 0), (0, 1, 0)), radius_d=None):
    """The sphere configurations: box n^3, sites whose centre lies within
    n/2 d of the box centre, incidence along +z."""
    return {"kind": "sphere", "box": (n, n, n), "radius_d": radius_d or n / 2.0, "m": m, "wavelength": wavelength,
            "mkd": mkd, "dirs": np.array([[0.0, 0.0, 1.0]]), "fixed_pols": [np.asarray(p, float) for p in pols]}


def ellipsoid128_spec(seed=0, mkd=0.6):
    """Large single solve: 128^3 box, semi-axes (64, 48, 40) d, Euler angles
    and m drawn from the seed."""
    rng = np.random.default_rng(seed)
    rot = euler_rotation(*rng.uniform(0, 2 * np.pi, size=3))
    m = complex(rng.uniform(1.3, 2.0), rng.uniform(0.0, 0.5))
    return {"kind": "ellipsoid", "box": (128, 128, 128), "semi_axes_d": (64.0, 48.0, 40.0), "rotation": rot,
            "m": m, "wavelength": 0.5, "mkd": mkd, "dirs": np.array([[0.0, 0.0, 1.0]]),
            "fixed_pols": [np.array([1.0, 0.0, 0.0])]}


def build_geometry(spec, device=None, dtype=_C128):
    """Voxelise a spec on the device and build its incident fields; returns
    (inv_alpha (nx,ny,nz), k, d, [E_inc (nx,ny,nz,3)])."""
    dev = _device(device)
    lam, m = spec["wavelength"], spec["m"]
    k = 2 * math.pi / lam
    d = spec["mkd"] / (abs(m) * k)
    ia = 1.0 / calculate_alpha(m, d, k, method="RR")
    box = tuple(int(b) for b in spec["box"])
    if spec["kind"] == "ellipsoid":
        center = [b * d / 2 for b in box]
        shapes = [Ellipsoid(0, center, [a * d for a in spec["semi_axes_d"]], m, rotation=spec["rotation"])]
    elif spec["kind"] == "sphere":
        shapes = [Sphere(0, [b * d / 2 for b in box], spec["radius_d"] * d, m)]
    elif spec["kind"] == "aggregate":
        off = np.asarray(spec["offset_d"])
        shapes = [Sphere(i, list((c + off) * d), float(r) * d, m)
                  for i, (c, r) in enumerate(zip(spec["centers_d"], spec["radii_d"]))]
    else:
        raise ValueError(f"unknown geometry kind {spec['kind']}")
    inv_alpha = voxelize_device(shapes, [ia] * len(shapes), box, d, dtype=dtype, device=dev)
    Es = []
    for kdir in spec["dirs"]:
        if "fixed_pols" in spec:
            pols = spec["fixed_pols"]
        else:
            pols = transverse_pair(kdir)[:spec.get("pols", 2)]
        for pol in pols:
            Es.append(incident_field_device(box, d, k * np.asarray(kdir), pol, dtype=dtype, device=dev))
    return inv_alpha, k, d, Es


def serving_stream(seed, rate=20.0, duration=60.0, mix=(0.4, 0.4, 0.2), edge=(16, 128), incidences=(1, 16)):
    """Poisson arrivals at ``rate`` per second over ``duration`` seconds:
    40% spheres, 40% ellipsoids, 20% aggregates of 4-32 touching spheres of
    radius 6-12 d; boxes 16^3-128^3; m Re in [1.3, 2], Im in [0, 0.5];
    lambda in [0.4, 0.8] um; 1-16 incidences each (one polarisation per
    incidence).  Returns [(arrival_s, spec)]."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > duration:
            break
        kind = rng.choice(3, p=list(mix))
        n_inc = int(rng.integers(incidences[0], incidences[1] + 1))
        if kind == 0:
            spec = random_sphere_spec(rng, edge=edge, n_dirs=n_inc)
        elif kind == 1:
            spec = random_ellipsoid_spec(rng, edge=edge, m_im=(0.0, 0.5), n_dirs=n_inc, cubic=True)
            spec["pols"] = 1
        else:
            spec = random_aggregate_spec(rng, max_edge=edge[1], n_dirs=n_inc)
        out.append((t, spec))
    return out
