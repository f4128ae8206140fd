"""Synthetic low-order meshes of the benchmark bodies.

Each generator returns an array (P, 4, 3) of quadrilateral panels whose right-hand-rule normal
``cross(v2 - v0, v3 - v1)`` points out of the body into the fluid; a triangle repeats its last
vertex.  The panel order and vertex order follow the procedural meshes of HydroBEM's test suite
(``tests/python/meshes.py:81-112`` cylinder, ``:49-78`` hemisphere, ``:27-46`` box), so a body built
here is the same mesh the reference solves.
"""

from __future__ import annotations

import numpy as np


def _outward(quad: np.ndarray, direction) -> np.ndarray:
    """The quad, with its vertex order reversed (v0 v3 v2 v1) when its normal points against
    ``direction``."""
    n = np.cross(quad[2] - quad[0], quad[3] - quad[1])
    if np.dot(n, direction) > 0:
        return quad
    return quad[[0, 3, 2, 1]]


def _spacing(n: int, cosine: bool) -> np.ndarray:
    """n intervals of [0, 1]: uniform, or refined at both ends by a cosine map."""
    if not cosine:
        return np.linspace(0.0, 1.0, n + 1)
    if n == 0:
        return np.zeros(1)
    return 0.5 * (1.0 - np.cos(np.pi * np.arange(n + 1) / n))


def cylinder(radius=1.0, draft=0.5, n_phi=32, n_z=8, n_r=8, quarter=False, cosine=False) -> np.ndarray:
    """Floating truncated vertical circular cylinder: n_z x n_phi side panels (waterline down),
    then n_r x n_phi bottom panels (rim inward; the ring at the axis are triangles)."""
    phi = np.linspace(0.0, 0.5 * np.pi if quarter else 2.0 * np.pi, n_phi + 1)
    z = -draft * _spacing(n_z, cosine)
    r = radius * (1.0 - _spacing(n_r, cosine))
    cp, sp = np.cos(phi), np.sin(phi)
    out = []
    for i in range(n_z):
        for j in range(n_phi):
            q = np.array([
                [radius * cp[j], radius * sp[j], z[i]],
                [radius * cp[j + 1], radius * sp[j + 1], z[i]],
                [radius * cp[j + 1], radius * sp[j + 1], z[i + 1]],
                [radius * cp[j], radius * sp[j], z[i + 1]],
            ])
            m = q.mean(axis=0)
            out.append(_outward(q, [m[0], m[1], 0.0]))
    for i in range(n_r):
        for j in range(n_phi):
            q = np.array([
                [r[i] * cp[j], r[i] * sp[j], -draft],
                [r[i] * cp[j + 1], r[i] * sp[j + 1], -draft],
                [r[i + 1] * cp[j + 1], r[i + 1] * sp[j + 1], -draft],
                [r[i + 1] * cp[j], r[i + 1] * sp[j], -draft],
            ])
            if i + 1 == n_r:
                q[3] = q[2]
            out.append(_outward(q, [0.0, 0.0, -1.0]))
    return np.array(out)


def hemisphere(radius=1.0, n_theta=8, n_phi=8, quarter=False, graded=False) -> np.ndarray:
    """Floating hemisphere z <= 0: n_theta polar rings from the waterline to the pole (the last
    ring triangles) times n_phi azimuthal divisions."""
    phi = np.linspace(0.0, 0.5 * np.pi if quarter else 2.0 * np.pi, n_phi + 1)
    s = np.linspace(0.0, 1.0, n_theta + 1)
    if graded:
        s = 1.0 - np.cos(0.5 * np.pi * s)
    theta = 0.5 * np.pi + 0.5 * np.pi * s

    def point(t, p):
        return radius * np.array([np.sin(t) * np.cos(p), np.sin(t) * np.sin(p), np.cos(t)])

    out = []
    for i in range(n_theta):
        for j in range(n_phi):
            a, b = point(theta[i], phi[j]), point(theta[i], phi[j + 1])
            c, d = point(theta[i + 1], phi[j + 1]), point(theta[i + 1], phi[j])
            q = np.array([a, b, c, d] if i + 1 < n_theta else [a, b, c, c])
            out.append(_outward(q, q.mean(axis=0)))
    return np.array(out)


def _face(origin, du, dv, nu, nv, direction):
    origin, du, dv = (np.asarray(v, dtype=float) for v in (origin, du, dv))
    a, b = du / nu, dv / nv
    out = []
    for i in range(nu):
        for j in range(nv):
            p = origin + a * i + b * j
            out.append(_outward(np.array([p, p + a, p + a + b, p + b]), direction))
    return out


def box(a=1.0, b=0.5, d=0.5, n=(4, 2, 2), quarter=False, lid=False) -> np.ndarray:
    """Surface-piercing box |x| <= a, |y| <= b, -d <= z <= 0: bottom (nx ny), x faces (ny nz),
    y faces (nx nz); lid: the interior water plane z = 0 (nx ny panels, normals up) appended."""
    nx, ny, nz = n
    x0, y0 = (0.0, 0.0) if quarter else (-a, -b)
    lx, ly = a - x0, b - y0
    p = []
    p += _face((x0, y0, -d), (lx, 0, 0), (0, ly, 0), nx, ny, (0, 0, -1))
    p += _face((a, y0, -d), (0, ly, 0), (0, 0, d), ny, nz, (1, 0, 0))
    p += _face((x0, b, -d), (lx, 0, 0), (0, 0, d), nx, nz, (0, 1, 0))
    if not quarter:
        p += _face((-a, y0, -d), (0, ly, 0), (0, 0, d), ny, nz, (-1, 0, 0))
        p += _face((x0, -b, -d), (lx, 0, 0), (0, 0, d), nx, nz, (0, -1, 0))
    if lid:
        p += _face((x0, y0, 0.0), (lx, 0, 0), (0, ly, 0), nx, ny, (0, 0, 1))
    return np.array(p)


def reflect_full(quarter_panels: np.ndarray) -> np.ndarray:
    """The full mesh of a quarter mesh symmetric about x = 0 and y = 0: the stored panels, then
    their x, y and xy reflections (geometry.rs:208-235 order e, sigma_x, sigma_y, sigma_x sigma_y),
    a reflection that reverses orientation taking the vertices as v0 v3 v2 v1."""
    out = [quarter_panels]
    for sx, sy in ((-1.0, 1.0), (1.0, -1.0), (-1.0, -1.0)):
        w = quarter_panels * np.array([sx, sy, 1.0])
        if sx * sy < 0:
            w = w[:, [0, 3, 2, 1]]
        out.append(w)
    return np.concatenate(out)


def config_cylinder(n_phi, n_z, n_r, radius=1.0, draft=0.5) -> np.ndarray:
    return cylinder(radius, draft, n_phi=n_phi, n_z=n_z, n_r=n_r, quarter=False)


GRAVITY = 9.80665


def uneven_bodies(count=64, seed=20261203):
    """The batched uneven workload: ``count`` bodies drawn from ``seed`` -- truncated cylinders (radius
    U[0.5, 3] m, draught U[0.3, 2] m) or hemispheres (radius U[0.5, 3] m) with panel counts N ~ U[800,
    6000] rounded to the generators' grids -- each with 16 frequencies of wavenumber K r ~ U[0.1, 10].
    Returns [(vertices, omegas)]; the grids are drawn first and a mesh is built only for the bodies
    asked for, so ``uneven_bodies(count)[i]`` is the same body for every count > i."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        r, d, n = rng.uniform(0.5, 3.0), rng.uniform(0.3, 2.0), int(rng.uniform(800, 6000))
        if rng.uniform() < 0.5:
            nphi = max(8, int(round(np.sqrt(n) / 4)) * 4)
            nz = max(2, int(round(n / (2 * nphi))))
            v = cylinder(r, d, nphi, nz, nz)
        else:
            nphi = max(8, int(round(np.sqrt(2 * n) / 4)) * 4)
            v = hemisphere(r, max(2, int(round(n / nphi))), nphi)
        omegas = np.sqrt(rng.uniform(0.1, 10.0, 16) / r * GRAVITY)
        out.append((v, omegas))
    return out


def cylinder_array(n_phi=64, n_z=32, n_r=32, spacing=4.0):
    """Three cylinders of radius 1 m and draught 1 m, ``spacing`` apart along x, each rotating about its own
    axis at the waterline: (vertices, panel body, rotation centres)."""
    one = cylinder(1.0, 1.0, n_phi, n_z, n_r)
    parts, body, centers = [], [], []
    for b, x in enumerate((-spacing, 0.0, spacing)):
        c = one.copy()
        c[..., 0] += x
        parts.append(c)
        body.append(np.full(len(c), b, np.int32))
        centers.append([x, 0.0, 0.0])
    return np.concatenate(parts), np.concatenate(body), centers


def barge(n=(64, 32, 75)):
    """The 80 m x 20 m barge of 10 m draught with its interior waterplane lid: (vertices, kinds) with the
    lid's nx ny panels last and of kind 1 (interior surface)."""
    v = box(40.0, 10.0, 10.0, n=n, lid=True)
    kinds = np.zeros(len(v), np.int32)
    kinds[-n[0] * n[1]:] = 1
    return v, kinds
