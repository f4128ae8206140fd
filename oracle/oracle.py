"""CPU oracle of the low-order frequency-domain BEM path -- TEST INFRASTRUCTURE ONLY.

This module is the checker: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it, and never as the thing measured or shipped.  It drives the plain-C FP64
restatement ``libhb_oracle.so`` (``hb_oracle.c``) of HydroBEM's diagnostic double-precision path
and adds, in numpy, the steps that are short formulas of ``crates/hydrobem/src/``:

- incident wave and boundary values  ``low_order.rs:1397-1485``, ``lo_frequency.rs:214-273``
- right-hand sides -S u and the dense solve  ``lo_frequency.rs:823-955`` (LU with partial pivoting:
  LAPACK ``zgesv`` through numpy, standing in for faer's blocked LU, ``linalg.rs:134-252``)
- pressure integration A, B, X, FK, SC  ``lo_frequency.rs:1039-1115``
- the Haskind exciting force HK from the radiation potentials  ``lo_frequency.rs:1118-1171``
- Kochin functions of the radiation and scattered waves  ``lo_frequency.rs:1277-1374``,
  ``low_order.rs:1417-1452``, and the mean drift by momentum conservation  ``response.rs:51-300``
- field points: the elevation or p / (rho g) of the radiation, incident, scattered and total waves at
  points in the fluid by Green's identity over the panels  ``lo_frequency.rs:1392-1470``
- hydrostatics, rigid inertia and the motion equation of each frequency  ``hydrostatics.rs:116-356``,
  ``motion.rs:121-158``
- symmetry sectors (a body given as one sector of its mirror-symmetric mesh): the matrices of the
  mirrored mesh's sector rows summed over the reflections with the group's characters, one system
  per sector, the potentials recombined  ``lo_geometry.rs:25-36``, ``lo_frequency.rs:276-346,823-943``

Parity: pinned against the reference's golden kernel files (``tests/data/green_inf_reference.txt``,
``green_fin_reference.txt``, ``panel_reference.txt``, ``dispersion_reference.txt``) and against the
reference's own solver outputs (``tests/data/regression/lo_cylinder_drift.npz``) -- see
``tests/test_oracle_golden.py``.
"""

from __future__ import annotations

import collections
import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libhb_oracle.so"
TABLES = HERE.parent / "hydrobem_b200" / "tables" / "green_tables.bin"
GRAVITY = 9.80665
DENSITY = 1000.0
WET, INTERIOR = 0, 1


class Panel(ctypes.Structure):
    _fields_ = [
        ("nv", ctypes.c_int32),
        ("pad", ctypes.c_int32),
        ("v", ctypes.c_double * 12),
        ("c", ctypes.c_double * 3),
        ("n", ctypes.c_double * 3),
        ("area", ctypes.c_double),
        ("radius", ctypes.c_double),
        ("elen", ctypes.c_double * 4),
        ("em", ctypes.c_double * 12),
        ("gx", ctypes.c_double * 27),
        ("gw", ctypes.c_double * 9),
        ("q", ctypes.c_double * 12),
    ]


_lib = None


def build() -> None:
    """Compile the oracle library (make in this directory)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        build()
    L = ctypes.CDLL(str(LIB))
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int32)
    pp = ctypes.POINTER(Panel)
    L.hbo_load_tables.argtypes = [ctypes.c_char_p]
    L.hbo_set_production.argtypes = [ctypes.c_int]
    L.hbo_make_panels_kinds.argtypes = [ctypes.c_int, dp, ip, pp]
    L.hbo_wave_kernel.argtypes = [ctypes.c_double, ctypes.c_double, dp]
    L.hbo_dispersion_x0.argtypes = [ctypes.c_double]
    L.hbo_dispersion_x0.restype = ctypes.c_double
    L.hbo_dispersion_xn.argtypes = [ctypes.c_double, ctypes.c_int]
    L.hbo_dispersion_xn.restype = ctypes.c_double
    L.hbo_finite_kernel.argtypes = [ctypes.c_double] * 2 + [ctypes.c_int] + [ctypes.c_double] * 3 + [dp]
    L.hbo_rankine.argtypes = [pp, dp, dp]
    L.hbo_rankine_any.argtypes = [pp, dp, dp]
    L.hbo_log_singularity.argtypes = [pp, dp, dp]
    L.hbo_log_in_plane.argtypes = [pp, dp]
    L.hbo_log_in_plane.restype = ctypes.c_double
    L.hbo_statics.argtypes = [ctypes.c_int, pp, ip, ctypes.c_double, ctypes.c_int, ctypes.c_double, dp]
    L.hbo_assemble.argtypes = [ctypes.c_int, pp, ip, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                               ctypes.c_int, dp, dp]
    fp = ctypes.POINTER(ctypes.c_float)
    L.hbo_assemble_c64.argtypes = [ctypes.c_int, pp, ip, dp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_int, fp, fp]
    L.hbo_wavenumber.argtypes = [ctypes.c_double] * 3
    L.hbo_wavenumber.restype = ctypes.c_double
    L.hbo_field_influence.argtypes = [ctypes.c_int, pp, ip, ctypes.c_int, dp, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_int, ctypes.c_double, dp, dp]
    rc = L.hbo_load_tables(str(TABLES).encode())
    if rc != 0:
        raise RuntimeError(f"oracle: cannot load the Green-function tables {TABLES} (code {rc})")
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


# ------------------------------------------------------------------ kernels (golden-vector tests)
def wave_kernel(X: float, Y: float) -> np.ndarray:
    out = np.zeros(7)
    lib().hbo_wave_kernel(X, Y, _dp(out))
    return out


def finite_kernel(h, K, mode, R, z, zeta) -> np.ndarray:
    out = np.zeros(8)
    lib().hbo_finite_kernel(h, K, mode, R, z, zeta, _dp(out))
    return out


def dispersion_x0(H):
    return lib().hbo_dispersion_x0(H)


def dispersion_xn(H, n):
    return lib().hbo_dispersion_xn(H, n)


# ------------------------------------------------------------------ panels and statics
def make_panels(verts: np.ndarray, kinds=None):
    v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 12)
    n = v.shape[0]
    k = None if kinds is None else np.ascontiguousarray(kinds, dtype=np.int32)
    arr = (Panel * n)()
    rc = lib().hbo_make_panels_kinds(n, _dp(v), None if k is None else _ip(k), arr)
    if rc != 0:
        raise ValueError(f"invalid panel {rc - 1}")
    return arr


def panel_arrays(panels):
    """Centroid, normal and area of every panel as numpy arrays."""
    c = np.array([list(p.c) for p in panels])
    n = np.array([list(p.n) for p in panels])
    a = np.array([p.area for p in panels])
    return c, n, a


def rankine(panel, x):
    out = np.zeros(2)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    lib().hbo_rankine(ctypes.byref(panel), _dp(xx), _dp(out))
    return out


def rankine_any(panel, x):
    out = np.zeros(2)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    lib().hbo_rankine_any(ctypes.byref(panel), _dp(xx), _dp(out))
    return out


def log_singularity(panel, image):
    out = np.zeros(2)
    xx = np.ascontiguousarray(image, dtype=np.float64)
    lib().hbo_log_singularity(ctypes.byref(panel), _dp(xx), _dp(out))
    return out


def statics(panels, kinds, depth, logint=True, tol=1e-4) -> np.ndarray:
    n = len(panels)
    out = np.zeros((n, n, 4))
    k = np.zeros(n, np.int32) if kinds is None else np.ascontiguousarray(kinds, dtype=np.int32)
    d = depth if (depth is not None and np.isfinite(depth) and depth > 0) else np.inf
    lib().hbo_statics(n, panels, _ip(k), d, int(logint), tol, _dp(out))
    return out


def assemble(panels, kinds, st, depth, omega, grav=GRAVITY, logint=True, dtype=np.complex128):
    """(S, A) N x N (entry [k, n], Fortran order) of one ordinary frequency, complex128 or (the production
    path's storage) complex64."""
    n = len(panels)
    S = np.empty((n, n), dtype=dtype, order="F")
    A = np.empty((n, n), dtype=dtype, order="F")
    k = np.zeros(n, np.int32) if kinds is None else np.ascontiguousarray(kinds, dtype=np.int32)
    d = depth if (depth is not None and np.isfinite(depth) and depth > 0) else np.inf
    if np.dtype(dtype) == np.complex64:
        fp = ctypes.POINTER(ctypes.c_float)
        lib().hbo_assemble_c64(n, panels, _ip(k), _dp(st), d, omega, grav, int(logint),
                               S.ctypes.data_as(fp), A.ctypes.data_as(fp))
    else:
        lib().hbo_assemble(n, panels, _ip(k), _dp(st), d, omega, grav, int(logint),
                           S.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                           A.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return S, A


def lu_solve(A, B):
    """A X = B by LAPACK ?gesv (LU with partial pivoting; scipy's threaded OpenBLAS: cgesv for complex64,
    zgesv for complex128), standing in for faer's blocked LU (linalg.rs:134-252, 321-354).  A is
    overwritten when it is a Fortran-ordered array of the solve's type."""
    from scipy.linalg import lapack

    gesv = lapack.cgesv if A.dtype == np.complex64 else lapack.zgesv
    lu, piv, x, info = gesv(A, np.asarray(B, dtype=A.dtype), overwrite_a=True, overwrite_b=False)
    if info != 0:
        raise np.linalg.LinAlgError(f"singular matrix (?gesv info {info})")
    return x


# ------------------------------------------------------------------ one frequency
def incident(c, depth, k, omega, beta, grav=GRAVITY):
    """(phi_I, grad phi_I) at the points c (low_order.rs:1441-1459, frame at the origin, yaw 0)."""
    cb, sb = np.cos(beta), np.sin(beta)
    phase = -k * (c[:, 0] * cb + c[:, 1] * sb)
    Z = np.exp(k * c[:, 2])
    Zz = k * Z
    if depth is not None and np.isfinite(depth) and depth > 0:
        b = np.exp(-k * (c[:, 2] + 2.0 * depth))
        dd = 1.0 + np.exp(-2.0 * k * depth)
        Zz = k * (Z - b) / dd
        Z = (Z + b) / dd
    e = (1j * grav / omega) * (np.cos(phase) + 1j * np.sin(phase))
    phi = e * Z
    grad = np.stack([phi * (-1j * k * cb), phi * (-1j * k * sb), e * Zz], axis=1)
    return phi, grad


def rigid_normals(c, n, kinds, panel_body=None, centers=None):
    """Generalized normals [N][6 n_bodies]: for body b's modes, (n, (c - R_b) x n) on its panels and 0
    elsewhere; 0 off the wetted surface (lo_geometry.rs:805-811, lo_frequency.rs:236-251). One body
    about the origin when panel_body and centers are None."""
    nb = 1 if panel_body is None else int(np.max(panel_body)) + 1
    if centers is not None:
        nb = max(nb, len(centers))
    body = np.zeros(len(c), int) if panel_body is None else np.asarray(panel_body)
    R = np.zeros((nb, 3)) if centers is None else np.asarray(centers, dtype=float).reshape(-1, 3)
    nj = np.zeros((len(c), 6 * nb))
    for b in range(nb):
        on = body == b
        nj[on, 6 * b:6 * b + 3] = n[on]
        nj[on, 6 * b + 3:6 * b + 6] = np.cross(c[on] - R[b], n[on])
    if kinds is not None:
        nj[np.asarray(kinds) != WET] = 0.0
    return nj


# ------------------------------------------------------------------ symmetry sectors
SYM_NONE, SYM_YZ, SYM_XZ, SYM_BOTH = 0, 1, 2, 3


def sector_count(symmetry: int) -> int:
    return {SYM_NONE: 1, SYM_YZ: 2, SYM_XZ: 2, SYM_BOTH: 4}[int(symmetry)]


def character(c: int, g: int) -> float:
    """chi_c(g) of the reflection group, elements e, x, y, xy reflections (lo_geometry.rs:25-36)."""
    return -1.0 if bin(c & g).count("1") % 2 else 1.0


def mirror_sector(verts, symmetry):
    """The panels of a sector followed by their images in the group's element order (image g of panel n
    at g Ns + n); a reflection that reverses orientation takes the vertices as v0 v3 v2 v1."""
    v = np.asarray(verts, dtype=np.float64).reshape(-1, 4, 3)
    refl = {SYM_NONE: [], SYM_YZ: [(-1.0, 1.0)], SYM_XZ: [(1.0, -1.0)],
            SYM_BOTH: [(-1.0, 1.0), (1.0, -1.0), (-1.0, -1.0)]}[int(symmetry)]
    out = [v]
    for sx, sy in refl:
        w = v * np.array([sx, sy, 1.0])
        out.append(w[:, [0, 3, 2, 1]] if sx * sy < 0 else w)
    return np.concatenate(out)


class ProductionMode:
    """Context in which the oracle computes the reference's default (production) arithmetic instead of
    its diagnostic double path: float32 Gauss tiers for the Rankine integrals, the direct 2-D tables of
    the wave kernel, float32 static rows (hbo_set_production), and -- in solve_frequency -- complex64
    matrices, right-hand sides and LU (LAPACK cgesv through numpy; linalg.rs:321-354 with R = f32)."""

    def __init__(self, on=True):
        self.on = bool(on)

    def __enter__(self):
        lib().hbo_set_production(int(self.on))
        return self

    def __exit__(self, *a):
        lib().hbo_set_production(0)


def sector_solve(S, A, u, G):
    """phi on every panel of the mirrored mesh from the G sector systems (lo_frequency.rs:823-943): for
    character c, S_c and A_c the sums over g of chi_c(g) times the column block g of the sector rows,
    right-hand sides -S_c U_c with U_c = (1/G) sum_g chi_c(g) u(g n), and phi(g n) = sum_c chi_c(g) x_c(n)."""
    Ns = S.shape[0] // G
    blk = lambda M, g: M[:Ns, g * Ns:(g + 1) * Ns]
    phi = np.zeros((S.shape[0], u.shape[1]), dtype=np.complex128)
    for c in range(G):
        Sc = sum(character(c, g) * blk(S, g) for g in range(G))
        Ac = sum(character(c, g) * blk(A, g) for g in range(G))
        Uc = sum(character(c, g) * u[g * Ns:(g + 1) * Ns] for g in range(G)) / G
        xc = lu_solve(np.asfortranarray(Ac), Sc @ (-Uc))
        for g in range(G):
            phi[g * Ns:(g + 1) * Ns] += character(c, g) * xc
    return phi


def depth_factor(z, depth, k):
    """(Z, dZ/dz) of the wave's vertical profile at depths z (low_order.rs:1401-1412): e^{kz} in infinite
    depth, cosh k(z + h) / cosh kh in depth h."""
    Z = np.exp(k * z)
    Zz = k * Z
    if depth is not None and np.isfinite(depth) and depth > 0:
        b = np.exp(-k * (z + 2.0 * depth))
        dd = 1.0 + np.exp(-2.0 * k * depth)
        Zz = k * (Z - b) / dd
        Z = (Z + b) / dd
    return Z, Zz


def kochin(c, n, area, wet, depth, k, phi, u, phiI, D, n_angles):
    """Kochin functions of one frequency on n_angles global angles theta_t = 2 pi t / n_angles
    (lo_frequency.rs:1277-1374 on this route's panels, the frame at the origin with no yaw): Green's
    identity with the far-field kernel (low_order.rs:1417-1431: g = Z e^{i k (x cos + y sin)}, its normal
    derivative gn and the theta-derivatives gt, gnt) over the wetted panels, the interior panels taking no
    part.  Radiation column c: H = sum_j phi_c Dx - Sx u_c; heading h (scattered formulation): H = sum_j
    (phi_S + phi_I) Dx.  Returns (kr, krt) [T][D] and (kd, kdt) [T][H], H_t the theta-derivative."""
    th = 2.0 * np.pi * np.arange(n_angles) / n_angles
    cs, sn = np.cos(th)[:, None], np.sin(th)[:, None]
    x, y = c[None, :, 0], c[None, :, 1]
    Z, Zz = depth_factor(c[:, 2], depth, k)
    e = np.exp(1j * k * (x * cs + y * sn))
    ik = 1j * k
    dt = -x * sn + y * cs
    dnt = -n[None, :, 0] * sn + n[None, :, 1] * cs
    g = Z[None] * e
    gn = e * (Z[None] * ik * (n[None, :, 0] * cs + n[None, :, 1] * sn) + Zz[None] * n[None, :, 2])
    gt = g * ik * dt
    gnt = gn * ik * dt + e * Z[None] * ik * dnt
    w = (area * wet)[None]
    Sx, Dx, St, Dt = w * g, w * gn, w * gt, w * gnt
    kr = Dx @ phi[:, :D] - Sx @ u[:, :D]
    krt = Dt @ phi[:, :D] - St @ u[:, :D]
    tot = phi[:, D:] + np.where(wet[:, None], phiI.T, 0.0)
    return kr, krt, Dx @ tot, Dt @ tot


def kochin_angle_count(verts, omegas, depth, grav=GRAVITY):
    """The reference's automatic count (response.rs:109-176): 8 ceil((2 ceil(k R) + 96) / 8) for the
    largest wave number k and the largest horizontal distance R of a vertex from the origin."""
    k = max(lib().hbo_wavenumber(w, depth if depth else np.inf, grav) for w in omegas)
    R = float(np.hypot(np.asarray(verts)[..., 0], np.asarray(verts)[..., 1]).max())
    n = 2 * int(np.ceil(k * R)) + 96
    return 8 * ((n + 7) // 8)


def momentum_drift(omegas, headings_deg, kd, kdt, kr, krt, xi, depth=np.inf, grav=GRAVITY, rho=DENSITY):
    """Mean drift forces by momentum conservation from the Kochin functions (response.rs:183-300):
    surge, sway force and yaw moment of every heading pair [F][H][H][3] (complex; the equal pairs are the
    real unidirectional coefficients).  kd, kdt [F][T][H]; kr, krt [F][T][K] and xi [F][H][K] the motions
    of the radiation columns (None: a fixed body)."""
    F, T, H = kd.shape
    th = 2.0 * np.pi * np.arange(T) / T
    dth = 2.0 * np.pi / T
    beta = np.radians(np.asarray(headings_deg, dtype=float))
    lo = -(T - 1) // 2 if T % 2 else -(T - 1) // 2
    modes = np.arange(lo, -lo + 1)

    def coefficients(v):  # the trigonometric interpolant's coefficients (and the Nyquist one for even T)
        c = np.array([(v * np.exp(-2j * np.pi * m * np.arange(T) / T)).sum() / T for m in modes])
        if T % 2 == 0:
            c = np.append(c, (v * (-1.0) ** np.arange(T)).sum() / T)
        return c

    def value(c, b):  # the interpolant at angle b
        e = np.exp(1j * modes * b)
        if T % 2 == 0:
            e = np.append(e, np.cos(T / 2 * b))
        return (c * e).sum()

    out = np.zeros((F, H, H, 3), dtype=np.complex128)
    for f, w in enumerate(omegas):
        K0 = w * w / grav
        k = lib().hbo_wavenumber(w, depth if depth else np.inf, grav)
        C, Ke = 2.0 * np.pi * K0, K0
        if depth is not None and np.isfinite(depth) and depth > 0:
            x = k * depth
            A0 = 2.0 * np.pi * k / (-np.expm1(-4.0 * x) + 4.0 * x * np.exp(-2.0 * x))
            C = A0 * (1.0 + np.exp(-2.0 * x)) ** 2
            Ke = K0 + k * k * depth / np.cosh(x) ** 2
        fac = -(1j * C / (4.0 * np.pi)) * np.sqrt(2.0 / (np.pi * k)) * np.exp(1j * np.pi / 4.0)
        a, e, q = 1j * grav / w, np.exp(-1j * np.pi / 4.0), np.sqrt(2.0 * np.pi / k)
        b = kd[f].T.astype(np.complex128)   # [H][T]
        bt = kdt[f].T.astype(np.complex128)
        if xi is not None and kr is not None:
            b = b + 1j * w * (xi[f] @ kr[f].T)
            bt = bt + 1j * w * (xi[f] @ krt[f].T)
        b, bt = fac * b, fac * bt
        cf = [coefficients(b[i]) for i in range(H)]
        cft = [coefficients(bt[i]) for i in range(H)]
        bb = np.array([[value(cf[i], beta[j]) for j in range(H)] for i in range(H)])
        bbt = np.array([[value(cft[i], beta[j]) for j in range(H)] for i in range(H)])
        s = rho * Ke / 4.0
        for i in range(H):
            for j in range(H):
                pij = b[i] * np.conj(b[j])
                sx, sy = (pij * np.cos(th)).sum(), (pij * np.sin(th)).sum()
                dd = (bt[i] * np.conj(b[j]) - b[i] * np.conj(bt[j])).sum() * (-0.5j)
                cx = -s * q * np.conj(a) * e * bb[i, j]
                cy = -s * q * a * np.conj(e) * np.conj(bb[j, i])
                o = out[f, i, j]
                o[0] = -s * sx * dth + cx * np.cos(beta[j]) + cy * np.cos(beta[i])
                o[1] = -s * sy * dth + cx * np.sin(beta[j]) + cy * np.sin(beta[i])
                o[2] = (s / k) * dd * dth - (s / k) * q * (1j * np.conj(a) * e * bbt[i, j]
                                                            - 1j * a * np.conj(e) * np.conj(bbt[j, i]))
                if i == j:
                    out[f, i, j] = o.real
    return out


def solve_frequency(panels, kinds, st, depth, omega, headings_rad, grav=GRAVITY, rho=DENSITY, logint=True,
                    want_matrices=False, panel_body=None, centers=None, sectors=1, points=None, tol=1e-4,
                    production=False, kochin_angles=0):
    """A, B [D][D], X, FK, SC, HK [H][D] of one frequency (D = 6 per body), all in float64 (complex128).
    sectors > 1: the panels are a mirrored mesh (mirror_sector) solved by its symmetry sectors.
    production: the reference's default path (class production) -- statics computed in that mode are
    expected; the matrices, right-hand sides and LU in complex64, the forces summed in float64."""
    c, n, area = panel_arrays(panels)
    N = len(panels)
    with ProductionMode(production):
        S, A = assemble(panels, kinds, st, depth, omega, grav, logint,
                        dtype=np.complex64 if production else np.complex128)
    if want_matrices:
        A0 = A.copy()
    k = lib().hbo_wavenumber(omega, depth if depth else np.inf, grav)
    wet = np.ones(N, bool) if kinds is None else (np.asarray(kinds) == WET)
    nj = rigid_normals(c, n, kinds, panel_body, centers)
    D = nj.shape[1]
    H = len(headings_rad)
    u = np.zeros((N, D + H), dtype=np.complex128)
    u[:, :D] = nj
    phiI = np.zeros((H, N), dtype=np.complex128)
    dphiI = np.zeros((H, N), dtype=np.complex128)
    for h, beta in enumerate(headings_rad):
        pI, gr = incident(c, depth, k, omega, beta, grav)
        phiI[h] = pI
        d = (gr * n).sum(axis=1)
        dphiI[h] = d
        u[:, D + h] = np.where(wet, -d, 0.0)
    uu = u.astype(S.dtype)
    rhs = S @ (-uu)
    phi = (lu_solve(A, rhs) if sectors == 1 else sector_solve(S, A, uu, sectors)).astype(np.complex128)
    w = (nj * area[:, None]) * wet[:, None]          # n_i A_j on the body panels
    z = -rho * (w.T @ phi[:, :D])                    # [i][c]
    out = {"A": z.real, "B": -omega * z.imag}
    if H:
        x = w.T @ (phi[:, D:] + phiI.T)              # [i][h]
        fk = w.T @ phiI.T
        iwr = 1j * omega * rho
        out["X"] = (iwr * x).T
        out["FK"] = (iwr * fk).T
        out["SC"] = (iwr * (x - fk)).T
        # Haskind relation (lo_frequency.rs:1118-1171): i w rho sum over wetted panels of
        # (n_c phi_I - phi_c dphi_I/dn) A_j, per radiation column c; given [h][c] as the other forces
        hk = w.T @ phiI.T - ((phi[:, :D] * (area * wet)[:, None]).T @ dphiI.T)
        out["HK"] = (iwr * hk).T
    if points is not None and len(points):
        out.update(field_values(panels, kinds, points, depth, omega, headings_rad, phi, u, phiI, D, grav, logint, tol))
    if kochin_angles and H:
        out["kr"], out["krt"], out["kd"], out["kdt"] = kochin(c, n, area, wet, depth, k, phi, u, phiI, D,
                                                               kochin_angles)
    if want_matrices:
        out["S"], out["Amat"], out["rhs"], out["phi"] = S, A0, rhs, phi
    return out


# ------------------------------------------------------------------ generated interior surface
def projected_lid(verts, z0=0.0):
    """interior.rs:79-138 projected: the downward-facing panels (unit normal of the diagonals' cross product
    with n_z < -1e-6) projected onto z = z0 with their vertex order reversed (facing up); panels in z0 and
    vertical ones skipped; an upward-facing panel (n_z > 1e-6) raises ValueError."""
    v = np.asarray(verts, dtype=np.float64).reshape(-1, 4, 3)
    tol = 1e-6 * max(1.0, np.abs(v).max())
    out = []
    for k, q in enumerate(v):
        if np.all(np.abs(q[:, 2] - z0) <= tol):
            continue
        n = np.cross(q[2] - q[0], q[3] - q[1])
        nz = n[2] / np.linalg.norm(n)
        if nz > 1e-6:
            raise ValueError(f"wetted element {k + 1} faces upward")
        if nz >= -1e-6:
            continue
        w = q[::-1].copy()
        w[:, 2] = z0
        out.append(w)
    if not out:
        raise ValueError("no wetted element faces downward")
    return np.array(out)


def _dist(a, b):
    return float(np.hypot(a[0] - b[0], a[1] - b[1]))


def _orient(o, a, b):
    return (a[0] - o[0]) * (b[1] - o[1]) - (a[1] - o[1]) * (b[0] - o[0])


def _seg_dist(x, a, b):
    """polygon.rs:94-99 the distance from x to the segment ab."""
    e = (b[0] - a[0], b[1] - a[1])
    w = (x[0] - a[0], x[1] - a[1])
    ee = e[0] * e[0] + e[1] * e[1]
    t = min(1.0, max(0.0, (w[0] * e[0] + w[1] * e[1]) / ee)) if ee > 0.0 else 0.0
    return _dist(x, (a[0] + t * e[0], a[1] + t * e[1]))


def _meet(p, q, a, b):
    """polygon.rs:81-90 whether the segments pq and ab cross or touch."""
    d1, d2, d3, d4 = _orient(a, b, p), _orient(a, b, q), _orient(p, q, a), _orient(p, q, b)
    if ((d1 > 0 and d2 < 0) or (d1 < 0 and d2 > 0)) and ((d3 > 0 and d4 < 0) or (d3 < 0 and d4 > 0)):
        return True

    def on(o, e, x, d):
        return d == 0.0 and min(o[0], e[0]) <= x[0] <= max(o[0], e[0]) and min(o[1], e[1]) <= x[1] <= max(o[1], e[1])

    return on(a, b, p, d1) or on(a, b, q, d2) or on(p, q, a, d3) or on(p, q, b, d4)


def _loops_meet(loops, tol):
    """polygon.rs:111-149 whether two loops, or two non-adjacent edges of one loop, cross or come within tol."""
    edges = [(li, k, lp[k], lp[(k + 1) % len(lp)]) for li, lp in enumerate(loops) for k in range(len(lp))]
    for i in range(len(edges)):
        for j in range(i + 1, len(edges)):
            e, f = edges[i], edges[j]
            if (min(e[2][0], e[3][0]) - tol > max(f[2][0], f[3][0]) + tol
                    or min(f[2][0], f[3][0]) - tol > max(e[2][0], e[3][0]) + tol
                    or min(e[2][1], e[3][1]) - tol > max(f[2][1], f[3][1]) + tol
                    or min(f[2][1], f[3][1]) - tol > max(e[2][1], e[3][1]) + tol):
                continue
            if e[0] == f[0]:
                n = len(loops[e[0]])
                if n <= 3 or (e[1] + 1) % n == f[1] or (f[1] + 1) % n == e[1]:
                    continue
            if (_meet(e[2], e[3], f[2], f[3]) or _seg_dist(e[2], f[2], f[3]) <= tol or _seg_dist(e[3], f[2], f[3]) <= tol
                    or _seg_dist(f[2], e[2], e[3]) <= tol or _seg_dist(f[3], e[2], e[3]) <= tol):
                return True
    return False


def _inside(loop, x):
    """polygon.rs:29-39 crossing-number test."""
    c = False
    n = len(loop)
    for k in range(n):
        p, q = loop[k], loop[(k + 1) % n]
        if (p[1] > x[1]) != (q[1] > x[1]) and x[0] < p[0] + (x[1] - p[1]) / (q[1] - p[1]) * (q[0] - p[0]):
            c = not c
    return c


def _signed_area(loop):
    n = len(loop)
    return 0.5 * sum(loop[k][0] * loop[(k + 1) % n][1] - loop[(k + 1) % n][0] * loop[k][1] for k in range(n))


def _waterplane_loops(verts, isx, isy, z0, reference_length, merge_collinear):
    """interior.rs:139-153 the closed waterline contours of the stored panels in the quadrant x, y >= 0:
    (loops, sx, sy, target = the mean waterline segment length, ax_x, ax_y, tol); with merge_collinear
    the collinear points of every loop are merged (the waterline generator), not for the fan."""
    v = np.asarray(verts, dtype=np.float64).reshape(-1, 4, 3)
    tol = 1e-6 * max(reference_length, float(np.abs(v).max()) if v.size else 0.0)
    segs = []
    total = 0.0
    for q in v:
        n = np.cross(q[2] - q[0], q[3] - q[1])
        nn = np.linalg.norm(n)
        n = n / nn if nn > 0 else n
        if np.hypot(n[0], n[1]) < 1e-6:
            continue
        d = (-n[1], n[0])
        for i in range(4):
            u, w = q[i], q[(i + 1) % 4]
            if abs(u[2] - z0) > tol or abs(w[2] - z0) > tol:
                continue
            a, b = (u[0], u[1]), (w[0], w[1])
            if _dist(a, b) <= tol:
                continue
            if (b[0] - a[0]) * d[0] + (b[1] - a[1]) * d[1] < 0.0:
                a, b = b, a
            segs.append([a, b])
            total += _dist(a, b)
    if not segs:
        raise ValueError("the wetted surface has no waterline")
    mx = sum(s[0][0] + s[1][0] for s in segs)
    my = sum(s[0][1] + s[1][1] for s in segs)
    sx = -1.0 if isx and mx < 0.0 else 1.0
    sy = -1.0 if isy and my < 0.0 else 1.0
    for s in segs:
        s[0] = (sx * s[0][0], sy * s[0][1])
        s[1] = (sx * s[1][0], sy * s[1][1])
        if sx * sy < 0.0:
            s[0], s[1] = s[1], s[0]
    # chains (from a segment without a predecessor) and closed loops
    n = len(segs)
    nxt, prv = [-1] * n, [-1] * n
    for i in range(n):
        for j in range(n):
            if i == j or _dist(segs[i][1], segs[j][0]) > tol:
                continue
            if nxt[i] >= 0 or prv[j] >= 0:
                raise ValueError("waterline contours touch or cross")
            nxt[i], prv[j] = j, i
    used = [False] * n
    chains, loops = [], []
    for s in range(n):
        if prv[s] >= 0:
            continue
        c, k = [segs[s][0]], s
        while k >= 0:
            used[k] = True
            c.append(segs[k][1])
            k = nxt[k]
        chains.append(c)
    for s in range(n):
        if used[s]:
            continue
        c, k = [], s
        while not used[k]:
            used[k] = True
            c.append(segs[k][0])
            k = nxt[k]
            if k < 0:
                raise RuntimeError("broken waterline loop")
        loops.append(c)
    ax_x, ax_y = bool(isy), bool(isx)

    def on_x(p):
        return ax_x and abs(p[1]) <= tol and (p[0] >= -tol or not ax_y)

    def on_y(p):
        return ax_y and abs(p[0]) <= tol and (p[1] >= -tol or not ax_x)

    def key_start(p):
        return (0, p[0]) if on_x(p) else (1, -p[1])

    def key_end(p):
        return (1, -p[1]) if on_y(p) else (0, p[0])

    for c in chains:
        if not (on_x(c[0]) or on_y(c[0])) or not (on_x(c[-1]) or on_y(c[-1])):
            raise ValueError("the waterline does not close")
    cused = [False] * len(chains)
    for c0 in range(len(chains)):
        if cused[c0]:
            continue
        lp, c = [], c0
        while True:
            cused[c] = True
            lp.extend(chains[c])
            ke = key_end(chains[c][-1])
            best, wrap = -1, False
            for pas in range(2):
                if best >= 0:
                    break
                for d in range(len(chains)):
                    if cused[d] and d != c0:
                        continue
                    ks = key_start(chains[d][0])
                    if pas == 0 and ks < ke:
                        continue
                    if best < 0 or ks < key_start(chains[best][0]):
                        best = d
                wrap = pas == 1
            if best < 0:
                raise ValueError("the waterline does not close")
            ks = key_start(chains[best][0])
            if ke[0] == 0 and ks[0] == 1 and not wrap:
                raise ValueError("the waterline does not close")
            if wrap:
                if not (ax_x and ax_y):
                    raise ValueError("the waterline does not close")
                lp.append((0.0, 0.0))
            if best == c0:
                break
            c = best
        loops.append(lp)
    for i, lp in enumerate(loops):
        c = []
        for p in lp:
            if not c or _dist(c[-1], p) > tol:
                c.append(p)
        while len(c) > 1 and _dist(c[0], c[-1]) <= tol:
            c.pop()
        loops[i] = _merge_collinear(c, tol) if merge_collinear else c
    if _loops_meet(loops, tol):
        raise ValueError("waterline contours cross or touch")
    return loops, sx, sy, total / len(segs), ax_x, ax_y, tol


def graded_lid(verts, isx=0, isy=0, z0=0.0, reference_length=1.0):
    """interior.rs:139-515 graded: the interior free surface fanned from the area centroid of each
    waterplane region to its waterline segments, the rays divided at t_k = sin(pi k / (2N)).

    ``verts`` [P][4][3] the stored panels of the mesh (one sector when isx / isy declare the planes
    x = 0 / y = 0); returns the generated panels [Q][4][3] in the same stored form (a triangle repeats its
    last vertex), facing up.  Steps:

    - waterline segments (interior.rs:158-214): the edges lying in z0 (within tol = 1e-6 max(reference
      length, |vertex coordinates|)) of the non-horizontal panels (|n_h| >= 1e-6), oriented along
      z x n_h, mapped to the quadrant x, y >= 0 by the sign of the coordinate sums on symmetric axes;
    - chains and loops (interior.rs:217-272), open chains closed along the symmetry axes through the
      quadrant corner (interior.rs:274-340), repeated points dropped (interior.rs:343-357);
    - contours that cross or touch, openings, or a region whose waterline a centroid ray meets twice
      raise ValueError, as the reference does."""
    v = np.asarray(verts, dtype=np.float64).reshape(-1, 4, 3)
    loops, sx, sy, _, ax_x, ax_y, tol = _waterplane_loops(v, isx, isy, z0, reference_length, False)
    outers = [lp for lp in loops if len(lp) >= 3 and _signed_area(lp) > 0.0]
    holes = [lp for lp in loops if len(lp) >= 3 and not _signed_area(lp) > 0.0]
    if not outers:
        raise ValueError("no enclosed region")
    for h in holes:
        if not any(_inside(o, h[0]) for o in outers):
            raise ValueError("a waterline contour lies outside the body")
        raise ValueError("a waterplane region has an opening (a moonpool)")
    out = []

    def mapped(cs):
        w = np.zeros((4, 3))
        for k, p in enumerate(cs):
            w[k] = (sx * p[0], sy * p[1], z0)
        if sx * sy < 0.0:
            w[:len(cs)] = w[:len(cs)][::-1]
        if len(cs) == 3:
            w[3] = w[2]
        return w

    for lp in outers:
        a = cx = cy = 0.0
        on_y0 = on_x0 = False
        m = len(lp)
        for i in range(m):
            p, q = lp[i], lp[(i + 1) % m]
            cr = p[0] * q[1] - p[1] * q[0]
            a += 0.5 * cr
            cx += (p[0] + q[0]) * cr / 6.0
            cy += (p[1] + q[1]) * cr / 6.0
            on_y0 = on_y0 or (ax_x and abs(p[1]) <= tol and abs(q[1]) <= tol)
            on_x0 = on_x0 or (ax_y and abs(p[0]) <= tol and abs(q[0]) <= tol)
        c = [cx / a, cy / a]
        if on_x0:
            c[0] = 0.0
        if on_y0:
            c[1] = 0.0
        fan, ray, seg = [], 0.0, 0.0
        for i in range(m):
            p, q = lp[i], lp[(i + 1) % m]
            s = _orient(c, p, q)
            if abs(s) <= tol * _dist(p, q):
                continue
            if s < 0.0:
                raise ValueError("a ray from the centroid of a waterplane region meets its waterline more than once")
            fan.append((p, q))
            ray += 0.5 * (_dist(c, p) + _dist(c, q))
            seg += _dist(p, q)
        if not fan:
            raise ValueError("no enclosed region")
        N = max(1, int(np.ceil(ray / seg - 1e-9)))
        t = [1.0 if k == N else float(np.sin(0.5 * np.pi * k / N)) for k in range(N + 1)]

        def at(p, s):
            return (c[0] + s * (p[0] - c[0]), c[1] + s * (p[1] - c[1]))

        for p, q in fan:
            out.append(mapped([tuple(c), at(p, t[1]), at(q, t[1])]))
            for k in range(1, N):
                out.append(mapped([at(p, t[k]), at(p, t[k + 1]), at(q, t[k + 1]), at(q, t[k])]))
    return np.array(out)


# ------------------------------------------------------------------ field points
def field_influence(panels, kinds, pts, depth, omega, grav=GRAVITY, logint=True, tol=1e-4):
    """(S, D) [P][N] complex128: the influence of every panel at every field point."""
    n = len(panels)
    p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    S = np.zeros((len(p), n), dtype=np.complex128)
    D = np.zeros((len(p), n), dtype=np.complex128)
    k = np.zeros(n, np.int32) if kinds is None else np.ascontiguousarray(kinds, dtype=np.int32)
    d = depth if (depth is not None and np.isfinite(depth) and depth > 0) else np.inf
    lib().hbo_field_influence(n, panels, _ip(k), len(p), _dp(p), d, omega, grav, int(logint), tol,
                              S.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                              D.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return S, D


def field_values(panels, kinds, pts, depth, omega, heads_rad, phi, u, phiI, nrad, grav=GRAVITY, logint=True,
                 tol=1e-4):
    """lo_frequency.rs:1392-1470: at each point the elevation (z = 0) or p / (rho g): radiation
    w^2/g (1/4 pi) sum_j (phi_c D - S u_c) [P][nrad]; per heading the incident wave (-i w / g) phi_I, the
    scattered (-i w / g) (1/4 pi) sum_j (phi_S + phi_I) D (phi_I on the wetted panels) and their sum
    [P][H]; the interior panels take no part.  phi, u [N][nrhs], phiI [H][N]."""
    S, D = field_influence(panels, kinds, pts, depth, omega, grav, logint, tol)
    interior = np.zeros(len(panels), bool) if kinds is None else np.asarray(kinds) != WET
    S[:, interior] = 0.0
    D[:, interior] = 0.0
    frad = (omega * omega / grav) * (D @ phi[:, :nrad] - S @ u[:, :nrad]) / (4.0 * np.pi)
    H = len(heads_rad)
    p = np.asarray(pts, dtype=np.float64).reshape(-1, 3)
    k = lib().hbo_wavenumber(omega, depth if depth else np.inf, grav)
    finc = np.zeros((len(p), H), dtype=np.complex128)
    fsca = np.zeros_like(finc)
    for h, beta in enumerate(heads_rad):
        pI, _ = incident(p, depth, k, omega, beta, grav)
        v = D @ (phi[:, nrad + h] + np.where(interior, 0.0, phiI[h]))
        finc[:, h] = pI * (-1j * omega / grav)
        fsca[:, h] = v / (4.0 * np.pi) * (-1j * omega / grav)
    return {"field_radiation": frad, "field_incident": finc, "field_scattering": fsca, "field_diffraction": finc + fsca}


# ------------------------------------------------------------------ hydrostatics and motions
def hydrostatics(c, n, area, kinds=None, panel_body=None, centers=None, rho=DENSITY, grav=GRAVITY, rigid=None):
    """The hydrostatics of every body (hydrostatics.rs:116-313; one quadrature point per panel, its centroid
    with n dS = area n, quadrature.rs:152-159) and, with rigid (the dict of native.Body), the motion matrices:
    (records, M, C, B_ext) with M the rigid inertia about the rotation centres (hydrostatics.rs:315-356), C
    the restoring matrix with the weight terms plus the additional stiffness, all D x D."""
    nb = 1 if panel_body is None else int(np.max(panel_body)) + 1
    if centers is not None:
        nb = max(nb, len(centers))
    body = np.zeros(len(c), int) if panel_body is None else np.asarray(panel_body)
    R = np.zeros((nb, 3)) if centers is None else np.asarray(centers, dtype=float).reshape(-1, 3)
    wet = np.ones(len(c), bool) if kinds is None else np.asarray(kinds) == WET
    D = 6 * nb
    M, C, Bx = np.zeros((D, D)), np.zeros((D, D)), np.zeros((D, D))
    recs = []
    for b in range(nb):
        on = wet & (body == b)
        x, y, z = c[on, 0] - R[b, 0], c[on, 1] - R[b, 1], c[on, 2]
        nds = area[on, None] * n[on]
        vx, vy, V = (x * nds[:, 0]).sum(), (y * nds[:, 1]).sum(), (z * nds[:, 2]).sum()
        mx, my, mz = (0.5 * x * x * nds[:, 0]).sum(), (0.5 * y * y * nds[:, 1]).sum(), (0.5 * z * z * nds[:, 2]).sum()
        aw, ax, ay = -nds[:, 2].sum(), -(x * nds[:, 2]).sum(), -(y * nds[:, 2]).sum()
        axx, ayy, axy = -(x * x * nds[:, 2]).sum(), -(y * y * nds[:, 2]).sum(), -(x * y * nds[:, 2]).sum()
        rg, Vzb = rho * grav, mz - R[b, 2] * V
        crg = np.zeros((6, 6))
        crg[2, 2] = rg * aw
        crg[2, 3] = crg[3, 2] = rg * ay
        crg[2, 4] = crg[4, 2] = -rg * ax
        crg[3, 3] = rg * (ayy + Vzb)
        crg[3, 4] = crg[4, 3] = -rg * axy
        crg[3, 5] = -rg * mx
        crg[4, 4] = rg * (axx + Vzb)
        crg[4, 5] = -rg * my
        cw = crg.copy()
        mass = np.nan
        Mb = np.zeros((6, 6))
        if rigid is not None:
            m0 = np.asarray(rigid["mass"], float).reshape(-1)[b]
            mass = rho * vx if np.isnan(m0) else m0
            cg = np.asarray(rigid["center_of_gravity"], float).reshape(-1, 3)[b]
            g = cg - R[b]
            mg = mass * grav
            cw[3, 3] -= mg * g[2]
            cw[3, 5] += mg * g[0]
            cw[4, 4] -= mg * g[2]
            cw[4, 5] += mg * g[1]
            J = np.asarray(rigid["inertia"], float).reshape(-1, 3, 3)[b].copy()
            if int(np.broadcast_to(np.asarray(rigid.get("inertia_kind", 0)), (nb,))[b]) == 1:  # radii of gyration
                J = mass * J * np.abs(J)
            a = cg - np.asarray(rigid["inertia_origin"], float).reshape(-1, 3)[b]
            J += -mass * (np.dot(a, a) * np.eye(3) - np.outer(a, a)) + mass * (np.dot(g, g) * np.eye(3) - np.outer(g, g))
            S = np.array([[0.0, -g[2], g[1]], [g[2], 0.0, -g[0]], [-g[1], g[0], 0.0]])
            Mb[:3, :3] = mass * np.eye(3)
            Mb[:3, 3:] = -mass * S
            Mb[3:, :3] = mass * S
            Mb[3:, 3:] = J
        M[6 * b:6 * b + 6, 6 * b:6 * b + 6] = Mb
        C[6 * b:6 * b + 6, 6 * b:6 * b + 6] = cw
        recs.append({"volumes": np.array([vx, vy, V]), "center_of_buoyancy": np.array([mx / V + R[b, 0], my / V + R[b, 1], mz / V]),
                     "waterplane_area": aw, "waterplane_centroid": np.array([ax / aw + R[b, 0], ay / aw + R[b, 1]]),
                     "stiffness_rho_g": crg, "stiffness": cw, "mass": mass, "displaced_mass": rho * vx})
    if rigid is not None:
        if rigid.get("stiffness") is not None:
            C += np.asarray(rigid["stiffness"], float)
        if rigid.get("damping") is not None:
            Bx += np.asarray(rigid["damping"], float)
    return recs, M, C, Bx


def motions(A, B, X, omega, M, C, Bx):
    """xi [H][D] of one frequency: (C - w^2 (M + A) + i w (B + B_ext)) xi = X (motion.rs:121-158)."""
    Z = C - omega * omega * (M + A) + 1j * omega * (B + Bx)
    return np.linalg.solve(Z, np.asarray(X).T).T


def solve_body(verts, omegas, headings_deg=(), depth=np.inf, kinds=None, grav=GRAVITY, rho=DENSITY, logint=True,
               tol=1e-4, panel_body=None, centers=None, symmetry=SYM_NONE, rigid=None, points=None,
               production=False, kochin_angles=0):
    """The whole path for one problem: statics once, then every frequency. Arrays [F][D][D], [F][H][D]
    (D = 6 per body; interacting bodies by panel_body and their rotation centers).  With symmetry the
    panels (and kinds, panel_body) are one sector: mirrored, then solved by sectors."""
    G = sector_count(symmetry)
    if G > 1:
        verts = mirror_sector(verts, symmetry)
        kinds = None if kinds is None else np.tile(np.asarray(kinds), G)
        panel_body = None if panel_body is None else np.tile(np.asarray(panel_body), G)
    panels = make_panels(verts, kinds)
    with ProductionMode(production):
        st = statics(panels, kinds, depth, logint, tol)
    heads = np.radians(np.asarray(headings_deg, dtype=float))
    if kochin_angles == "auto":
        kochin_angles = kochin_angle_count(verts, omegas, depth, grav)
    res = [solve_frequency(panels, kinds, st, depth, w, heads, grav, rho, logint, panel_body=panel_body,
                           centers=centers, sectors=G, points=points, tol=tol, production=production,
                           kochin_angles=kochin_angles)
           for w in omegas]
    out = {k: np.array([r[k] for r in res]) for k in res[0]}
    c, n, area = panel_arrays(panels)
    recs, M, C, Bx = hydrostatics(c, n, area, kinds, panel_body, centers, rho, grav, rigid)
    out["hydrostatics"] = recs
    if rigid is not None and len(heads):
        out["motions"] = np.array([motions(out["A"][i], out["B"][i], out["X"][i], w, M, C, Bx)
                                   for i, w in enumerate(omegas)])
    if kochin_angles and len(heads):
        out["kochin_angles"] = 2.0 * np.pi * np.arange(kochin_angles) / kochin_angles
        out["drift"] = momentum_drift(omegas, headings_deg, out["kd"], out["kdt"], out["kr"], out["krt"],
                                      out.get("motions"), depth, grav, rho)
    return out


# ------------------------------------------------------------------ the waterline generator
# polygon.rs: holes bridged to the outer loop, ear clipping, Lawson flips, Delaunay refinement;
# interior.rs:408-434 the regions triangulated and mapped to stored panels.
_NONE = -1
REFINE_MIN_ANGLE = 25.0
MAX_GENERATED = 200000


def _merge_collinear(loop, tol):
    """polygon.rs:154-170 the loop without the vertices within tol of the line through their neighbours
    (the first such vertex, again from the start, until none), at least three kept."""
    c = list(loop)
    changed = True
    while changed and len(c) > 3:
        changed = False
        for i in range(len(c)):
            n = len(c)
            a, b, d = c[(i + n - 1) % n], c[i], c[(i + 1) % n]
            if abs(_orient(a, b, d)) <= tol * _dist(a, d):
                del c[i]
                changed = True
                break
    return c


def _bridge(outer, holes, eps):
    """polygon.rs:220-258 the holes merged into the outer loop, the rightmost hole first, each by a bridge
    from its rightmost vertex to the nearest visible vertex of the polygon so far (to its right if any)."""
    poly = list(outer)

    def right(lp):
        r = -np.inf
        for p in lp:
            r = max(r, p[0])
        return r

    hs = sorted(holes, key=right, reverse=True)  # stable, as sort_by
    for hi, h in enumerate(hs):
        mi = 0
        for i in range(len(h)):  # max_by: the last of equal maxima
            if h[i][0] >= h[mi][0]:
                mi = i
        m = h[mi]
        n = len(poly)
        later = hs[hi + 1:]

        def visible(k):
            p = poly[k]
            for e in range(n):
                if not (e == k or (e + 1) % n == k) and _meet(m, p, poly[e], poly[(e + 1) % n]):
                    return False
            for e in range(len(h)):
                if not (e == mi or (e + 1) % len(h) == mi) and _meet(m, p, h[e], h[(e + 1) % len(h)]):
                    return False
            for lp in later:
                for e in range(len(lp)):
                    if _meet(m, p, lp[e], lp[(e + 1) % len(lp)]):
                        return False
            return True

        def nearest(cands):  # min_by: the first of equal minima
            best = None
            for k in cands:
                if best is None or _dist(poly[k], m) < _dist(poly[best], m):
                    best = k
            return best

        best = nearest([k for k in range(n) if poly[k][0] >= m[0] - eps and visible(k)])
        if best is None:
            best = nearest([k for k in range(n) if visible(k)])
        if best is None:
            raise RuntimeError("polygon triangulation: a hole without a bridge")
        poly = poly[:best + 1] + [h[(mi + k) % len(h)] for k in range(len(h) + 1)] + poly[best:]
    return poly


def _ears(poly, eps):
    """polygon.rs:262-306 ear clipping of the counter-clockwise bridged polygon (index triples); a
    straight corner (sine below 1e-12) is dropped."""
    def straight(a, b, c):
        return abs(_orient(a, b, c)) <= 1e-12 * _dist(a, b) * _dist(b, c)

    out = []
    idx = list(range(len(poly)))
    while len(idx) > 3:
        n = len(idx)
        clipped = False
        for i in range(n):
            ia, ib, ic = idx[(i + n - 1) % n], idx[i], idx[(i + 1) % n]
            a, b, c = poly[ia], poly[ib], poly[ic]
            if straight(a, b, c):
                del idx[i]
                clipped = True
                break
            if _orient(a, b, c) < 0.0:
                continue

            def at(x, y):
                return abs(x[0] - y[0]) <= eps and abs(x[1] - y[1]) <= eps

            ear = True
            for k in idx:
                x = poly[k]
                if not (at(x, a) or at(x, b) or at(x, c)
                        or not (_orient(a, b, x) > 0.0 and _orient(b, c, x) > 0.0 and _orient(c, a, x) > 0.0)):
                    ear = False
                    break
            if ear:
                out.append([ia, ib, ic])
                del idx[i]
                clipped = True
                break
        if not clipped:
            raise RuntimeError("polygon triangulation: the ear clipping failed")
    if len(idx) == 3 and not straight(poly[idx[0]], poly[idx[1]], poly[idx[2]]):
        out.append([idx[0], idx[1], idx[2]])
    return out


def _incircle(pa, pb, pc, pd):
    adx, ady, bdx, bdy = pa[0] - pd[0], pa[1] - pd[1], pb[0] - pd[0], pb[1] - pd[1]
    cdx, cdy = pc[0] - pd[0], pc[1] - pd[1]
    return ((adx * adx + ady * ady) * (bdx * cdy - cdx * bdy) - (bdx * bdx + bdy * bdy) * (adx * cdy - cdx * ady)
            + (cdx * cdx + cdy * cdy) * (adx * bdy - bdx * ady))


def _key(a, b):
    return (min(a, b), max(a, b))


def _delaunay_flips(p, tris):
    """polygon.rs:310-388 Lawson flips to the constrained Delaunay triangulation, in place: passes over
    the triangles, each inner edge at its later triangle, until a pass flips none."""
    owners, fixed = {}, []
    for t, q in enumerate(tris):
        for e in range(3):
            k = _key(q[e], q[(e + 1) % 3])
            o = owners.setdefault(k, [_NONE, _NONE])
            if o[0] == _NONE:
                o[0] = t
            elif o[1] == _NONE:
                o[1] = t
            else:
                fixed.append(k)
    for k in fixed:
        owners[k] = [_NONE, _NONE]
    limit = max(len(tris) * len(tris), 16)
    flips = 0
    while True:
        flipped = False
        for t in range(len(tris)):
            for e in range(3):
                a, b, c = tris[t][e], tris[t][(e + 1) % 3], tris[t][(e + 2) % 3]
                o = owners[_key(a, b)]
                u = o[1] if o[0] == t else o[0]
                if u == _NONE or u > t:
                    continue
                f = next((f for f in range(3) if tris[u][f] == b and tris[u][(f + 1) % 3] == a), None)
                if f is None:
                    raise RuntimeError("polygon triangulation: two triangles turned the same way")
                d = tris[u][(f + 2) % 3]
                ob = _orient(p[a], p[b], p[c])
                if (_incircle(p[a], p[b], p[c], p[d]) > 1e-12 * ob * ob and _orient(p[c], p[d], p[b]) > 0.0
                        and _orient(p[d], p[c], p[a]) > 0.0):
                    tris[t] = [c, d, b]
                    tris[u] = [d, c, a]
                    del owners[_key(a, b)]
                    owners[_key(c, d)] = [t, u]
                    for edge, frm, to in ((_key(d, b), u, t), (_key(c, a), t, u)):
                        o = owners[edge]
                        for x in range(2):
                            if o[x] == frm:
                                o[x] = to
                    flipped = True
                    flips += 1
                    if flips > limit:
                        raise RuntimeError("polygon triangulation: the Delaunay flips do not end")
                    break
        if not flipped:
            return


def _circumcentre(a, b, c):
    bx, by, cx, cy = b[0] - a[0], b[1] - a[1], c[0] - a[0], c[1] - a[1]
    d = 2.0 * (bx * cy - by * cx)
    b2, c2 = bx * bx + by * by, cx * cx + cy * cy
    return (a[0] + (cy * b2 - by * c2) / d, a[1] + (bx * c2 - cx * b2) / d)


class _Mesh2:
    """polygon.rs:428-576 a triangulation under refinement: triangles (dead ones kept), the map of each
    edge to its two triangles, the boundary segments with the length of the edge each was split from."""

    def __init__(self, p):
        self.p, self.t, self.alive, self.owners, self.segs = p, [], [], {}, {}

    def add_tri(self, q):
        i = len(self.t)
        self.t.append(q)
        self.alive.append(True)
        for e in range(3):
            o = self.owners.setdefault(_key(q[e], q[(e + 1) % 3]), [_NONE, _NONE])
            if o[0] == _NONE:
                o[0] = i
            else:
                o[1] = i
        return i

    def kill(self, i):
        self.alive[i] = False
        q = self.t[i]
        for e in range(3):
            k = _key(q[e], q[(e + 1) % 3])
            o = self.owners.get(k)
            if o is not None:
                for x in range(2):
                    if o[x] == i:
                        o[x] = _NONE
                if o[0] == _NONE and o[1] == _NONE:
                    del self.owners[k]

    def across(self, t, a, b):
        o = self.owners.get(_key(a, b))
        if o is None:
            return _NONE
        return o[1] if o[0] == t else o[0]

    def locate(self, t, c):
        """('inside', t) for the triangle holding c, walked from t along the line from its centroid,
        ('segment', u, v) for the first boundary edge the line meets, or ('lost',)."""
        p = self.p
        q = self.t[t]
        g = ((p[q[0]][0] + p[q[1]][0] + p[q[2]][0]) / 3.0, (p[q[0]][1] + p[q[1]][1] + p[q[2]][1]) / 3.0)
        cur, frm = t, _NONE
        for _ in range(len(self.t) + 3):
            q = self.t[cur]
            crossed = []
            for e in range(3):
                u, v = q[e], q[(e + 1) % 3]
                su, sv = _orient(g, c, p[u]), _orient(g, c, p[v])
                if _orient(p[u], p[v], c) < 0.0 and ((su <= 0.0 and sv >= 0.0) or (su >= 0.0 and sv <= 0.0)):
                    crossed.append((u, v, self.across(cur, u, v)))
            ex = next((x for x in crossed if x[2] != frm), crossed[0] if crossed else None)
            if ex is None:
                if all(_orient(p[q[e]], p[q[(e + 1) % 3]], c) >= 0.0 for e in range(3)):
                    return ("inside", cur)
                return ("lost",)
            u, v, n = ex
            if _key(u, v) in self.segs or n == _NONE:
                return ("segment", u, v)
            frm, cur = cur, n
        return ("lost",)

    def cavity(self, t, x):
        p = self.p
        cav = [t]
        k = 0
        while k < len(cav):
            q = self.t[cav[k]]
            for e in range(3):
                u, v = q[e], q[(e + 1) % 3]
                if _key(u, v) in self.segs:
                    continue
                n = self.across(cav[k], u, v)
                if n == _NONE or n in cav:
                    continue
                r = self.t[n]
                if _incircle(p[r[0]], p[r[1]], p[r[2]], x) > 0.0:
                    cav.append(n)
            k += 1
        bnd = []
        for c in cav:
            q = self.t[c]
            for e in range(3):
                u, v = q[e], q[(e + 1) % 3]
                n = self.across(c, u, v)
                if n == _NONE or n not in cav or _key(u, v) in self.segs:
                    bnd.append((u, v))
        return cav, bnd

    def insert(self, cav, bnd, x, skip):
        fan = [(u, v) for (u, v) in bnd if (u, v) != skip]
        for u, v in fan:
            pu, pv = self.p[u], self.p[v]
            l2 = (pu[0] - pv[0]) * (pu[0] - pv[0]) + (pu[1] - pv[1]) * (pu[1] - pv[1])
            if _orient(pu, pv, x) <= 1e-9 * l2:
                return None
        i = len(self.p)
        self.p.append(x)
        for c in cav:
            self.kill(c)
        return [self.add_tri([u, v, i]) for (u, v) in fan]


def _triangulate_refined(outer, holes, eps, size, cap):
    """polygon.rs:593-700 the triangles (counter-clockwise) of a region refined to `size` and the smallest
    angle REFINE_MIN_ANGLE (Ruppert's refinement with Shewchuk's rules, in one fixed order)."""
    poly = _bridge(outer, holes, eps)
    tris = _ears(poly, eps)
    p, id_of, ids = [], {}, []
    for x in poly:  # the two ends of a bridge are exact copies: one vertex
        k = (float(x[0]), float(x[1]))
        if k not in id_of:
            id_of[k] = len(p)
            p.append(k)
        ids.append(id_of[k])
    t = [[ids[q[0]], ids[q[1]], ids[q[2]]] for q in tris]
    _delaunay_flips(p, t)
    m = _Mesh2(p)
    for q in t:
        m.add_tri(q)
    shortest = np.inf
    for i in range(len(m.t)):
        q = m.t[i]
        for e in range(3):
            u, v = q[e], q[(e + 1) % 3]
            if m.across(i, u, v) == _NONE:
                ln = _dist(m.p[u], m.p[v])
                m.segs[_key(u, v)] = ln
                shortest = min(shortest, ln)
    ratio = 0.5 / math.sin(REFINE_MIN_ANGLE * math.pi / 180.0)
    queue = collections.deque(range(len(m.t)))
    live = len(m.t)
    while queue:
        i = queue.popleft()
        if not m.alive[i] or live > cap:
            continue
        q = m.t[i]
        a, b, c = m.p[q[0]], m.p[q[1]], m.p[q[2]]
        ls = [_dist(b, c), _dist(c, a), _dist(a, b)]
        lo, hi = min(min(ls[0], ls[1]), ls[2]), max(max(ls[0], ls[1]), ls[2])
        cc = _circumcentre(a, b, c)
        big = hi > size
        skinny = _dist(cc, a) > ratio * lo and lo >= 0.25 * shortest
        if not big and not skinny:
            continue
        fan = None
        loc = m.locate(i, cc)
        if loc[0] == "lost":
            continue
        if loc[0] == "segment":
            split = (loc[1], loc[2])
        else:
            cav, bnd = m.cavity(loc[1], cc)
            split = None
            for u, v in bnd:
                if _key(u, v) in m.segs:
                    pu, pv = m.p[u], m.p[v]
                    if (pu[0] - cc[0]) * (pv[0] - cc[0]) + (pu[1] - cc[1]) * (pv[1] - cc[1]) < 0.0:
                        split = (u, v)
                        break
            if split is None:
                new = m.insert(cav, bnd, cc, None)
                fan = None if new is None else (new, len(cav))
        if split is not None:
            u, v = split
            ln = _dist(m.p[u], m.p[v])
            if not (ln > size or ln >= 0.75 * min(0.5 * size, m.segs[_key(u, v)])):
                continue
            s = m.owners[_key(u, v)]
            ts = s[0] if s[0] != _NONE else s[1]
            qs = m.t[ts]
            u, v = next((qs[e], qs[(e + 1) % 3]) for e in range(3) if _key(qs[e], qs[(e + 1) % 3]) == _key(u, v))
            mid = (0.5 * (m.p[u][0] + m.p[v][0]), 0.5 * (m.p[u][1] + m.p[v][1]))
            cav, bnd = m.cavity(ts, mid)
            frm = m.segs[_key(u, v)]
            new = m.insert(cav, bnd, mid, (u, v))
            if new is not None:
                x = len(m.p) - 1
                del m.segs[_key(u, v)]
                m.segs[_key(u, x)] = frm
                m.segs[_key(x, v)] = frm
                live += len(new) - len(cav)
                queue.extend(new)
                if m.alive[i]:
                    queue.append(i)
        elif fan is not None:
            live += len(fan[0]) - fan[1]
            queue.extend(fan[0])
    return [[m.p[m.t[i][0]], m.p[m.t[i][1]], m.p[m.t[i][2]]] for i in range(len(m.t)) if m.alive[i]]


def waterline_lid(verts, isx=0, isy=0, z0=0.0, reference_length=1.0):
    """interior.rs:408-434 waterline: the waterplane regions (their contours with collinear points merged,
    holes -- moonpools -- kept, each hole with the smallest outer contour around it) triangulated with
    their holes and refined to edges of at most twice the mean waterline segment length and angles of at
    least REFINE_MIN_ANGLE; the triangles as stored panels [Q][4][3] (the last vertex repeated), facing up.
    More than MAX_GENERATED triangles raise ValueError, as the reference does."""
    v = np.asarray(verts, dtype=np.float64).reshape(-1, 4, 3)
    loops, sx, sy, target, ax_x, ax_y, tol = _waterplane_loops(v, isx, isy, z0, reference_length, True)
    outers = [lp for lp in loops if len(lp) >= 3 and _signed_area(lp) > 0.0]
    holes = [lp for lp in loops if len(lp) >= 3 and not _signed_area(lp) > 0.0]
    if not outers:
        raise ValueError("no enclosed region")
    hole_of = [[] for _ in outers]
    for h in holes:
        owner = -1
        for o in range(len(outers)):
            if _inside(outers[o], h[0]) and (owner < 0 or abs(_signed_area(outers[o])) < abs(_signed_area(outers[owner]))):
                owner = o
        if owner < 0:
            raise ValueError("a waterline contour lies outside the body")
        hole_of[owner].append(h)
    done = []
    for o in range(len(outers)):
        done.extend(_triangulate_refined(outers[o], hole_of[o], tol, 2.0 * target, MAX_GENERATED - len(done)))
        if len(done) > MAX_GENERATED:
            raise ValueError(f"the waterplane needs more than {MAX_GENERATED} panels of twice the mean waterline "
                             "segment length; use 'graded' or a mesh of its own")
    out = []
    for tri in done:
        w = np.zeros((4, 3))
        for k in range(3):
            w[k] = (sx * tri[k][0], sy * tri[k][1], z0)
        if sx * sy < 0.0:
            w[:3] = w[:3][::-1]
        w[3] = w[2]
        out.append(w)
    return np.array(out)
