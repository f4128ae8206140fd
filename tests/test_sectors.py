"""Symmetry sectors (the reference's reflection characters, lo_geometry.rs:25-36 and
lo_frequency.rs:276-346, 823-943): a body mirrored in the yz and/or xz planes is solved as G systems
of one sector's unknowns per frequency.

CPU: on the oracle's own matrices of the mirrored mesh, the character method reproduces the whole-mesh
solve (element order e, x, y, xy reflections; chi_c(g) = (-1)^popc(c & g); right-hand sides projected
with 1/G; potentials recombined without it) -- exactly with the log-singularity correction off, and with
it on up to that quadrature's mirror asymmetry (the rule integrates a mirrored panel, vertices reversed,
to a few 1e-12, so the whole mirrored mesh is not exactly symmetric; the reference's character path
inherits the same difference).  GPU: both forms with symmetry against the oracle's character method,
statics and sector matrices entry by entry, and a 4096-panel body against its whole mesh.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from hydrobem_b200 import meshes
from oracle import oracle as O

FP64_TOL = 1e-9
MIXED_TOL = 1e-5


def scaled_error(got, ref, floor=1e-3):
    ref = np.asarray(ref)
    peak = np.abs(ref).max()
    scale = np.maximum(np.abs(ref).max(axis=0, keepdims=True), floor * peak)
    return float((np.abs(np.asarray(got) - ref) / scale).max())


def half_from_quarter(q: np.ndarray, plane: str) -> np.ndarray:
    """The sector of one symmetry plane from a quarter mesh (x, y >= 0): x >= 0 for the yz plane (the
    quarter and its y mirror), y >= 0 for the xz plane (the quarter and its x mirror)."""
    return O.mirror_sector(q, O.SYM_XZ if plane == "yz" else O.SYM_YZ)


@pytest.mark.parametrize("sym,depth", [(3, math.inf), (1, 4.0), (2, math.inf)])
def test_oracle_character_method_against_the_whole_mesh(sym, depth):
    q = meshes.cylinder(1.0, 0.5, 4, 2, 2, quarter=True)
    sector = q if sym == 3 else half_from_quarter(q, "yz" if sym == 1 else "xz")
    G = O.sector_count(sym)
    v = O.mirror_sector(sector, sym)
    Ns, N = len(sector), len(v)
    panels = O.make_panels(v)
    omega, beta = 1.7, 0.6
    c, n, _ = O.panel_arrays(panels)
    k = O.lib().hbo_wavenumber(omega, depth, O.GRAVITY)
    u = np.zeros((N, 7), dtype=np.complex128)
    u[:, :6] = O.rigid_normals(c, n, None)
    _, gr = O.incident(c, depth, k, omega, beta)
    u[:, 6] = -(gr * n).sum(axis=1)
    for logint, tol in ((False, 1e-11), (True, 1e-9)):
        st = O.statics(panels, None, depth, logint=logint)
        S, A = O.assemble(panels, None, st, depth, omega, logint=logint)
        full = np.linalg.solve(A, S @ (-u))
        phi = O.sector_solve(S, A, u, G)
        assert np.abs(phi - full).max() <= tol * np.abs(full).max(), logint
    # every radiation mode lives in one sector at most (a vertical cylinder's yaw normal vanishes)
    for m in range(6):
        live = [cc for cc in range(G)
                if np.abs(sum(O.character(cc, g) * u[g * Ns:(g + 1) * Ns, m] for g in range(G))).max() > 1e-12]
        assert len(live) <= 1 and (m == 5 or len(live) == 1), (m, live)


def _gpu():
    from hydrobem_b200 import native as nv
    return nv


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("sym,depth", [(3, math.inf), (3, 3.0), (1, math.inf), (2, 5.0)])
def test_gpu_sectors_against_the_oracle(precision, sym, depth):
    nv = _gpu()
    q = meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True)
    sector = q if sym == 3 else half_from_quarter(q, "yz" if sym == 1 else "xz")
    omegas = np.array([0.8, 1.9, 3.1, 6.0])
    heads = [0.0, 35.0, 90.0]
    prec = nv.HBG_MIXED if precision == "mixed" else nv.HBG_FP64
    gpu = nv.solve(sector, omegas, heads, symmetry=sym, depth=depth, precision=prec)
    ref = O.solve_body(sector, omegas, heads, depth=depth, symmetry=sym)
    errs = {k: scaled_error(gpu[k], ref[k]) for k in ("A", "B", "X", "FK", "SC", "HK")}
    assert max(errs.values()) <= (MIXED_TOL if precision == "mixed" else FP64_TOL), errs


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_sectors_with_an_interior_lid(precision):
    """A quarter box with its quarter lid (kind interior in the sector and in every image)."""
    nv = _gpu()
    q = meshes.box(1.0, 0.5, 0.5, n=(4, 2, 2), quarter=True, lid=True)
    kinds = np.zeros(len(q), np.int32)
    kinds[-8:] = 1
    omegas = np.array([1.0, 2.5])
    prec = nv.HBG_MIXED if precision == "mixed" else nv.HBG_FP64
    gpu = nv.solve(q, omegas, [20.0], kinds=kinds, symmetry=nv.SYM_BOTH, precision=prec)
    ref = O.solve_body(q, omegas, [20.0], kinds=kinds, symmetry=O.SYM_BOTH)
    errs = {k: scaled_error(gpu[k], ref[k]) for k in ("A", "B", "X", "HK")}
    assert max(errs.values()) <= (MIXED_TOL if precision == "mixed" else FP64_TOL), errs


@pytest.mark.gpu
def test_gpu_sectors_two_bodies():
    """Two cylinders at y = -2.5 and y = +2.5, each symmetric about the yz plane: the sector holds the
    x >= 0 halves of both, each image keeps its body, each body rotates about its own centre."""
    nv = _gpu()
    half = half_from_quarter(meshes.cylinder(1.0, 0.5, 6, 3, 3, quarter=True), "yz")
    sector = np.concatenate([half + np.array([0.0, -2.5, 0.0]), half + np.array([0.0, 2.5, 0.0])])
    body = np.repeat([0, 1], len(half)).astype(np.int32)
    centers = np.array([[0.0, -2.5, 0.0], [0.0, 2.5, -0.1]])
    omegas = np.array([1.2, 2.4])
    gpu = nv.solve(sector, omegas, [0.0, 60.0], panel_body=body, rotation_centers=centers, symmetry=nv.SYM_YZ)
    ref = O.solve_body(sector, omegas, [0.0, 60.0], panel_body=body, centers=centers, symmetry=O.SYM_YZ)
    assert gpu["A"].shape == (2, 12, 12)
    errs = {k: scaled_error(gpu[k], ref[k]) for k in ("A", "B", "X", "HK")}
    assert max(errs.values()) <= FP64_TOL, errs


@pytest.mark.gpu
@pytest.mark.parametrize("sym,depth", [(1, math.inf), (3, math.inf), (3, 4.0)])
def test_gpu_sector_statics_and_matrices_against_the_oracle(sym, depth):
    """The statics of the sector rows and the G sector matrices of one frequency, entry by entry, against
    the oracle's statics and matrices of the mirrored mesh (its first n rows, character sums of its
    column blocks)."""
    nv = _gpu()
    q = meshes.cylinder(1.0, 0.5, 6, 3, 3, quarter=True)
    sector = q if sym == 3 else half_from_quarter(q, "yz")
    G = O.sector_count(sym)
    n = len(sector)
    omega = 4.0
    st, S, A = nv.debug_matrices(sector, omega, symmetry=sym, depth=depth)
    panels = O.make_panels(O.mirror_sector(sector, sym))
    st_ref = O.statics(panels, None, depth)
    S_ref, A_ref = O.assemble(panels, None, st_ref, depth, omega)
    for q_ in range(4):
        ref = st_ref[:n, :, q_]
        assert np.abs(st[:, :, q_] - ref).max() <= 1e-13 * np.abs(ref).max(), q_
    blk = lambda M, g: M[:n, g * n:(g + 1) * n]
    for cc in range(G):
        Sc = sum(O.character(cc, g) * blk(S_ref, g) for g in range(G))
        Ac = sum(O.character(cc, g) * blk(A_ref, g) for g in range(G))
        assert np.abs(S[cc] - Sc).max() <= 1e-12 * np.abs(Sc).max(), cc
        assert np.abs(A[cc] - Ac).max() <= 1e-12 * np.abs(Ac).max(), cc


@pytest.mark.gpu
def test_gpu_sectors_equal_the_whole_mesh_at_size():
    """A 4096-panel cylinder (the benchmark's mesh) given as its 1024-panel quarter: the sector solve
    against the solve of the whole mirrored mesh, both on the GPU."""
    nv = _gpu()
    q = meshes.cylinder(1.0, 0.5, 16, 32, 32, quarter=True)
    assert len(q) == 1024
    omegas = np.array([0.7, 2.0, 5.0])
    heads = [0.0, 45.0]
    whole = nv.solve(O.mirror_sector(q, O.SYM_BOTH), omegas, heads, depth=5.0)
    for prec, tol in ((nv.HBG_FP64, 1e-9), (nv.HBG_MIXED, MIXED_TOL)):
        sec = nv.solve(q, omegas, heads, symmetry=nv.SYM_BOTH, depth=5.0, precision=prec)
        errs = {k: scaled_error(sec[k], whole[k]) for k in ("A", "B", "X", "HK")}
        assert max(errs.values()) <= tol, (prec, errs)


@pytest.mark.gpu
def test_gpu_symmetry_argument_checked():
    nv = _gpu()
    q = meshes.cylinder(1.0, 0.5, 4, 2, 2, quarter=True)
    with pytest.raises(nv.HydroBEMError) as e:
        nv.solve(q, [1.0], [0.0], symmetry=5)
    assert e.value.status == 1  # HB_ERR_VALUE
