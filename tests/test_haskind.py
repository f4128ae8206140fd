"""The Haskind exciting force (lo_frequency.rs:1118-1171): the exciting force from the radiation
potentials and the incident wave, beside the pressure integration of the diffraction potential.

The reference's identity tests (tests/python/test_low_order.py:70-107) solve the hemisphere of radius 1
with 24 panels a quadrant edge (its quarter with two symmetry planes) at K a = 0.4, 1.0, 1.8 and headings
every 15 degrees, and state what the discretization leaves: Haskind against pressure 3.6e-4 of the
peak (bound 1e-3), the energy relation 1.2e-3 (bound 2e-3).  The oracle reproduces those figures (CPU);
the GPU forms match the oracle's Haskind force at 1e-9 (FP64) and 1e-5 (mixed) -- these and the
parametrised parity tests of the other files, which compare HK beside A, B, X.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from hydrobem_b200 import meshes
from oracle import oracle as O

G, RHO = 9.80665, 1000.0
OMEGAS = np.sqrt(np.array([0.4, 1.0, 1.8]) * G)
HEADS = np.arange(0.0, 360.0, 15.0)


def peak(a):
    return float(np.abs(a).max())


def haskind_error(r):
    return peak(r["HK"] - r["X"]) / peak(r["X"])


def energy_error(r):
    """Newman (1977, eq. 6.173): B_jj = k / (8 pi rho g Cg) int |X_j(theta)|^2 dtheta, Cg = g / (2 w), from
    the Haskind force over the headings (periodic trapezoid); yaw radiates no waves for a body of
    revolution."""
    worst = 0.0
    for f, w in enumerate(OMEGAS):
        k = w * w / G
        integral = (np.abs(r["HK"][f]) ** 2).mean(axis=0) * 2 * math.pi
        b = k / (8 * math.pi * RHO * G * (G / (2 * w))) * integral
        diag = np.diag(r["B"][f])[:5]
        worst = max(worst, np.abs(b[:5] - diag).max() / peak(r["B"][f]))
    return worst


@pytest.fixture(scope="module")
def hemi_oracle():
    quarter = meshes.hemisphere(1.0, 24, 24, quarter=True)
    return O.solve_body(quarter, OMEGAS, HEADS, symmetry=O.SYM_BOTH)


def test_oracle_haskind_equals_pressure_excitation(hemi_oracle):
    e = haskind_error(hemi_oracle)
    assert e <= 1e-3
    assert 3.5e-4 <= e <= 3.7e-4, e  # the reference's stated 3.6e-4 on this mesh


def test_oracle_energy_relation(hemi_oracle):
    e = energy_error(hemi_oracle)
    assert e <= 2e-3
    assert 1.1e-3 <= e <= 1.3e-3, e  # the reference's stated 1.2e-3


def test_oracle_haskind_is_reciprocal_in_the_interior_lid():
    """Interior (irregular-frequency) panels take no part in the Haskind sum; a box with a lid still
    satisfies the identity to its discretization level."""
    v = meshes.box(1.0, 0.5, 0.5, n=(8, 4, 4), lid=True)
    kinds = np.zeros(len(v), np.int32)
    kinds[-32:] = 1
    r = O.solve_body(v, np.array([1.5, 2.5]), [0.0, 60.0], kinds=kinds)
    assert haskind_error(r) <= 2e-2


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_haskind_identity_hemisphere(precision, hemi_oracle):
    """The reference's identity problem on the GPU (the quarter solved by its four sectors)."""
    from hydrobem_b200 import native as nv

    quarter = meshes.hemisphere(1.0, 24, 24, quarter=True)
    prec = nv.HBG_MIXED if precision == "mixed" else nv.HBG_FP64
    gpu = nv.solve(quarter, OMEGAS, HEADS, symmetry=nv.SYM_BOTH, precision=prec)
    ref = hemi_oracle
    scale = np.maximum(np.abs(ref["HK"]).max(axis=0, keepdims=True), 1e-3 * peak(ref["HK"]))
    err = float((np.abs(gpu["HK"] - ref["HK"]) / scale).max())
    assert err <= (1e-9 if precision == "fp64" else 1e-5), err
    assert haskind_error(gpu) <= 1e-3
    assert energy_error(gpu) <= 2e-3


@pytest.mark.gpu
def test_gpu_haskind_through_the_model_abi():
    """excitation_haskind (HB_C64 [F][H][K]) and its _f64 copy through hb_model_solve, finite depth."""
    from hydrobem_b200 import native as nv

    v = meshes.cylinder(1.0, 0.5, 16, 4, 4)
    omegas = np.array([0.9, 2.1])
    heads = np.array([0.0, 45.0])
    with nv.Model() as m:
        m.add("meshes", "cyl")
        m.reals("meshes/cyl", "vertices", v)
        m.add("bodies", "body")
        m.text("bodies/body", "mesh", "cyl")
        m.reals("environment", "omegas", omegas)
        m.reals("environment", "headings", heads)
        m.real("environment", "depth", 4.0)
        res = m.solve()
        hk = res.quantity("excitation_haskind_f64")
        hk32 = res.quantity("excitation_haskind")
        res.free()
    ref = O.solve_body(v, omegas, heads, depth=4.0)
    assert hk.shape == (2, 2, 6) and hk32.dtype == np.complex64
    scale = np.maximum(np.abs(ref["HK"]).max(axis=0, keepdims=True), 1e-3 * peak(ref["HK"]))
    assert float((np.abs(hk - ref["HK"]) / scale).max()) <= 1e-9
    assert float((np.abs(hk32 - ref["HK"]) / scale).max()) <= 1e-6


GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden" / "lo_cylinder_drift.npz"


def _scaled(got, ref, floor=1e-3):
    ref = np.asarray(ref)
    scale = np.maximum(np.abs(ref).max(axis=0, keepdims=True), floor * np.abs(ref).max())
    return float((np.abs(np.asarray(got) - ref) / scale).max())


def test_oracle_haskind_against_the_reference_solve():
    """The reference's stored Haskind force of its regression problem lo_cylinder_drift (a quarter
    cylinder with two symmetry planes; float32 outputs of its production path): the oracle's to 2e-5."""
    g = np.load(GOLDEN)
    quarter = meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True)
    ref = O.solve_body(quarter, g["omegas"], g["headings"], symmetry=O.SYM_BOTH)
    assert ref["HK"].shape == g["excitation_haskind"].shape
    assert _scaled(ref["HK"], g["excitation_haskind"]) <= 2e-5


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_haskind_against_the_reference_solve(precision):
    from hydrobem_b200 import native as nv

    g = np.load(GOLDEN)
    with nv.Model() as m:
        m.add("meshes", "cyl")
        m.reals("meshes/cyl", "vertices", meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True))
        m.text("meshes/cyl", "symmetry", "xz_and_yz")
        m.add("bodies", "body")
        m.text("bodies/body", "mesh", "cyl")
        m.reals("environment", "omegas", g["omegas"])
        m.reals("environment", "headings", g["headings"])
        m.text("options", "gpu_precision", precision)
        res = m.solve()
        hk = res.quantity("excitation_haskind_f64")
        res.free()
    assert _scaled(hk, g["excitation_haskind"]) <= 2e-5
