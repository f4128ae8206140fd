"""Kochin functions and the mean drift by momentum conservation (lo_frequency.rs:1277-1374,
low_order.rs:1417-1452, response.rs:51-300), pinned on the reference's stored outputs of its regression
problem lo_cylinder_drift (a floating quarter cylinder with two symmetry planes, its mass and inertia,
two frequencies, headings 0 and 30 degrees; float32 outputs of its production path): the 104 automatic
angles exactly, the Kochin functions and their angular derivatives, and the drift force and moment of
each heading."""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

from hydrobem_b200 import meshes
from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden" / "lo_cylinder_drift.npz"
MASS = 1000.0 * math.pi * 0.5
FREE = {"mass": [MASS], "center_of_gravity": [[0.0, 0.0, -0.2]], "inertia_kind": [0],
        "inertia": [np.diag([MASS * 0.36, MASS * 0.36, MASS * 0.49])], "inertia_origin": [[0.0, 0.0, -0.2]]}
PAIRS = {"kr": "kochin_radiation", "krt": "kochin_radiation_derivative", "kd": "kochin_diffraction",
         "kdt": "kochin_diffraction_derivative"}


def peak_error(got, ref):
    ref = np.asarray(ref)
    return float(np.abs(np.asarray(got) - ref).max() / np.abs(ref).max())


def unidirectional(drift):
    """The equal heading pairs [F][H][3] of a [F][H][H][3] drift."""
    H = drift.shape[1]
    return np.stack([drift[:, h, h] for h in range(H)], axis=1)


@pytest.fixture(scope="module")
def oracle_drift():
    g = np.load(GOLDEN)
    quarter = meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True)
    return g, O.solve_body(quarter, g["omegas"], g["headings"], symmetry=O.SYM_BOTH, rigid=FREE,
                           kochin_angles="auto")


def test_oracle_kochin_against_the_reference(oracle_drift):
    g, r = oracle_drift
    assert np.array_equal(r["kochin_angles"], g["kochin_angles"])
    for k, name in PAIRS.items():
        assert peak_error(r[k], g[name]) <= 1e-6, name


def test_oracle_momentum_drift_against_the_reference(oracle_drift):
    g, r = oracle_drift
    assert peak_error(unidirectional(r["drift"]), g["drift_momentum_conservation"]) <= 1e-6


def test_oracle_drift_of_a_fixed_body_is_the_diffraction_part():
    """Without motions the drift comes from the scattered wave alone; it differs from the free body's."""
    g = np.load(GOLDEN)
    quarter = meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True)
    fixed = O.solve_body(quarter, g["omegas"], g["headings"], symmetry=O.SYM_BOTH, kochin_angles=104)
    assert "motions" not in fixed
    d = unidirectional(fixed["drift"])
    assert np.all(np.isfinite(d)) and peak_error(d, g["drift_momentum_conservation"]) > 1e-3


def _scaled(got, ref, floor=1e-3):
    ref = np.asarray(ref)
    scale = np.maximum(np.abs(ref).max(axis=0, keepdims=True), floor * np.abs(ref).max())
    return float((np.abs(np.asarray(got) - ref) / scale).max())


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-5)])
def test_gpu_kochin_and_drift_against_the_oracle(precision, tol, oracle_drift):
    """The free cylinder by its four sectors (the potentials recombined before the far-field sums)."""
    from hydrobem_b200 import native as nv

    g, ref = oracle_drift
    quarter = meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True)
    prec = nv.HBG_MIXED if precision == "mixed" else nv.HBG_FP64
    gpu = nv.solve(quarter, g["omegas"], g["headings"], symmetry=nv.SYM_BOTH, rigid=FREE, kochin_angles=104,
                   precision=prec)
    for k in ("kr", "krt", "kd", "kdt"):
        assert _scaled(gpu[k], ref[k]) <= tol, k
    assert peak_error(gpu["drift"], ref["drift"]) <= tol


@pytest.mark.gpu
def test_gpu_kochin_finite_depth_two_bodies_bidirectional():
    """Finite depth, two interacting bodies, three headings, every heading pair; fixed bodies (no motions)."""
    from hydrobem_b200 import native as nv

    v = meshes.cylinder(1.0, 0.5, 16, 4, 4)
    two = np.concatenate([v + [-2.0, 0.0, 0.0], v + [2.0, 0.0, 0.0]])
    body = np.repeat([0, 1], len(v)).astype(np.int32)
    centers = [[-2.0, 0.0, 0.0], [2.0, 0.0, 0.0]]
    omegas, heads = np.array([1.1, 2.3]), [0.0, 45.0, 120.0]
    gpu = nv.solve(two, omegas, heads, panel_body=body, rotation_centers=centers, depth=4.0, kochin_angles=120)
    ref = O.solve_body(two, omegas, heads, depth=4.0, panel_body=body, centers=centers, kochin_angles=120)
    for k in ("kr", "krt", "kd", "kdt"):
        assert _scaled(gpu[k], ref[k]) <= 1e-9, k
    assert peak_error(gpu["drift"], ref["drift"]) <= 1e-9


@pytest.mark.gpu
def test_gpu_drift_through_the_model_abi():
    """drift_momentum_conservation with its automatic angles through hb_model_solve, the motions on:
    against the reference's stored drift of lo_cylinder_drift (its float32 production path) to 2e-5 of
    the peak, the 104 angles exactly."""
    from hydrobem_b200 import native as nv

    g = np.load(GOLDEN)
    with nv.Model() as m:
        m.add("meshes", "cyl")
        m.reals("meshes/cyl", "vertices", meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True))
        m.text("meshes/cyl", "symmetry", "xz_and_yz")
        m.add("bodies", "body")
        m.text("bodies/body", "mesh", "cyl")
        m.reals("bodies/body", "center_of_gravity", [0.0, 0.0, -0.2])
        m.real("bodies/body", "mass", MASS)
        m.text("bodies/body", "inertia_input", "components")
        for k, val in (("Ixx", MASS * 0.36), ("Iyy", MASS * 0.36), ("Izz", MASS * 0.49)):
            m.real("bodies/body", k, val)
        m.text("bodies/body", "inertia_origin", "center_of_gravity")
        m.boolean("options", "motion", True)
        m.boolean("options", "drift_momentum_conservation", True)
        m.reals("environment", "omegas", g["omegas"])
        m.reals("environment", "headings", g["headings"])
        res = m.solve()
        ang = res.quantity("kochin_angles")
        drift = res.quantity("drift_momentum_conservation")
        pairs = res.quantity("drift_heading_pairs")
        kd = res.quantity("kochin_diffraction")
        res.free()
    assert np.array_equal(ang, g["kochin_angles"])
    assert np.array_equal(pairs, g["drift_heading_pairs"])
    assert kd.dtype == np.complex64 and peak_error(kd, g["kochin_diffraction"]) <= 2e-5
    assert peak_error(drift, g["drift_momentum_conservation"]) <= 2e-5
