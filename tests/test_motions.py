"""Hydrostatics and rigid-body motions (crates/hydrobem/src/hydrostatics.rs, motion.rs): the restoring
matrix with the weight terms, the rigid inertia about the rotation centre, and the motion equation
(C - w^2 (M + A) + i w (B + B_ext)) xi = X of each frequency.

Pinned on the reference's own outputs of its regression problem lo_cylinder_drift (a free cylinder,
r = 1 m, draught 0.5 m, mass pi/2 t, G at z = -0.2 m, inertia components about G): the oracle's
hydrostatics against the stored ones, the oracle's motion equation on the stored A, B, X against the
stored motions; then the GPU (both forms, the batched entry and the object model) against the oracle
and the stored outputs.
"""
from __future__ import annotations

import ctypes
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


def scaled_error(got, ref, floor=1e-3):
    ref = np.asarray(ref)
    peak = np.abs(ref).max()
    scale = np.maximum(np.abs(ref).max(axis=0, keepdims=True), floor * peak)
    return float((np.abs(np.asarray(got) - ref) / scale).max())


def quarter():
    return meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True)


def test_oracle_hydrostatics_against_the_reference():
    g = np.load(GOLDEN)
    panels = O.make_panels(O.mirror_sector(quarter(), O.SYM_BOTH))
    c, n, area = O.panel_arrays(panels)
    (h,), M, C, _ = O.hydrostatics(c, n, area, rigid=FREE)
    assert np.allclose(h["volumes"], g["hydrostatics_volumes"][0], rtol=1e-12, atol=0)
    assert np.allclose(h["center_of_buoyancy"], g["hydrostatics_center_of_buoyancy"][0], rtol=1e-12, atol=1e-15)
    assert h["waterplane_area"] == pytest.approx(g["hydrostatics_waterplane_area"][0], rel=1e-12)
    assert np.allclose(h["waterplane_centroid"], g["hydrostatics_waterplane_centroid"][0], atol=1e-14)
    for k, key in (("stiffness_rho_g", "hydrostatics_stiffness_rho_g"), ("stiffness", "hydrostatics_stiffness")):
        ref = g[key][0]
        assert np.abs(h[k] - ref).max() <= 1e-12 * np.abs(ref).max(), k
    assert h["mass"] == g["hydrostatics_mass"][0]
    assert h["displaced_mass"] == pytest.approx(g["hydrostatics_displaced_mass"][0], rel=1e-12)
    # the rigid inertia about the rotation centre (the origin) and the restoring matrix in use
    assert M[0, 0] == MASS and M[3, 3] == pytest.approx(MASS * 0.36 + MASS * 0.04, rel=1e-15)
    assert M[0, 4] == pytest.approx(MASS * -0.2, rel=1e-15) and M[4, 0] == M[0, 4]
    assert np.array_equal(C, h["stiffness"])


def test_oracle_motion_equation_on_the_reference_outputs():
    """The motion equation solved on the reference's own stored A, B, X (float32, as its motion solve
    reads them) reproduces its stored motions to their float32 rounding."""
    g = np.load(GOLDEN)
    panels = O.make_panels(O.mirror_sector(quarter(), O.SYM_BOTH))
    c, n, area = O.panel_arrays(panels)
    _, M, C, Bx = O.hydrostatics(c, n, area, rigid=FREE)
    xi = np.array([O.motions(g["added_mass"][i].astype(np.float64), g["radiation_damping"][i].astype(np.float64),
                             g["excitation_diffraction"][i].astype(np.complex128), w, M, C, Bx)
                   for i, w in enumerate(g["omegas"])])
    assert scaled_error(xi, g["motion"]) <= 1e-5


def test_oracle_motions_against_the_reference_solve():
    """The whole oracle path (its own FP64 A, B, X) against the reference's stored motions."""
    g = np.load(GOLDEN)
    ref = O.solve_body(quarter(), g["omegas"], g["headings"], symmetry=O.SYM_BOTH, rigid=FREE)
    assert scaled_error(ref["motions"], g["motion"]) <= 2e-5


def _gpu():
    from hydrobem_b200 import native as nv
    return nv


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_motions_against_the_oracle(precision):
    nv = _gpu()
    g = np.load(GOLDEN)
    omegas = np.r_[g["omegas"], 1.4, 3.0]
    heads = [0.0, 30.0, 75.0]
    prec = nv.HBG_MIXED if precision == "mixed" else nv.HBG_FP64
    gpu = nv.solve(quarter(), omegas, heads, symmetry=nv.SYM_BOTH, rigid=FREE, precision=prec)
    ref = O.solve_body(quarter(), omegas, heads, symmetry=O.SYM_BOTH, rigid=FREE)
    tol = 1e-5 if precision == "mixed" else 1e-9
    assert scaled_error(gpu["motions"], ref["motions"]) <= tol
    h, r = gpu["hydrostatics"][0], ref["hydrostatics"][0]
    for k in ("volumes", "center_of_buoyancy", "stiffness_rho_g", "stiffness"):
        assert np.abs(h[k] - r[k]).max() <= 1e-12 * max(np.abs(r[k]).max(), 1.0), k
    assert h["mass"] == r["mass"] and h["displaced_mass"] == pytest.approx(r["displaced_mass"], rel=1e-13)
    # the stored motions of the reference (float32 solve) within the regression bar
    assert scaled_error(gpu["motions"][:2, :2], g["motion"]) <= 2e-5


@pytest.mark.gpu
def test_gpu_motions_two_bodies_displaced_gyration_and_additional_matrices():
    """Two interacting cylinders: the first with its displaced mass and radii of gyration about its
    rotation centre, the second with a given mass and inertia components about a point; additional
    stiffness and damping couple them."""
    nv = _gpu()
    a = meshes.cylinder(1.0, 0.5, 16, 4, 4).copy()
    b = a.copy()
    a[..., 0] -= 3.0
    b[..., 0] += 3.0
    v = np.concatenate([a, b])
    body = np.r_[np.zeros(len(a), np.int32), np.ones(len(b), np.int32)]
    centers = [[-3.0, 0.0, 0.0], [3.0, 0.0, -0.1]]
    D = 12
    rng = np.random.default_rng(7)
    K = rng.standard_normal((D, D)) * 200.0
    rigid = {"mass": [np.nan, 1400.0], "center_of_gravity": [[-3.0, 0.0, -0.15], [3.0, 0.05, -0.2]],
             "inertia_kind": [1, 0],
             "inertia": [np.diag([0.6, 0.6, 0.7]), [[500.0, 3.0, 0.0], [3.0, 520.0, 1.0], [0.0, 1.0, 700.0]]],
             "inertia_origin": [[-3.0, 0.0, 0.0], [3.1, 0.0, -0.3]],
             "stiffness": K + K.T, "damping": np.abs(K) * 0.1}
    omegas = np.array([0.9, 1.7, 2.6])
    heads = [0.0, 45.0]
    gpu = nv.solve(v, omegas, heads, panel_body=body, rotation_centers=centers, rigid=rigid)
    ref = O.solve_body(v, omegas, heads, panel_body=body, centers=centers, rigid=rigid)
    assert gpu["motions"].shape == (3, 2, 12)
    assert scaled_error(gpu["motions"], ref["motions"]) <= 1e-9
    for hb, rb in zip(gpu["hydrostatics"], ref["hydrostatics"]):
        assert hb["mass"] == pytest.approx(rb["mass"], rel=1e-13)
        assert np.abs(hb["stiffness"] - rb["stiffness"]).max() <= 1e-12 * np.abs(rb["stiffness"]).max()


@pytest.mark.gpu
def test_gpu_motions_through_the_model_abi():
    """lo_cylinder_drift through hb_model_solve with its mass properties and motion = true: the motion
    and hydrostatics quantities against the reference's stored ones."""
    nv = _gpu()
    g = np.load(GOLDEN)
    L = nv.lib()
    m = ctypes.c_void_p()
    assert L.hb_model_new(ctypes.byref(m)) == 0
    try:
        def obj(path):
            o = ctypes.c_uint64()
            assert L.hb_object(m, path.encode(), ctypes.byref(o)) == 0, L.hb_last_error_message()
            return o.value

        L.hb_add.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                             ctypes.c_int64, ctypes.POINTER(ctypes.c_uint64)]
        L.hb_set_reals.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, nv.dp,
                                   ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t]
        L.hb_set_text.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_char_p]
        L.hb_set_real.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_double]
        L.hb_set_bool.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_int32]
        out = ctypes.c_uint64()

        def reals(o, name, arr):
            a = np.ascontiguousarray(arr, dtype=np.float64)
            assert L.hb_set_reals(m, o, name, a.ctypes.data_as(nv.dp), (ctypes.c_size_t * a.ndim)(*a.shape),
                                  a.ndim) == 0, L.hb_last_error_message()

        assert L.hb_add(m, 0, b"meshes", None, b"cyl", -1, ctypes.byref(out)) == 0
        reals(obj("meshes/cyl"), b"vertices", quarter())
        assert L.hb_set_text(m, obj("meshes/cyl"), b"symmetry", b"xz_and_yz") == 0
        assert L.hb_add(m, 0, b"bodies", None, b"body", -1, ctypes.byref(out)) == 0
        bo = obj("bodies/body")
        assert L.hb_set_text(m, bo, b"mesh", b"cyl") == 0
        reals(bo, b"center_of_gravity", [0.0, 0.0, -0.2])
        assert L.hb_set_real(m, bo, b"mass", MASS) == 0
        assert L.hb_set_text(m, bo, b"inertia_input", b"components") == 0
        for k, val in (("Ixx", MASS * 0.36), ("Iyy", MASS * 0.36), ("Izz", MASS * 0.49)):
            assert L.hb_set_real(m, bo, k.encode(), val) == 0
        assert L.hb_set_text(m, bo, b"inertia_origin", b"center_of_gravity") == 0
        assert L.hb_set_bool(m, obj("options"), b"motion", 1) == 0
        env = obj("environment")
        reals(env, b"omegas", g["omegas"])
        reals(env, b"headings", g["headings"])
        res = ctypes.c_void_p()
        L.hb_model_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        assert L.hb_model_solve(m, None, None, ctypes.byref(res)) == 0, L.hb_last_error_message()
        L.hb_results_quantity.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(nv.HbColumn)]

        def quantity(name, dtype):
            col = nv.HbColumn()
            assert L.hb_results_quantity(res, name.encode(), ctypes.byref(col)) == 0, name
            shape = tuple(col.shape[i] for i in range(col.ndim))
            ct = ctypes.c_float if dtype in (np.float32, np.complex64) else ctypes.c_double
            n = col.count * (2 if dtype in (np.complex64, np.complex128) else 1)
            return np.ctypeslib.as_array(ctypes.cast(col.data, ctypes.POINTER(ct)), shape=(n,)).copy().view(
                dtype).reshape(shape)

        mo = quantity("motion_f64", np.complex128)
        mo32 = quantity("motion", np.complex64)
        hs = {k: quantity(k, np.float64) for k in (
            "hydrostatics_volumes", "hydrostatics_center_of_buoyancy", "hydrostatics_waterplane_area",
            "hydrostatics_stiffness_rho_g", "hydrostatics_stiffness", "hydrostatics_mass",
            "hydrostatics_displaced_mass", "hydrostatics_center_of_gravity", "hydrostatics_metacentric_height")}
        L.hb_results_free(res)
        # the motions need the mass properties of every body
        m2 = ctypes.c_void_p()
        assert L.hb_model_new(ctypes.byref(m2)) == 0
        assert L.hb_add(m2, 0, b"meshes", None, b"cyl", -1, ctypes.byref(out)) == 0
        o2 = ctypes.c_uint64()
        assert L.hb_object(m2, b"meshes/cyl", ctypes.byref(o2)) == 0
        q = np.ascontiguousarray(quarter())
        assert L.hb_set_reals(m2, o2.value, b"vertices", q.ctypes.data_as(nv.dp), (ctypes.c_size_t * 3)(*q.shape), 3) == 0
        assert L.hb_add(m2, 0, b"bodies", None, b"body", -1, ctypes.byref(out)) == 0
        assert L.hb_object(m2, b"bodies/body", ctypes.byref(o2)) == 0
        assert L.hb_set_text(m2, o2.value, b"mesh", b"cyl") == 0
        assert L.hb_object(m2, b"options", ctypes.byref(o2)) == 0
        assert L.hb_set_bool(m2, o2.value, b"motion", 1) == 0
        assert L.hb_object(m2, b"environment", ctypes.byref(o2)) == 0
        w = np.ascontiguousarray([1.0])
        assert L.hb_set_reals(m2, o2.value, b"omegas", w.ctypes.data_as(nv.dp), (ctypes.c_size_t * 1)(1), 1) == 0
        assert L.hb_set_reals(m2, o2.value, b"headings", w.ctypes.data_as(nv.dp), (ctypes.c_size_t * 1)(1), 1) == 0
        res2 = ctypes.c_void_p()
        assert L.hb_model_solve(m2, None, None, ctypes.byref(res2)) == 1  # HB_ERR_VALUE
        L.hb_model_free(m2)
    finally:
        L.hb_model_free(m)
    assert mo.shape == g["motion"].shape and mo32.dtype == np.complex64
    assert scaled_error(mo, g["motion"]) <= 2e-5
    for k, v in hs.items():
        ref = g[k]
        assert v.shape == ref.shape, k
        assert np.allclose(v, ref, rtol=1e-11, atol=1e-11 * max(np.abs(ref).max(), 1.0)), k
