"""Field points (crates/hydrobem/src/lo_frequency.rs:1392-1470 field_values): the elevation at z = 0 or
p / (rho g) below it, of the radiation waves per unit displacement and of the incident, scattered and
total waves per unit amplitude, by Green's identity over the panels at each point.

Pinned on the reference's own outputs of its regression problem lo_cylinder_field_body_points (the
cylinder r = 1 m, draught 0.5 m held fixed; three points, one on the free surface): the oracle against
them, then the GPU (both forms, symmetry sectors, finite depth, two bodies, the object model) against the
oracle and them.
"""
from __future__ import annotations

import ctypes
import math
from pathlib import Path

import numpy as np
import pytest

from hydrobem_b200 import meshes
from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden" / "lo_cylinder_field.npz"
KEYS = (("field_radiation", "field_points_pressure_radiation"), ("field_incident", "field_points_pressure_incident"),
        ("field_scattering", "field_points_pressure_scattering"),
        ("field_diffraction", "field_points_pressure_diffraction"))


def scaled_error(got, ref, floor=1e-3):
    ref = np.asarray(ref)
    peak = np.abs(ref).max()
    scale = np.maximum(np.abs(ref).max(axis=0, keepdims=True), floor * peak)
    return float((np.abs(np.asarray(got) - ref) / scale).max())


def quarter():
    return meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True)


def test_oracle_field_points_against_the_reference():
    g = np.load(GOLDEN)
    ref = O.solve_body(quarter(), g["omegas"], g["headings"], symmetry=O.SYM_BOTH, points=g["field_points"])
    for mine, theirs in KEYS:
        assert scaled_error(ref[mine], g[theirs]) <= 2e-5, mine


def test_oracle_field_incident_wave_is_the_boundary_formula():
    """The incident elevation at a point on z = 0 has modulus 1 (unit amplitude) in infinite depth."""
    g = np.load(GOLDEN)
    ref = O.solve_body(quarter(), g["omegas"], g["headings"], symmetry=O.SYM_BOTH, points=g["field_points"])
    assert np.allclose(np.abs(ref["field_incident"][:, 0, :]), 1.0, rtol=1e-13)


def _gpu():
    from hydrobem_b200 import native as nv
    return nv


POINTS = np.array([[3.0, 0.5, 0.0], [2.0, 2.0, -0.4], [-2.5, 1.0, -0.2], [0.3, -1.6, 0.0], [1.2, 0.1, -0.7],
                   [-0.4, 0.2, -0.9]])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("sym,depth", [(0, math.inf), (3, math.inf), (3, 3.0), (1, 5.0)])
def test_gpu_field_points_against_the_oracle(precision, sym, depth):
    nv = _gpu()
    q = quarter()
    body = q if sym == 3 else O.mirror_sector(q, O.SYM_XZ) if sym == 1 else O.mirror_sector(q, O.SYM_BOTH)
    omegas = np.array([1.1, 2.2, 4.0])
    heads = [0.0, 40.0]
    prec = nv.HBG_MIXED if precision == "mixed" else nv.HBG_FP64
    gpu = nv.solve(body, omegas, heads, symmetry=sym, depth=depth, points=POINTS, precision=prec)
    ref = O.solve_body(body, omegas, heads, depth=depth, symmetry=sym, points=POINTS)
    tol = 1e-5 if precision == "mixed" else 1e-9
    for mine, _ in KEYS:
        assert gpu[mine].shape == ref[mine].shape
        assert scaled_error(gpu[mine], ref[mine]) <= tol, mine


@pytest.mark.gpu
def test_gpu_field_points_two_bodies_and_a_lid():
    """Two cylinders (12 radiation columns), the second with an interior lid (no part in the sums)."""
    nv = _gpu()
    a = meshes.cylinder(1.0, 0.5, 16, 4, 4).copy()
    lid = meshes.box(0.6, 0.6, 0.5, n=(4, 4, 1), lid=True)[-16:]
    b = np.concatenate([a, lid])
    a[..., 0] -= 3.0
    b[..., 0] += 3.0
    v = np.concatenate([a, b])
    body = np.r_[np.zeros(len(a), np.int32), np.ones(len(b), np.int32)]
    kinds = np.r_[np.zeros(len(a) + len(a), np.int32), np.ones(16, np.int32)]
    centers = [[-3.0, 0.0, 0.0], [3.0, 0.0, 0.0]]
    omegas = np.array([1.3, 2.5])
    pts = np.array([[0.0, 0.0, 0.0], [0.0, 2.0, -0.3], [6.0, 1.0, -0.1]])
    gpu = nv.solve(v, omegas, [15.0], kinds=kinds, panel_body=body, rotation_centers=centers, points=pts)
    ref = O.solve_body(v, omegas, [15.0], kinds=kinds, panel_body=body, centers=centers, points=pts)
    assert gpu["field_radiation"].shape == (2, 3, 12)
    for mine, _ in KEYS:
        assert scaled_error(gpu[mine], ref[mine]) <= 1e-9, mine


@pytest.mark.gpu
def test_gpu_field_points_through_the_model_abi():
    """lo_cylinder_field_body_points through hb_model_solve (first_order.field_points, field_pressure):
    the field quantities against the reference's stored ones."""
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
        assert L.hb_set_text(m, obj("bodies/body"), b"mesh", b"cyl") == 0
        fo = obj("first_order")
        reals(fo, b"field_points", g["field_points"])
        assert L.hb_set_bool(m, fo, b"field_pressure", 1) == 0
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

        got = {theirs: quantity(theirs + "_f64", np.complex128) for _, theirs in KEYS}
        got32 = quantity("field_points_pressure_radiation", np.complex64)
        pts = quantity("field_points", np.float64)
        L.hb_results_free(res)
    finally:
        L.hb_model_free(m)
    assert np.array_equal(pts, g["field_points"]) and got32.dtype == np.complex64
    for _, theirs in KEYS:
        assert got[theirs].shape == g[theirs].shape
        assert scaled_error(got[theirs], g[theirs]) <= 2e-5, theirs


@pytest.mark.gpu
def test_gpu_field_point_arguments_checked():
    nv = _gpu()
    with pytest.raises(nv.HydroBEMError) as e:
        nv.solve(quarter(), [1.0], [0.0], symmetry=nv.SYM_BOTH, points=[[2.0, 0.0, 0.5]])
    assert e.value.status == 1  # HB_ERR_VALUE: above the free surface
