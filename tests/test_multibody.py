"""Interacting bodies: several rigid bodies in one problem, 6 modes each (the reference's several bodies
of one model: crates/hydrobem/src/lo_frequency.rs:236-251 radiation columns per body, 1039-1115 forces
per coordinate, low_order.rs:313 generalized normals about each body's rotation centre).

The oracle is checked on CPU by linearity (a rigid body split into two bodies that rotate about the same
point: the single body's matrices are the sums of the two-body blocks); the GPU forms against the oracle
on two cylinders that interact.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from hydrobem_b200 import meshes
from oracle import oracle as O

OMEGAS = 2.0 * math.pi / np.array([2.0, 4.0, 7.0])
HEADS = [0.0, 45.0]


def scaled_error(got, ref, floor=1e-3):
    ref = np.asarray(ref)
    got = np.asarray(got)
    peak = np.abs(ref).max()
    scale = np.maximum(np.abs(ref).max(axis=0, keepdims=True), floor * peak)
    return float((np.abs(got - ref) / scale).max())


def two_cylinders(gap=3.0):
    """Two cylinders (r 1 m, draft 0.5 m, 128 panels each) at x = -gap and x = +gap."""
    a = meshes.cylinder(1.0, 0.5, 16, 4, 4).copy()
    b = a.copy()
    a[..., 0] -= gap
    b[..., 0] += gap
    v = np.concatenate([a, b])
    body = np.r_[np.zeros(len(a), np.int32), np.ones(len(b), np.int32)]
    return v, body, [[-gap, 0.0, 0.0], [gap, 0.0, 0.0]]


def split_cylinder():
    """One cylinder whose panels are assigned to two bodies by the sign of the centroid's x."""
    v = meshes.cylinder(1.0, 0.5, 16, 4, 4)
    body = (v.mean(axis=1)[:, 0] > 0.0).astype(np.int32)
    return v, body


def block_sums(r, F, H):
    """The 12-mode results of a split body summed over the body blocks (6 modes)."""
    out = {"A": r["A"].reshape(F, 2, 6, 2, 6).sum(axis=(1, 3)), "B": r["B"].reshape(F, 2, 6, 2, 6).sum(axis=(1, 3))}
    for k in ("X", "FK", "SC", "HK"):
        out[k] = r[k].reshape(F, H, 2, 6).sum(axis=2)
    return out


def test_oracle_split_body_is_linear():
    v, body = split_cylinder()
    one = O.solve_body(v, OMEGAS[:2], HEADS, depth=math.inf)
    two = O.solve_body(v, OMEGAS[:2], HEADS, depth=math.inf, panel_body=body, centers=[[0, 0, 0], [0, 0, 0]])
    assert two["A"].shape == (2, 12, 12) and two["X"].shape == (2, 2, 12)
    summed = block_sums(two, 2, len(HEADS))
    for k in ("A", "B", "X", "FK", "SC", "HK"):
        assert scaled_error(summed[k], one[k]) <= 1e-10, k


def test_oracle_rotation_centre_shifts_moments():
    """Moving the rotation centre by r changes the roll/pitch/yaw normals by -(r x n): the translation
    columns of A are unchanged and the moment rows pick up -(r x F)."""
    v = meshes.cylinder(1.0, 0.5, 16, 4, 4)
    r = np.array([0.3, -0.2, 0.1])
    base = O.solve_body(v, OMEGAS[:1], [], depth=math.inf)
    moved = O.solve_body(v, OMEGAS[:1], [], depth=math.inf, panel_body=np.zeros(len(v), np.int32), centers=[r])
    assert np.allclose(moved["A"][:, :3, :3], base["A"][:, :3, :3], rtol=1e-12, atol=0.0)
    # row i >= 3 (moment about R): M_R = M_0 - r x F for the translation columns
    F0 = base["A"][0, :3, :3]
    expect = base["A"][0, 3:, :3] - np.cross(r, F0.T).T
    assert np.allclose(moved["A"][0, 3:, :3], expect, rtol=1e-10, atol=1e-12 * np.abs(F0).max())


@pytest.mark.gpu
@pytest.mark.parametrize("depth", [math.inf, 3.0])
def test_gpu_two_interacting_bodies(depth):
    from hydrobem_b200 import native as nv

    v, body, centers = two_cylinders()
    gpu = nv.solve(v, OMEGAS, HEADS, depth=depth, panel_body=body, rotation_centers=centers)
    ref = O.solve_body(v, OMEGAS, HEADS, depth=depth, panel_body=body, centers=centers)
    assert gpu["A"].shape == (3, 12, 12) and gpu["X"].shape == (3, 2, 12)
    errs = {k: scaled_error(gpu[k], ref[k]) for k in ("A", "B", "X", "FK", "SC", "HK")}
    assert max(errs.values()) <= 1e-9, errs
    # the two bodies are mirror images about x = 0 and the heading-0 wave comes along x: their heave
    # added masses agree
    assert abs(gpu["A"][0, 2, 2] - gpu["A"][0, 8, 8]) <= 1e-9 * abs(gpu["A"][0, 2, 2])


@pytest.mark.gpu
def test_gpu_mixed_two_interacting_bodies():
    from hydrobem_b200 import native as nv

    v, body, centers = two_cylinders()
    gpu = nv.solve(v, OMEGAS, HEADS, depth=3.0, panel_body=body, rotation_centers=centers, precision=nv.HBG_MIXED)
    ref = O.solve_body(v, OMEGAS, HEADS, depth=3.0, panel_body=body, centers=centers)
    errs = {k: scaled_error(gpu[k], ref[k]) for k in ("A", "B", "X")}
    assert max(errs.values()) <= 1e-5, errs


@pytest.mark.gpu
def test_gpu_split_body_is_linear():
    from hydrobem_b200 import native as nv

    v, body = split_cylinder()
    one = nv.solve(v, OMEGAS, HEADS)
    two = nv.solve(v, OMEGAS, HEADS, panel_body=body, rotation_centers=[[0, 0, 0], [0, 0, 0]])
    summed = block_sums(two, len(OMEGAS), len(HEADS))
    for k in ("A", "B", "X", "FK", "SC", "HK"):
        assert scaled_error(summed[k], one[k]) <= 1e-10, k


@pytest.mark.gpu
def test_gpu_body_arguments_checked():
    import ctypes

    from hydrobem_b200 import native as nv

    v, body, centers = two_cylinders()
    bad = body.copy()
    bad[5] = 7
    b = nv.Body(v, OMEGAS[:1], [], panel_body=bad, rotation_centers=centers)
    b.n_bodies = 2
    arr = (nv.HbgProblem * 1)(b.problem())
    opt = nv.default_options()
    assert nv.lib().hbg_solve_batch(arr, 1, ctypes.byref(opt)) == 1  # HB_ERR_VALUE
    # more right-hand sides than the solve takes: 6 bodies (36 modes)
    many = nv.Body(np.concatenate([v, v, v]), OMEGAS[:1], [], panel_body=np.r_[body, body + 2, body + 4])
    arr = (nv.HbgProblem * 1)(many.problem())
    assert nv.lib().hbg_solve_batch(arr, 1, ctypes.byref(opt)) == 3  # HB_ERR_UNSUPPORTED


@pytest.mark.gpu
def test_gpu_two_bodies_through_the_model_abi():
    """Two bodies of one mesh placed by position, rotation centres body-local: the model layer's solve
    equals the batched entry's with the panels moved and labelled by hand."""
    import ctypes

    from hydrobem_b200 import native as nv

    cyl = np.ascontiguousarray(meshes.cylinder(1.0, 0.5, 16, 4, 4))
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
        out = ctypes.c_uint64()
        assert L.hb_add(m, 0, b"meshes", None, b"cyl", -1, ctypes.byref(out)) == 0
        assert L.hb_set_reals(m, obj("meshes/cyl"), b"vertices", cyl.ctypes.data_as(nv.dp),
                              (ctypes.c_size_t * 3)(*cyl.shape), 3) == 0
        rc_local = np.array([0.1, 0.0, -0.2])
        for name, x in ((b"west", -3.0), (b"east", 3.0)):
            assert L.hb_add(m, 0, b"bodies", None, name, -1, ctypes.byref(out)) == 0
            b = obj("bodies/" + name.decode())
            assert L.hb_set_text(m, b, b"mesh", b"cyl") == 0
            pos = np.array([x, 0.0, 0.0])
            assert L.hb_set_reals(m, b, b"position", pos.ctypes.data_as(nv.dp), (ctypes.c_size_t * 1)(3), 1) == 0
            assert L.hb_set_reals(m, b, b"rotation_center", rc_local.ctypes.data_as(nv.dp),
                                  (ctypes.c_size_t * 1)(3), 1) == 0
            assert L.hb_set_real(m, b, b"yaw", 0.0) == 0
            assert L.hb_set_real(m, b, b"yaw", 10.0) == 3  # a rotated body is not on this route
        env = obj("environment")
        w = np.ascontiguousarray(OMEGAS)
        h = np.ascontiguousarray(HEADS, dtype=np.float64)
        assert L.hb_set_reals(m, env, b"omegas", w.ctypes.data_as(nv.dp), (ctypes.c_size_t * 1)(w.size), 1) == 0
        assert L.hb_set_reals(m, env, b"headings", h.ctypes.data_as(nv.dp), (ctypes.c_size_t * 1)(h.size), 1) == 0
        res = ctypes.c_void_p()
        L.hb_model_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        assert L.hb_model_solve(m, None, None, ctypes.byref(res)) == 0, L.hb_last_error_message()
        L.hb_results_quantity.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(nv.HbColumn)]
        c = nv.HbColumn()
        assert L.hb_results_quantity(res, b"added_mass_f64", ctypes.byref(c)) == 0
        shape = tuple(c.shape[i] for i in range(c.ndim))
        A = np.ctypeslib.as_array(ctypes.cast(c.data, ctypes.POINTER(ctypes.c_double)), shape=shape).copy()
        L.hb_results_free(res)
    finally:
        L.hb_model_free(m)
    assert A.shape == (len(OMEGAS), 12, 12)
    v, body, _ = two_cylinders()
    direct = nv.solve(v, OMEGAS, HEADS, panel_body=body,
                      rotation_centers=[[-3.0 + rc_local[0], 0.0, rc_local[2]], [3.0 + rc_local[0], 0.0, rc_local[2]]])
    assert np.abs(A - direct["A"]).max() <= 1e-12 * np.abs(direct["A"]).max()


def three_cylinder_array(n_phi=16, n_z=4, n_r=4):
    """The array of the surrogate configuration at a reduced panel count: three cylinders of radius 1 m
    and draft 1 m, 4 m apart along x, each rotating about its own axis at the waterline."""
    one = meshes.cylinder(1.0, 1.0, n_phi, n_z, n_r)
    parts, body, centers = [], [], []
    for b, x in enumerate((-4.0, 0.0, 4.0)):
        c = one.copy()
        c[..., 0] += x
        parts.append(c)
        body.append(np.full(len(c), b, np.int32))
        centers.append([x, 0.0, 0.0])
    return np.concatenate(parts), np.concatenate(body), centers


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_three_cylinder_array(precision):
    """18 modes and one heading: 19 right-hand sides, beyond the 16 of the persistent sweeps and the TMA
    residual, so the stepwise solves and the register-form products run."""
    from hydrobem_b200 import native as nv

    v, body, centers = three_cylinder_array()
    omegas = OMEGAS[:2]
    prec = nv.HBG_MIXED if precision == "mixed" else nv.HBG_FP64
    gpu = nv.solve(v, omegas, [0.0], panel_body=body, rotation_centers=centers, precision=prec)
    ref = O.solve_body(v, omegas, [0.0], depth=math.inf, panel_body=body, centers=centers)
    assert gpu["A"].shape == (2, 18, 18)
    keys = ("A", "B", "X", "FK", "SC", "HK") if precision == "fp64" else ("A", "B", "X", "HK")
    errs = {k: scaled_error(gpu[k], ref[k]) for k in keys}
    assert max(errs.values()) <= (1e-9 if precision == "fp64" else 1e-5), errs
