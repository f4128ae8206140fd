"""The generated interior surface interior_surface = "projected" (crates/hydrobem/src/interior.rs:79-138): the
downward-facing wetted panels projected onto the free surface, facing up, as interior panels that remove
the irregular frequencies.  The object model generates it; the oracle restates the rule and solves the body
with the lid given explicitly."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from hydrobem_b200 import meshes
from hydrobem_b200 import native as nv
from oracle import oracle as O


def _model(mesh, symmetry="none", interior="projected", position=None):
    L = nv.lib()
    m = ctypes.c_void_p()
    assert L.hb_model_new(ctypes.byref(m)) == 0
    L.hb_add.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                         ctypes.c_int64, ctypes.POINTER(ctypes.c_uint64)]
    L.hb_set_reals.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, nv.dp,
                               ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t]
    L.hb_set_text.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_char_p]
    out = ctypes.c_uint64()
    assert L.hb_add(m, 0, b"meshes", None, b"hull", -1, ctypes.byref(out)) == 0
    q = np.ascontiguousarray(mesh, dtype=np.float64)
    assert L.hb_set_reals(m, out.value, b"vertices", q.ctypes.data_as(nv.dp), (ctypes.c_size_t * 3)(*q.shape), 3) == 0
    assert L.hb_set_text(m, out.value, b"symmetry", symmetry.encode()) == 0
    assert L.hb_add(m, 0, b"bodies", None, b"body", -1, ctypes.byref(out)) == 0
    assert L.hb_set_text(m, out.value, b"mesh", b"hull") == 0
    assert L.hb_set_text(m, out.value, b"interior_surface", interior.encode()) == 0
    if position is not None:
        p = np.ascontiguousarray(position, dtype=np.float64)
        assert L.hb_set_reals(m, out.value, b"position", p.ctypes.data_as(nv.dp), (ctypes.c_size_t * 1)(3), 1) == 0
    env = ctypes.c_uint64()
    assert L.hb_object(m, b"environment", ctypes.byref(env)) == 0
    w = np.ascontiguousarray([1.0, 2.4])
    h = np.ascontiguousarray([0.0, 30.0])
    assert L.hb_set_reals(m, env.value, b"omegas", w.ctypes.data_as(nv.dp), (ctypes.c_size_t * 1)(2), 1) == 0
    assert L.hb_set_reals(m, env.value, b"headings", h.ctypes.data_as(nv.dp), (ctypes.c_size_t * 1)(2), 1) == 0
    return L, m


def _solve(L, m):
    res = ctypes.c_void_p()
    L.hb_model_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    st = L.hb_model_solve(m, None, None, ctypes.byref(res))
    return st, res


def test_oracle_projected_lid_of_a_cylinder():
    v = meshes.cylinder(1.0, 0.5, 8, 2, 3)
    lid = O.projected_lid(v)
    assert lid.shape == (8 * 3, 4, 3) and np.all(lid[..., 2] == 0.0)
    c, n, _ = O.panel_arrays(O.make_panels(lid, np.ones(len(lid), np.int32)))
    assert np.all(n[:, 2] > 0.99)  # facing up
    # the projected bottom covers the waterplane disc (area of the inscribed polygon)
    _, _, area = O.panel_arrays(O.make_panels(lid, np.ones(len(lid), np.int32)))
    assert area.sum() == pytest.approx(0.5 * 8 * np.sin(2 * np.pi / 8), rel=1e-12)


def test_model_refuses_what_cannot_be_projected():
    # a closed box sunk below the free surface: its top face points up into the fluid above it
    box = meshes.box(1.0, 0.5, 0.5, n=(2, 1, 1), lid=True).copy()
    box[..., 2] -= 1.0
    first_top = len(box) - 2 + 1  # the lid panels come last (nx ny = 2); 1-based
    with pytest.raises(ValueError, match=f"wetted element {first_top} faces upward"):
        O.projected_lid(box)
    L, m = _model(box)
    try:
        st, _ = _solve(L, m)
        msg = L.hb_last_error_message().decode()
        assert st == 1 and f"wetted element {first_top} faces upward" in msg, msg
    finally:
        L.hb_model_free(m)
    # a box without bottom: vertical walls only
    box = meshes.box(1.0, 0.5, 0.5, n=(2, 1, 1))
    walls = box[2:]  # drop the bottom panels (nx ny = 2)
    L, m = _model(walls)
    try:
        st, _ = _solve(L, m)
        assert st == 1 and "no wetted element faces downward" in L.hb_last_error_message().decode()
    finally:
        L.hb_model_free(m)


@pytest.mark.gpu
@pytest.mark.parametrize("symmetry", ["none", "xz_and_yz"])
def test_gpu_projected_lid_through_the_model(symmetry):
    q = meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True)
    mesh = q if symmetry != "none" else O.mirror_sector(q, O.SYM_BOTH)
    L, m = _model(mesh, symmetry)
    try:
        st, res = _solve(L, m)
        assert st == 0, L.hb_last_error_message()
        L.hb_results_quantity.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(nv.HbColumn)]
        got = {}
        for name, key, dt in (("added_mass_f64", "A", np.float64), ("radiation_damping_f64", "B", np.float64),
                              ("excitation_diffraction_f64", "X", np.complex128)):
            col = nv.HbColumn()
            assert L.hb_results_quantity(res, name.encode(), ctypes.byref(col)) == 0
            n = col.count * (2 if dt == np.complex128 else 1)
            got[key] = np.ctypeslib.as_array(ctypes.cast(col.data, ctypes.POINTER(ctypes.c_double)),
                                             shape=(n,)).copy().view(dt)
        L.hb_results_free(res)
    finally:
        L.hb_model_free(m)
    full = O.mirror_sector(q, O.SYM_BOTH)
    lid = O.projected_lid(full)
    verts = np.concatenate([full, lid])
    kinds = np.r_[np.zeros(len(full), np.int32), np.ones(len(lid), np.int32)]
    if symmetry == "none":
        ref = O.solve_body(verts, [1.0, 2.4], [0.0, 30.0], kinds=kinds)
    else:  # the sector's lid, mirrored with the sector
        sl = O.projected_lid(q)
        ref = O.solve_body(np.concatenate([q, sl]), [1.0, 2.4], [0.0, 30.0],
                           kinds=np.r_[np.zeros(len(q), np.int32), np.ones(len(sl), np.int32)], symmetry=O.SYM_BOTH)
    for k in ("A", "B", "X"):
        r = np.asarray(ref[k]).reshape(-1)
        assert np.abs(got[k] - r).max() <= 1e-9 * np.abs(r).max(), k
