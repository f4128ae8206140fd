"""Parity of the GPU FP64 form with the CPU oracle, through the C ABI (libhydrobem_gpu.so).

Bar (the plain FP64 form is the correctness oracle of the mixed form): statics, S and A entry by
entry within 1e-10 of their scale; A, B, X, FK, SC within 1e-9 of each entry's scale -- its largest
modulus over the frequencies, floor 1e-3 of the quantity's peak: the measure of the reference's
regression test (tests/python/test_regression.py:34-78) at a 1e-9 bound.  The floor keeps the
couplings that vanish by symmetry (roll-heave of a cylinder, ~1e-14 of the peak in both codes) from
turning rounding noise into a relative error.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from hydrobem_b200 import meshes
from hydrobem_b200 import native as nv
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-9


def scaled_error(got, ref, floor=1e-3):
    ref = np.asarray(ref)
    got = np.asarray(got)
    peak = np.abs(ref).max()
    scale = np.maximum(np.abs(ref).max(axis=0, keepdims=True), floor * peak)
    return float((np.abs(got - ref) / scale).max())


def compare(gpu, ref, keys=("A", "B", "X", "FK", "SC", "HK")):
    errs = {k: scaled_error(gpu[k], ref[k]) for k in keys if k in ref and np.asarray(ref[k]).size}
    assert max(errs.values()) <= TOL, errs
    return errs


C1 = dict(mesh=lambda: meshes.cylinder(1.0, 0.5, 32, 8, 8), periods=np.arange(2.0, 12.0), heads=[0.0], depth=math.inf)


@pytest.mark.parametrize("depth", [math.inf, 5.0, 1.5])
def test_statics_and_matrices_match_oracle(depth):
    v = meshes.cylinder(1.0, 0.5, 16, 4, 4)
    omega = 2.0 * math.pi / 3.0
    st, S, A = nv.debug_matrices(v, omega, depth=depth)
    pan = O.make_panels(v)
    st_o = O.statics(pan, None, depth)
    S_o, A_o = O.assemble(pan, None, st_o, depth, omega)
    for q in range(4):
        scale = max(np.abs(st_o[..., q]).max(), 1e-300)
        assert np.abs(st[..., q] - st_o[..., q]).max() <= 1e-10 * scale, q
    assert np.abs(S - S_o).max() <= 1e-10 * np.abs(S_o).max()
    assert np.abs(A - A_o).max() <= 1e-10 * np.abs(A_o).max()


def test_config1_cylinder_infinite_depth():
    """The reference's CPU-runnable configuration: cylinder r 1 m, draft 0.5 m, 512 panels, infinite
    depth, periods 2..11 s, heading 0."""
    v = C1["mesh"]()
    omegas = 2.0 * math.pi / C1["periods"]
    gpu = nv.solve(v, omegas, C1["heads"])
    ref = O.solve_body(v, omegas, C1["heads"], depth=math.inf)
    compare(gpu, ref)


@pytest.mark.parametrize("depth", [5.0, 1.5])
def test_finite_depth_cylinder(depth):
    """Finite depth (h = 5: every pair in the tiled integral form; h = 1.5: pairs beyond h/2 in the
    eigenfunction series), four headings."""
    v = meshes.cylinder(1.0, 0.5, 32, 8, 8)
    omegas = 2.0 * math.pi / np.array([1.5, 3.0, 7.0, 20.0])
    heads = [0.0, 30.0, 60.0, 90.0]
    gpu = nv.solve(v, omegas, heads, depth=depth)
    ref = O.solve_body(v, omegas, heads, depth=depth)
    compare(gpu, ref)


def test_many_headings():
    """12 headings: 18 right-hand sides (the wide substitution variant)."""
    v = meshes.cylinder(1.0, 0.5, 16, 4, 4)
    heads = list(np.linspace(0.0, 330.0, 12))
    omegas = np.array([0.9, 2.2])
    gpu = nv.solve(v, omegas, heads, depth=3.0)
    ref = O.solve_body(v, omegas, heads, depth=3.0)
    compare(gpu, ref)


def test_interior_lid_box():
    """A box with an interior free-surface lid (kind interior: column K S, free term -4 pi, the
    in-plane log integral for pairs both in z = 0)."""
    v = meshes.box(1.0, 0.5, 0.5, n=(8, 4, 4), lid=True)
    n_lid = 8 * 4
    kinds = np.zeros(len(v), np.int32)
    kinds[-n_lid:] = 1
    omegas = np.array([1.0, 2.0, 3.5])
    heads = [0.0, 45.0]
    gpu = nv.solve(v, omegas, heads, kinds=kinds)
    ref = O.solve_body(v, omegas, heads, depth=math.inf, kinds=kinds)
    compare(gpu, ref)


def test_batched_bodies_of_uneven_size():
    """Several bodies of different panel counts and frequencies in one call."""
    bodies = [nv.Body(meshes.cylinder(1.0, 0.5, 16, 4, 4), [0.8, 1.7], [0.0]),
              nv.Body(meshes.hemisphere(1.3, 6, 12), [1.1], [0.0, 90.0]),
              nv.Body(meshes.cylinder(2.0, 1.0, 24, 6, 6), [0.5, 1.0, 2.0], [30.0])]
    out = nv.solve_batch(bodies, max_batch=2)
    for b, g in zip(bodies, out):
        ref = O.solve_body(b.vertices, b.omegas, b.headings, depth=math.inf)
        compare(g, ref)


def test_reference_solver_outputs_through_the_model_abi():
    """The regression problem lo_cylinder_drift through hb_model_solve (quarter mesh with two
    symmetry planes): within 2e-5 of the reference's own outputs and 1e-9 of the oracle."""
    import ctypes
    from pathlib import Path

    g = np.load(Path(__file__).resolve().parent / "golden" / "lo_cylinder_drift.npz")
    quarter = meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True)
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
        out = ctypes.c_uint64()
        assert L.hb_add(m, 0, b"meshes", None, b"cyl", -1, ctypes.byref(out)) == 0
        q = np.ascontiguousarray(quarter)
        assert L.hb_set_reals(m, obj("meshes/cyl"), b"vertices", q.ctypes.data_as(nv.dp),
                              (ctypes.c_size_t * 3)(*q.shape), 3) == 0
        assert L.hb_set_text(m, obj("meshes/cyl"), b"symmetry", b"xz_and_yz") == 0
        assert L.hb_add(m, 0, b"bodies", None, b"body", -1, ctypes.byref(out)) == 0
        assert L.hb_set_text(m, obj("bodies/body"), b"mesh", b"cyl") == 0
        env = obj("environment")
        w = np.ascontiguousarray(g["omegas"])
        h = np.ascontiguousarray(g["headings"])
        assert L.hb_set_reals(m, env, b"omegas", w.ctypes.data_as(nv.dp), (ctypes.c_size_t * 1)(w.size), 1) == 0
        assert L.hb_set_reals(m, env, b"headings", h.ctypes.data_as(nv.dp), (ctypes.c_size_t * 1)(h.size), 1) == 0
        res = ctypes.c_void_p()
        L.hb_model_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        assert L.hb_model_solve(m, None, None, ctypes.byref(res)) == 0, L.hb_last_error_message()
        L.hb_results_quantity.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(nv.HbColumn)]

        def quantity(name, dtype):
            c = nv.HbColumn()
            assert L.hb_results_quantity(res, name.encode(), ctypes.byref(c)) == 0
            shape = tuple(c.shape[i] for i in range(c.ndim))
            return np.ctypeslib.as_array(ctypes.cast(c.data, ctypes.POINTER(ctypes.c_double if dtype != np.float32
                                                                               else ctypes.c_float)),
                                         shape=(c.count * (2 if dtype == np.complex128 else 1),)).copy().view(
                dtype).reshape(shape)

        A = quantity("added_mass_f64", np.float64)
        B = quantity("radiation_damping_f64", np.float64)
        X = quantity("excitation_diffraction_f64", np.complex128)
        A32 = quantity("added_mass", np.float32)
        assert A32.dtype == np.float32 and A32.shape == A.shape
        L.hb_results_free(res)
    finally:
        L.hb_model_free(m)
    full = meshes.reflect_full(quarter)
    ref = O.solve_body(full, g["omegas"], g["headings"], depth=math.inf)
    compare({"A": A, "B": B, "X": X}, ref, keys=("A", "B", "X"))
    assert scaled_error(A, g["added_mass"], 1e-3) <= 2e-5
    assert scaled_error(B, g["radiation_damping"], 1e-3) <= 2e-5
    assert scaled_error(X, g["excitation_diffraction"], 1e-3) <= 2e-5


def test_error_paths():
    """Invalid inputs come back as the reference's status codes, with nothing run on them."""
    v = meshes.cylinder(1.0, 0.5, 8, 2, 2).copy()
    with pytest.raises(nv.HydroBEMError) as e:
        nv.solve(v, [0.0], [0.0])
    assert e.value.status == 1 and e.value.location["frequency"] == 0
    bad = v.copy()
    bad[3] = bad[3][[0, 0, 0, 0]]  # a degenerate panel
    with pytest.raises(nv.HydroBEMError) as e:
        nv.solve(bad, [1.0], [0.0])
    assert e.value.status == 1 and "panel 4" in e.value.message
    # the mixed form reads the flag only at the end of its solve; its assembly skips the work
    for depth in (float("inf"), 3.0):
        with pytest.raises(nv.HydroBEMError) as e:
            nv.solve(bad, [1.0, 1.5], [0.0], precision=nv.HBG_MIXED, depth=depth)
        assert e.value.status == 1 and "panel 4" in e.value.message
    g = nv.solve(v, [1.0], [0.0], precision=nv.HBG_MIXED)  # the context is still usable
    assert np.isfinite(g["A"]).all()
    import ctypes

    flag = (ctypes.c_int32 * 1)(1)
    body = nv.Body(v, [1.0], [0.0])
    arr = (nv.HbgProblem * 1)(body.problem())
    opt = nv.default_options()
    opt.cancel = ctypes.cast(flag, nv.ip)
    assert nv.lib().hbg_solve_batch(arr, 1, ctypes.byref(opt)) == 5  # HB_ERR_CANCELLED
