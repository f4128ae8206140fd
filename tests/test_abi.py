"""The C-ABI library without a GPU: it loads, exports every symbol include/hydrobem_gpu.h declares,
and its host-side model layer follows the reference's conventions (hydrobem.h status codes,
out-pointers checked first, per-thread last error, refusals of items off this route)."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from hydrobem_b200 import native as nv

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    text = (ROOT / "include" / "hydrobem_gpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(hbg?_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = nv.lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert sorted(nv.EXPORTS) == names


def test_abi_version_and_defaults():
    L = nv.lib()
    # the reference's HB_ABI_VERSION (crates/hydrobem-c/src/info.rs:15): a caller built against
    # hydrobem.h compares hb_abi_version() with it
    assert L.hb_abi_version() == 8
    assert L.hbg_library_version() == 9
    o = nv.default_options()
    assert o.precision == nv.HBG_FP64 and o.logarithmic == 1
    assert o.log_tolerance == 1e-4 and o.gravity == 9.80665 and o.density == 1000.0
    assert np.isinf(o.depth) and o.max_batch == 0


def _model():
    L = nv.lib()
    m = ctypes.c_void_p()
    assert L.hb_model_new(ctypes.byref(m)) == 0
    return L, m


def _obj(L, m, path):
    o = ctypes.c_uint64()
    rc = L.hb_object(m, path.encode(), ctypes.byref(o))
    return rc, o.value


def test_model_layer_items_and_refusals():
    L, m = _model()
    try:
        rc, env = _obj(L, m, "environment")
        assert rc == 0
        rc, _ = _obj(L, m, "bodies/nothing")
        assert rc == 1  # HB_ERR_VALUE
        assert b"no object" in L.hb_last_error_message()
        w = np.array([0.5, 1.0])
        shape = (ctypes.c_size_t * 1)(2)
        L.hb_set_reals.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, nv.dp,
                                   ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t]
        assert L.hb_set_reals(m, env, b"omegas", w.ctypes.data_as(nv.dp), shape, 1) == 0
        bad = np.array([-1.0])
        assert L.hb_set_reals(m, env, b"omegas", bad.ctypes.data_as(nv.dp), (ctypes.c_size_t * 1)(1), 1) == 1
        L.hb_set_real.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_double]
        assert L.hb_set_real(m, env, b"depth", 5.0) == 0
        assert L.hb_set_real(m, env, b"depth", -1.0) == 1
        assert L.hb_set_real(m, env, b"wind_speed", 1.0) == 3  # HB_ERR_UNSUPPORTED
        # a mesh and a body
        L.hb_add.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                             ctypes.c_int64, ctypes.POINTER(ctypes.c_uint64)]
        mesh = ctypes.c_uint64()
        assert L.hb_add(m, 0, b"meshes", None, b"hull", -1, ctypes.byref(mesh)) == 0
        assert L.hb_add(m, 0, b"meshes", None, b"hull", -1, ctypes.byref(mesh)) == 1  # duplicate name
        assert L.hb_add(m, 0, b"lids", None, b"l", -1, ctypes.byref(mesh)) == 3
        v = np.zeros((2, 4, 2))
        s3 = (ctypes.c_size_t * 3)(2, 4, 2)
        rc, mid = _obj(L, m, "meshes/hull")
        assert rc == 0
        assert L.hb_set_reals(m, mid, b"vertices", v.ctypes.data_as(nv.dp), s3, 3) == 1  # wrong shape
        L.hb_set_text.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_char_p]
        assert L.hb_set_text(m, mid, b"symmetry", b"xz_and_yz") == 0
        assert L.hb_set_text(m, mid, b"symmetry", b"diagonal") == 1
        # null out-pointers are refused and change nothing
        assert L.hb_object(m, b"environment", None) == 7
        assert L.hb_model_new(None) == 7
        # a body item outside the route, and a model without a body
        rc, _ = _obj(L, m, "bodies/nothing")
        assert rc == 1
        L.hb_model_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        assert L.hb_model_solve(m, None, None, None) == 1
        assert b"no body" in L.hb_last_error_message()
    finally:
        assert L.hb_model_free(m) == 0


def test_results_quantity_refusals():
    L = nv.lib()
    col = nv.HbColumn()
    L.hb_results_quantity.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(nv.HbColumn)]
    assert L.hb_results_quantity(None, b"added_mass", ctypes.byref(col)) == 7


def test_batch_entry_refuses_null_arguments():
    L = nv.lib()
    opt = nv.default_options()
    assert L.hbg_solve_batch(None, 1, ctypes.byref(opt)) == 7
    p = nv.HbgProblem()
    assert L.hbg_solve_batch(ctypes.byref(p), 1, None) == 7
    assert L.hbg_solve_batch(ctypes.byref(p), 1, ctypes.byref(opt)) == 7  # null vertices


def test_no_gpu_means_a_loud_refusal_not_a_cpu_fallback():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from hydrobem_b200 import meshes

    with pytest.raises(nv.HydroBEMError) as e:
        nv.solve(meshes.cylinder(1.0, 0.5, 8, 2, 2), [1.0], [0.0])
    assert e.value.status == 3 and "GPU" in e.value.message
