"""The low-order GDF reader (crates/hydrobem/src/gdf.rs:200-535, text.rs:205-345) through the C ABI: the
header, Fortran list-directed records (commas as spaces, D exponents, comments after a line's numbers), the
trailing record of zeros, and the reference's error reports; then a mesh of the object model read from a
GDF file, solved against the reference's stored outputs (GPU).

The cases follow the reference's own reader tests (tests/python/test_readers.py: the zero trailer, D
exponents and commas); the files are written here from the meshes of this package.
"""
from __future__ import annotations

import ctypes
import math
from pathlib import Path

import numpy as np
import pytest

from hydrobem_b200 import meshes
from hydrobem_b200 import native as nv


def _fmt(values):
    return " ".join(repr(float(v)) for v in values)


def _write(path, q, header=("box", "1.0 9.80665", "1 1"), npan=None, extra=()):
    lines = list(header) + [f"{len(q) if npan is None else npan}"] + [_fmt(v) for v in q.reshape(-1, 3)] + list(extra)
    Path(path).write_text("\n".join(lines) + "\n")


def _error(path, **kw):
    with pytest.raises(nv.HydroBEMError) as e:
        nv.read_gdf(path, **kw)
    return e.value


def test_round_trip_is_bit_exact(tmp_path):
    q = meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True)
    _write(tmp_path / "c.gdf", q, header=("quarter cylinder", "1.0 9.80665", "1 1"))
    g = nv.read_gdf(tmp_path / "c.gdf")
    assert g["label"] == "quarter cylinder" and g["ulen"] == 1.0 and g["gravity"] == 9.80665
    assert (g["isx"], g["isy"]) == (1, 1)
    assert g["vertices"].tobytes() == np.ascontiguousarray(q, dtype=np.float64).tobytes()


def test_zero_trailer_is_accepted_when_asked(tmp_path):
    q = meshes.box(1.0, 0.5, 0.5, n=(2, 1, 1), quarter=True)
    _write(tmp_path / "plain.gdf", q)
    _write(tmp_path / "zeros.gdf", q, extra=["0 0 0 0 0 0 0 0 0 0 0 0"])
    e = _error(tmp_path / "zeros.gdf")
    assert e.status == 1 and f"trailing record of zeros after NPAN = {len(q)}" in e.message
    a, b = nv.read_gdf(tmp_path / "plain.gdf"), nv.read_gdf(tmp_path / "zeros.gdf", zero_trailer=True)
    assert a["vertices"].tobytes() == b["vertices"].tobytes()
    e = _error(tmp_path / "missing.gdf")
    assert e.status == 9 and "missing.gdf" in e.message  # HB_ERR_IO


def test_d_exponents_commas_and_comments(tmp_path):
    q = np.array([[[0.0, 0.0, -0.5], [1.0, 0.0, -0.5], [1.0, 1.0, -0.5], [0.0, 1.0, -0.5]],
                  [[1.0e-3, 2.5e+2, -1.0], [3.0, 4.0, -1.0], [3.0, 5.0, -1.0], [1.0e-3, 5.0, -1.0]]])
    rows = []
    for p in q:
        for k, v in enumerate(p):
            row = " , ".join(repr(float(x)).replace("e", "D") for x in v)
            rows.append(row + ("   end of panel" if k == 3 else ""))
    Path(tmp_path / "c.gdf").write_text("\n".join(["plate", "1.0D0 9.80665  ULEN GRAV", "0, 0", "2  NPAN"] + rows) + "\n")
    g = nv.read_gdf(tmp_path / "c.gdf")
    assert np.array_equal(g["vertices"], q) and (g["isx"], g["isy"]) == (0, 0)
    # panels over any number of lines, several per line
    flat = " ".join(repr(float(x)) for x in q.reshape(-1))
    Path(tmp_path / "d.gdf").write_text("\n".join(["plate", "1 9.81", "0 0", "2", flat]) + "\n")
    assert np.array_equal(nv.read_gdf(tmp_path / "d.gdf")["vertices"], q)


def test_malformed_files_are_reported(tmp_path):
    q = meshes.box(1.0, 0.5, 0.5, n=(2, 1, 1), quarter=True)
    cases = [
        (dict(header=("b", "1.0", "1 1")), "expected ULEN GRAV on the line '1.0'"),
        (dict(header=("b", "1.0 -9.8", "1 1")), "GRAV must be a positive finite number"),
        (dict(header=("b", "1.0 9.8", "2 0")), "ISX must be 0 or 1, not 2"),
        (dict(header=("b", "1.0 9.8", "0 0.5")), "ISY must be an integer, got 0.5"),
        (dict(npan=0), "NPAN must be >= 1"),
        (dict(npan=len(q) + 1), f"the file ends after {len(q)} of NPAN = {len(q) + 1} records"),
        (dict(extra=["1 2 3"]), f"unexpected data after NPAN = {len(q)}"),
        (dict(extra=["end 1 2 3"]), "invalid number 'end'"),
    ]
    for i, (kw, msg) in enumerate(cases):
        f = tmp_path / f"bad{i}.gdf"
        _write(f, q, **kw)
        e = _error(f)
        assert e.status == 1 and msg in e.message, (msg, e.message)
    Path(tmp_path / "short.gdf").write_text("b\n1 9.8\n0 0\n")
    assert "needs a header, ULEN GRAV, ISX ISY and NPAN lines" in _error(tmp_path / "short.gdf").message


def test_model_refuses_higher_order_files(tmp_path):
    L = nv.lib()
    m = ctypes.c_void_p()
    assert L.hb_model_new(ctypes.byref(m)) == 0
    try:
        q = meshes.box(1.0, 0.5, 0.5, n=(2, 1, 1), quarter=True)
        _write(tmp_path / "b.gdf", q)
        opts = (ctypes.c_int32 * 2)(1, 0)  # higher_order, zero_trailer
        out = ctypes.c_uint64()
        L.hb_model_load_mesh.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p,
                                         ctypes.POINTER(ctypes.c_uint64)]
        assert L.hb_model_load_mesh(m, b"hull", str(tmp_path / "b.gdf").encode(), None, ctypes.byref(out)) == 0
        assert L.hb_model_load_mesh(m, b"hull", str(tmp_path / "b.gdf").encode(), None, ctypes.byref(out)) == 1
        # a null-terminated options struct with higher_order set (the remaining fields zero)
        buf = ctypes.create_string_buffer(128)
        ctypes.memmove(buf, opts, 8)
        assert L.hb_model_load_mesh(m, b"h2", str(tmp_path / "b.gdf").encode(), buf, ctypes.byref(out)) == 3
    finally:
        L.hb_model_free(m)


@pytest.mark.gpu
def test_gpu_model_from_a_gdf_file(tmp_path):
    """The regression problem lo_cylinder_drift with its quarter mesh read from a GDF file (ISX = ISY = 1:
    the model solves it by symmetry sectors): the reference's stored A, B, X."""
    g = np.load(Path(__file__).resolve().parent / "golden" / "lo_cylinder_drift.npz")
    q = meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True)
    _write(tmp_path / "cyl.gdf", q, header=("cylinder r = 1, draught 0.5", "1.0 9.80665", "1 1"))
    L = nv.lib()
    m = ctypes.c_void_p()
    assert L.hb_model_new(ctypes.byref(m)) == 0
    try:
        mesh = ctypes.c_uint64()
        L.hb_model_load_mesh.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_void_p,
                                         ctypes.POINTER(ctypes.c_uint64)]
        assert L.hb_model_load_mesh(m, b"cyl", str(tmp_path / "cyl.gdf").encode(), None, ctypes.byref(mesh)) == 0
        L.hb_add.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                             ctypes.c_int64, ctypes.POINTER(ctypes.c_uint64)]
        L.hb_set_reals.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, nv.dp,
                                   ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t]
        L.hb_set_text.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_char_p]
        body = ctypes.c_uint64()
        assert L.hb_add(m, 0, b"bodies", None, b"body", -1, ctypes.byref(body)) == 0
        assert L.hb_set_text(m, body.value, b"mesh", b"cyl") == 0
        env = ctypes.c_uint64()
        assert L.hb_object(m, b"environment", ctypes.byref(env)) == 0
        for name, arr in ((b"omegas", g["omegas"]), (b"headings", g["headings"])):
            a = np.ascontiguousarray(arr, dtype=np.float64)
            assert L.hb_set_reals(m, env.value, name, a.ctypes.data_as(nv.dp), (ctypes.c_size_t * 1)(a.size), 1) == 0
        res = ctypes.c_void_p()
        L.hb_model_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        assert L.hb_model_solve(m, None, None, ctypes.byref(res)) == 0, L.hb_last_error_message()
        L.hb_results_quantity.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(nv.HbColumn)]
        col = nv.HbColumn()
        assert L.hb_results_quantity(res, b"added_mass_f64", ctypes.byref(col)) == 0
        A = np.ctypeslib.as_array(ctypes.cast(col.data, ctypes.POINTER(ctypes.c_double)), shape=(col.count,)).copy()
        L.hb_results_free(res)
    finally:
        L.hb_model_free(m)
    ref = g["added_mass"].astype(np.float64).reshape(-1)
    peak = np.abs(ref).max()
    assert np.abs(A - ref).max() <= 2e-5 * peak
