"""ctypes binding of libhydrobem_gpu.so (include/hydrobem_gpu.h).

Plain pointers and sizes cross the boundary; numpy arrays own the host memory.  The library runs
the whole path on the GPU and has no CPU fallback: without a CUDA device its solve entry returns
HB_ERR_UNSUPPORTED, which this module raises.
"""

from __future__ import annotations

import ctypes
import math
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libhydrobem_gpu.so"

HB_OK = 0
STATUS_NAMES = {1: "HB_ERR_VALUE", 2: "HB_ERR_TYPE", 3: "HB_ERR_UNSUPPORTED", 4: "HB_ERR_STATE",
                5: "HB_ERR_CANCELLED", 6: "HB_ERR_INTERNAL", 7: "HB_ERR_ARGUMENT", 8: "HB_ERR_NUMERICAL",
                9: "HB_ERR_IO", 10: "HB_ERR_EXISTS"}
HBG_FP64, HBG_MIXED = 0, 1
HBG_STATICS_ACCURATE, HBG_STATICS_PRODUCTION = 0, 1
HBG_WET, HBG_INTERIOR = 0, 1

dp = ctypes.POINTER(ctypes.c_double)
ip = ctypes.POINTER(ctypes.c_int32)


class HbgBody(ctypes.Structure):
    _fields_ = [("n_panels", ctypes.c_int64), ("vertices", dp), ("kinds", ip), ("panel_body", ip),
                ("n_bodies", ctypes.c_int32), ("rotation_centers", dp), ("symmetry", ctypes.c_int32)]


# HbgBody.symmetry: one sector's panels given, their mirror images added by the library
SYM_NONE, SYM_YZ, SYM_XZ, SYM_BOTH = 0, 1, 2, 3


class HbgOutputs(ctypes.Structure):
    _fields_ = [("added_mass", dp), ("radiation_damping", dp), ("excitation", dp), ("froude_krylov", dp),
                ("scattering", dp), ("motions", dp), ("hydrostatics", dp), ("field_radiation", dp),
                ("field_incident", dp), ("field_scattering", dp), ("field_diffraction", dp), ("haskind", dp),
                ("kochin_radiation", dp), ("kochin_radiation_derivative", dp), ("kochin_diffraction", dp),
                ("kochin_diffraction_derivative", dp), ("drift", dp)]


class HbgRigid(ctypes.Structure):
    _fields_ = [("mass", dp), ("center_of_gravity", dp), ("inertia_kind", ip), ("inertia", dp),
                ("inertia_origin", dp), ("stiffness", dp), ("damping", dp)]


class HbgProblem(ctypes.Structure):
    _fields_ = [("body", HbgBody), ("omegas", dp), ("n_omega", ctypes.c_int64), ("headings_deg", dp),
                ("n_heading", ctypes.c_int64), ("out", HbgOutputs), ("rigid", ctypes.POINTER(HbgRigid)),
                ("field_points", dp), ("n_field_points", ctypes.c_int64), ("kochin_angles", ctypes.c_int32)]


# HbgRigid.inertia_kind, and the record of HbgOutputs.hydrostatics (HBG_HS doubles per body)
INERTIA_COMPONENTS, INERTIA_GYRATION = 0, 1
HBG_HS = 83


def hydrostatics_record(h):
    """The fields of one body's hydrostatics record (global frame)."""
    h = np.asarray(h, dtype=np.float64)
    return {"volumes": h[0:3], "center_of_buoyancy": h[3:6], "waterplane_area": h[6],
            "waterplane_centroid": h[7:9], "stiffness_rho_g": h[9:45].reshape(6, 6),
            "stiffness": h[45:81].reshape(6, 6), "mass": h[81], "displaced_mass": h[82]}


class HbgOptions(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("logarithmic", ctypes.c_int32), ("log_tolerance", ctypes.c_double),
                ("gravity", ctypes.c_double), ("density", ctypes.c_double), ("depth", ctypes.c_double),
                ("max_batch", ctypes.c_int32), ("device", ctypes.c_int32), ("cancel", ip),
                ("surrogate", ctypes.POINTER(ctypes.c_float)), ("statics_rule", ctypes.c_int32),
                ("concurrency", ctypes.c_int32)]


class HbLocation(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("body", "mesh", "element", "field_point", "lid", "frequency")]


class HbColumn(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("dtype", ctypes.c_int32), ("ndim", ctypes.c_size_t),
                ("shape", ctypes.POINTER(ctypes.c_size_t)), ("count", ctypes.c_size_t), ("data", ctypes.c_void_p)]


# every symbol include/hydrobem_gpu.h declares
EXPORTS = ["hbg_default_options", "hbg_solve_batch", "hbg_debug_matrices", "hbg_debug_gemm_tf32",
           "hbg_last_ir_iterations", "hbg_last_profile", "hbg_last_launch_count",
           "hbg_profile_kernels", "hbg_kernel_profile", "hbg_release_workspace", "hb_abi_version",
           "hbg_library_version",
           "hb_last_error_message", "hb_last_error_location", "hb_model_new", "hb_model_free", "hb_model_cancel",
           "hb_object", "hb_add", "hb_set_bool", "hb_set_int", "hb_set_real", "hb_set_text", "hb_set_reals",
           "hb_set_ints", "hb_model_solve", "hb_results_free", "hb_results_has", "hb_results_quantity",
           "hbg_statics_noalloc", "hbg_measure_peaks", "hbg_last_ir_history", "hbg_surrogate_train",
           "hbg_surrogate_grad", "hbg_surrogate_eval", "hbg_last_surrogate_pairs", "hbg_read_gdf", "hbg_gdf_free",
           "hb_model_load_mesh", "hbg_last_fallback_count", "hbg_debug_lu_f64", "hb_model_panels", "hbg_tuned_tiles", "hbg_last_fallback_time"]

_lib = None


class HydroBEMError(RuntimeError):
    def __init__(self, status, message, location=None):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message
        self.location = location


def lib():
    """The loaded library (built on first use when absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        from . import build as _b

        _b.build()
    L = ctypes.CDLL(str(LIB_PATH))
    L.hbg_default_options.argtypes = [ctypes.POINTER(HbgOptions)]
    L.hbg_default_options.restype = None
    L.hbg_solve_batch.argtypes = [ctypes.POINTER(HbgProblem), ctypes.c_int64, ctypes.POINTER(HbgOptions)]
    L.hbg_solve_batch.restype = ctypes.c_int32
    L.hbg_debug_matrices.argtypes = [ctypes.POINTER(HbgBody), ctypes.c_double, ctypes.POINTER(HbgOptions), dp, dp, dp]
    L.hbg_debug_matrices.restype = ctypes.c_int32
    fp = ctypes.POINTER(ctypes.c_float)
    L.hbg_debug_gemm_tf32.argtypes = [ctypes.c_int32] * 3 + [fp, fp, fp, ctypes.c_int32]
    L.hbg_last_ir_iterations.argtypes = [ctypes.POINTER(ctypes.c_int32)]
    L.hbg_debug_lu_f64.argtypes = [ctypes.c_int32, ctypes.c_int32, dp, ctypes.c_int32, dp, dp]
    L.hbg_debug_lu_f64.restype = ctypes.c_int32
    L.hbg_measure_peaks.argtypes = [dp]
    L.hbg_last_ir_history.argtypes = [dp, ctypes.POINTER(ctypes.c_int32)]
    L.hbg_surrogate_train.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                      ctypes.c_uint64, ctypes.c_int64, fp, fp, dp]
    L.hbg_surrogate_grad.argtypes = [fp, ctypes.c_int32, fp, fp, fp, dp]
    L.hbg_surrogate_eval.argtypes = [fp, fp, ctypes.c_int32, dp, dp, dp, dp]
    L.hbg_last_surrogate_pairs.argtypes = [ctypes.POINTER(ctypes.c_int64)]
    L.hbg_statics_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
                                      ctypes.c_int32, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    L.hbg_statics_noalloc.restype = ctypes.c_int32
    L.hbg_last_profile.argtypes = [dp]
    L.hbg_profile_kernels.argtypes = [ctypes.c_int32]
    L.hbg_kernel_profile.argtypes = [ctypes.c_int32, dp, ctypes.POINTER(ctypes.c_int64), dp]
    L.hbg_last_launch_count.argtypes = [ctypes.POINTER(ctypes.c_int64)]
    L.hb_last_error_message.restype = ctypes.c_char_p
    L.hb_last_error_location.argtypes = [ctypes.POINTER(HbLocation)]
    L.hb_abi_version.restype = ctypes.c_uint32
    L.hbg_library_version.restype = ctypes.c_uint32
    _lib = L
    return L


def check(status):
    if status != HB_OK:
        L = lib()
        loc = HbLocation()
        L.hb_last_error_location(ctypes.byref(loc))
        raise HydroBEMError(status, L.hb_last_error_message().decode(errors="replace"),
                            {f: getattr(loc, f) for f, _ in HbLocation._fields_})


def default_options(**kw) -> HbgOptions:
    o = HbgOptions()
    lib().hbg_default_options(ctypes.byref(o))
    for k, v in kw.items():
        if k == "depth" and (v is None or not np.isfinite(v)):
            v = float("inf")
        if k == "surrogate":
            if v is None:
                continue
            o._surrogate_keep = np.ascontiguousarray(v, np.float32)  # alive as long as the options
            v = o._surrogate_keep.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        setattr(o, k, v)
    return o


class Body:
    """The inputs and output arrays of one problem of a batch (kept alive across the call): the panels of
    one rigid body, or of interacting bodies with panel_body (the body of each panel) and
    rotation_centers [n_bodies][3] (None: the origin); 6 rigid modes per body, D = 6 n_bodies.  With
    symmetry (SYM_YZ, SYM_XZ, SYM_BOTH) the panels are one sector of a body mirrored in those planes.
    rigid: the mass properties for the motions, a dict of mass [n_bodies] (NaN: displaced),
    center_of_gravity [n_bodies][3], inertia [n_bodies][3][3] about inertia_origin [n_bodies][3],
    inertia_kind [n_bodies] (INERTIA_COMPONENTS / INERTIA_GYRATION), optional stiffness, damping [D][D].
    points: field points [P][3] (global, z <= 0) for the elevation or p / (rho g) there."""

    def __init__(self, vertices, omegas, headings_deg=(), kinds=None, panel_body=None, rotation_centers=None,
                 symmetry=SYM_NONE, rigid=None, points=None, kochin_angles=0, motions=None):
        self.symmetry = int(symmetry)
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 4, 3)
        self.kinds = None if kinds is None else np.ascontiguousarray(kinds, dtype=np.int32)
        self.panel_body = None if panel_body is None else np.ascontiguousarray(panel_body, dtype=np.int32)
        self.n_bodies = 1 if self.panel_body is None else int(self.panel_body.max()) + 1
        self.centers = None if rotation_centers is None else \
            np.ascontiguousarray(rotation_centers, dtype=np.float64).reshape(-1, 3)
        if self.centers is not None:
            self.n_bodies = max(self.n_bodies, self.centers.shape[0])
        self.omegas = np.ascontiguousarray(omegas, dtype=np.float64).reshape(-1)
        self.headings = np.ascontiguousarray(headings_deg, dtype=np.float64).reshape(-1)
        F, H, D = self.omegas.size, self.headings.size, 6 * self.n_bodies
        self.A = np.zeros((F, D, D))
        self.B = np.zeros((F, D, D))
        self.X = np.zeros((F, H, D), dtype=np.complex128)
        self.FK = np.zeros((F, H, D), dtype=np.complex128)
        self.SC = np.zeros((F, H, D), dtype=np.complex128)
        self.HK = np.zeros((F, H, D), dtype=np.complex128)
        T = int(kochin_angles) if H else 0
        self.kochin_angles = T
        self.KR = np.zeros((F, T, D), dtype=np.complex128)
        self.KRT = np.zeros((F, T, D), dtype=np.complex128)
        self.KD = np.zeros((F, T, H), dtype=np.complex128)
        self.KDT = np.zeros((F, T, H), dtype=np.complex128)
        self.DRIFT = np.zeros((F, H, H, 3), dtype=np.complex128)
        self.HS = np.zeros((self.n_bodies, HBG_HS))
        self.points = None if points is None else np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        P = 0 if self.points is None else self.points.shape[0]
        self.FR = np.zeros((F, P, D), dtype=np.complex128)
        self.FI = np.zeros((F, P, H), dtype=np.complex128)
        self.FS = np.zeros((F, P, H), dtype=np.complex128)
        self.FD = np.zeros((F, P, H), dtype=np.complex128)
        # the motions when rigid data are given (motions=False leaves them out: then a drift is that of the
        # fixed body)
        want_mo = rigid is not None if motions is None else bool(motions)
        self.MO = np.zeros((F, H, D), dtype=np.complex128) if want_mo else None
        self._rigid = None
        if rigid is not None:
            nb = self.n_bodies
            arr = lambda k, shape: np.ascontiguousarray(np.broadcast_to(np.asarray(rigid[k], dtype=np.float64), shape))
            self._rig_keep = {
                "mass": arr("mass", (nb,)), "cg": arr("center_of_gravity", (nb, 3)),
                "kind": np.ascontiguousarray(np.broadcast_to(np.asarray(rigid.get("inertia_kind", 0), np.int32), (nb,))),
                "inertia": arr("inertia", (nb, 3, 3)), "origin": arr("inertia_origin", (nb, 3)),
                "stiffness": None if rigid.get("stiffness") is None else arr("stiffness", (D, D)),
                "damping": None if rigid.get("damping") is None else arr("damping", (D, D))}
            k = self._rig_keep
            self._rigid = HbgRigid(k["mass"].ctypes.data_as(dp), k["cg"].ctypes.data_as(dp), k["kind"].ctypes.data_as(ip),
                                   k["inertia"].ctypes.data_as(dp), k["origin"].ctypes.data_as(dp),
                                   None if k["stiffness"] is None else k["stiffness"].ctypes.data_as(dp),
                                   None if k["damping"] is None else k["damping"].ctypes.data_as(dp))

    def problem(self) -> HbgProblem:
        p = HbgProblem()
        p.body.n_panels = self.vertices.shape[0]
        p.body.vertices = self.vertices.ctypes.data_as(dp)
        p.body.kinds = None if self.kinds is None else self.kinds.ctypes.data_as(ip)
        p.body.panel_body = None if self.panel_body is None else self.panel_body.ctypes.data_as(ip)
        p.body.n_bodies = self.n_bodies
        p.body.rotation_centers = None if self.centers is None else self.centers.ctypes.data_as(dp)
        p.body.symmetry = self.symmetry
        p.omegas = self.omegas.ctypes.data_as(dp)
        p.n_omega = self.omegas.size
        p.headings_deg = self.headings.ctypes.data_as(dp)
        p.n_heading = self.headings.size
        p.out.added_mass = self.A.ctypes.data_as(dp)
        p.out.radiation_damping = self.B.ctypes.data_as(dp)
        p.out.excitation = self.X.ctypes.data_as(dp)
        p.out.froude_krylov = self.FK.ctypes.data_as(dp)
        p.out.scattering = self.SC.ctypes.data_as(dp)
        p.out.haskind = self.HK.ctypes.data_as(dp)
        if self.kochin_angles:
            p.kochin_angles = self.kochin_angles
            p.out.kochin_radiation = self.KR.ctypes.data_as(dp)
            p.out.kochin_radiation_derivative = self.KRT.ctypes.data_as(dp)
            p.out.kochin_diffraction = self.KD.ctypes.data_as(dp)
            p.out.kochin_diffraction_derivative = self.KDT.ctypes.data_as(dp)
            p.out.drift = self.DRIFT.ctypes.data_as(dp)
        p.out.motions = None if self.MO is None else self.MO.ctypes.data_as(dp)
        p.out.hydrostatics = self.HS.ctypes.data_as(dp)
        p.rigid = None if self._rigid is None else ctypes.pointer(self._rigid)
        if self.points is not None and self.points.shape[0]:
            p.field_points = self.points.ctypes.data_as(dp)
            p.n_field_points = self.points.shape[0]
            p.out.field_radiation = self.FR.ctypes.data_as(dp)
            p.out.field_incident = self.FI.ctypes.data_as(dp)
            p.out.field_scattering = self.FS.ctypes.data_as(dp)
            p.out.field_diffraction = self.FD.ctypes.data_as(dp)
        return p

    def results(self):
        out = {"A": self.A, "B": self.B, "X": self.X, "FK": self.FK, "SC": self.SC, "HK": self.HK,
               "hydrostatics": [hydrostatics_record(h) for h in self.HS]}
        if self.MO is not None:
            out["motions"] = self.MO
        if self.kochin_angles:
            out.update({"kr": self.KR, "krt": self.KRT, "kd": self.KD, "kdt": self.KDT, "drift": self.DRIFT,
                        "kochin_angles": 2.0 * np.pi * np.arange(self.kochin_angles) / self.kochin_angles})
        if self.points is not None:
            out.update({"field_radiation": self.FR, "field_incident": self.FI, "field_scattering": self.FS,
                        "field_diffraction": self.FD})
        return out


class HbgGdf(ctypes.Structure):
    _fields_ = [("label", ctypes.c_char * 256), ("ulen", ctypes.c_double), ("gravity", ctypes.c_double),
                ("isx", ctypes.c_int32), ("isy", ctypes.c_int32), ("n_panels", ctypes.c_int64), ("vertices", dp)]


def read_gdf(path, zero_trailer=False):
    """A low-order GDF file through hbg_read_gdf: dict of label, ulen, gravity, isx, isy and vertices [P][4][3]."""
    g = HbgGdf()
    L = lib()
    check(L.hbg_read_gdf(str(path).encode(), int(bool(zero_trailer)), ctypes.byref(g)))
    try:
        v = np.ctypeslib.as_array(g.vertices, shape=(g.n_panels * 12,)).copy().reshape(-1, 4, 3)
    finally:
        L.hbg_gdf_free(ctypes.byref(g))
    return {"label": g.label.decode(), "ulen": g.ulen, "gravity": g.gravity, "isx": g.isx, "isy": g.isy, "vertices": v}


def solve_batch(bodies, **options):
    """Solve a list of Body on the GPU through hbg_solve_batch; returns the list of result dicts."""
    arr = (HbgProblem * len(bodies))(*[b.problem() for b in bodies])
    opt = default_options(**options)
    check(lib().hbg_solve_batch(arr, len(bodies), ctypes.byref(opt)))
    return [b.results() for b in bodies]


def solve(vertices, omegas, headings_deg=(), kinds=None, panel_body=None, rotation_centers=None,
          symmetry=SYM_NONE, rigid=None, points=None, kochin_angles=0, **options):
    """One problem through the GPU path: dict of A, B [F][D][D], X, FK, SC [F][H][D], D = 6 per body, the
    hydrostatics records of the bodies, with rigid the motions [F][H][D], with points the field values
    field_radiation [F][P][D] and field_incident, field_scattering, field_diffraction [F][P][H]; with
    kochin_angles = T > 0 the Kochin functions kr, krt [F][T][D], kd, kdt [F][T][H] and the momentum drift
    [F][H][H][3] (the motions included with rigid)."""
    return solve_batch([Body(vertices, omegas, headings_deg, kinds, panel_body, rotation_centers, symmetry, rigid,
                             points, kochin_angles)], **options)[0]


def last_profile():
    v = (ctypes.c_double * 6)()
    lib().hbg_last_profile(v)
    return dict(zip(("statics", "assembly", "lu", "substitution", "forces", "total"), list(v)))


def last_fallback_count() -> int:
    """Frequencies of the last solve that the mixed form handed to the FP64 form."""
    c = ctypes.c_int64()
    lib().hbg_last_fallback_count(ctypes.byref(c))
    return c.value


def last_fallback_time() -> float:
    """Device milliseconds of the FP64 solves of those frequencies in the last solve."""
    v = ctypes.c_double()
    lib().hbg_last_fallback_time(ctypes.byref(v))
    return v.value


def last_launch_count() -> int:
    c = ctypes.c_int64()
    lib().hbg_last_launch_count(ctypes.byref(c))
    return c.value


def debug_matrices(vertices, omega, kinds=None, symmetry=SYM_NONE, **options):
    """(statics [N][N][4] with entry [k][j], S, A complex128 [N][N] with entry [k][n]) of one
    body at one frequency, FP64 form (test support).  With symmetry (G sectors of the n given panels):
    statics [n][G n][4] (the sector rows against every panel) and S, A [G][n][n] (the sector matrices)."""
    v = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 4, 3)
    k = None if kinds is None else np.ascontiguousarray(kinds, dtype=np.int32)
    n = v.shape[0]
    G = {SYM_NONE: 1, SYM_YZ: 2, SYM_XZ: 2, SYM_BOTH: 4}.get(int(symmetry), 1)
    body = HbgBody(n, v.ctypes.data_as(dp), None if k is None else k.ctypes.data_as(ip))
    body.symmetry = int(symmetry)
    st = np.zeros((4, G * n, n))   # plane, j, k  (entry (k, j) at k + j n)
    S = np.zeros((G, n, n), dtype=np.complex128)   # [c][n][k] (column-major)
    A = np.zeros((G, n, n), dtype=np.complex128)
    opt = default_options(**options)
    check(lib().hbg_debug_matrices(ctypes.byref(body), omega, ctypes.byref(opt), st.ctypes.data_as(dp),
                                   S.ctypes.data_as(dp), A.ctypes.data_as(dp)))
    if G == 1:
        return st.transpose(2, 1, 0), S[0].T, A[0].T
    return st.transpose(2, 1, 0), S.transpose(0, 2, 1), A.transpose(0, 2, 1)


KERNEL_FAMILIES = ["geometry", "statics", "statics_adaptive", "fd_tiles", "assemble", "boundary", "rhs", "lu_panel",
                   "lu_laswp", "lu_trsm", "lu_gemm", "lu_solve", "forces", "mixed_convert", "mixed_gemm",
                   "mixed_residual"]
FLOP_FAMILIES = {"lu_panel", "lu_trsm", "lu_gemm", "mixed_gemm"}


def profile_kernels(on: bool) -> None:
    lib().hbg_profile_kernels(1 if on else 0)


def kernel_profile():
    """{family: (ms, launches, work)} of the last solve of this thread."""
    out = {}
    for i, name in enumerate(KERNEL_FAMILIES):
        ms, n, w = ctypes.c_double(), ctypes.c_int64(), ctypes.c_double()
        lib().hbg_kernel_profile(i, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(w))
        out[name] = (ms.value, n.value, w.value)
    return out


def debug_lu_f64(A, B):
    """X = A^-1 B by the FP64 form's LU on the GPU: A [batch][n][n], B [batch][n][nrhs] complex."""
    A = np.asarray(A, dtype=np.complex128)
    B = np.asarray(B, dtype=np.complex128)
    batch, n, _ = A.shape
    nrhs = B.shape[2]
    Ac = np.ascontiguousarray(A.transpose(0, 2, 1))  # column-major per matrix
    Bc = np.ascontiguousarray(B.transpose(0, 2, 1))  # [batch][nrhs][n]
    X = np.zeros_like(Bc)
    check(lib().hbg_debug_lu_f64(n, batch, Ac.ctypes.data_as(dp), nrhs, Bc.ctypes.data_as(dp), X.ctypes.data_as(dp)))
    return X.transpose(0, 2, 1)


def debug_gemm_tf32(A, B, C=None):
    """C = A B^T, or C - A B^T when C is given, through the tcgen05 TF32 kernel (test support);
    A [M][K], B [N][K], C [M][N] float32."""
    A = np.ascontiguousarray(A, dtype=np.float32)
    B = np.ascontiguousarray(B, dtype=np.float32)
    M, K = A.shape
    N = B.shape[0]
    sub = C is not None
    C = np.array(C, dtype=np.float32, order="C", copy=True) if sub else np.zeros((M, N), dtype=np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    check(lib().hbg_debug_gemm_tf32(M, N, K, A.ctypes.data_as(fp), B.ctypes.data_as(fp), C.ctypes.data_as(fp),
                                    int(sub)))
    return C


def statics_noalloc(d_vertices: int, d_kinds: int | None, n_panels: int, d_statics: int, depth: float = math.inf,
                    logarithmic: bool = True, log_tolerance: float = 1e-4, stream: int | None = None) -> None:
    """The statics of a panel set into caller-owned device memory, with no device allocation by the
    library (its scratch is a fixed array for at most 2048 panels).  Arguments are raw device
    addresses on the current device: vertices [N][4][3] FP64, kinds [N] int32 or None, statics
    [4][N][N] FP64 with entry (k, j) of plane q at q N^2 + k + j N."""
    check(lib().hbg_statics_noalloc(d_vertices, d_kinds, n_panels, depth, 1 if logarithmic else 0, log_tolerance,
                                    d_statics, stream))


def measure_peaks() -> dict:
    """Measured dense peaks of the current device in TFLOP/s: fp64_fma, fp64_mma, tf32_tcgen05."""
    out = np.zeros(3)
    check(lib().hbg_measure_peaks(out.ctypes.data_as(dp)))
    return {"fp64_fma": float(out[0]), "fp64_mma": float(out[1]), "tf32_tcgen05": float(out[2])}


def tuned_tiles(device: int = 0) -> dict:
    """The FP64 products' tile widths the library's tuner chose on a device: state (0 not tuned yet, 1
    default, 2 measured), and per width bucket (n <= 8, 16, ..., 2048, 4096) the choice (64 or 32 columns)
    and the two timings in microseconds."""
    state = ctypes.c_int32()
    wide = np.zeros(10, np.int32)
    us = np.zeros(20, np.float32)
    check(lib().hbg_tuned_tiles(device, ctypes.byref(state), wide.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                us.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
    widths = [8 << b for b in range(10)]
    return {"state": state.value, "columns": {w: (64 if x else 32) for w, x in zip(widths, wide)},
            "us": {w: (float(us[2 * b]), float(us[2 * b + 1])) for b, w in enumerate(widths)}}


def last_ir_history() -> list:
    """Largest relative correction per refinement iteration of the last mixed-precision batch."""
    out = np.zeros(32)
    n = ctypes.c_int32()
    check(lib().hbg_last_ir_history(out.ctypes.data_as(dp), ctypes.byref(n)))
    return [float(v) for v in out[: n.value]]


SURROGATE_PARAMS = 50822
SURROGATE_OUTPUTS = ["g", "g_X", "g_Y", "I", "I_X", "I_Y"]


def surrogate_train(n_train=1 << 22, batch=8192, steps=3000, lr=2e-3, seed=1, n_val=1 << 16):
    """Train the wave-term surrogate on the current device; returns (params, norm, report dict)."""
    p = np.zeros(SURROGATE_PARAMS, np.float32)
    nm = np.zeros(12, np.float32)
    rep = np.zeros(15)
    fpp = ctypes.POINTER(ctypes.c_float)
    check(lib().hbg_surrogate_train(n_train, batch, steps, lr, seed, n_val, p.ctypes.data_as(fpp),
                                    nm.ctypes.data_as(fpp), rep.ctypes.data_as(dp)))
    report = {"loss_first": rep[0], "loss_last": rep[1], "train_ms": rep[2],
              "val_rms_over_spread": dict(zip(SURROGATE_OUTPUTS, rep[3:9].tolist())),
              "val_max_over_max": dict(zip(SURROGATE_OUTPUTS, rep[9:15].tolist()))}
    return p, nm, report


def surrogate_grad(params, inputs, targets):
    """(loss, grads) of the training loss from the device training kernels (test support)."""
    fpp = ctypes.POINTER(ctypes.c_float)
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(inputs, np.float32)
    t = np.ascontiguousarray(targets, np.float32)
    g = np.zeros(SURROGATE_PARAMS, np.float32)
    loss = ctypes.c_double()
    check(lib().hbg_surrogate_grad(p.ctypes.data_as(fpp), len(x), x.ctypes.data_as(fpp), t.ctypes.data_as(fpp),
                                   g.ctypes.data_as(fpp), ctypes.byref(loss)))
    return loss.value, g


def surrogate_eval(params, norm, xy):
    """(network [n][6], table [n][6], (ms network, ms table)) at points xy [n][2] in [0, 100) x [0, 50)."""
    fpp = ctypes.POINTER(ctypes.c_float)
    p = np.ascontiguousarray(params, np.float32)
    nm = np.ascontiguousarray(norm, np.float32)
    x = np.ascontiguousarray(xy, np.float64)
    n = len(x)
    on = np.zeros((n, 6))
    ot = np.zeros((n, 6))
    ms = np.zeros(2)
    check(lib().hbg_surrogate_eval(p.ctypes.data_as(fpp), nm.ctypes.data_as(fpp), n, x.ctypes.data_as(dp),
                                   on.ctypes.data_as(dp), ot.ctypes.data_as(dp), ms.ctypes.data_as(dp)))
    return on, ot, (float(ms[0]), float(ms[1]))


def last_surrogate_pairs() -> int:
    """Pairs whose wave term came from the network in the last mixed solve with a surrogate."""
    n = ctypes.c_int64()
    check(lib().hbg_last_surrogate_pairs(ctypes.byref(n)))
    return n.value


def surrogate_blob(params, norm):
    """The HbgOptions.surrogate array: parameters then the outputs' means and spreads (float32)."""
    return np.ascontiguousarray(np.concatenate([np.asarray(params, np.float32), np.asarray(norm, np.float32)]))


def last_ir_iterations() -> int:
    n = ctypes.c_int32()
    lib().hbg_last_ir_iterations(ctypes.byref(n))
    return n.value


_HB_DTYPES = {1: np.float64, 2: np.float32, 3: np.int32, 4: np.int64, 5: np.uint64, 6: np.complex64, 7: np.complex128}


class Model:
    """The reference's object model through the C ABI: hb_model_new, hb_object, hb_add, hb_set_*,
    hb_model_solve (crates/hydrobem-c/include/hydrobem.h:507-814).  Items are set by object path
    ("" the model, "environment", "options", "meshes/<name>", "bodies/<name>"); every call checks its
    status and raises HydroBEMError with the library's message."""

    def __init__(self):
        self.L = L = lib()
        L.hb_add.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                             ctypes.c_int64, ctypes.POINTER(ctypes.c_uint64)]
        L.hb_object.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64)]
        L.hb_set_reals.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, dp,
                                   ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t]
        L.hb_set_ints.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64),
                                  ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t]
        L.hb_set_text.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_char_p]
        L.hb_set_real.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_double]
        L.hb_set_int.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_int64]
        L.hb_set_bool.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_int32]
        L.hb_model_solve.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
        L.hb_model_free.argtypes = [ctypes.c_void_p]
        L.hb_results_quantity.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(HbColumn)]
        L.hb_results_free.argtypes = [ctypes.c_void_p]
        L.hb_model_panels.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]
        self.m = ctypes.c_void_p()
        check(L.hb_model_new(ctypes.byref(self.m)))

    def close(self):
        if self.m:
            self.L.hb_model_free(self.m)
            self.m = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def obj(self, path: str) -> int:
        o = ctypes.c_uint64()
        check(self.L.hb_object(self.m, path.encode(), ctypes.byref(o)))
        return o.value

    def add(self, lst: str, name: str, parent: str = "") -> int:
        o = ctypes.c_uint64()
        check(self.L.hb_add(self.m, self.obj(parent), lst.encode(), None, name.encode(), -1, ctypes.byref(o)))
        return o.value

    def reals(self, path: str, item: str, values):
        a = np.ascontiguousarray(values, dtype=np.float64)
        shape = (ctypes.c_size_t * max(a.ndim, 1))(*(a.shape or (1,)))
        check(self.L.hb_set_reals(self.m, self.obj(path), item.encode(), a.ctypes.data_as(dp), shape, a.ndim))

    def real(self, path: str, item: str, value: float):
        check(self.L.hb_set_real(self.m, self.obj(path), item.encode(), float(value)))

    def text(self, path: str, item: str, value: str):
        check(self.L.hb_set_text(self.m, self.obj(path), item.encode(), value.encode()))

    def boolean(self, path: str, item: str, value: bool):
        check(self.L.hb_set_bool(self.m, self.obj(path), item.encode(), int(bool(value))))

    def panels(self, role: str | None = None, include_reflections: bool = False) -> dict:
        """hb_model_panels (host work, no device): vertices [P][4][3], body [P], kind [P] of the roles
        ("wetted", "lid", comma separated; None both), stored symmetric form unless include_reflections."""
        r = ctypes.c_void_p()
        check(self.L.hb_model_panels(self.m, None if role is None else role.encode(), int(bool(include_reflections)),
                                     ctypes.byref(r)))
        res = Results(self.L, r)
        try:
            return {k: res.quantity(k) for k in ("vertices", "body", "kind")}
        finally:
            res.free()

    def solve(self) -> "Results":
        r = ctypes.c_void_p()
        check(self.L.hb_model_solve(self.m, None, None, ctypes.byref(r)))
        return Results(self.L, r)


class Results:
    """hb_results_quantity views copied into numpy arrays of the column's element type."""

    def __init__(self, L, handle):
        self.L, self.r = L, handle

    def quantity(self, name: str) -> np.ndarray:
        col = HbColumn()
        check(self.L.hb_results_quantity(self.r, name.encode(), ctypes.byref(col)))
        dt = np.dtype(_HB_DTYPES[col.dtype])
        shape = tuple(col.shape[i] for i in range(col.ndim))
        buf = (ctypes.c_char * (col.count * dt.itemsize)).from_address(col.data)
        return np.frombuffer(buf, dtype=dt).copy().reshape(shape)

    def free(self):
        if self.r:
            self.L.hb_results_free(self.r)
            self.r = ctypes.c_void_p()
