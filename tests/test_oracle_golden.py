"""Pin the CPU oracle against the reference's own golden vectors and solver outputs.

The oracle (oracle/hb_oracle.c + oracle/oracle.py) is the checker of every GPU parity test, so it
is itself checked here, with the error measures and targets of the reference's tests:

- wave kernel vs mpmath  (crates/hydrobem/tests/core.rs:119-150: 2e-6 of max(|v|, local scale))
- finite-depth kernel    (core.rs:152-195: 2e-6 of max(|v|, scale))
- dispersion roots       (core.rs:387-407: 2 ulp)
- panel integrals        (crates/hydrobem/tests/lo_a.rs:48-86: 1e-6)
- whole solve vs the reference's own outputs of the regression problem lo_cylinder_drift
  (tests/python/test_regression.py:34-78 compares at 1e-5 of each entry's max over the first
  axis, floor 1e-3 of the peak; the reference's production f32 path is within 1e-5 of its double
  path, tests/python/test_double_precision_mode.py:48-55)
"""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

from hydrobem_b200 import meshes
from oracle import oracle as O

G = Path(__file__).resolve().parent / "golden"


def bessel_j_ref(n, x):
    """J_n by the trapezoidal rule of its integral (core.rs:100-109), exact for these x."""
    m = int(x) + 64
    h = math.pi / m
    t = np.arange(1, m) * h
    return (0.5 * (1.0 + math.cos(n * math.pi)) + np.cos(n * t - x * np.sin(t)).sum()) / m


def test_wave_kernel_golden():
    d = np.load(G / "green_inf.npz")["xyff"]
    worst_f = worst_x = worst_i = 0.0
    for X, Y, F, FX in d:
        w = O.wave_kernel(X, Y)
        R0 = math.hypot(X, Y)
        scale = 2.0 * math.exp(-Y) * abs(math.log(Y + R0)) + 1.0 / R0
        scale_x = 2.0 * math.exp(-Y) / R0 + 1.0 / (R0 * R0)
        worst_f = max(worst_f, abs(w[0] - F) / max(abs(F), scale))
        worst_x = max(worst_x, abs(w[1] - FX) / max(abs(FX), scale_x))
        s = 2.0 * math.pi * math.exp(-Y)
        worst_i = max(worst_i, abs(w[3] + s * bessel_j_ref(0, X)) / s, abs(w[4] - s * bessel_j_ref(1, X)) / s)
    assert len(d) > 1000
    assert worst_f <= 2e-6 and worst_x <= 2e-6, (worst_f, worst_x)
    assert worst_i <= 1e-7, worst_i


def test_finite_kernel_golden():
    g = np.load(G / "green_fin.npz")
    modes, vals = g["mode"], g["vals"]
    worst = np.zeros(4)
    for mode, v in zip(modes, vals):
        h, K, R, z, ze = v[:5]
        ref = v[5:13]
        scale, scale_d = v[13], v[14]
        got = O.finite_kernel(h, K, int(mode), R, z, ze)
        for i in range(8):
            grp = (0 if i < 4 else 2) + (0 if i % 4 == 0 else 1)
            e = abs(got[i] - ref[i]) / max(abs(ref[i]), scale_d if grp % 2 else scale)
            worst[grp] = max(worst[grp], e)
    assert len(vals) > 1500
    assert worst.max() <= 2e-6, worst


def test_dispersion_golden():
    d = np.load(G / "dispersion.npz")
    worst = 0.0
    for H, n, x in zip(d["H"], d["n"], d["x"]):
        got = O.dispersion_x0(H) if n == 0 else O.dispersion_xn(H, int(n))
        ulp = np.nextafter(x, np.inf) - x
        worst = max(worst, abs(got - x) / ulp)
    assert len(d["x"]) > 2000
    assert worst <= 2.0, worst
    assert O.dispersion_x0(0.0) == 0.0 and O.dispersion_xn(math.inf, 3) == 2.5 * math.pi


def test_panel_integrals_golden():
    d = np.load(G / "panel.npz")
    worst_r = worst_l = 0.0
    for kind, v in zip(d["kind"], d["vals"]):
        verts = v[:12]
        p = np.array(v[12:15])
        a, b = v[15], v[16]
        pan = O.make_panels(verts.reshape(1, 4, 3))[0]
        c = np.array(list(pan.c))
        dist = np.linalg.norm(p - c)
        if kind == "R":
            S, D = O.rankine(pan, p)
            sS = pan.area / (dist + pan.radius)
            sD = pan.area / (dist * dist + pan.radius * pan.radius)
            worst_r = max(worst_r, abs(S - a) / max(abs(a), sS), abs(D - b) / max(abs(b), sD))
        else:
            L, Ld = O.log_singularity(pan, p)
            sL = pan.area * (abs(math.log(dist + pan.radius)) + 1.0)
            sD = pan.area / (dist + pan.radius)
            worst_l = max(worst_l, abs(L - a) / max(abs(a), sL), abs(Ld - b) / max(abs(b), sD))
    assert worst_r <= 1e-6 and worst_l <= 1e-6, (worst_r, worst_l)


def test_meshes_match_reference():
    import hashlib

    g = np.load(G / "meshes.npz")
    cases = {
        "c1": meshes.cylinder(1.0, 0.5, 32, 8, 8),
        "c2": meshes.cylinder(1.0, 0.5, 64, 32, 32),
        "drift_quarter": meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True),
        "hemi": meshes.hemisphere(1.0, 8, 8, quarter=True),
        "box_lid": meshes.box(80.0, 20.0, 10.0, n=(8, 4, 3), lid=True),
    }
    for k, v in cases.items():
        v = np.ascontiguousarray(v, dtype="<f8")
        assert tuple(g[k + "_shape"]) == v.shape, k
        assert hashlib.sha256(v.tobytes()).hexdigest() == str(g[k + "_sha256"]), k


def regression_error(got, ref):
    """test_regression.py's measure: |got - ref| over max(max |ref| over the first axis,
    1e-3 of the peak); returns the worst."""
    ref = np.asarray(ref)
    peak = np.abs(ref).max()
    scale = np.maximum(np.abs(ref).max(axis=0, keepdims=True), 1e-3 * peak)
    return float((np.abs(np.asarray(got) - ref) / scale).max())


@pytest.fixture(scope="module")
def drift_solution():
    g = np.load(G / "lo_cylinder_drift.npz")
    full = meshes.reflect_full(meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True))
    out = O.solve_body(full, g["omegas"], g["headings"], depth=math.inf)
    return g, out


def test_oracle_matches_reference_solver(drift_solution):
    """A, B, X, FK, SC of the reference's own solve of a floating cylinder (its f32 production
    path; the quarter mesh with two symmetry planes solved here as the full mesh)."""
    g, out = drift_solution
    errs = {
        "A": regression_error(out["A"], g["added_mass"]),
        "B": regression_error(out["B"], g["radiation_damping"]),
        "X": regression_error(out["X"], g["excitation_diffraction"]),
        "FK": regression_error(out["FK"], g["excitation_froude_krylov"]),
        "SC": regression_error(out["SC"], g["excitation_scattering"]),
    }
    # the reference's own production-vs-double bound is 1e-5 of the peak; f32 storage of the
    # baseline adds ~6e-8
    assert max(errs.values()) <= 2e-5, errs
