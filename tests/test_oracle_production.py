"""The oracle's production mode: the reference's default arithmetic (float32 Gauss tiers of the Rankine
integrals, panel_integrals.rs:288-363; the direct wave-kernel tables, green_inf.rs:316-330; float32 static
rows; complex64 matrices and LU) beside its diagnostic double path.  It is the CPU reference arm of the
benchmark, so it is pinned here on what the reference states for it:

- the tier rule errs by at most 1e-6 of each Rankine integral (panel_integrals.rs:288-290: "1e-6
  relative, measured 9.7e-7");
- the production solve equals the diagnostic one within 1e-5 of each quantity's peak, and the two
  really differ (tests/python/test_double_precision_mode.py:48-55, on its mesh and frequencies).
"""

from __future__ import annotations

import numpy as np

from hydrobem_b200 import meshes
from oracle import oracle as O


def test_tier_rule_within_its_stated_error():
    """Points around a quadrilateral and a triangle at 2 to 60 panel radii in every direction: the float32
    tier (orders 6, 5, 4, 3 by distance) against the closed forms."""
    rng = np.random.default_rng(7)
    quads = meshes.cylinder(1.0, 0.5, 16, 4, 4)
    panels = O.make_panels(quads)
    worst = 0.0
    for j in (0, 70, len(quads) - 1):  # side quads and a bottom triangle
        p = panels[j]
        c, rad = np.array(p.c), p.radius
        for r in np.concatenate([np.linspace(2.0, 9.0, 15), [12.0, 20.0, 40.0, 60.0]]):
            for _ in range(6):
                d = rng.standard_normal(3)
                x = c + r * rad * d / np.linalg.norm(d)
                with O.ProductionMode():
                    got = O.rankine_any(p, x)
                ref = O.rankine(p, x)  # the closed forms (diagnostic mode: to 1000 radii)
                # the dipole's scale is that of the source over the distance (area / dist^2): the
                # dipole itself vanishes for points in the panel's plane
                worst = max(worst, abs(got[0] - ref[0]) / abs(ref[0]),
                            abs(got[1] - ref[1]) / (abs(ref[0]) / (r * rad)))
    assert worst <= 1e-6, worst
    assert worst > 1e-9  # the tiers ran (not the closed forms again)


def test_production_equals_double_precision():
    quarter = meshes.cylinder(1.0, 1.0, 8, 6, 4, quarter=True, cosine=True)
    w = np.sqrt(np.array([0.5, 1.2, 2.0]) * 9.80665)
    diag = O.solve_body(quarter, w, [0.0, 45.0], symmetry=O.SYM_BOTH)
    prod = O.solve_body(quarter, w, [0.0, 45.0], symmetry=O.SYM_BOTH, production=True)
    for k in ("A", "B", "X", "HK"):
        ref = np.abs(diag[k]).max()
        assert np.abs(prod[k] - diag[k]).max() <= 1e-5 * ref, k
    assert np.abs(prod["A"] - diag["A"]).max() > 0.0


def test_production_statics_float32_rows():
    """The static rows of the production mode are float32 values and agree with the diagnostic rows to
    the tier rule's error."""
    v = meshes.cylinder(1.0, 0.5, 16, 4, 4)
    pan = O.make_panels(v)
    diag = O.statics(pan, None, 5.0)
    with O.ProductionMode():
        prod = O.statics(pan, None, 5.0)
    assert np.array_equal(prod, prod.astype(np.float32).astype(np.float64))
    for q in range(4):
        assert np.abs(prod[..., q] - diag[..., q]).max() <= 2e-6 * np.abs(diag[..., q]).max(), q
