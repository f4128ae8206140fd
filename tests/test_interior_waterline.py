"""The 'waterline' interior free surface (interior.rs:408-434 on polygon.rs:154-700): the waterplane
regions, holes (moonpools) included, triangulated -- holes bridged to the outer contour, ear clipping,
Lawson flips to the constrained Delaunay triangulation -- and refined (circumcentre insertion, Ruppert /
Shewchuk) to edges of at most twice the mean waterline segment and angles of at least 25 degrees.

No stored output of the reference uses this generator, so its parity is unpinned: the oracle restates
the reference's steps in their order (the same triangles on every run), the library's host code equals
the oracle triangle for triangle, and the solve with it removes the irregular-frequency error as the
graded surface does (within the lid's discretization of the reference's own graded result)."""

from __future__ import annotations

import numpy as np
import pytest

from hydrobem_b200 import meshes
from oracle import oracle as O
from test_interior_graded import GOLDEN, KEYS, SYM, half_cylinder, moonpool_box, peak_error, quarter_cylinder


def library_lid(stored, symmetry, position=(0.0, 0.0, 0.0), reflections=False):
    from hydrobem_b200 import native as nv

    with nv.Model() as m:
        m.add("meshes", "m")
        m.reals("meshes/m", "vertices", stored)
        m.text("meshes/m", "symmetry", symmetry)
        m.add("bodies", "b")
        m.text("bodies/b", "mesh", "m")
        m.reals("bodies/b", "position", list(position))
        m.text("bodies/b", "interior_surface", "waterline")
        return m.panels("lid", reflections)


def up_area(lid):
    n = np.cross(lid[:, 2] - lid[:, 0], lid[:, 3] - lid[:, 1])
    return n, 0.5 * n[:, 2].sum()


SHAPES = {
    "quarter_cylinder": (quarter_cylinder, "xz_and_yz"),
    "half_cylinder": (half_cylinder, "xz"),
    "full_cylinder": (lambda: meshes.cylinder(1.0, 0.5, 12, 2, 3), "none"),
    "fine_cylinder": (lambda: meshes.cylinder(1.0, 0.5, 64, 4, 8), "none"),
    "quarter_box": (lambda: meshes.box(2.0, 1.0, 0.5, (4, 3, 2), quarter=True), "xz_and_yz"),
    "moonpool_box": (moonpool_box, "none"),
}


def min_angle_deg(tri):
    a, b, c = tri[0, :2], tri[1, :2], tri[2, :2]
    out = []
    for p, q, r in ((a, b, c), (b, c, a), (c, a, b)):
        u, v = q - p, r - p
        out.append(np.degrees(np.arccos(np.clip(u @ v / np.linalg.norm(u) / np.linalg.norm(v), -1, 1))))
    return min(out)


def test_oracle_waterline_tiles_the_waterplane_and_is_refined():
    """The 64-sector cylinder: the triangles face up, tile the polygonal waterplane exactly, and are refined
    to edges of at most twice the mean waterline segment (the chord 2 sin(pi / 64)); no angle is sharp."""
    v = meshes.cylinder(1.0, 0.5, 64, 4, 8)
    lid = O.waterline_lid(v, 0, 0, 0.0)
    n, area = up_area(lid)
    assert (n[:, 2] > 0.0).all()
    assert abs(area - 32.0 * np.sin(2.0 * np.pi / 64.0)) < 1e-12
    assert np.abs(lid[:, :, 2]).max() == 0.0 and np.array_equal(lid[:, 3], lid[:, 2])
    size = 2.0 * 2.0 * np.sin(np.pi / 64.0)
    edges = np.linalg.norm(lid[:, [1, 2, 0], :2] - lid[:, [0, 1, 2], :2], axis=2)
    assert edges.max() <= size * (1.0 + 1e-12)
    assert min(min_angle_deg(t) for t in lid) > 15.0


def test_oracle_waterline_keeps_a_moonpool_open():
    """A box with a square moonpool (which the graded fan refuses): the triangles cover the waterplane less
    the opening, and none lies inside the opening."""
    lid = O.waterline_lid(moonpool_box(), 0, 0, 0.0)
    n, area = up_area(lid)
    assert (n[:, 2] > 0.0).all()
    assert abs(area - (4.0 - 0.64)) < 1e-12
    cent = lid[:, :3, :2].mean(axis=1)
    assert not ((np.abs(cent[:, 0]) < 0.4) & (np.abs(cent[:, 1]) < 0.4)).any()
    with pytest.raises(ValueError, match="opening"):
        O.graded_lid(moonpool_box(), 0, 0, 0.0)


@pytest.mark.parametrize("shape", list(SHAPES))
def test_library_waterline_equals_the_oracle(shape):
    make, symmetry = SHAPES[shape]
    stored = make()
    ref = O.waterline_lid(stored, *SYM[symmetry], 0.0)
    got = library_lid(stored, symmetry)
    assert got["vertices"].shape == ref.shape
    assert np.array_equal(got["vertices"], ref)
    assert (got["kind"] == 1).all()


def test_library_waterline_of_a_raised_body_and_its_reflections():
    q = quarter_cylinder() + np.array([0.0, 0.0, 0.1])
    ref = O.waterline_lid(q, 1, 1, 0.1)
    got = library_lid(q, "xz_and_yz", position=(0.0, 0.0, -0.1))
    assert np.abs(got["vertices"] - (ref - np.array([0.0, 0.0, 0.1]))).max() <= 1e-15
    full = library_lid(q, "xz_and_yz", position=(0.0, 0.0, -0.1), reflections=True)
    assert np.abs(full["vertices"] - (meshes.reflect_full(ref) - np.array([0.0, 0.0, 0.1]))).max() <= 1e-15


def test_waterline_refusals_match():
    """A stored quarter declared without its planes: the waterline does not close, in both."""
    from hydrobem_b200 import native as nv

    with pytest.raises(ValueError, match="does not close"):
        O.waterline_lid(quarter_cylinder(), 0, 0, 0.0)
    with pytest.raises(nv.HydroBEMError, match="does not close"):
        library_lid(quarter_cylinder(), "none")


def test_oracle_solve_with_the_waterline_surface_removes_the_irregular_frequency_error():
    """The quarter cylinder at the reference's regression frequencies: with the waterline surface the
    solve is within the lid discretization (3e-3 of the peak) of the reference's graded-surface result,
    ten times closer than without an interior surface."""
    g = np.load(GOLDEN)
    q = quarter_cylinder()
    lid = O.waterline_lid(q, 1, 1, 0.0)
    kinds = np.r_[np.full(len(q), O.WET), np.full(len(lid), O.INTERIOR)].astype(np.int32)
    r = O.solve_body(np.concatenate([q, lid]), g["omegas"], g["headings"], kinds=kinds, symmetry=O.SYM_BOTH)
    bare = O.solve_body(q, g["omegas"], g["headings"], symmetry=O.SYM_BOTH)
    for k, name in KEYS.items():
        if k == "FK":
            continue
        err, err0 = peak_error(r[k], g[name]), peak_error(bare[k], g[name])
        assert err <= 3e-3 and err * 5.0 <= err0, (k, err, err0)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 2e-5)])
def test_gpu_waterline_interior_through_the_model_abi(precision, tol):
    """The library's solve with its own waterline surface against the oracle's solve on the oracle's
    surface (the same panels): FP64 to 1e-9 of the peak, the mixed form to 2e-5."""
    from hydrobem_b200 import native as nv

    g = np.load(GOLDEN)
    q = quarter_cylinder()
    lid = O.waterline_lid(q, 1, 1, 0.0)
    kinds = np.r_[np.full(len(q), O.WET), np.full(len(lid), O.INTERIOR)].astype(np.int32)
    ref = O.solve_body(np.concatenate([q, lid]), g["omegas"], g["headings"], kinds=kinds, symmetry=O.SYM_BOTH)
    with nv.Model() as m:
        m.add("meshes", "cyl")
        m.reals("meshes/cyl", "vertices", q)
        m.text("meshes/cyl", "symmetry", "xz_and_yz")
        m.add("bodies", "body")
        m.text("bodies/body", "mesh", "cyl")
        m.text("bodies/body", "interior_surface", "waterline")
        m.text("options", "gpu_precision", precision)
        m.reals("environment", "omegas", g["omegas"])
        m.reals("environment", "headings", g["headings"])
        res = m.solve()
        got = {k: res.quantity(name + "_f64") for k, name in KEYS.items()}
        res.free()
    for k in KEYS:
        assert peak_error(got[k], ref[k]) <= tol, k
