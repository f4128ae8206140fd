"""The 'graded' interior free surface (interior.rs:139-515): the waterplane of each region fanned from
its area centroid to the waterline segments, the rays cut at t_k = sin(pi k / (2N)).

Pinned on the reference's stored outputs of its regression problem lo_cylinder_interior (the quarter
cylinder n_phi = 8, n_z = 4, n_r = 4 with two symmetry planes, held fixed, the interior surface
generated by 'graded', omegas sqrt(g) sqrt(1, 2.5), headings 0 and 30 degrees): the oracle's generator
and solve to 1e-6 of the peak, the library's generator (hb_model_panels, host code) equal to the
oracle's panel for panel, and the library's solve through hb_model_solve to 2e-5 of the peak (the
reference stores float32)."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from hydrobem_b200 import meshes
from oracle import oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden" / "lo_cylinder_interior.npz"
KEYS = {"A": "added_mass", "B": "radiation_damping", "X": "excitation_diffraction",
        "FK": "excitation_froude_krylov", "SC": "excitation_scattering", "HK": "excitation_haskind"}
SYM = {"none": (0, 0), "yz": (1, 0), "xz": (0, 1), "xz_and_yz": (1, 1)}


def peak_error(got, ref):
    ref = np.asarray(ref)
    return float(np.abs(np.asarray(got) - ref).max() / np.abs(ref).max())


def quarter_cylinder():
    return meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True)


def half_cylinder():
    """The y >= 0 half of a 16-sector cylinder (stored form of a mesh symmetric about y = 0)."""
    full = meshes.cylinder(1.0, 0.6, 16, 3, 3)
    return full[full.mean(axis=1)[:, 1] > 0.0]


def moonpool_box():
    """A box |x|, |y| <= 1 of draft 0.5 with a square moonpool |x|, |y| <= 0.4 through it: the outer
    walls, the moonpool walls facing into the pool, and the bottom ring."""
    p = []
    a, h, d = 1.0, 0.4, 0.5
    for (o, du, dv, nrm) in (((a, -a, -d), (0, 2 * a, 0), (0, 0, d), (1, 0, 0)),
                             ((-a, -a, -d), (0, 2 * a, 0), (0, 0, d), (-1, 0, 0)),
                             ((-a, a, -d), (2 * a, 0, 0), (0, 0, d), (0, 1, 0)),
                             ((-a, -a, -d), (2 * a, 0, 0), (0, 0, d), (0, -1, 0)),
                             ((h, -h, -d), (0, 2 * h, 0), (0, 0, d), (-1, 0, 0)),
                             ((-h, -h, -d), (0, 2 * h, 0), (0, 0, d), (1, 0, 0)),
                             ((-h, h, -d), (2 * h, 0, 0), (0, 0, d), (0, -1, 0)),
                             ((-h, -h, -d), (2 * h, 0, 0), (0, 0, d), (0, 1, 0))):
        p += meshes._face(o, du, dv, 2, 1, nrm)
    for (x0, y0, lx, ly) in ((-a, -a, 2 * a, a - h), (-a, h, 2 * a, a - h), (-a, -h, a - h, 2 * h), (h, -h, a - h, 2 * h)):
        p += meshes._face((x0, y0, -d), (lx, 0, 0), (0, ly, 0), 2, 1, (0, 0, -1))
    return np.array(p)


def library_lid(stored, symmetry, position=(0.0, 0.0, 0.0), reflections=False):
    from hydrobem_b200 import native as nv

    with nv.Model() as m:
        m.add("meshes", "m")
        m.reals("meshes/m", "vertices", stored)
        m.text("meshes/m", "symmetry", symmetry)
        m.add("bodies", "b")
        m.text("bodies/b", "mesh", "m")
        m.reals("bodies/b", "position", list(position))
        m.text("bodies/b", "interior_surface", "graded")
        return m.panels("lid", reflections)


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def test_oracle_graded_lid_covers_the_waterplane():
    """The fan of the quarter cylinder: N = ceil(1 / (2 sin(pi/32))) = 6 cells per segment, 8 segments;
    the panels face up and tile the polygonal quarter waterplane exactly."""
    lid = O.graded_lid(quarter_cylinder(), 1, 1, 0.0)
    assert lid.shape == (48, 4, 3)
    n = np.cross(lid[:, 2] - lid[:, 0], lid[:, 3] - lid[:, 1])
    assert (n[:, 2] > 0.0).all()
    assert abs(0.5 * n[:, 2].sum() - 4.0 * np.sin(np.pi / 16.0)) < 1e-13
    assert np.abs(lid[:, :, 2]).max() == 0.0


def test_oracle_solve_with_graded_lid_against_the_reference(golden):
    q = quarter_cylinder()
    lid = O.graded_lid(q, 1, 1, 0.0)
    v = np.concatenate([q, lid])
    kinds = np.r_[np.full(len(q), O.WET), np.full(len(lid), O.INTERIOR)].astype(np.int32)
    r = O.solve_body(v, golden["omegas"], golden["headings"], kinds=kinds, symmetry=O.SYM_BOTH)
    for k, name in KEYS.items():
        assert peak_error(r[k], golden[name]) <= 1e-6, name


@pytest.mark.parametrize("shape,symmetry", [("quarter_cylinder", "xz_and_yz"), ("half_cylinder", "xz"),
                                            ("full_cylinder", "none"), ("quarter_box", "xz_and_yz"),
                                            ("half_box_x", "yz")])
def test_library_graded_lid_equals_the_oracle(shape, symmetry):
    stored = {"quarter_cylinder": quarter_cylinder, "half_cylinder": half_cylinder,
              "full_cylinder": lambda: meshes.cylinder(1.0, 0.5, 12, 2, 3),
              "quarter_box": lambda: meshes.box(2.0, 1.0, 0.5, (4, 3, 2), quarter=True),
              "half_box_x": lambda: (lambda b: b[b.mean(axis=1)[:, 0] > 0.0])(meshes.box(1.5, 1.0, 0.4, (4, 4, 2)))}[shape]()
    isx, isy = SYM[symmetry]
    ref = O.graded_lid(stored, isx, isy, 0.0)
    got = library_lid(stored, symmetry)
    assert got["vertices"].shape == ref.shape
    assert np.abs(got["vertices"] - ref).max() <= 1e-15
    assert (got["kind"] == 1).all() and (got["body"] == 0).all()


def test_library_graded_lid_of_a_raised_body_and_its_reflections():
    """A mesh raised by 0.1 and placed at z = -0.1: the free surface is z0 = 0.1 in body coordinates and
    the lid lies at z = 0 globally; with the reflections the lid is the stored one mirrored."""
    q = quarter_cylinder() + np.array([0.0, 0.0, 0.1])
    ref = O.graded_lid(q, 1, 1, 0.1)
    got = library_lid(q, "xz_and_yz", position=(0.0, 0.0, -0.1))
    assert np.abs(got["vertices"] - (ref - np.array([0.0, 0.0, 0.1]))).max() <= 1e-15
    full = library_lid(q, "xz_and_yz", position=(0.0, 0.0, -0.1), reflections=True)
    mirrored = meshes.reflect_full(ref) - np.array([0.0, 0.0, 0.1])
    assert np.abs(full["vertices"] - mirrored).max() <= 1e-15


@pytest.mark.parametrize("case,why", [("moonpool", "opening"), ("open", "does not close")])
def test_graded_refusals_match(case, why):
    """A waterplane with an opening, and a stored quarter declared without its planes (the waterline
    does not close), are refused by the oracle and by the library with the reference's reasons."""
    from hydrobem_b200 import native as nv

    stored, symmetry = (moonpool_box(), "none") if case == "moonpool" else (quarter_cylinder(), "none")
    with pytest.raises(ValueError, match=why):
        O.graded_lid(stored, *SYM[symmetry], 0.0)
    with pytest.raises(nv.HydroBEMError, match=why):
        library_lid(stored, symmetry)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 2e-5), ("mixed", 2e-5)])
def test_gpu_graded_interior_through_the_model_abi(golden, precision, tol):
    from hydrobem_b200 import native as nv

    with nv.Model() as m:
        m.add("meshes", "cyl")
        m.reals("meshes/cyl", "vertices", quarter_cylinder())
        m.text("meshes/cyl", "symmetry", "xz_and_yz")
        m.add("bodies", "body")
        m.text("bodies/body", "mesh", "cyl")
        m.text("bodies/body", "interior_surface", "graded")
        m.text("options", "gpu_precision", precision)
        m.reals("environment", "omegas", golden["omegas"])
        m.reals("environment", "headings", golden["headings"])
        res = m.solve()
        got = {name: res.quantity(name) for name in KEYS.values()}
        res.free()
    for name in KEYS.values():
        assert got[name].dtype == golden[name].dtype, name
        assert peak_error(got[name], golden[name]) <= tol, name
