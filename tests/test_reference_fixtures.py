"""Whole solves pinned on numbers the reference holds for them: the floating hemisphere against
Hulme (1982) (tests/data/hulme1982_full.txt; test_low_order.py:417-440, A4) and the truncated cylinder
in finite depth against the eigenfunction-matching solution (tests/data/cylinder_finite_depth.txt;
test_finite_depth_and_limits.py:34-82, A5).  The fixtures are compact copies made by
tests/golden/make_golden.py.

The reference states what its discretization leaves on these meshes, and the oracle reproduces those
figures (CPU tests below); the GPU forms run the reference's own test configurations (GPU tests).
"""

from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

from hydrobem_b200 import meshes
from oracle import oracle as O

G, RHO = 9.80665, 1000.0
GOLD = Path(__file__).resolve().parent / "golden"


def hulme_rows(ka=(0.5, 1.0, 2.0)):
    ref = np.load(GOLD / "hulme.npz")["vals"]
    return ref[[int(np.flatnonzero(np.isclose(ref[:, 0], k, rtol=0, atol=1e-9))[0]) for k in ka]]


def hulme_errors(solve, n):
    """Heave A, B and surge A, B of the hemisphere a = 1 with n x n panels a quadrant, Ka = 0.5, 1, 2,
    normalised by the displaced mass (B also by w), against Hulme's tables: the largest difference per
    quantity over its largest published value."""
    ref = hulme_rows()
    w = np.sqrt(ref[:, 0] * G)
    m0 = RHO * 2 / 3 * math.pi
    r = solve(meshes.hemisphere(1.0, n, n, quarter=True), w, depth=math.inf)
    A, B = r["A"], r["B"]
    vals = np.c_[A[:, 2, 2] / m0, B[:, 2, 2] / (w * m0), A[:, 0, 0] / m0, B[:, 0, 0] / (w * m0)]
    return np.abs(vals - ref[:, 1:]).max(axis=0) / np.abs(ref[:, 1:]).max(axis=0)


def cylinder_fd_errors(solve, n):
    """Heave and surge A, B / w of the floating cylinder a = 1, draft 1 (graded: cosine spacing, n panels a
    quarter circle, n vertical, n / 2 radial), depths 2 and 4, Ka = 0.4, 0.8, 1.5, over rho, against the
    eigenfunction-matching reference: the largest difference per quantity over its largest value."""
    ref = np.load(GOLD / "cylinder_fd.npz")["vals"]
    vals, exact = [], []
    for h in (2.0, 4.0):
        sel = ref[ref[:, 0] == h]
        w = np.sqrt(sel[:, 2] * G)
        v = meshes.cylinder(1.0, 1.0, n, n, n // 2, quarter=True, cosine=True)
        r = solve(v, w, depth=h)
        A, B = r["A"] / RHO, r["B"] / RHO
        vals.append(np.c_[A[:, 2, 2], B[:, 2, 2] / w, A[:, 0, 0], B[:, 0, 0] / w])
        exact.append(sel[:, 3:])
    vals, exact = np.vstack(vals), np.vstack(exact)
    return np.abs(vals - exact).max(axis=0) / np.abs(exact).max(axis=0)


def oracle_solve(v, w, depth):
    return O.solve_body(v, w, [], depth=depth, symmetry=O.SYM_BOTH)


def test_oracle_hulme_converges_at_second_order():
    """O(h^2) panels: halving the panel size divides each error by about four."""
    e16, e32 = hulme_errors(oracle_solve, 16), hulme_errors(oracle_solve, 32)
    order = np.log(e16 / e32) / np.log(2.0)
    assert np.all(e32 < e16) and np.all(e32 <= 1.5e-3), (e16, e32)
    assert np.all((order >= 1.5) & (order <= 2.5)), order


def test_oracle_cylinder_finite_depth_A5():
    """The reference's A5 test: within 3e-3 at 32 panels a quarter circle (it states 2.8e-3 to 7.7e-4
    found) and converging at an order between 1.5 and 2.2 from 24 to 32 (1.74 to 1.91 found)."""
    e24, e32 = cylinder_fd_errors(oracle_solve, 24), cylinder_fd_errors(oracle_solve, 32)
    order = np.log(e24 / e32) / np.log(32 / 24)
    assert np.all(e32 <= 3e-3), e32
    assert np.all((order >= 1.5) & (order <= 2.2)), order
    assert 2.7e-3 <= e32.max() <= 2.9e-3 and 7.5e-4 <= e32.min() <= 7.9e-4, e32


def _gpu_solver(precision):
    from hydrobem_b200 import native as nv

    prec = nv.HBG_MIXED if precision == "mixed" else nv.HBG_FP64

    def solve(v, w, depth):
        return nv.solve(v, w, [], symmetry=nv.SYM_BOTH, depth=depth, precision=prec)

    return solve


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_hulme_A4(precision):
    """The reference's A4 test on the GPU: meshes of 16, 32 and 48 panels a quadrant edge, each error
    smaller than the last and within 1e-3 at the finest."""
    solve = _gpu_solver(precision)
    errs = np.array([hulme_errors(solve, n) for n in (16, 32, 48)])
    assert np.all(errs[1] < errs[0]) and np.all(errs[2] < errs[1]), errs
    assert np.all(errs[2] <= 1e-3), errs[2]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_cylinder_finite_depth_A5(precision):
    """The reference's A5 test on the GPU (finite depth: the tiled integral form and the eigenfunction
    series, depth 2 and 4)."""
    solve = _gpu_solver(precision)
    e24, e32 = cylinder_fd_errors(solve, 24), cylinder_fd_errors(solve, 32)
    order = np.log(e24 / e32) / np.log(32 / 24)
    assert np.all(e32 <= 3e-3), e32
    assert np.all((order >= 1.5) & (order <= 2.2)), order
