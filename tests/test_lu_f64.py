"""The FP64 form's dense solve (LU with partial pivoting: 128-column panels factored recursively down to
8-column strips, the trailing update on FP64 warp MMA, then the substitution) on matrices that need
pivoting, against LAPACK through numpy.  The reference's solve (Real::lu_solve, linalg.rs:100-201 and
321-354 on faer's partial-pivoting LU) is met to rounding, as its own test asks of the complex128 path
(linalg.rs:448-488: solution error <= 1e-10)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("n", [1, 7, 37, 130, 300, 517])
def test_random_systems_need_pivoting(n):
    from hydrobem_b200 import native as nv

    rng = np.random.default_rng(n)
    A = _rand(rng, 3, n, n)
    if n > 1:
        A[:, 0, 0] = 0.0  # the first pivot must come from another row
    B = _rand(rng, 3, n, 5)
    X = nv.debug_lu_f64(A, B)
    ref = np.linalg.solve(A, B)
    err = np.abs(X - ref).max() / np.abs(ref).max()
    assert err <= 1e-10, err
    res = np.abs(A @ X - B).max() / (np.abs(A).max() * np.abs(X).max() * n)
    assert res <= 1e-15, res


def test_permutation_matrix_and_many_right_hand_sides():
    """A permuted identity plus a small perturbation: every column's pivot lies off the diagonal; 32
    right-hand sides (the widest substitution)."""
    from hydrobem_b200 import native as nv

    rng = np.random.default_rng(3)
    n = 200
    P = np.eye(n)[rng.permutation(n)]
    A = (P + 1e-3 * _rand(rng, n, n))[None]
    B = _rand(rng, 1, n, 32)
    X = nv.debug_lu_f64(A, B)
    ref = np.linalg.solve(A, B)
    assert np.abs(X - ref).max() <= 1e-12 * np.abs(ref).max()


def test_singular_matrix_reported():
    from hydrobem_b200 import native as nv

    n = 40
    A = np.eye(n, dtype=np.complex128)[None].copy()
    A[0, :, 5] = 0.0
    with pytest.raises(nv.HydroBEMError) as e:
        nv.debug_lu_f64(A, np.ones((1, n, 1)))
    assert e.value.status == 8  # HB_ERR_NUMERICAL


@pytest.mark.gpu
def test_product_tiles_are_tuned_on_the_device():
    """The tuner times both tile widths of the FP64 product per width bucket when the device is first used;
    the choice follows the timings, and the narrow products of the panel recursion (8 to 32 columns, whose
    64-column tiles would be mostly empty) take the 32-column tile."""
    from hydrobem_b200 import native as nv

    rng = np.random.default_rng(3)
    A = rng.standard_normal((1, 40, 40)) + 1j * rng.standard_normal((1, 40, 40))
    B = rng.standard_normal((1, 40, 2)) + 1j * rng.standard_normal((1, 40, 2))
    nv.debug_lu_f64(A, B)  # the device is in use from here on
    t = nv.tuned_tiles(0)
    assert t["state"] == 2
    for n, (narrow, wide) in t["us"].items():
        assert narrow > 0.0 and wide > 0.0
        assert t["columns"][n] == (64 if wide < 0.98 * narrow else 32)
    assert all(t["columns"][n] == 32 for n in (8, 16, 32))
