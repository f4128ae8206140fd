"""The mixed form's statics by the reference's production rule (`HbgOptions.statics_rule`
HBG_STATICS_PRODUCTION) (panel_integrals.rs:190-216,
288-363, 380-392; lo_static.rs:82-88): the Rankine integrals by float32 Gauss tiers of orders 6, 5, 4, 3
from 2, 3, 4 and 8 panel radii (the closed forms within 2), the deep finite-depth images and the far log
integrals by the panels' 3 x 3 rule beyond 12 radii, the rows stored in float32.  The device's rows
against the oracle's production mode: the same float32 arithmetic in the same order, so equal to within
one float32 rounding of the stored value, at infinite and finite depth, with an interior lid and with
symmetry sectors."""

from __future__ import annotations

import math

import numpy as np
import pytest

from hydrobem_b200 import meshes
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def oracle_production_statics(v, kinds, depth):
    pan = O.make_panels(v, kinds)
    with O.ProductionMode(True):
        return O.statics(pan, kinds, depth)


def within_one_rounding(got, ref):
    """Every entry of every plane within one float32 unit of the reference entry (a different last
    rounding of a double-precision closed form), plus a floor far below the plane's scale."""
    for q in range(4):
        err = np.abs(got[..., q] - ref[..., q])
        bound = 1.2e-7 * np.abs(ref[..., q]) + 1e-12 * np.abs(ref[..., q]).max()
        assert (err <= bound).all(), (q, float((err / np.maximum(bound, 1e-300)).max()))


@pytest.mark.parametrize("depth", [math.inf, 3.0])
def test_gpu_production_statics_equal_the_oracle(depth):
    from hydrobem_b200 import native as nv

    v = meshes.cylinder(1.0, 0.5, 24, 8, 8)
    got, _, _ = nv.debug_matrices(v, 1.0, depth=depth, statics_rule=nv.HBG_STATICS_PRODUCTION)
    ref = oracle_production_statics(v, None, 0.0 if math.isinf(depth) else depth)
    assert np.array_equal(got, got.astype(np.float32).astype(np.float64))  # float32 rows
    within_one_rounding(got, ref)
    fp64, _, _ = nv.debug_matrices(v, 1.0, depth=depth)
    assert np.abs(got[..., 0] - fp64[..., 0]).max() > 0.0  # the tiers ran


def test_gpu_production_statics_interior_lid_and_sectors():
    from hydrobem_b200 import native as nv

    v = meshes.box(1.0, 0.5, 0.5, n=(8, 4, 4), lid=True)
    kinds = np.zeros(len(v), np.int32)
    kinds[-32:] = 1
    got, _, _ = nv.debug_matrices(v, 2.0, kinds=kinds, statics_rule=nv.HBG_STATICS_PRODUCTION)
    within_one_rounding(got, oracle_production_statics(v, kinds, 0.0))
    quarter = meshes.cylinder(1.0, 0.5, 8, 4, 4, quarter=True)
    got, _, _ = nv.debug_matrices(quarter, 1.0, symmetry=nv.SYM_BOTH, statics_rule=nv.HBG_STATICS_PRODUCTION)
    ref = oracle_production_statics(meshes.reflect_full(quarter), None, 0.0)[: len(quarter)]
    within_one_rounding(got, ref)


def test_gpu_production_rule_through_the_solve():
    """A mixed solve with the production rule stays within the reference's own production-versus-double
    bound of the FP64 form (1e-5 of each quantity's peak); the FP64 form refuses the rule."""
    from hydrobem_b200 import native as nv

    v = meshes.cylinder(1.0, 0.5, 24, 8, 8)
    omegas = np.array([0.8, 1.6, 3.0])
    ref = nv.solve(v, omegas, [0.0, 45.0], depth=3.0)
    got = nv.solve(v, omegas, [0.0, 45.0], depth=3.0, precision=nv.HBG_MIXED, statics_rule=nv.HBG_STATICS_PRODUCTION)
    for k in ("A", "B", "X"):
        assert np.abs(got[k] - ref[k]).max() <= 1e-5 * np.abs(ref[k]).max(), k
    with pytest.raises(nv.HydroBEMError):
        nv.solve(v, omegas, [0.0], statics_rule=nv.HBG_STATICS_PRODUCTION)
