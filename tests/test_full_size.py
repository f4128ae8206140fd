"""The benchmark configuration at full size against the oracle: the 4096-panel cylinder (radius 1 m,
draft 0.5 m, 64 x 32 side and 64 x 32 bottom panels) in depth 5 m with 4 headings, at three of its 40
periods (1.5 s, 8.1 s and 20 s: the shortest, one in the middle, the longest).  The FP64 form within 1e-9
and the mixed form within 1e-5 of each entry's scale (the regression measure), A, B, X, FK, SC and the
Haskind force; the oracle's statics are computed once for both forms."""

from __future__ import annotations

import math

import numpy as np
import pytest

from hydrobem_b200 import meshes
from oracle import oracle as O

pytestmark = pytest.mark.gpu

HEADS = [0.0, 30.0, 60.0, 90.0]
DEPTH = 5.0
PERIODS = np.linspace(1.5, 20.0, 40)[[0, 14, 39]]


def scaled_error(got, ref, floor=1e-3):
    ref = np.asarray(ref)
    peak = np.abs(ref).max()
    scale = np.maximum(np.abs(ref).max(axis=0, keepdims=True), floor * peak)
    return float((np.abs(np.asarray(got) - ref) / scale).max())


@pytest.fixture(scope="module")
def c2_oracle():
    v = meshes.cylinder(1.0, 0.5, 64, 32, 32)
    assert len(v) == 4096
    omegas = 2.0 * math.pi / PERIODS
    pan = O.make_panels(v)
    st = O.statics(pan, None, DEPTH)
    heads = np.radians(HEADS)
    res = [O.solve_frequency(pan, None, st, DEPTH, w, heads) for w in omegas]
    return v, omegas, {k: np.array([r[k] for r in res]) for k in res[0]}


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-5)])
def test_benchmark_cylinder_full_size(c2_oracle, precision, tol):
    from hydrobem_b200 import native as nv

    v, omegas, ref = c2_oracle
    prec = nv.HBG_MIXED if precision == "mixed" else nv.HBG_FP64
    gpu = nv.solve(v, omegas, HEADS, depth=DEPTH, precision=prec)
    keys = ("A", "B", "X", "FK", "SC", "HK")
    errs = {k: scaled_error(gpu[k], ref[k]) for k in keys}
    print(precision, errs)
    assert max(errs.values()) <= tol, errs
