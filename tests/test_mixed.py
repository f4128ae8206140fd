"""The mixed-precision form: the tcgen05 TF32 product kernel against exact and FP64 products, and the
whole mixed solve against the CPU oracle at the bar of the benchmark metric (A, B, X within 1e-5 of
each entry's scale -- the regression measure, floor 1e-3 of the peak)."""

from __future__ import annotations

import math

import numpy as np
import pytest

from hydrobem_b200 import meshes
from hydrobem_b200 import native as nv
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-5


def scaled_error(got, ref, floor=1e-3):
    ref = np.asarray(ref)
    peak = np.abs(ref).max()
    scale = np.maximum(np.abs(ref).max(axis=0, keepdims=True), floor * peak)
    return float((np.abs(np.asarray(got) - ref) / scale).max())


def test_tf32_gemm_exact_on_small_integers():
    """Small integers are exact in TF32 and their sums exact in FP32: any layout, swizzle or
    descriptor mistake shows as a mismatch."""
    rng = np.random.default_rng(1)
    for M, N, K in ((128, 128, 32), (128, 256, 32), (256, 512, 256), (384, 256, 96), (1152, 1408, 64)):
        A = rng.integers(-3, 4, size=(M, K)).astype(np.float32)
        B = rng.integers(-3, 4, size=(N, K)).astype(np.float32)
        C = nv.debug_gemm_tf32(A, B)
        assert np.array_equal(C, A @ B.T), (M, N, K)


def test_tf32_gemm_subtract_exact_on_small_integers():
    """The trailing-update form C -= A B^T: C tiles prefetched by TMA, updated, stored by TMA."""
    rng = np.random.default_rng(3)
    for M, N, K in ((128, 128, 32), (640, 896, 256)):
        A = rng.integers(-3, 4, size=(M, K)).astype(np.float32)
        B = rng.integers(-3, 4, size=(N, K)).astype(np.float32)
        C0 = rng.integers(-100, 100, size=(M, N)).astype(np.float32)
        C = nv.debug_gemm_tf32(A, B, C0)
        assert np.array_equal(C, C0 - A @ B.T), (M, N, K)


def test_tf32_gemm_against_fp64():
    rng = np.random.default_rng(2)
    A = rng.standard_normal((256, 256)).astype(np.float32)
    B = rng.standard_normal((512, 256)).astype(np.float32)
    C = nv.debug_gemm_tf32(A, B)
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    # TF32 keeps 10 mantissa bits: products to ~5e-4, sums of 256 random terms to ~1e-2 absolute
    err = np.abs(C - ref).max() / np.abs(ref).max()
    assert err < 5e-3, err
    assert err > 1e-7  # the operands were rounded to TF32 (not an FP32 path in disguise)


def test_mixed_config1_cylinder():
    v = meshes.cylinder(1.0, 0.5, 32, 8, 8)
    omegas = 2.0 * math.pi / np.arange(2.0, 12.0)
    gpu = nv.solve(v, omegas, [0.0], precision=nv.HBG_MIXED)
    its = nv.last_ir_iterations()
    ref = O.solve_body(v, omegas, [0.0], depth=math.inf)
    errs = {k: scaled_error(gpu[k], ref[k]) for k in ("A", "B", "X", "HK")}
    assert max(errs.values()) <= MIXED_TOL, (errs, its)
    assert 1 <= its <= 12


def test_mixed_finite_depth_four_headings():
    v = meshes.cylinder(1.0, 0.5, 32, 8, 8)
    omegas = 2.0 * math.pi / np.array([1.5, 3.0, 7.0, 20.0])
    heads = [0.0, 30.0, 60.0, 90.0]
    gpu = nv.solve(v, omegas, heads, depth=5.0, precision=nv.HBG_MIXED)
    ref = O.solve_body(v, omegas, heads, depth=5.0)
    errs = {k: scaled_error(gpu[k], ref[k]) for k in ("A", "B", "X", "HK")}
    assert max(errs.values()) <= MIXED_TOL, errs


def test_mixed_padding_and_uneven_bodies():
    """Panel counts that are not multiples of the 128-column LU block (identity padding)."""
    bodies = [nv.Body(meshes.hemisphere(1.3, 6, 12), [1.1, 2.0], [0.0, 90.0]),
              nv.Body(meshes.cylinder(2.0, 1.0, 24, 6, 6), [0.5, 1.0], [30.0])]
    out = nv.solve_batch(bodies, precision=nv.HBG_MIXED)
    for b, g in zip(bodies, out):
        ref = O.solve_body(b.vertices, b.omegas, b.headings, depth=math.inf)
        errs = {k: scaled_error(g[k], ref[k]) for k in ("A", "B", "X", "HK")}
        assert max(errs.values()) <= MIXED_TOL, errs


def test_mixed_interior_lid():
    v = meshes.box(1.0, 0.5, 0.5, n=(8, 4, 4), lid=True)
    kinds = np.zeros(len(v), np.int32)
    kinds[-32:] = 1
    omegas = np.array([1.0, 2.0, 3.5])
    gpu = nv.solve(v, omegas, [0.0, 45.0], kinds=kinds, precision=nv.HBG_MIXED)
    ref = O.solve_body(v, omegas, [0.0, 45.0], depth=math.inf, kinds=kinds)
    errs = {k: scaled_error(gpu[k], ref[k]) for k in ("A", "B", "X", "HK")}
    assert max(errs.values()) <= MIXED_TOL, errs


def test_mixed_many_headings():
    """12 headings (18 right-hand sides: the wide refinement and triangular-solve variants)."""
    v = meshes.cylinder(1.0, 0.5, 16, 4, 4)
    heads = list(np.linspace(0.0, 330.0, 12))
    omegas = np.array([0.9, 2.2])
    gpu = nv.solve(v, omegas, heads, depth=3.0, precision=nv.HBG_MIXED)
    ref = O.solve_body(v, omegas, heads, depth=3.0)
    errs = {k: scaled_error(gpu[k], ref[k]) for k in ("A", "B", "X", "HK")}
    assert max(errs.values()) <= MIXED_TOL, errs


def test_mixed_large_barge_with_lid():
    """An 80 m x 20 m barge of 10 m draught: 16448 wetted panels and a 2048-panel interior lid (18496
    unknowns), 8 headings.  Too large for the oracle; the FP64 form, pinned on the oracle at smaller
    sizes, is the reference here, and the refinement must still converge in a few corrections."""
    v = meshes.box(40.0, 10.0, 10.0, n=(64, 32, 75), lid=True)
    kinds = np.zeros(len(v), np.int32)
    kinds[-64 * 32:] = 1
    omegas = np.array([0.3, 0.8])
    heads = list(np.arange(8) * 22.5)
    mixed = nv.solve(v, omegas, heads, kinds=kinds, precision=nv.HBG_MIXED)
    hist = nv.last_ir_history()
    fp64 = nv.solve(v, omegas, heads, kinds=kinds)
    errs = {k: scaled_error(mixed[k], fp64[k]) for k in ("A", "B", "X", "HK")}
    assert max(errs.values()) <= MIXED_TOL, (errs, hist)
    # converged by the refinement's own test (the last correction times its contraction below 1e-9)
    assert len(hist) <= 12 and hist[-1] * min(1.0, hist[-1] / hist[-2]) <= 1e-9, hist


def _c3_body(index):
    """Body `index` of the 64-body configuration (meshes.uneven_bodies: seed 20261203, cylinders or
    hemispheres of radius U[0.5, 3], draught U[0.3, 2], N ~ U[800, 6000] rounded to the generators'
    grids, 16 frequencies with K r ~ U[0.1, 10])."""
    return meshes.uneven_bodies(index + 1)[index]


def _shallow_cylinder():
    """Body 30 of the 64-body configuration (r = 2.7 m, draught 0.31 m, 2912 panels, no interior lid) at
    its 16 frequencies and two more next to its irregular frequencies (K r = 9.09 and 9.40, where a scan of
    K r in steps of 0.01 found the reduced-precision refinement diverging; it converges, in up to 20
    corrections, at most others around them)."""
    v, omegas = _c3_body(30)
    r = float(np.hypot(v[..., 0], v[..., 1]).max())
    near = np.sqrt(np.array([9.09, 9.40]) / r * meshes.GRAVITY)
    return v, np.concatenate([omegas, near])


def test_mixed_falls_back_to_fp64_where_refinement_cannot_converge():
    """A shallow cylinder without an interior lid (r = 2.7 m, draught 0.31 m, 2912 panels) over K r up to
    10: next to its irregular frequencies the reduced-precision factors no longer contract the error, and
    those frequencies are solved by the FP64 form; the whole answer stays within the bar."""
    v, omegas = _shallow_cylinder()
    assert len(v) == 2912
    gpu = nv.solve(v, omegas, [0.0, 45.0], precision=nv.HBG_MIXED)
    assert 1 <= nv.last_fallback_count() < len(omegas)
    assert 0.0 < nv.last_fallback_time() < nv.last_profile()["total"]
    ref = nv.solve(v, omegas, [0.0, 45.0])
    errs = {k: scaled_error(gpu[k], ref[k]) for k in ("A", "B", "X", "HK")}
    assert max(errs.values()) <= MIXED_TOL, errs


def test_mixed_fallback_after_corrections_beyond_the_first_look():
    """Each problem's refinement queues three corrections before the host first looks at their norms
    (a 128-panel body converges within them: two entries of history).  The shallow cylinder's batch needs
    more: its systems that converge only in the corrections the host adds one by one must report the
    outputs of their last iterate, not those read back at the first look, while the ones that cannot
    converge go to the FP64 form.  The count does not carry over from the problem solved before."""
    small = meshes.cylinder(1.0, 0.5, 16, 4, 4)
    assert len(small) == 128
    nv.solve(small, np.array([1.0, 2.0]), [0.0], precision=nv.HBG_MIXED)
    assert len(nv.last_ir_history()) == 2, nv.last_ir_history()
    v, omegas = _shallow_cylinder()
    gpu = nv.solve(v, omegas, [0.0, 45.0], precision=nv.HBG_MIXED)
    assert len(nv.last_ir_history()) > 3, nv.last_ir_history()
    assert 1 <= nv.last_fallback_count() < len(omegas)
    ref = nv.solve(v, omegas, [0.0, 45.0])
    errs = {k: scaled_error(gpu[k], ref[k]) for k in ("A", "B", "X", "HK")}
    assert max(errs.values()) <= MIXED_TOL, errs
    nv.solve(small, np.array([1.0, 2.0]), [0.0], precision=nv.HBG_MIXED)
    again = nv.solve(v, omegas, [0.0, 45.0], precision=nv.HBG_MIXED)  # the same path after another problem
    for k in ("A", "B", "X", "HK"):
        assert np.array_equal(np.asarray(again[k]), np.asarray(gpu[k])), k
