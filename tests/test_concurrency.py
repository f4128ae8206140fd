"""Several problems of one hbg_solve_batch call on concurrent pipelines (the option `concurrency`): the
reference's worker pool over independent bodies (parallel.rs:31-109, solve_driver.rs:275-282).  Each
problem is solved by the same kernels whatever the pipeline, so the FP64 results equal those of the
one-after-another solve to the bit, the mixed ones to its refinement tolerance; a failing problem is
reported with its own index."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from hydrobem_b200 import meshes
from hydrobem_b200 import native as nv

QUANTS = ("A", "B", "X", "FK", "SC", "HK")
HB_ERR_VALUE = 1  # hydrobem.h


def uneven_bodies():
    """Five cylinders of 48 to 320 panels, three frequencies and two headings each."""
    shapes = [(1.0, 0.5, 12, 2, 2), (0.8, 0.6, 16, 4, 3), (1.2, 0.4, 20, 6, 4), (0.6, 0.3, 8, 3, 3), (1.0, 1.0, 24, 4, 4)]
    out = []
    for i, (r, d, nphi, nz, nr) in enumerate(shapes):
        omegas = np.sqrt(9.80665 * np.array([0.4, 1.1, 2.3]) * (1.0 + 0.1 * i))
        out.append(dict(vertices=meshes.cylinder(r, d, nphi, nz, nr), omegas=omegas, headings_deg=[0.0, 40.0]))
    return out


def solve_all(problems, **options):
    return nv.solve_batch([nv.Body(**p) for p in problems], **options)


def test_concurrency_option_default_and_range():
    """The default leaves the choice to the tuner (0); values outside 0..8 are refused before any device
    work."""
    o = nv.default_options()
    assert o.concurrency == 0
    b = nv.Body(**uneven_bodies()[0])
    arr = (nv.HbgProblem * 1)(b.problem())
    for bad in (-1, 9):
        o = nv.default_options(concurrency=bad)
        assert nv.lib().hbg_solve_batch(arr, 1, ctypes.byref(o)) == HB_ERR_VALUE
        assert "concurrency" in nv.lib().hb_last_error_message().decode()


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(nv.HBG_FP64, 0.0), (nv.HBG_MIXED, 1e-7)])
def test_concurrent_pipelines_match_one_after_another(precision, tol):
    probs = uneven_bodies()
    one = solve_all(probs, precision=precision, concurrency=1)
    prof1 = nv.last_profile()
    for k in (2, 3, 5):
        got = solve_all(probs, precision=precision, concurrency=k)
        prof = nv.last_profile()
        assert prof["total"] > 0.0 and prof["assembly"] > 0.0 and prof["lu"] > 0.0
        assert nv.last_launch_count() > 0
        for p, (a, b) in enumerate(zip(got, one)):
            for q in QUANTS:
                x, y = np.asarray(a[q]), np.asarray(b[q])
                err = np.abs(x - y).max() / max(np.abs(y).max(), 1e-300)
                assert err <= tol, (k, p, q, err)
    assert prof1["total"] > 0.0


@pytest.mark.gpu
def test_concurrent_failure_reports_its_problem():
    """Problem 3 of five has a non-positive frequency: the call fails with HB_ERR_VALUE located at problem 3
    whatever the number of pipelines."""
    probs = uneven_bodies()
    probs[3] = dict(probs[3], omegas=np.array([1.0, -2.0, 3.0]))
    for k in (1, 3):
        bodies = [nv.Body(**p) for p in probs]
        arr = (nv.HbgProblem * len(bodies))(*[b.problem() for b in bodies])
        o = nv.default_options(concurrency=k)
        assert nv.lib().hbg_solve_batch(arr, len(bodies), ctypes.byref(o)) == HB_ERR_VALUE
        loc = nv.HbLocation()
        nv.lib().hb_last_error_location(ctypes.byref(loc))
        assert loc.body == 3
        assert "omega" in nv.lib().hb_last_error_message().decode()


@pytest.mark.gpu
def test_release_frees_the_pipelines_buffers():
    """hbg_release_workspace also frees what the pipelines hold: a later call solves again."""
    import torch

    probs = uneven_bodies()
    solve_all(probs, precision=nv.HBG_MIXED, concurrency=3)
    before = torch.cuda.mem_get_info()[0]
    nv.check(nv.lib().hbg_release_workspace())
    after = torch.cuda.mem_get_info()[0]
    assert after >= before
    again = solve_all(probs, precision=nv.HBG_MIXED, concurrency=3)
    assert np.isfinite(np.asarray(again[0]["A"])).all()


@pytest.mark.gpu
def test_cancelled_batch_on_pipelines():
    """A set cancel flag stops every pipeline before its first batch: HB_ERR_CANCELLED, and the pipelines
    solve again afterwards."""
    flag = (ctypes.c_int32 * 1)(1)
    bodies = [nv.Body(**p) for p in uneven_bodies()]
    arr = (nv.HbgProblem * len(bodies))(*[b.problem() for b in bodies])
    o = nv.default_options(concurrency=3)
    o.cancel = ctypes.cast(flag, nv.ip)
    assert nv.lib().hbg_solve_batch(arr, len(bodies), ctypes.byref(o)) == 5  # HB_ERR_CANCELLED
    flag[0] = 0
    nv.check(nv.lib().hbg_solve_batch(arr, len(bodies), ctypes.byref(o)))
    assert all(np.isfinite(np.asarray(b.results()["A"])).all() for b in bodies)


@pytest.mark.gpu
def test_pipelines_and_the_calling_thread_hand_over_the_memory():
    """A concurrent call after a solve on the calling thread, and a solve on the calling thread after a
    concurrent call, each get the device memory: the buffers of the other mode are freed first."""
    import torch

    probs = uneven_bodies()
    nv.solve_batch([nv.Body(**probs[4])], precision=nv.HBG_MIXED)  # buffers on the calling thread
    solve_all(probs, precision=nv.HBG_MIXED, concurrency=2)
    after_concurrent = torch.cuda.mem_get_info()[0]
    nv.solve_batch([nv.Body(**probs[4])], precision=nv.HBG_MIXED, concurrency=1)
    after_single = torch.cuda.mem_get_info()[0]
    # the pipelines' buffers are gone once the calling thread solves again (its own are smaller)
    assert after_single >= after_concurrent
