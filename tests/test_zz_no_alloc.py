"""The allocation-free statics entry (hbg_statics_noalloc): the same statics as the allocating path
(hbg_debug_matrices), from the library's fixed device scratch into caller-owned device memory, on
two calls in a row (the second reuses the scratch the first left behind)."""

from __future__ import annotations

import math

import numpy as np
import pytest

from hydrobem_b200 import meshes
from hydrobem_b200 import native as nv

pytestmark = pytest.mark.gpu

TOL = 1e-12  # of the largest entry of each plane: the same kernels on the same inputs


def _device_statics(torch, v, kinds, depth):
    N = len(v)
    dv = torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64).reshape(-1)).cuda()
    dk = None if kinds is None else torch.from_numpy(np.asarray(kinds, dtype=np.int32)).cuda()
    out = []
    for _ in range(2):
        dst = torch.full((4 * N * N,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        nv.statics_noalloc(dv.data_ptr(), None if dk is None else dk.data_ptr(), N, dst.data_ptr(), depth=depth,
                           stream=torch.cuda.current_stream().cuda_stream)
        # plane q, entry (k, j) at q N^2 + k + j N  ->  [k][j][q]
        out.append(dst.cpu().numpy().reshape(4, N, N).transpose(2, 1, 0))
    return out


@pytest.mark.parametrize("depth", [math.inf, 3.0])
def test_statics_noalloc_matches_allocating_path(depth):
    torch = pytest.importorskip("torch")
    v = meshes.cylinder(1.0, 0.5, 24, 8, 8)
    ref, _, _ = nv.debug_matrices(v, 1.0, depth=depth)
    for got in _device_statics(torch, v, None, depth):
        assert np.isfinite(got).all()
        for q in range(4):
            scale = np.abs(ref[..., q]).max()
            assert np.abs(got[..., q] - ref[..., q]).max() <= TOL * scale, q


def test_statics_noalloc_interior_lid():
    torch = pytest.importorskip("torch")
    v = meshes.box(1.0, 0.5, 0.5, n=(8, 4, 4), lid=True)
    kinds = np.zeros(len(v), np.int32)
    kinds[-32:] = 1
    ref, _, _ = nv.debug_matrices(v, 2.0, kinds=kinds)
    for got in _device_statics(torch, v, kinds, math.inf):
        for q in range(4):
            scale = np.abs(ref[..., q]).max()
            assert np.abs(got[..., q] - ref[..., q]).max() <= TOL * scale, q


def test_statics_noalloc_rejects_more_panels_than_its_scratch():
    torch = pytest.importorskip("torch")
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    with pytest.raises(nv.HydroBEMError) as e:
        nv.statics_noalloc(buf.data_ptr(), None, 2049, buf.data_ptr())
    assert nv.STATUS_NAMES[e.value.status] == "HB_ERR_VALUE"
    assert "2048" in e.value.message


def test_statics_noalloc_allocates_no_device_memory():
    """After warm-up calls (module loading), further calls leave the device's free memory unchanged:
    the entry writes only the caller's buffer and its fixed device scratch."""
    torch = pytest.importorskip("torch")
    v = meshes.cylinder(1.0, 0.5, 24, 8, 8)
    N = len(v)
    dv = torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64).reshape(-1)).cuda()
    dst = torch.empty(4 * N * N, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for depth in (3.0, math.inf):  # both depth forms loaded (lazy module loading may allocate)
        nv.statics_noalloc(dv.data_ptr(), None, N, dst.data_ptr(), depth=depth, stream=stream)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for depth in (3.0, math.inf):
        nv.statics_noalloc(dv.data_ptr(), None, N, dst.data_ptr(), depth=depth, stream=stream)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
