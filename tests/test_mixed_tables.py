"""The mixed form's FP32 copies of TABLE_1D and TABLE_2D carry their Chebyshev series cut short.

The degrees kept are read from the device header; the tests re-expand the stored power-basis
coefficients of every cell in Chebyshev polynomials and bound the dropped terms.  Dropped terms of
a Chebyshev series bound the truncation error on the cell (|T_n| <= 1), so the FP32 copies stay
within a few FP32 roundings of the double-precision tables the FP64 form uses.  The finite-depth
tiles are built per frequency on the device; the GPU parity tests cover their truncation.
"""
from __future__ import annotations

import re
import struct
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "hydrobem_b200" / "csrc" / "hbg_device.cuh"
BLOB = ROOT / "hydrobem_b200" / "tables" / "green_tables.bin"


def _const(name: str) -> int:
    m = re.search(rf"\b{name}\s*=\s*(\d+)", HEADER.read_text())
    assert m, name
    return int(m.group(1))


def _arrays():
    b = BLOB.read_bytes()
    assert b[:8] == b"HBGTBL01"
    cnt = struct.unpack("<Q", b[8:16])[0]
    off, out = 16 + 8 * 24, []
    for i in range(cnt):
        n = struct.unpack("<Q", b[16 + i * 24 + 16:16 + i * 24 + 24])[0]
        out.append(np.frombuffer(b, dtype="<f8", count=n, offset=off))
        off += n * 8
    return out


def _cheb_from_power(n: int) -> np.ndarray:
    """Matrix taking power-basis coefficients on [-1, 1] to Chebyshev coefficients."""
    cp = np.zeros((n, n))  # cp[j, k]: coefficient of t^k in T_j
    cp[0, 0] = 1.0
    if n > 1:
        cp[1, 1] = 1.0
    for j in range(2, n):
        cp[j, 1:] = 2.0 * cp[j - 1, :-1]
        cp[j] -= cp[j - 2]
    return np.linalg.inv(cp.T)


def test_table1d_truncation_bound():
    t1 = _arrays()[0].reshape(30, 17, 4)  # [cell][term][J0, J1, Yt, Yt']
    keep = _const("T1D_FN")
    c = np.einsum("jk,xkq->xjq", _cheb_from_power(17), t1)
    dropped = np.abs(c[:, keep:, :]).sum(axis=1)
    assert dropped.max() < 1e-9, dropped.max()
    # the values themselves are O(1): the cut sits far below FP32 rounding
    assert np.abs(c[:, 0, :]).max() > 0.1


def test_table2d_truncation_bound():
    t2 = _arrays()[1].reshape(30, 30, 2, 8, 8)  # [iy][ix][V, V_X][tx power][ty power]
    kx, ky = _const("T2D_FX"), _const("T2D_FY")
    ti = _cheb_from_power(8)
    c = np.einsum("jk,yxqkl,ml->yxqjm", ti, t2, ti)
    d = np.abs(c).copy()
    d[..., :kx, :ky] = 0.0
    dropped = d.sum(axis=(3, 4))
    assert dropped.max() < 1e-7, dropped.max()


def test_truncation_padding_fits_float4():
    assert _const("T1D_FN") >= 1
    kx, ky = _const("T2D_FX"), _const("T2D_FY")
    fb = (kx * ky + 3) // 4 * 4
    assert fb % 4 == 0 and fb >= kx * ky
