"""Extract the Green-function coefficient tables into one binary blob.

The infinite- and finite-depth wave Green functions of HydroBEM are evaluated from tables of
Chebyshev/power coefficients that the reference generates with mpmath
(``scripts/gen_green_tables.py`` and ``scripts/gen_green_finite_tables.py``) and ships as array
literals in ``crates/hydrobem/src/tables/green_inf_tables.rs`` and ``green_fin_tables.rs``.
They are data, not code: the coefficients define the numerical method, so this project reads the
same numbers to reproduce the reference's kernels.  This script parses the literals, checks the
reference's own FNV-1a checksums (``green_inf.rs:268-283``, ``green_fin.rs:853-868``, algorithm
``constants.rs:9-16``) and writes ``green_tables.bin`` beside itself:

    magic  b"HBGTBL01"           8 bytes
    count  uint64                number of arrays (8)
    per array: name (16 bytes, NUL padded), length (uint64)
    the arrays, float64 little endian, in the order of the header

Order: TABLE_1D, TABLE_2D, TABLE_2D_DIRECT, ASYMPTOTIC (infinite depth, checksum 0xCAC816A5E6E5C8F2)
then REGION_META, Q, L0, BESSEL_K (finite depth, checksum 0x4982F563A8976372).

Usage: python extract_tables.py [REFERENCE_ROOT]
"""

from __future__ import annotations

import re
import struct
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "green_tables.bin"

INF = ("TABLE_1D", "TABLE_2D", "TABLE_2D_DIRECT", "ASYMPTOTIC")
FIN = ("REGION_META", "Q", "L0", "BESSEL_K")
CONSTS_INF = {"XT": 30, "YT": 30, "N1": 16, "N2": 7, "N3": 6, "HANKEL_TERMS": 14, "STRUVE_TERMS": 14}
CONSTS_FIN = {"M": 9, "NW": 12, "REGIONS": 13, "NK": 17}
CHECK_INF = 0xCAC816A5E6E5C8F2
CHECK_FIN = 0x4982F563A8976372
FNV_OFFSET = 0xCBF29CE484222325
FNV_PRIME = 0x100000001B3
MASK = (1 << 64) - 1


def fnv1a(arrays, h=FNV_OFFSET):
    """FNV-1a over the little-endian bytes of the doubles (the reference's table checksum)."""
    for a in arrays:
        for byte in np.ascontiguousarray(a, dtype="<f8").tobytes():
            h ^= byte
            h = (h * FNV_PRIME) & MASK
    return h


def parse(text: str, name: str) -> np.ndarray:
    m = re.search(r"pub static " + name + r": \[f64; (\d+)\] = \[(.*?)\];", text, re.S)
    if not m:
        raise SystemExit(f"table {name} not found")
    n = int(m.group(1))
    vals = [float(t) for t in m.group(2).replace("\n", " ").split(",") if t.strip()]
    if len(vals) != n:
        raise SystemExit(f"table {name}: {len(vals)} values, {n} declared")
    return np.array(vals, dtype="<f8")


def consts(text: str, names: dict) -> None:
    for k, v in names.items():
        m = re.search(r"pub const " + k + r": i32 = (-?\d+);", text)
        if not m or int(m.group(1)) != v:
            raise SystemExit(f"constant {k} differs from the layout this project is written for")


def main(argv):
    root = Path(argv[1]) if len(argv) > 1 else Path("/root/reference")
    tdir = root / "crates/hydrobem/src/tables"
    tinf = (tdir / "green_inf_tables.rs").read_text()
    tfin = (tdir / "green_fin_tables.rs").read_text()
    consts(tinf, CONSTS_INF)
    consts(tfin, CONSTS_FIN)
    arrays = {n: parse(tinf, n) for n in INF}
    arrays.update({n: parse(tfin, n) for n in FIN})
    hi = fnv1a([arrays[n] for n in INF])
    hf = fnv1a([arrays[n] for n in FIN])
    if hi != CHECK_INF or hf != CHECK_FIN:
        raise SystemExit(f"checksum mismatch: inf {hi:#x} fin {hf:#x}")
    with open(OUT, "wb") as f:
        f.write(b"HBGTBL01")
        names = INF + FIN
        f.write(struct.pack("<Q", len(names)))
        for n in names:
            f.write(n.encode().ljust(16, b"\0"))
            f.write(struct.pack("<Q", arrays[n].size))
        for n in names:
            f.write(arrays[n].tobytes())
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes), checksums ok")


if __name__ == "__main__":
    main(sys.argv)
