"""Build libhydrobem_gpu.so in-tree for sm_100a (nvcc cross-compiles without a GPU).

The Green-function tables (tables/green_tables.bin, checksum-verified data) are embedded in the
library with an assembler ``.incbin``, so the shared object is self-contained.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG.parent / "_build"
LIB = PKG / "libhydrobem_gpu.so"
TABLES = PKG / "tables" / "green_tables.bin"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd[:3]))
    return r


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [
        PKG.parent / "include" / "hydrobem_gpu.h", TABLES]


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and LIB.exists():
        t = LIB.stat().st_mtime
        if all(s.stat().st_mtime <= t for s in sources()):
            return LIB
    BUILD.mkdir(exist_ok=True)
    asm = BUILD / "tables_blob.S"
    asm.write_text(
        '    .section .rodata\n'
        '    .global hbg_tables_blob\n    .global hbg_tables_blob_end\n'
        '    .balign 64\n'
        f'hbg_tables_blob:\n    .incbin "{TABLES}"\n'
        'hbg_tables_blob_end:\n    .byte 0\n'
        '    .section .note.GNU-stack,"",@progbits\n')
    obj = BUILD / "tables_blob.o"
    _run(["gcc", "-c", "-fPIC", str(asm), "-o", str(obj)])
    common = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-Xptxas", "-v" if verbose else "-O3"]
    # geometry and statics without contraction: their threshold decisions follow the reference bit for bit
    st_obj = BUILD / "hbg_statics.o"
    r1 = _run(["nvcc", *common, "-fmad=false", "-c", str(CSRC / "hbg_statics.cu"), "-o", str(st_obj)])
    r = _run(["nvcc", *common, "-shared", "-o", str(LIB), str(CSRC / "hbg_all.cu"), str(st_obj), str(obj)])
    if verbose:
        sys.stderr.write(r1.stderr + r.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
