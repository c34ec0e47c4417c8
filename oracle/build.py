"""Build recipe of the CPU checker ``oracle/libdvr3d_oracle.so`` (test infrastructure).

Compiles the oracle's C++ sources with g++; LAPACK (dsyev and friends) is resolved at run
time from scipy's OpenBLAS by ``oracle.oracle.load``. Usage: ``python -m oracle.build``.
"""
from __future__ import annotations

import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
SOURCES = [HERE / "dvr3d_oracle.cpp", HERE / "deck_reader.cpp", HERE / "dipole3_oracle.cpp", HERE / "rotlev3_oracle.cpp"]
DEPS = SOURCES + [HERE / "dvr3d_oracle.h", ROOT / "include" / "dvr3d_b200.h"]
LIB = HERE / "libdvr3d_oracle.so"


def build(force: bool = False) -> Path:
    if not force and LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in DEPS):
        return LIB
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-o", str(LIB), *map(str, SOURCES), "-ldl"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("oracle build failed: " + " ".join(cmd[:4]) + " ...")
    return LIB


if __name__ == "__main__":
    print(build("--force" in sys.argv[1:]))
