"""Build the in-tree shared libraries.

* ``dvr3d_b200/libdvr3d_b200.so`` -- the product: CUDA kernels for sm_100a plus the host
  code behind the C ABI of ``include/dvr3d_b200.h``; compiled with nvcc only for
  ``-gencode arch=compute_100a,code=sm_100a``.

The CPU checker (``oracle/libdvr3d_oracle.so``, test infrastructure) has its own recipe in
``oracle/build.py``.

Usage: ``python -m dvr3d_b200.build [--force]``. Object files go to ``_build/``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "dvr3d_b200"
CSRC = PKG / "csrc"
BUILD = ROOT / "_build"
LIB = PKG / "libdvr3d_b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libdvr3d_b200.so")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:4]) + " ...")


def build_product(force: bool = False, verbose: bool = False) -> Path:
    srcs = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    hdrs = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [ROOT / "include" / "dvr3d_b200.h"]
    if not force and not _stale(LIB, srcs + hdrs):
        return LIB
    BUILD.mkdir(exist_ok=True)
    nvcc = _nvcc()
    objs = []
    for s in srcs:
        o = BUILD / (s.stem + ".o")
        if force or _stale(o, [s] + hdrs):
            cmd = [nvcc, *NVCC_FLAGS, "-c", str(s), "-o", str(o)]
            if s.suffix == ".cpp":
                cmd = [nvcc, "-x", "cu", *NVCC_FLAGS, "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
        objs.append(str(o))
    _run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(LIB), *objs,
          "-lcudart"])
    return LIB


def main(argv: list[str]) -> int:
    force = "--force" in argv
    build_product(force, verbose="-v" in argv)
    print(LIB)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
