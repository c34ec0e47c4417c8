"""ctypes wrapper of the CPU oracle (``oracle/libdvr3d_oracle.so``).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the CPU-baseline
leg of bench.py to check / time the reference algorithm; never by the product package.
The oracle restates source/dvr3drjz_segmented.f90 of the reference (see dvr3d_oracle.cpp)
and calls LAPACK dsyev from the OpenBLAS library bundled with scipy.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
LIB = Path(__file__).resolve().parent / "libdvr3d_oracle.so"

import sys  # noqa: E402

if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
from dvr3d_b200._abi import Deck, Result  # noqa: E402  (interface structs only)


class Quad(C.Structure):
    _fields_ = [("npnt1", C.c_int), ("npnt2", C.c_int), ("nang2", C.c_int), ("nidvr", C.c_int),
                ("y1", C.c_double * 128), ("wt1", C.c_double * 128), ("r1", C.c_double * 128),
                ("csx1", C.c_double), ("csa1", C.c_double), ("tsx1", C.c_double), ("tsa1", C.c_double),
                ("y2", C.c_double * 128), ("wt2", C.c_double * 128), ("r2", C.c_double * 128),
                ("csx2", C.c_double), ("csa2", C.c_double), ("tsx2", C.c_double), ("tsa2", C.c_double),
                ("xhalf", C.c_double * 128), ("whalf", C.c_double * 128),
                ("cswalf", C.c_double), ("tswalf", C.c_double),
                ("xalf", C.c_double * 256), ("walf", C.c_double * 256),
                ("ur1", C.c_double), ("ur2", C.c_double), ("urr1", C.c_double), ("urr2", C.c_double),
                ("beta1", C.c_double), ("beta2", C.c_double), ("a1", C.c_double), ("a2", C.c_double),
                ("g1", C.c_double), ("g2", C.c_double), ("iu1", C.c_int), ("iu2", C.c_int),
                ("status", C.c_int)]


class Trace(C.Structure):
    _fields_ = [("nblocks", C.c_int), ("npnta", C.c_int), ("npntb", C.c_int), ("npntc", C.c_int),
                ("max2d", C.c_int), ("max3d", C.c_int), ("kz", C.c_int), ("ipar", C.c_int),
                ("iv1", C.POINTER(C.c_int)), ("iv1_cap", C.c_int),
                ("iv2", C.POINTER(C.c_int)), ("iv2_cap", C.c_int),
                ("n2d", C.POINTER(C.c_int)), ("n2d_cap", C.c_int),
                ("eig2all", C.POINTER(C.c_double)), ("eig2all_cap", C.c_int),
                ("eigs2d", C.POINTER(C.c_double)), ("eigs2d_cap", C.c_int),
                ("h3", C.POINTER(C.c_double)), ("h3_cap", C.c_size_t),
                ("stage_s", C.c_double * 4), ("nham3", C.c_int)]


def _lapack_path() -> str:
    import scipy

    base = Path(scipy.__file__).resolve().parent.parent / "scipy.libs"
    cands = sorted(glob.glob(str(base / "libscipy_openblas*.so")))
    cands = [c for c in cands if "64_" not in os.path.basename(c)]
    if not cands:
        raise RuntimeError("scipy's OpenBLAS (LAPACK dsyev) not found")
    return cands[0]


_lib = None


def load(build: bool = True) -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if build or not LIB.exists():
        from dvr3d_b200.build import build_oracle

        build_oracle()
    lib = C.CDLL(str(LIB))
    P = C.POINTER
    lib.oracle_load_lapack.argtypes = [C.c_char_p, C.c_char_p]
    lib.oracle_quadrature.argtypes = [P(Deck), C.c_int, P(Quad)]
    lib.oracle_solve_block.argtypes = [P(Deck), C.c_int, C.c_int, P(C.c_double), C.c_int, P(C.c_double),
                                       C.c_size_t, C.c_int, P(Trace), P(Result)]
    lib.oracle_sizes.argtypes = [P(Deck), C.c_int, P(C.c_int)]
    lib.oracle_pes_morse_sum.argtypes = [P(C.c_double), C.c_double, C.c_double, C.c_double]
    lib.oracle_pes_morse_sum.restype = C.c_double
    lib.oracle_time_dsyev.argtypes = [C.c_int, C.c_int, C.c_int]
    lib.oracle_time_dsyev.restype = C.c_double
    rc = lib.oracle_load_lapack(_lapack_path().encode(), b"scipy_")
    if rc != 0:
        raise RuntimeError("could not bind LAPACK dsyev for the oracle")
    _lib = lib
    return lib


def quadrature(deck: Deck, kk: int = 0) -> Quad:
    q = Quad()
    load().oracle_quadrature(C.byref(deck), kk, C.byref(q))
    return q


def sizes(deck: Deck, kk: int = 0) -> dict:
    o = (C.c_int * 16)()
    rc = load().oracle_sizes(C.byref(deck), kk, o)
    if rc != 0:
        raise RuntimeError(f"oracle_sizes failed: {rc}")
    keys = ["npnt1", "npnt2", "nalf", "idvr", "npnta", "npntb", "npntc", "max2d", "max3d", "neval",
            "kz", "ipar", "nidvr", "lincr", "kd", "ku"]
    return dict(zip(keys, list(o)))


@dataclass
class OracleResult:
    status: int
    eval: np.ndarray
    nham3: int
    iv2: np.ndarray
    iv1: np.ndarray | None
    n2d: np.ndarray
    eigs2d: np.ndarray | None
    h3: np.ndarray | None
    stage_s: np.ndarray
    kz: int
    ipar: int


def solve(deck: Deck, kk: int = 0, pes=None, vgrid=None, final_mode: int = 0, want_h3: bool = False,
          want_eigs2d: bool = True, h3_cap: int = 0) -> OracleResult:
    """Run the oracle on one k block. pes: 13 MORSE_SUM parameters, or vgrid: table."""
    lib = load()
    s = sizes(deck, kk)
    nblk = max(s["nalf"], s["npntc"], 1)
    neval = max(s["neval"], 1)
    ev = np.zeros(neval + 8)
    iv2 = np.zeros(nblk + 8, dtype=np.int32)
    n2d = np.zeros(nblk + 8, dtype=np.int32)
    r = Result()
    r.eval = ev.ctypes.data_as(C.POINTER(C.c_double))
    r.eval_cap = ev.size
    t = Trace()
    t.iv2 = iv2.ctypes.data_as(C.POINTER(C.c_int))
    t.iv2_cap = iv2.size
    t.n2d = n2d.ctypes.data_as(C.POINTER(C.c_int))
    t.n2d_cap = n2d.size
    iv1 = None
    if deck.idia != -2:
        iv1 = np.zeros(s["npntc"] * s["npntb"] + 8, dtype=np.int32)
        t.iv1 = iv1.ctypes.data_as(C.POINTER(C.c_int))
        t.iv1_cap = iv1.size
    e2 = None
    maxn = max(s["max3d"], 1)
    if want_eigs2d:
        e2 = np.zeros(maxn + 8)
        t.eigs2d = e2.ctypes.data_as(C.POINTER(C.c_double))
        t.eigs2d_cap = e2.size
    h3 = None
    if want_h3:
        cap = h3_cap or maxn * maxn
        h3 = np.zeros(cap)
        t.h3 = h3.ctypes.data_as(C.POINTER(C.c_double))
        t.h3_cap = h3.size
    kind, pp, npes, vg, nvg = 0, None, 0, None, 0
    if pes is not None:
        p = np.ascontiguousarray(np.asarray(pes, dtype=np.float64))
        kind, pp, npes = 1, p.ctypes.data_as(C.POINTER(C.c_double)), p.size
        keep_p = p
    if vgrid is not None:
        g = np.ascontiguousarray(np.asarray(vgrid, dtype=np.float64).ravel())
        kind, vg, nvg = 2, g.ctypes.data_as(C.POINTER(C.c_double)), g.size
        keep_g = g
    rc = lib.oracle_solve_block(C.byref(deck), kk, kind, pp, npes, vg, nvg, final_mode, C.byref(t), C.byref(r))
    n = t.nham3
    return OracleResult(status=rc, eval=ev[:r.meval].copy(), nham3=n, iv2=iv2[:t.nblocks].copy(),
                        iv1=None if iv1 is None else iv1[:s["npntc"] * s["npntb"]].copy(),
                        n2d=n2d[:t.nblocks].copy(),
                        eigs2d=None if e2 is None else e2[:n].copy(),
                        h3=None if h3 is None or n == 0 else h3[:n * n].reshape(n, n, order="F").copy(),
                        stage_s=np.array(t.stage_s[:]), kz=t.kz, ipar=t.ipar)


def pes_morse_sum(p, r1: float, r2: float, x: float) -> float:
    pp = np.ascontiguousarray(np.asarray(p, dtype=np.float64))
    return load().oracle_pes_morse_sum(pp.ctypes.data_as(C.POINTER(C.c_double)), r1, r2, x)


def time_dsyev(n: int, reps: int = 1, mode: int = 0) -> float:
    return load().oracle_time_dsyev(n, reps, mode)
