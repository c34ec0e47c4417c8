"""ctypes wrapper of the CPU oracle (``oracle/libdvr3d_oracle.so``).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the CPU legs of
bench.py to check / time the reference algorithm; never by the product package, and it never
imports the product package itself: it has its own deck reader (deck_reader.cpp), its own
build recipe (oracle/build.py) and its own mirrors of the two interface structures of
include/dvr3d_b200.h that it fills (struct dvr3d_deck, struct dvr3d_result).
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

_DECK_INTS = ["zpham", "zprad", "zp1d", "zp2d", "zpmin", "zpvec", "zlmat", "zcut", "zrot", "zperp", "zembed",
              "zlin", "zmors1", "zmors2", "zladd", "ztwod", "zvec", "zall", "ztheta", "zr2r1", "ztran", "zquad2",
              "zdiag", "zpfun", "zx", "zs0", "zs1", "ncoord", "npnt2", "jrot", "neval", "nalf", "max2d", "max3d",
              "idia", "kmin", "npnt1", "ipar", "max3d2"]


class Deck(C.Structure):
    """struct dvr3d_deck (include/dvr3d_b200.h), as the oracle's deck reader fills it."""

    _fields_ = ([(n, C.c_int) for n in _DECK_INTS] +
                [("title", C.c_char * 80), ("fixcos", C.c_double),
                 ("xmass", C.c_double * 3), ("xmassr", C.c_double * 3),
                 ("emax1", C.c_double), ("emax2", C.c_double),
                 ("re1", C.c_double), ("diss1", C.c_double), ("we1", C.c_double),
                 ("re2", C.c_double), ("diss2", C.c_double), ("we2", C.c_double),
                 ("ezero", C.c_double), ("have_ezero", C.c_int)])


class Result(C.Structure):
    """struct dvr3d_result (include/dvr3d_b200.h): the oracle writes eval, meval and status."""

    _fields_ = [("kz", C.c_int), ("ipar", C.c_int), ("nham3", C.c_int), ("meval", C.c_int),
                ("nblocks", C.c_int), ("iterations", C.c_int), ("fallback", C.c_int),
                ("stage_ms", C.c_double * 6), ("max_resid", C.c_double),
                ("dom_ms", C.c_double), ("dom_bytes", C.c_double), ("dom_flops", C.c_double),
                ("dom_launches", C.c_int), ("launches", C.c_int),
                ("h2d_bytes", C.c_longlong), ("d2h_bytes", C.c_longlong),
                ("dom_kernel", C.c_char * 48),
                ("eval", C.POINTER(C.c_double)), ("eval_cap", C.c_int),
                ("iv2", C.POINTER(C.c_int)), ("iv2_cap", C.c_int),
                ("resid", C.POINTER(C.c_double)), ("resid_cap", C.c_int),
                ("evec", C.POINTER(C.c_double)), ("evec_cap", C.c_size_t),
                ("h3", C.POINTER(C.c_double)), ("h3_cap", C.c_size_t),
                ("path", C.c_int), ("matvecs", C.c_int), ("lp_pairs", C.c_int),
                ("lp_loss_first", C.c_double), ("lp_loss_last", C.c_double)]


class DipoleResult(C.Structure):
    """struct dvr3d_dipole_result (include/dvr3d_b200.h)."""

    _fields_ = [("cap1", C.c_int), ("cap2", C.c_int),
                ("e1", C.POINTER(C.c_double)), ("e2", C.POINTER(C.c_double)),
                ("tz", C.POINTER(C.c_double)), ("tx", C.POINTER(C.c_double)),
                ("sint", C.POINTER(C.c_double)),
                ("neval1", C.c_int), ("neval2", C.c_int), ("j1", C.c_int), ("j2", C.c_int),
                ("kmin1", C.c_int), ("kmin2", C.c_int), ("nblocks", C.c_int),
                ("dev_ms", C.c_double), ("flops", C.c_double)]


DIPD_FN = C.CFUNCTYPE(C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_void_p)
DIPSA_FN = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double, C.c_double, C.c_double,
                       C.c_void_p)


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
                ("stage_s", C.c_double * 4), ("nham3", C.c_int),
                ("psi", C.POINTER(C.c_double)), ("psi_cap", C.c_size_t),
                ("psi_len", C.c_longlong), ("psi_nlev", C.c_int),
                ("pleg_walf", C.POINTER(C.c_double)), ("pleg_cap", C.c_size_t),
                ("maxleg", C.c_int), ("nidvr", C.c_int), ("lincr", C.c_int)]


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
        from oracle.build import build as build_oracle

        build_oracle()
    lib = C.CDLL(str(LIB))
    P = C.POINTER
    lib.oracle_load_lapack.argtypes = [C.c_char_p, C.c_char_p]
    lib.oracle_parse_deck.argtypes = [C.c_char_p, P(Deck)]
    lib.oracle_quadrature.argtypes = [P(Deck), C.c_int, P(Quad)]
    lib.oracle_solve_block.argtypes = [P(Deck), C.c_int, C.c_int, P(C.c_double), C.c_int, P(C.c_double),
                                       C.c_size_t, C.c_int, P(Trace), P(Result)]
    lib.oracle_sizes.argtypes = [P(Deck), C.c_int, P(C.c_int)]
    lib.oracle_pes_morse_sum.argtypes = [P(C.c_double), C.c_double, C.c_double, C.c_double]
    lib.oracle_pes_morse_sum.restype = C.c_double
    lib.oracle_session_begin.argtypes = [P(Deck), C.c_int, C.c_int, P(C.c_double), C.c_int, P(C.c_double),
                                         C.c_size_t, C.c_int, P(C.c_void_p)]
    lib.oracle_session_units.argtypes = [C.c_void_p]
    lib.oracle_session_step.argtypes = [C.c_void_p, C.c_int]
    lib.oracle_session_counts.argtypes = [C.c_void_p, P(C.c_int), P(C.c_int), C.c_int]
    lib.oracle_session_end.argtypes = [C.c_void_p, P(Trace), P(Result)]
    lib.oracle_time_dsyev.argtypes = [C.c_int, C.c_int, C.c_int]
    lib.oracle_time_dsyev.restype = C.c_double
    lib.oracle_rotlev3b.argtypes = [C.c_char_p, C.c_char_p, P(C.c_double), C.c_int, P(C.c_int)]
    lib.oracle_rotlev3b_trans.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, P(C.c_double), C.c_int, P(C.c_int)]
    lib.oracle_rotlev3b_pair.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, P(C.c_double), C.c_int,
                                         P(C.c_int), P(C.c_double), C.c_int, P(C.c_int)]
    lib.oracle_rotlev3.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, P(C.c_double), C.c_int,
                                   P(C.c_int), P(C.c_double), C.c_int, P(C.c_int)]
    lib.oracle_dipole3.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, DIPD_FN, DIPSA_FN, C.c_void_p, C.c_char_p,
                                   P(DipoleResult), C.c_char_p, C.c_size_t, P(C.c_size_t)]
    lib.oracle_dipole_quadrature.argtypes = [C.c_int, P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_double)]
    lib.oracle_threej.argtypes = [C.c_int] * 6
    lib.oracle_threej.restype = C.c_double
    lib.oracle_rot_quadrature.argtypes = [C.c_int, C.c_int, P(C.c_double), P(C.c_double), P(C.c_double),
                                          P(C.c_double)]
    rc = lib.oracle_load_lapack(_lapack_path().encode(), b"scipy_")
    if rc != 0:
        raise RuntimeError("could not bind LAPACK dsyev for the oracle")
    _lib = lib
    return lib


def parse_deck(text: str) -> Deck:
    """Read a job deck with the oracle's own reader (deck_reader.cpp)."""
    d = Deck()
    rc = load().oracle_parse_deck(text.encode(), C.byref(d))
    if rc != 0:
        raise ValueError(f"oracle deck reader rejected the deck ({rc})")
    return d


def as_deck(deck) -> Deck:
    """A deck for the oracle: deck text is read by the oracle's reader; a structure of the
    same C layout (struct dvr3d_deck) is copied byte for byte."""
    if isinstance(deck, str):
        return parse_deck(deck)
    if isinstance(deck, Deck):
        return deck
    if C.sizeof(deck) != C.sizeof(Deck):
        raise TypeError("not a struct dvr3d_deck")
    d = Deck()
    C.memmove(C.byref(d), C.byref(deck), C.sizeof(Deck))
    return d


def k_blocks(deck) -> list[int]:
    """k-loop indices [kd .. ku] of ccmain (:811-819) for a deck (from oracle_sizes)."""
    deck = as_deck(deck)
    for kk in range(0, 3):  # the loop may start at k = 1 (kmin = 1 without zbisc, or f parity)
        try:
            s = sizes(deck, kk)
        except RuntimeError:
            continue
        return list(range(s["kd"], s["ku"] + 1))
    raise RuntimeError("oracle_sizes failed for k = 0, 1, 2")


def quadrature(deck, kk: int = 0) -> Quad:
    q = Quad()
    load().oracle_quadrature(C.byref(as_deck(deck)), kk, C.byref(q))
    return q


def sizes(deck, kk: int = 0) -> dict:
    deck = as_deck(deck)
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
    psi: np.ndarray | None = None  # (levels, record length): amplitudes as trans / transr write them
    pleg_walf: np.ndarray | None = None  # ((maxleg + 1) x nidvr, column-major) the block's angular record
    maxleg: int = 0
    nidvr: int = 0
    lincr: int = 0


def solve(deck: Deck, kk: int = 0, pes=None, vgrid=None, final_mode: int = 0, want_h3: bool = False,
          want_eigs2d: bool = True, h3_cap: int = 0, want_psi: bool = False) -> OracleResult:
    """Run the oracle on one k block. pes: 13 MORSE_SUM parameters, or vgrid: table.
    deck: deck text (read by the oracle's reader) or a struct dvr3d_deck."""
    lib = load()
    deck = as_deck(deck)
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
    psi = None
    if want_psi:
        cap = max(s["idvr"] * s["npnt1"] * s["npnt2"], s["nalf"] * max(s["max2d"], 1)) * neval
        psi = np.zeros(cap)
        t.psi = psi.ctypes.data_as(C.POINTER(C.c_double))
        t.psi_cap = psi.size
        pleg = np.zeros(256 * 256)
        t.pleg_walf = pleg.ctypes.data_as(C.POINTER(C.c_double))
        t.pleg_cap = pleg.size
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
                        stage_s=np.array(t.stage_s[:]), kz=t.kz, ipar=t.ipar,
                        psi=None if psi is None or t.psi_nlev == 0 else
                        psi[:t.psi_len * t.psi_nlev].reshape(t.psi_nlev, t.psi_len).copy(),
                        pleg_walf=None if psi is None else pleg[:(t.maxleg + 1) * t.nidvr].copy(),
                        maxleg=t.maxleg, nidvr=t.nidvr, lincr=t.lincr)


def pes_morse_sum(p, r1: float, r2: float, x: float) -> float:
    pp = np.ascontiguousarray(np.asarray(p, dtype=np.float64))
    return load().oracle_pes_morse_sum(pp.ctypes.data_as(C.POINTER(C.c_double)), r1, r2, x)


def rotlev3b(deck_text: str, wave_path: str) -> np.ndarray:
    """ROTLEV3B's lowest levels (Eh) for one parity from a first-step wavefunction file."""
    lv = np.zeros(20000)
    n = C.c_int(0)
    rc = load().oracle_rotlev3b(deck_text.encode(), str(wave_path).encode(),
                                lv.ctypes.data_as(C.POINTER(C.c_double)), lv.size, C.byref(n))
    if rc != 0:
        raise RuntimeError(f"oracle_rotlev3b failed: {rc}")
    return lv[:n.value].copy()


def rotlev3b_trans(deck_text: str, wave_path: str, kvec_path: str) -> np.ndarray:
    """ROTLEV3B with ZTRAN: the levels, and the transformed vectors written to kvec_path."""
    lv = np.zeros(20000)
    n = C.c_int(0)
    rc = load().oracle_rotlev3b_trans(deck_text.encode(), str(wave_path).encode(), str(kvec_path).encode(),
                                      lv.ctypes.data_as(C.POINTER(C.c_double)), lv.size, C.byref(n))
    if rc != 0:
        raise RuntimeError(f"oracle_rotlev3b_trans failed: {rc}")
    return lv[:n.value].copy()


def rotlev3b_pair(deck_text: str, wave_path: str, kvec_path: str | None = None, kvec2_path: str | None = None):
    """ROTLEV3B with KMIN = 2: (e levels, f levels) in Eh; with paths, the two vector files."""
    lv, lv2 = np.zeros(20000), np.zeros(20000)
    n, n2 = C.c_int(0), C.c_int(0)
    P = C.POINTER(C.c_double)
    rc = load().oracle_rotlev3b_pair(deck_text.encode(), str(wave_path).encode(), (kvec_path or "").encode(),
                                     (kvec2_path or "").encode(), lv.ctypes.data_as(P), lv.size, C.byref(n),
                                     lv2.ctypes.data_as(P), lv2.size, C.byref(n2))
    if rc != 0:
        raise RuntimeError(f"oracle_rotlev3b_pair failed: {rc}")
    return lv[:n.value].copy(), lv2[:n2.value].copy()


def rotlev3(deck_text: str, wave_path: str, kvec_path: str | None = None, kvec2_path: str | None = None):
    """ROTLEV3 (z along r1 or r2): (first set, KMIN = 2 f set) of levels in Eh; with paths, the
    vector files (J = 1 f with KMIN = 0 writes kvec2_path)."""
    lv, lv2 = np.zeros(20000), np.zeros(20000)
    n, n2 = C.c_int(0), C.c_int(0)
    P = C.POINTER(C.c_double)
    rc = load().oracle_rotlev3(deck_text.encode(), str(wave_path).encode(), (kvec_path or "").encode(),
                               (kvec2_path or "").encode(), lv.ctypes.data_as(P), lv.size, C.byref(n),
                               lv2.ctypes.data_as(P), lv2.size, C.byref(n2))
    if rc != 0:
        raise RuntimeError(f"oracle_rotlev3 failed: {rc}")
    return lv[:n.value].copy(), lv2[:n2.value].copy()


def dipole3(deck_text: str, ket_path: str, bra_path: str, dipd=None, dipsa=None, tra_path: str | None = None,
            cap: int = 4096) -> dict:
    """DIPOLE3 on two wavefunction files with a Python dipole plug-in: dipd(r1, r2, xcos, nu) -> float
    or dipsa(q1, q2, cost) -> (dipx, dipy). Returns e1, e2, tz, tx, sint (neval1 x neval2), the
    sizes and the printed text."""
    if (dipd is None) == (dipsa is None):
        raise ValueError("give exactly one of dipd, dipsa")
    e1, e2 = np.zeros(cap), np.zeros(cap)
    tz, tx, si = (np.zeros((cap, cap), order="F") for _ in range(3))
    P = C.POINTER(C.c_double)
    res = DipoleResult(cap1=cap, cap2=cap, e1=e1.ctypes.data_as(P), e2=e2.ctypes.data_as(P),
                       tz=tz.ctypes.data_as(P), tx=tx.ctypes.data_as(P), sint=si.ctypes.data_as(P))
    f1 = DIPD_FN(lambda r1, r2, x, nu, u: float(dipd(r1, r2, x, nu))) if dipd else DIPD_FN()

    def _sa(px, py, q1, q2, ct, u):
        dx, dy = dipsa(q1, q2, ct)
        px[0] = dx
        py[0] = dy

    f2 = DIPSA_FN(_sa) if dipsa else DIPSA_FN()
    out = C.create_string_buffer(1 << 22)
    olen = C.c_size_t(0)
    rc = load().oracle_dipole3(deck_text.encode(), str(ket_path).encode(), str(bra_path).encode(), f1, f2, None,
                               (tra_path or "").encode(), C.byref(res), out, len(out), C.byref(olen))
    if rc != 0:
        raise RuntimeError(f"oracle_dipole3 failed: {rc}")
    n1, n2 = res.neval1, res.neval2
    return dict(e1=e1[:n1].copy(), e2=e2[:n2].copy(), tz=tz[:n1, :n2].copy(), tx=tx[:n1, :n2].copy(),
                sint=si[:n1, :n2].copy(), neval1=n1, neval2=n2, j1=res.j1, j2=res.j2, kmin1=res.kmin1,
                kmin2=res.kmin2, nblocks=res.nblocks, text=out.value.decode())


def dipole_quadrature(npot: int):
    """DIPOLE3's angular rule: the npot/2 largest Gauss-Legendre points, weights, and the
    computed and exact half sums."""
    x, w = np.zeros(npot // 2), np.zeros(npot // 2)
    cs, ts = C.c_double(0), C.c_double(0)
    P = C.POINTER(C.c_double)
    rc = load().oracle_dipole_quadrature(npot, x.ctypes.data_as(P), w.ctypes.data_as(P), C.byref(cs), C.byref(ts))
    if rc != 0:
        raise RuntimeError(f"oracle_dipole_quadrature failed: {rc}")
    return x, w, cs.value, ts.value


def threej(j1: int, j2: int, j3: int, m1: int, m2: int, m3: int) -> float:
    return load().oracle_threej(j1, j2, j3, m1, m2, m3)


def rot_quadrature(npnt: int, k: int):
    """ROTLEV3B's Gauss-associated Legendre half-range rule: (x, w, computed sum, exact sum)."""
    n2 = (npnt + 1) // 2
    x, w = np.zeros(n2), np.zeros(n2)
    cs, ts = C.c_double(0), C.c_double(0)
    P = C.POINTER(C.c_double)
    rc = load().oracle_rot_quadrature(npnt, k, x.ctypes.data_as(P), w.ctypes.data_as(P), C.byref(cs), C.byref(ts))
    if rc != 0:
        raise RuntimeError(f"oracle_rot_quadrature failed: {rc}")
    return x, w, cs.value, ts.value


def time_dsyev(n: int, reps: int = 1, mode: int = 0) -> float:
    return load().oracle_time_dsyev(n, reps, mode)


class Session:
    """One k-block solve of the oracle run in steps (oracle_session_*): ``units`` units of
    work in total (per block of the 1D and 2D stages, the selection, per block row of the
    assembly, the final diagonalisation); ``step(n)`` runs the next n of them and returns
    the units left; ``finish()`` returns the result of a complete run (or cancels an
    unfinished one and returns None)."""

    def __init__(self, deck, kk: int = 0, pes=None, vgrid=None, final_mode: int = 0):
        lib = load()
        self._deck = as_deck(deck)
        self._keep = []
        kind, pp, npes, vg, nvg = 0, None, 0, None, 0
        if pes is not None:
            p = np.ascontiguousarray(np.asarray(pes, dtype=np.float64))
            kind, pp, npes = 1, p.ctypes.data_as(C.POINTER(C.c_double)), p.size
            self._keep.append(p)
        if vgrid is not None:
            g = np.ascontiguousarray(np.asarray(vgrid, dtype=np.float64).ravel())
            kind, vg, nvg = 2, g.ctypes.data_as(C.POINTER(C.c_double)), g.size
            self._keep.append(g)
        self._h = C.c_void_p()
        rc = lib.oracle_session_begin(C.byref(self._deck), kk, kind, pp, npes, vg, nvg, final_mode,
                                      C.byref(self._h))
        if rc != 0:
            raise RuntimeError(f"oracle_session_begin failed: {rc}")
        self.units = lib.oracle_session_units(self._h)
        self._s = sizes(self._deck, kk)

    def step(self, n: int) -> int:
        rc = load().oracle_session_step(self._h, int(n))
        if rc < 0:
            raise RuntimeError(f"oracle session step failed: {rc}")
        return rc

    def counts(self):
        """(iv2, n2d) per block once the selection unit has run, else None."""
        cap = max(self._s["nalf"], self._s["npntc"], 1) + 8
        iv2 = np.zeros(cap, dtype=np.int32)
        n2d = np.zeros(cap, dtype=np.int32)
        ip = C.POINTER(C.c_int)
        nb = load().oracle_session_counts(self._h, iv2.ctypes.data_as(ip), n2d.ctypes.data_as(ip), cap)
        if nb <= 0:
            return None
        return iv2[:nb].copy(), n2d[:nb].copy()

    def finish(self):
        lib = load()
        neval = max(self._s["neval"], 1)
        nblk = max(self._s["nalf"], self._s["npntc"], 1)
        ev = np.zeros(neval + 8)
        iv2 = np.zeros(nblk + 8, dtype=np.int32)
        r = Result()
        r.eval = ev.ctypes.data_as(C.POINTER(C.c_double))
        r.eval_cap = ev.size
        t = Trace()
        t.iv2 = iv2.ctypes.data_as(C.POINTER(C.c_int))
        t.iv2_cap = iv2.size
        rc = lib.oracle_session_end(self._h, C.byref(t), C.byref(r))
        self._h = None
        if rc != 0:
            return None
        return OracleResult(status=rc, eval=ev[:r.meval].copy(), nham3=r.nham3, iv2=iv2[:t.nblocks].copy(), iv1=None,
                            n2d=np.zeros(0, dtype=np.int32), eigs2d=None, h3=None, stage_s=np.array(t.stage_s[:]),
                            kz=r.kz, ipar=r.ipar)
