"""ctypes mirror of ``include/dvr3d_b200.h`` and the loader of ``libdvr3d_b200.so``.

The structures here must match the header field for field; ``tests/test_abi.py`` checks
their sizes against the compiled library's expectations and that every declared entry
point is exported.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
ROOT = PKG_DIR.parent
LIB_PATH = PKG_DIR / "libdvr3d_b200.so"
HEADER = ROOT / "include" / "dvr3d_b200.h"

# error codes (enum dvr3d_status)
DVR3D_OK = 0
DVR3D_ERR_ARG = -1
DVR3D_ERR_CORE_MAX2D = -2
DVR3D_ERR_CORE_MAX3D = -3
DVR3D_ERR_QUADRATURE = -4
DVR3D_ERR_NOCONV = -5
DVR3D_ERR_CUDA = -6
DVR3D_ERR_NOMEM = -7
DVR3D_ERR_UNSUPPORTED = -8
DVR3D_ERR_THETA0 = -9
DVR3D_ERR_PES = -10
DVR3D_ERR_DECK = -11
DVR3D_ERR_NO_DEVICE = -12
DVR3D_ERR_BUFFER = -13
DVR3D_ERR_SCRATCH = -14
DVR3D_NOALLOC_SCRATCH_BYTES = 64 * 1024 * 1024

DVR3D_PES_NONE = 0
DVR3D_PES_MORSE_SUM = 1
DVR3D_PES_GRID = 2
DVR3D_PES_MORSE_SUM_NPARAM = 13

DVR3D_PREC_FP64 = 0
DVR3D_PREC_MIXED_DAVIDSON = 1
DVR3D_PREC_SPLIT_BF16 = 2

_DECK_INTS_1 = ["zpham", "zprad", "zp1d", "zp2d", "zpmin", "zpvec", "zlmat", "zcut", "zrot",
                "zperp", "zembed", "zlin", "zmors1", "zmors2", "zladd", "ztwod", "zvec", "zall",
                "ztheta", "zr2r1", "ztran", "zquad2", "zdiag", "zpfun", "zx", "zs0", "zs1",
                "ncoord", "npnt2", "jrot", "neval", "nalf", "max2d", "max3d", "idia", "kmin",
                "npnt1", "ipar", "max3d2"]


class Deck(C.Structure):
    """struct dvr3d_deck: the job deck of DVR3DRJZ (namelist PRT and cards 2-10)."""

    _fields_ = ([(n, C.c_int) for n in _DECK_INTS_1] +
                [("title", C.c_char * 80),
                 ("fixcos", C.c_double),
                 ("xmass", C.c_double * 3), ("xmassr", C.c_double * 3),
                 ("emax1", C.c_double), ("emax2", C.c_double),
                 ("re1", C.c_double), ("diss1", C.c_double), ("we1", C.c_double),
                 ("re2", C.c_double), ("diss2", C.c_double), ("we2", C.c_double),
                 ("ezero", C.c_double), ("have_ezero", C.c_int)])

    def copy(self) -> "Deck":
        d = Deck()
        C.memmove(C.byref(d), C.byref(self), C.sizeof(Deck))
        return d


DVR3D_LP_NPARAM = 369
DVR3D_PATH_DENSE, DVR3D_PATH_SHIFT_INVERT, DVR3D_PATH_DAVIDSON = 0, 1, 2


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("nlevels", C.c_int), ("tol_cm", C.c_double),
                ("max_iter", C.c_int), ("block", C.c_int), ("learned_precond", C.c_int),
                ("want_vectors", C.c_int), ("want_h3", C.c_int)]


class Result(C.Structure):
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
                ("lp_loss_first", C.c_double), ("lp_loss_last", C.c_double),
                ("low_iterations", C.c_int), ("low_matvecs", C.c_int)]


class DipoleResult(C.Structure):
    """struct dvr3d_dipole_result"""

    _fields_ = [("cap1", C.c_int), ("cap2", C.c_int),
                ("e1", C.POINTER(C.c_double)), ("e2", C.POINTER(C.c_double)),
                ("tz", C.POINTER(C.c_double)), ("tx", C.POINTER(C.c_double)),
                ("sint", C.POINTER(C.c_double)),
                ("neval1", C.c_int), ("neval2", C.c_int), ("j1", C.c_int), ("j2", C.c_int),
                ("kmin1", C.c_int), ("kmin2", C.c_int), ("nblocks", C.c_int),
                ("dev_ms", C.c_double), ("flops", C.c_double)]


# dvr3d_dipd_fn, dvr3d_dipsa_fn
DIPD_FN = C.CFUNCTYPE(C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_void_p)
DIPSA_FN = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double, C.c_double, C.c_double,
                       C.c_void_p)


def header_entry_points() -> list[str]:
    """Names of the functions declared in include/dvr3d_b200.h."""
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(dvr3d_b200_[a-z_]+)\s*\(", text)))


_lib = None


def load_library(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load libdvr3d_b200.so (built in-tree). Raises if it is missing: there is no
    fallback implementation of the hot path."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python -m dvr3d_b200.build` "
                           "(the CUDA extension is required; there is no CPU fallback)")
    lib = C.CDLL(str(p))
    P = C.POINTER
    vp = C.c_void_p
    sig = {
        "dvr3d_b200_init": (C.c_int, [C.c_int, P(vp)]),
        "dvr3d_b200_destroy": (None, [vp]),
        "dvr3d_b200_strerror": (C.c_char_p, [C.c_int]),
        "dvr3d_b200_last_error": (C.c_char_p, [vp]),
        "dvr3d_b200_set_stream": (C.c_int, [vp, vp]),
        "dvr3d_b200_set_wait_limit": (C.c_int, [vp, C.c_longlong]),
        "dvr3d_b200_rotlev3b": (C.c_int, [vp, C.c_char_p, C.c_char_p, P(C.c_double), C.c_int, P(C.c_int),
                                          C.c_char_p, C.c_size_t, P(C.c_size_t)]),
        "dvr3d_b200_rotlev3b_trans": (C.c_int, [vp, C.c_char_p, C.c_char_p, C.c_char_p, P(C.c_double), C.c_int,
                                                P(C.c_int), C.c_char_p, C.c_size_t, P(C.c_size_t)]),
        "dvr3d_b200_rotlev3b_pair": (C.c_int, [vp, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, P(C.c_double),
                                               C.c_int, P(C.c_int), P(C.c_double), C.c_int, P(C.c_int), C.c_char_p,
                                               C.c_size_t, P(C.c_size_t)]),
        "dvr3d_b200_rotlev3": (C.c_int, [vp, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, P(C.c_double),
                                         C.c_int, P(C.c_int), P(C.c_double), C.c_int, P(C.c_int), C.c_char_p,
                                         C.c_size_t, P(C.c_size_t)]),
        "dvr3d_b200_dipole3": (C.c_int, [vp, C.c_char_p, C.c_char_p, C.c_char_p, DIPD_FN, DIPSA_FN, vp, C.c_char_p,
                                         P(DipoleResult), C.c_char_p, C.c_size_t, P(C.c_size_t)]),
        "dvr3d_b200_split_gemm": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, P(C.c_double), C.c_longlong,
                                            P(C.c_double), C.c_longlong, C.c_int, P(C.c_double),
                                            C.c_longlong]),
        "dvr3d_b200_ozaki_gemm": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                            C.c_int, C.c_double, P(C.c_double), C.c_longlong, P(C.c_double),
                                            C.c_longlong, C.c_double, P(C.c_double), C.c_longlong, C.c_int]),
        "dvr3d_b200_parse_deck": (C.c_int, [C.c_char_p, P(Deck)]),
        "dvr3d_b200_set_pes": (C.c_int, [vp, C.c_int, P(C.c_double), C.c_int]),
        "dvr3d_b200_set_pes_grid": (C.c_int, [vp, P(C.c_double), C.c_size_t]),
        "dvr3d_b200_set_pes_grid_k": (C.c_int, [vp, C.c_int, P(C.c_double), C.c_size_t]),
        "dvr3d_b200_grid": (C.c_int, [vp, P(Deck), C.c_int, P(C.c_double), C.c_int,
                                      P(C.c_double), C.c_int, P(C.c_double), C.c_int]),
        "dvr3d_b200_solve_block": (C.c_int, [vp, P(Deck), C.c_int, P(Options), P(Result)]),
        "dvr3d_b200_solve_batch": (C.c_int, [vp, P(Deck), P(C.c_double), C.c_int, P(Options),
                                             P(Result)]),
        "dvr3d_b200_run_deck": (C.c_int, [vp, C.c_char_p, P(Options), C.c_char_p, C.c_size_t,
                                          P(C.c_size_t), C.c_char_p, C.c_size_t,
                                          P(C.c_size_t)]),
        "dvr3d_b200_run_deck_wave": (C.c_int, [vp, C.c_char_p, P(Options), C.c_char_p, C.c_size_t,
                                               P(C.c_size_t), C.c_char_p, C.c_size_t, P(C.c_size_t),
                                               C.c_char_p]),
        "dvr3d_b200_diag_batched": (C.c_int, [vp, C.c_int, P(C.c_int), P(C.c_longlong),
                                              P(C.c_longlong), vp, vp, C.c_int]),
        "dvr3d_b200_diag_batched_noalloc": (C.c_int, [vp, C.c_int, P(C.c_int), P(C.c_longlong),
                                                      P(C.c_longlong), vp, vp, C.c_int]),
        "dvr3d_b200_lp_get_weights": (C.c_int, [vp, P(C.c_double), C.c_int]),
        "dvr3d_b200_lp_set_weights": (C.c_int, [vp, P(C.c_double), C.c_int]),
        "dvr3d_b200_lp_eval": (C.c_int, [vp, P(C.c_double), C.c_int, C.c_int, P(C.c_double), P(C.c_double),
                                         P(C.c_double), P(C.c_double), C.c_double, P(C.c_double),
                                         P(C.c_double), P(C.c_double), P(C.c_double)]),
        "dvr3d_b200_lp_train_loss": (C.c_int, [vp, P(C.c_double), P(C.c_double), P(C.c_double)]),
    }
    for name, (res, args) in sig.items():
        if hasattr(lib, name):
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
    if path is None:
        _lib = lib
    return lib
