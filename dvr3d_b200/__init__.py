"""dvr3d_b200 -- B200-native DVR3DRJZ hot path behind a C ABI.

Python mirror of the library's C entry points (include/dvr3d_b200.h). The numerical work
runs in ``libdvr3d_b200.so`` (CUDA kernels for sm_100a); this module only marshals
arguments. Importing it does not need a GPU; creating a :class:`Context` does, and fails
with an error when no usable device or no built library is present (there is no CPU
fallback of the hot path).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import (DVR3D_LP_NPARAM, DVR3D_PATH_DAVIDSON, DVR3D_PATH_DENSE, DVR3D_PATH_SHIFT_INVERT,
                   DVR3D_PES_GRID, DVR3D_PES_MORSE_SUM, DVR3D_PES_MORSE_SUM_NPARAM, DVR3D_PREC_FP64,
                   DVR3D_PREC_MIXED_DAVIDSON, DVR3D_PREC_SPLIT_BF16, Deck, Options, Result)

AUTOCM = 2.19474624e5  # hartree -> cm-1, as diag3d (:2681)

__all__ = ["Context", "Deck", "DVR3DError", "SolveResult", "parse_deck", "AUTOCM",
           "DVR3D_PES_MORSE_SUM", "DVR3D_PES_GRID", "DVR3D_PREC_FP64",
           "DVR3D_PREC_MIXED_DAVIDSON", "DVR3D_PREC_SPLIT_BF16", "DVR3D_LP_NPARAM", "DVR3D_PATH_DENSE", "DVR3D_PATH_SHIFT_INVERT",
           "DVR3D_PATH_DAVIDSON", "k_blocks", "host_grid"]


class DVR3DError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _strerror(code: int) -> str:
    return _abi.load_library().dvr3d_b200_strerror(code).decode()


def parse_deck(text: str) -> Deck:
    """Read a DVR3DRJZ job deck (namelist PRT + cards) into a :class:`Deck`."""
    lib = _abi.load_library()
    d = Deck()
    rc = lib.dvr3d_b200_parse_deck(text.encode(), C.byref(d))
    if rc != 0:
        raise DVR3DError(rc, _strerror(rc))
    return d


def k_blocks(deck: Deck) -> list[int]:
    """k-loop indices of ccmain (:811-819) for a deck: [kd .. ku]."""
    jrot, kmin = abs(deck.jrot), deck.kmin
    zrot = bool(deck.zrot) and jrot != 0
    if jrot == 0:
        kmin = 0
    if deck.zperp and deck.idia == -2:  # KMIN carries the Q symmetry; k starts at 0 (:257-261)
        kmin = 1 if jrot else 0
    if zrot:
        zbisc = deck.idia == -2
        if kmin != 0 and not zbisc:
            kmin = 1
        if kmin not in (0, 1):
            kmin = 2
        kd, ku = 1 - min(kmin, 1), jrot + (1 if kmin == 2 else 0)
    else:
        kd = ku = kmin
    return list(range(kd, ku + 1))


def host_grid(deck: Deck, kk: int = 0):
    """DVR grid (r1, r2, cos theta) of one k block from the library's host set-up
    (dvr3d_b200_grid with no device context; needs no GPU)."""
    lib = _abi.load_library()
    r1 = np.zeros(256)
    r2 = np.zeros(256)
    xa = np.zeros(512)
    dp = C.POINTER(C.c_double)
    rc = lib.dvr3d_b200_grid(None, C.byref(deck), kk, r1.ctypes.data_as(dp), 256, r2.ctypes.data_as(dp), 256,
                             xa.ctypes.data_as(dp), 512)
    if rc != 0:
        raise DVR3DError(rc, _strerror(rc))
    n1 = deck.npnt2 if deck.idia == -2 else deck.npnt1
    na = deck.nalf // 2 if deck.idia == 2 else deck.nalf
    return r1[:n1].copy(), r2[:deck.npnt2].copy(), xa[:na].copy()


@dataclass
class SolveResult:
    eval: np.ndarray                 # levels (Eh), ascending, length meval
    nham3: int
    iv2: np.ndarray                  # per-block selection counts
    kz: int
    ipar: int
    stage_ms: np.ndarray
    max_resid: float
    iterations: int = 0
    fallback: int = 0
    resid: np.ndarray | None = None
    evec: np.ndarray | None = None
    h3: np.ndarray | None = None
    extra: dict = field(default_factory=dict)

    @property
    def eval_cm(self) -> np.ndarray:
        return self.eval * AUTOCM


def _counters(r: Result) -> dict:
    return {"dom_ms": r.dom_ms, "dom_bytes": r.dom_bytes, "dom_flops": r.dom_flops,
            "dom_launches": r.dom_launches, "launches": r.launches, "h2d_bytes": r.h2d_bytes,
            "d2h_bytes": r.d2h_bytes, "dom_kernel": r.dom_kernel.decode(), "path": r.path,
            "matvecs": r.matvecs, "lp_pairs": r.lp_pairs, "lp_loss_first": r.lp_loss_first,
            "lp_loss_last": r.lp_loss_last, "low_iterations": r.low_iterations,
            "low_matvecs": r.low_matvecs}


class Context:
    """One CUDA device context of the library (dvr3d_b200_init)."""

    def __init__(self, device: int = 0):
        self._lib = _abi.load_library()
        h = C.c_void_p()
        rc = self._lib.dvr3d_b200_init(int(device), C.byref(h))
        if rc != 0:
            raise DVR3DError(rc, _strerror(rc) + " (the CUDA path is required; no CPU fallback)")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.dvr3d_b200_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        if rc != 0:
            msg = self._lib.dvr3d_b200_last_error(self._h).decode()
            raise DVR3DError(rc, _strerror(rc) + (": " + msg if msg else ""))

    def set_stream(self, stream_ptr: int) -> None:
        self._check(self._lib.dvr3d_b200_set_stream(self._h, C.c_void_p(stream_ptr)))

    def set_wait_limit(self, polls: int) -> None:
        """Poll limit of every bounded device wait of later solves (0: the defaults)."""
        self._check(self._lib.dvr3d_b200_set_wait_limit(self._h, int(polls)))

    def rotlev3b(self, deck_text: str, wave_path: str) -> tuple[np.ndarray, str]:
        """The second variational step (ROTLEV3B) on a first-step wavefunction file
        (dvr3d_b200_rotlev3b): the lowest levels (Eh) and the printed level table."""
        lv = np.zeros(20000)
        n = C.c_int(0)
        ln = C.c_size_t(0)
        self._check(self._lib.dvr3d_b200_rotlev3b(self._h, deck_text.encode(), str(wave_path).encode(),
                                                  lv.ctypes.data_as(C.POINTER(C.c_double)), lv.size,
                                                  C.byref(n), None, 0, C.byref(ln)))
        buf = C.create_string_buffer(ln.value)
        self._check(self._lib.dvr3d_b200_rotlev3b(self._h, deck_text.encode(), str(wave_path).encode(),
                                                  None, 0, C.byref(n), buf, ln.value, None))
        return lv[:n.value].copy(), buf.value.decode()

    def rotlev3b_trans(self, deck_text: str, wave_path: str, kvec_path: str) -> tuple[np.ndarray, str]:
        """ROTLEV3B with ZTRAN (dvr3d_b200_rotlev3b_trans): the levels and the printed table; the
        eigenvectors transformed back to the first step's basis are written to kvec_path."""
        lv = np.zeros(20000)
        n = C.c_int(0)
        ln = C.c_size_t(0)
        buf = C.create_string_buffer(1 << 20)
        self._check(self._lib.dvr3d_b200_rotlev3b_trans(self._h, deck_text.encode(), str(wave_path).encode(),
                                                        str(kvec_path).encode(),
                                                        lv.ctypes.data_as(C.POINTER(C.c_double)), lv.size,
                                                        C.byref(n), buf, len(buf), C.byref(ln)))
        return lv[:n.value].copy(), buf.value.decode()

    def rotlev3b_pair(self, deck_text: str, wave_path: str, kvec_path: str | None = None,
                      kvec2_path: str | None = None) -> tuple[np.ndarray, np.ndarray, str]:
        """ROTLEV3B with KMIN = 2 (dvr3d_b200_rotlev3b_pair): the e levels, the f levels of the
        second pass and both printed tables; with paths, the e and f vector files (ZTRAN)."""
        le, lf = np.zeros(20000), np.zeros(20000)
        ne, nf = C.c_int(0), C.c_int(0)
        ln = C.c_size_t(0)
        buf = C.create_string_buffer(1 << 21)
        P = C.POINTER(C.c_double)
        self._check(self._lib.dvr3d_b200_rotlev3b_pair(self._h, deck_text.encode(), str(wave_path).encode(),
                                                       (kvec_path or "").encode(), (kvec2_path or "").encode(),
                                                       le.ctypes.data_as(P), le.size, C.byref(ne),
                                                       lf.ctypes.data_as(P), lf.size, C.byref(nf), buf, len(buf),
                                                       C.byref(ln)))
        return le[:ne.value].copy(), lf[:nf.value].copy(), buf.value.decode()

    def rotlev3(self, deck_text: str, wave_path: str, kvec_path: str | None = None,
                kvec2_path: str | None = None) -> tuple[np.ndarray, np.ndarray, str]:
        """ROTLEV3, z along r1 or r2 (dvr3d_b200_rotlev3): the first set of levels (e for KMIN =
        1, 2; f for KMIN = 0), the f set of KMIN = 2 (empty otherwise) and the printed lists; with
        paths, the vector files (ZTRAN; J = 1 f with KMIN = 0 writes kvec2_path)."""
        le, lf = np.zeros(20000), np.zeros(20000)
        ne, nf = C.c_int(0), C.c_int(0)
        ln = C.c_size_t(0)
        buf = C.create_string_buffer(1 << 21)
        P = C.POINTER(C.c_double)
        self._check(self._lib.dvr3d_b200_rotlev3(self._h, deck_text.encode(), str(wave_path).encode(),
                                                 (kvec_path or "").encode(), (kvec2_path or "").encode(),
                                                 le.ctypes.data_as(P), le.size, C.byref(ne),
                                                 lf.ctypes.data_as(P), lf.size, C.byref(nf), buf, len(buf),
                                                 C.byref(ln)))
        return le[:ne.value].copy(), lf[:nf.value].copy(), buf.value.decode()

    def dipole3(self, deck_text: str, ket_path: str, bra_path: str, dipd=None, dipsa=None,
                tra_path: str | None = None, cap: int = 4096) -> dict:
        """DIPOLE3 (dvr3d_b200_dipole3) on two wavefunction files with a Python dipole plug-in:
        dipd(r1, r2, xcos, nu) -> component nu, or dipsa(q1, q2, cost) -> (dipx, dipy) for the
        reference's own coordinate transform. Returns the energies e1, e2 (Eh), the transition
        moments tz, tx and S(f-i) (neval1 x neval2, a.u.), the sizes and the printed table."""
        if (dipd is None) == (dipsa is None):
            raise ValueError("give exactly one of dipd, dipsa")
        P = C.POINTER(C.c_double)
        e1, e2 = np.zeros(cap), np.zeros(cap)
        tz, tx, si = (np.zeros((cap, cap), order="F") for _ in range(3))
        res = _abi.DipoleResult(cap1=cap, cap2=cap, e1=e1.ctypes.data_as(P), e2=e2.ctypes.data_as(P),
                                tz=tz.ctypes.data_as(P), tx=tx.ctypes.data_as(P), sint=si.ctypes.data_as(P))
        err = []

        def _d(r1, r2, x, nu, u):
            try:
                return float(dipd(r1, r2, x, nu))
            except Exception as e:  # noqa: BLE001 -- reported after the call
                err.append(e)
                return float("nan")

        def _s(px, py, q1, q2, ct, u):
            try:
                dx, dy = dipsa(q1, q2, ct)
                px[0], py[0] = float(dx), float(dy)
            except Exception as e:  # noqa: BLE001
                err.append(e)
                px[0] = py[0] = float("nan")

        f1 = _abi.DIPD_FN(_d) if dipd else _abi.DIPD_FN()
        f2 = _abi.DIPSA_FN(_s) if dipsa else _abi.DIPSA_FN()
        out = C.create_string_buffer(1 << 22)
        ln = C.c_size_t(0)
        rc = self._lib.dvr3d_b200_dipole3(self._h, deck_text.encode(), str(ket_path).encode(),
                                          str(bra_path).encode(), f1, f2, None, (tra_path or "").encode(),
                                          C.byref(res), out, len(out), C.byref(ln))
        if err:
            raise err[0]
        self._check(rc)
        n1, n2 = res.neval1, res.neval2
        return dict(e1=e1[:n1].copy(), e2=e2[:n2].copy(), tz=tz[:n1, :n2].copy(), tx=tx[:n1, :n2].copy(),
                    sint=si[:n1, :n2].copy(), neval1=n1, neval2=n2, j1=res.j1, j2=res.j2, kmin1=res.kmin1,
                    kmin2=res.kmin2, nblocks=res.nblocks, dev_ms=res.dev_ms, flops=res.flops,
                    text=out.value.decode())

    def ozaki_gemm(self, a, b, *, ta: bool = False, tb: bool = False, tri: int = 0, tri_b: int = 0,
                   lower_out: bool = False, alpha: float = 1.0, beta: float = 0.0, c=None,
                   nslice: int = 8) -> np.ndarray:
        """alpha op(a) op(b) + beta c on the int8 tensor cores from Ozaki slices
        (dvr3d_b200_ozaki_gemm); nslice = 0 runs the FP64 DMMA GEMM on the same operands."""
        a = np.asfortranarray(np.asarray(a, dtype=np.float64))
        b = np.asfortranarray(np.asarray(b, dtype=np.float64))
        m, k = (a.shape[1], a.shape[0]) if ta else a.shape
        n = b.shape[0] if tb else b.shape[1]
        if (b.shape[1] if tb else b.shape[0]) != k:
            raise ValueError("op(a) is m x k and op(b) must be k x n")
        if c is None:
            c = np.zeros((m, n), dtype=np.float64, order="F")
        c = np.asfortranarray(np.array(c, dtype=np.float64))
        lda, ldb = a.shape[0], b.shape[0]
        if lda % 2 or ldb % 2:  # even leading dimensions: pad the stored rows
            a = np.asfortranarray(np.vstack([a, np.zeros((lda % 2, a.shape[1]))]))
            b = np.asfortranarray(np.vstack([b, np.zeros((ldb % 2, b.shape[1]))]))
            lda, ldb = a.shape[0], b.shape[0]
        dp = C.POINTER(C.c_double)
        self._check(self._lib.dvr3d_b200_ozaki_gemm(
            self._h, int(ta), int(tb), int(tri), int(tri_b), int(lower_out), m, n, k, float(alpha),
            a.ctypes.data_as(dp), lda, b.ctypes.data_as(dp), ldb, float(beta), c.ctypes.data_as(dp), max(m, 1),
            int(nslice)))
        return c

    def split_gemm(self, a, b, nslice: int = 2) -> np.ndarray:
        """a^T b on the tensor cores from split-BF16 operands (dvr3d_b200_split_gemm):
        a is k x m, b is k x n (FP64); nslice 1 = one BF16 product, 2 = BF16x3."""
        a = np.asfortranarray(np.asarray(a, dtype=np.float64))
        b = np.asfortranarray(np.asarray(b, dtype=np.float64))
        if a.ndim != 2 or b.ndim != 2 or a.shape[0] != b.shape[0]:
            raise ValueError("a (k x m) and b (k x n) must share k")
        k, m = a.shape
        n = b.shape[1]
        c = np.zeros((m, n), dtype=np.float64, order="F")
        dp = C.POINTER(C.c_double)
        self._check(self._lib.dvr3d_b200_split_gemm(
            self._h, m, n, k, a.ctypes.data_as(dp), k, b.ctypes.data_as(dp), k, int(nslice),
            c.ctypes.data_as(dp), max(m, 1)))
        return c

    def set_pes(self, params) -> None:
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float64))
        if p.size != DVR3D_PES_MORSE_SUM_NPARAM:
            raise ValueError("MORSE_SUM takes 13 parameters")
        self._check(self._lib.dvr3d_b200_set_pes(
            self._h, DVR3D_PES_MORSE_SUM, p.ctypes.data_as(C.POINTER(C.c_double)), p.size))

    def set_pes_grid(self, table) -> None:
        t = np.ascontiguousarray(np.asarray(table, dtype=np.float64).ravel())
        self._check(self._lib.dvr3d_b200_set_pes_grid(
            self._h, t.ctypes.data_as(C.POINTER(C.c_double)), t.size))

    def set_pes_grid_k(self, kz: int, table) -> None:
        """The PES table of k block kz alone, on that block's grid (dvr3d_b200_set_pes_grid_k);
        an empty table removes it."""
        t = np.ascontiguousarray(np.asarray(table, dtype=np.float64).ravel())
        self._check(self._lib.dvr3d_b200_set_pes_grid_k(
            self._h, int(kz), t.ctypes.data_as(C.POINTER(C.c_double)), t.size))

    def grid(self, deck: Deck, kk: int = 0):
        r1 = np.zeros(256)
        r2 = np.zeros(256)
        xa = np.zeros(512)
        dp = C.POINTER(C.c_double)
        self._check(self._lib.dvr3d_b200_grid(self._h, C.byref(deck), kk, r1.ctypes.data_as(dp), 256,
                                              r2.ctypes.data_as(dp), 256, xa.ctypes.data_as(dp), 512))
        n1 = deck.npnt2 if deck.idia == -2 else deck.npnt1
        n2 = deck.npnt2
        na = deck.nalf // 2 if deck.idia == 2 else deck.nalf
        return r1[:n1].copy(), r2[:n2].copy(), xa[:na].copy()

    def solve(self, deck: Deck, kk: int | None = None, *, precision: int = DVR3D_PREC_FP64,
              nlevels: int = 0, tol_cm: float = 0.0, max_iter: int = 0, block: int = 0,
              learned_precond: int = 0, want_vectors: bool = False, want_h3: bool = False,
              want_resid: bool = False) -> SolveResult:
        """Solve one k block (dvr3d_b200_solve_block)."""
        if kk is None:
            kk = k_blocks(deck)[0]
        neval = max(int(deck.neval), 10, int(nlevels))
        nalf = max(int(deck.nalf), int(deck.npnt1), int(deck.npnt2), 1)
        ev = np.zeros(neval + 8)
        iv2 = np.zeros(nalf + 8, dtype=np.int32)
        r = Result()
        r.eval = ev.ctypes.data_as(C.POINTER(C.c_double))
        r.eval_cap = ev.size
        r.iv2 = iv2.ctypes.data_as(C.POINTER(C.c_int))
        r.iv2_cap = iv2.size
        rs = None
        if want_resid:
            rs = np.zeros(neval + 8)
            r.resid = rs.ctypes.data_as(C.POINTER(C.c_double))
            r.resid_cap = rs.size
        o = Options(precision=precision, nlevels=nlevels, tol_cm=tol_cm, max_iter=max_iter,
                    block=block, learned_precond=int(learned_precond),
                    want_vectors=int(want_vectors), want_h3=int(want_h3))
        h3 = evec = None
        if want_h3 or want_vectors:
            # size is only known after the 2D stage: solve once to learn N, then allocate
            probe = self.solve(deck, kk, precision=precision, nlevels=nlevels, tol_cm=tol_cm,
                               max_iter=max_iter, block=block, learned_precond=learned_precond)
            n = probe.nham3
            m = len(probe.eval)
            if want_h3:
                h3 = np.zeros((n, n), order="F")
                r.h3 = h3.ctypes.data_as(C.POINTER(C.c_double))
                r.h3_cap = h3.size
            if want_vectors:
                evec = np.zeros((n, max(m, 1)), order="F")
                r.evec = evec.ctypes.data_as(C.POINTER(C.c_double))
                r.evec_cap = evec.size
        self._check(self._lib.dvr3d_b200_solve_block(self._h, C.byref(deck), kk, C.byref(o), C.byref(r)))
        m = r.meval
        return SolveResult(eval=ev[:m].copy(), nham3=r.nham3, iv2=iv2[:r.nblocks].copy(), kz=r.kz,
                           ipar=r.ipar, stage_ms=np.array(r.stage_ms[:]), max_resid=r.max_resid,
                           iterations=r.iterations, fallback=r.fallback,
                           resid=None if rs is None else rs[:m].copy(),
                           evec=None if evec is None else evec[:, :m], h3=h3, extra=_counters(r))

    # ---- learned Davidson preconditioner
    def lp_get_weights(self) -> np.ndarray:
        w = np.zeros(DVR3D_LP_NPARAM)
        rc = self._lib.dvr3d_b200_lp_get_weights(self._h, w.ctypes.data_as(C.POINTER(C.c_double)), w.size)
        if rc < 0:
            self._check(rc)
        return w

    def lp_set_weights(self, w) -> None:
        w = np.ascontiguousarray(np.asarray(w, dtype=np.float64))
        self._check(self._lib.dvr3d_b200_lp_set_weights(self._h, w.ctypes.data_as(C.POINTER(C.c_double)), w.size))

    def lp_eval(self, w, lam, f1, f2, f3, scale, theta, delta) -> tuple[np.ndarray, np.ndarray]:
        """Network outputs g (nmode x ncol) and sum(delta * dg/dw), by the device kernels."""
        P = C.POINTER(C.c_double)
        arr = [np.ascontiguousarray(np.asarray(x, dtype=np.float64)) for x in (w, lam, f1, f2, f3, theta)]
        d = np.asfortranarray(np.asarray(delta, dtype=np.float64))
        nmode, ncol = d.shape
        g = np.zeros((nmode, ncol), order="F")
        grad = np.zeros(DVR3D_LP_NPARAM)
        self._check(self._lib.dvr3d_b200_lp_eval(
            self._h, arr[0].ctypes.data_as(P), nmode, ncol, arr[1].ctypes.data_as(P), arr[2].ctypes.data_as(P),
            arr[3].ctypes.data_as(P), arr[4].ctypes.data_as(P), float(scale), arr[5].ctypes.data_as(P),
            d.ctypes.data_as(P), g.ctypes.data_as(P), grad.ctypes.data_as(P)))
        return g, grad

    def lp_train_loss(self, w, want_grad: bool = True) -> tuple[float, np.ndarray | None]:
        P = C.POINTER(C.c_double)
        w = np.ascontiguousarray(np.asarray(w, dtype=np.float64))
        loss = np.zeros(1)
        grad = np.zeros(DVR3D_LP_NPARAM) if want_grad else None
        self._check(self._lib.dvr3d_b200_lp_train_loss(self._h, w.ctypes.data_as(P), loss.ctypes.data_as(P),
                                                       grad.ctypes.data_as(P) if want_grad else None))
        return float(loss[0]), grad

    def solve_batch(self, decks: list[Deck], pes_rows, precision: int = DVR3D_PREC_FP64,
                    nlevels: int = 0) -> list[SolveResult]:
        n = len(decks)
        arr = (Deck * n)(*decks)
        P = np.ascontiguousarray(np.asarray(pes_rows, dtype=np.float64).reshape(n, DVR3D_PES_MORSE_SUM_NPARAM))
        res = (Result * n)()
        bufs = []
        for i, d in enumerate(decks):
            ev = np.zeros(max(d.neval, 10) + 8)
            iv2 = np.zeros(max(d.nalf, d.npnt1, d.npnt2) + 8, dtype=np.int32)
            bufs.append((ev, iv2))
            res[i].eval = ev.ctypes.data_as(C.POINTER(C.c_double))
            res[i].eval_cap = ev.size
            res[i].iv2 = iv2.ctypes.data_as(C.POINTER(C.c_int))
            res[i].iv2_cap = iv2.size
        o = Options(precision=precision, nlevels=nlevels)
        self._check(self._lib.dvr3d_b200_solve_batch(self._h, arr, P.ctypes.data_as(C.POINTER(C.c_double)), n,
                                                     C.byref(o), res))
        out = []
        for i in range(n):
            ev, iv2 = bufs[i]
            r = res[i]
            out.append(SolveResult(eval=ev[:r.meval].copy(), nham3=r.nham3, iv2=iv2[:r.nblocks].copy(),
                                   kz=r.kz, ipar=r.ipar, stage_ms=np.array(r.stage_ms[:]),
                                   max_resid=r.max_resid))
        return out

    def run_deck(self, text: str, precision: int = DVR3D_PREC_FP64, wave_path: str | None = None) -> tuple[str, str]:
        """Run a job like program DVR3DRJZ; returns (printed output, fort.14 levels text).
        With wave_path (and ZTRAN in the deck) the wavefunction file is written there."""
        o = Options(precision=precision)
        need = C.c_size_t(0)
        needl = C.c_size_t(0)
        # the first call sizes the text buffers (and writes no wavefunction file)
        self._check(self._lib.dvr3d_b200_run_deck(self._h, text.encode(), C.byref(o), None, 0, C.byref(need),
                                                  None, 0, C.byref(needl)))
        out = C.create_string_buffer(need.value + 1)
        lev = C.create_string_buffer(needl.value + 1)
        if wave_path is None:
            self._check(self._lib.dvr3d_b200_run_deck(self._h, text.encode(), C.byref(o), out, len(out),
                                                      C.byref(need), lev, len(lev), C.byref(needl)))
        else:
            self._check(self._lib.dvr3d_b200_run_deck_wave(self._h, text.encode(), C.byref(o), out, len(out),
                                                           C.byref(need), lev, len(lev), C.byref(needl),
                                                           str(wave_path).encode()))
        return out.value.decode(), lev.value.decode()
