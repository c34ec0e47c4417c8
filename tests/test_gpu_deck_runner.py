"""GPU tests of the whole-job runner and of failure reporting, through the C ABI.

* dvr3d_b200_run_deck against text that the oracle's levels give through the reference's
  format statements: the level tables of diag3d (format 1020, 5d24.12/, :2703-2730), the band
  origins (format 1021, 5f15.6/, :2748-2761) and the fort.14 levels file of zpfun (formats
  1125 6i4 and 1126 4d20.12, :2708-2719), for J = 0 and for J = 2 k blocks.
* Radau J > 0 with the bisector embedding (testiv, :3380-3451) against the oracle per k block.
* Bounded device waits that are made to run out (a poll limit of one) end the solve with
  DVR3D_ERR_NOCONV and leave the context usable.
* Inverse iteration that cannot converge (a block with a non-finite entry) is reported as
  DVR3D_ERR_NOCONV by the batched eigensolver instead of returning NaN vectors.
"""
from __future__ import annotations

import math
import re

import numpy as np
import pytest

import dvr3d_b200
from dvr3d_b200 import AUTOCM, configs, parse_deck

pytestmark = pytest.mark.gpu

TOL_CM = 1e-6


def fortran_d(x: float, w: int, d: int) -> str:
    """Fortran Dw.d output (0.ddddD+ee, right-justified in w columns)."""
    if x == 0.0:
        s = "0." + "0" * d + "D+00"
    else:
        e = math.floor(math.log10(abs(x))) + 1
        m = round(abs(x) / 10.0 ** e, d)
        if m >= 1.0:
            m /= 10.0
            e += 1
        s = ("-" if x < 0 else "") + f"{m:.{d}f}" + ("D+" if e >= 0 else "D-") + f"{abs(e):02d}"
    return s.rjust(w)


def table(vals, per: int, fmt) -> list[str]:
    """Rows of a Fortran '(<per><fmt>/)' write: `per` values a line, then an empty line."""
    out = []
    for i in range(0, len(vals), per):
        out.append("".join(fmt(v) for v in vals[i:i + per]))
        out.append("")
    return out


def numbers(lines):
    return np.array([float(t.replace("D", "E")) for ln in lines for t in ln.split()])


def section(text: str, header: str) -> list[str]:
    """Lines after `header` up to the next header line (one containing letters)."""
    lines = text.splitlines()
    i = next(k for k, ln in enumerate(lines) if header in ln)
    out = []
    for ln in lines[i + 1:]:
        if re.search(r"[A-Za-z]", ln.replace("D+", "").replace("D-", "")):
            break
        out.append(ln)
    while out and not out[0].strip():
        out.pop(0)
    while out and not out[-1].strip():
        out.pop()
    return out


def oracle_levels(oracle_mod, w, k):
    ref = oracle_mod.solve(w.deck, k, pes=w.pes, final_mode=1)
    assert ref.status == 0
    return ref


def expected_fort14(oracle_mod, w) -> str:
    """fort.14 of zpfun from the oracle's levels, written as diag3d writes it: a block for
    every k when jrot = 0 or jrot - kmin = 1 (:2708-2710). Covers J = 0 and J > 0 with the
    rotational k loop of a non-bisector embedding, where insize maps kmin != 0 to 1 (:526)."""
    d = oracle_mod.parse_deck(w.deck)
    jrot = d.jrot
    assert jrot == 0 or (d.zrot and d.idia != -2)
    kmin = 0 if jrot == 0 else (1 if d.kmin != 0 else 0)
    ip = jrot - kmin
    if not (jrot == 0 or ip == 1):
        return ""
    out = []
    for k in oracle_mod.k_blocks(d):
        ref = oracle_levels(oracle_mod, w, k)
        jdia = max(0, d.idia)
        jpar = min(jdia, ref.ipar)
        isym = abs(min(0, d.idia))
        if ref.ipar == 1:
            isym = -isym
        out.append("".join(f"{v:4d}" for v in (jrot, ip, jdia, jpar, isym, len(ref.eval))))
        for i in range(0, len(ref.eval), 4):
            out.append("".join(fortran_d(v, 20, 12) for v in ref.eval[i:i + 4]))
    return "\n".join(out) + "\n"


def test_fortran_d_formatter():
    assert fortran_d(0.0313630673207, 24, 12) == "      0.313630673207D-01"
    assert fortran_d(6304.370931, 20, 12) == "  0.630437093100D+04"
    assert fortran_d(-1.5, 20, 12) == " -0.150000000000D+01"


def test_run_deck_j0_tables_band_origins_and_fort14(ctx, oracle_mod):
    w = configs.radau_water_like(12, 16, 30000.0, 12, title="runner J0")
    w.deck = w.deck.replace("ZPMIN=.TRUE.", "ZPMIN=.FALSE., ZPFUN=.TRUE.")
    ctx.set_pes(w.pes)
    out, lev = ctx.run_deck(w.deck)
    ref = oracle_levels(oracle_mod, w, 0)
    ev = ref.eval
    got_h = section(out, "eigenvalues in hartrees")
    want_h = table(list(ev), 5, lambda v: fortran_d(v, 24, 12))
    while want_h and not want_h[-1]:
        want_h.pop()
    assert len(got_h) == len(want_h)
    np.testing.assert_allclose(numbers(got_h), ev, rtol=0, atol=TOL_CM / AUTOCM)
    # the layout (column widths, 5 a line, blank lines) is the reference's
    assert [len(ln) for ln in got_h] == [len(ln) for ln in want_h]
    got_cm = section(out, "eigenvalues in wavenumbers")
    np.testing.assert_allclose(numbers(got_cm), ev * AUTOCM, rtol=0, atol=TOL_CM)
    got_bo = section(out, "Band origins in wavenumbers")
    want_bo = (ev[1:] - ev[0]) * AUTOCM
    np.testing.assert_allclose(numbers(got_bo), want_bo, rtol=0, atol=2e-6)
    assert [len(ln) for ln in got_bo] == [len(ln) for ln in table(list(want_bo), 5, lambda v: f"{v:15.6f}")[:-1]]
    want14 = expected_fort14(oracle_mod, w)
    assert lev.splitlines()[0] == want14.splitlines()[0]  # header 6i4
    np.testing.assert_allclose(numbers(lev.splitlines()[1:]), ev, rtol=0, atol=TOL_CM / AUTOCM)
    assert [len(ln) for ln in lev.splitlines()] == [len(ln) for ln in want14.splitlines()]


def _jacobi_j2(kmin: int):
    w = configs.jacobi_h3p_like(9, 10, 14, 45000.0, 40000.0, 8, title="runner J2")
    lines = w.deck.splitlines()
    c3 = list(lines[2])
    c3[5:10] = list(f"{2:5d}")      # jrot = 2
    c3[35:40] = list(f"{kmin:5d}")  # kmin
    lines[2] = "".join(c3)
    w.deck = "\n".join(lines).replace("ZPMIN=.TRUE.", "ZPMIN=.TRUE., ZROT=.TRUE., ZPFUN=.TRUE.") + "\n"
    return w


def test_run_deck_j2_writes_fort14_for_every_k_block(ctx, oracle_mod):
    """J = 2, kmin = 1: ip = jrot - kmin = 1, so diag3d writes a fort.14 block for each k."""
    w = _jacobi_j2(1)
    ctx.set_pes(w.pes)
    out, lev = ctx.run_deck(w.deck)
    want = expected_fort14(oracle_mod, w)
    got_lines, want_lines = lev.splitlines(), want.splitlines()
    assert len(got_lines) == len(want_lines) and len(want_lines) > 0
    heads = [i for i, ln in enumerate(want_lines) if "D" not in ln]
    assert len(heads) == 3  # k = 0, 1, 2
    for i, (g, r) in enumerate(zip(got_lines, want_lines)):
        if i in heads:
            assert g == r
        else:
            assert len(g) == len(r)
            np.testing.assert_allclose(numbers([g]), numbers([r]), rtol=0, atol=TOL_CM / AUTOCM)
    assert out.count("Solutions with J =  2 k =") == 3


def test_run_deck_j2_kmin0_writes_no_fort14(ctx, oracle_mod):
    """J = 2, kmin = 0: ip = 2, diag3d skips the levels file (:2710)."""
    w = _jacobi_j2(0)
    ctx.set_pes(w.pes)
    _, lev = ctx.run_deck(w.deck)
    assert lev == "" and expected_fort14(oracle_mod, w) == ""


def test_radau_j1_bisector_embedding_matches_oracle(ctx, oracle_mod):
    """Radau J = 1 with zrot (bisector embedding, testiv): every k block against the oracle."""
    w = configs.radau_water_like(12, 16, 30000.0, 15, title="radau J1")
    lines = w.deck.splitlines()
    c3 = list(lines[2])
    c3[5:10] = list(f"{1:5d}")      # jrot = 1
    c3[35:40] = list(f"{1:5d}")     # kmin = 1
    lines[2] = "".join(c3)
    w.deck = "\n".join(lines).replace("ZPMIN=.TRUE.", "ZPMIN=.TRUE., ZROT=.TRUE.") + "\n"
    d = parse_deck(w.deck)
    ks = dvr3d_b200.k_blocks(d)
    assert ks == oracle_mod.k_blocks(w.deck) and len(ks) == 2
    ctx.set_pes(w.pes)
    for k in ks:
        ref = oracle_levels(oracle_mod, w, k)
        got = ctx.solve(d, k, want_resid=True)
        assert got.nham3 == ref.nham3 and got.kz == ref.kz and got.ipar == ref.ipar
        np.testing.assert_array_equal(got.iv2, ref.iv2)
        err = np.abs(got.eval - ref.eval) * AUTOCM
        assert err.max() <= TOL_CM, f"k={k}: {err.max():.3e} cm-1"
        assert got.max_resid < 1e-9


def test_bounded_waits_run_out_and_context_recovers(ctx):
    """A poll limit of one makes the grid barriers of the dense reduction and the hand-off
    waits of the bulge chase run out: each solve returns DVR3D_ERR_NOCONV; with the default
    limits restored the same context solves both again, with the same levels."""
    w = configs.jacobi_h3p_like(14, 14, 24, 50000.0, 45000.0, 150, title="waits")
    d = parse_deck(w.deck)
    ctx.set_pes(w.pes)
    ref = ctx.solve(d, 0)
    ref_mixed = ctx.solve(d, 0, precision=dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON)
    assert ref_mixed.extra["path"] == dvr3d_b200.DVR3D_PATH_SHIFT_INVERT
    try:
        ctx.set_wait_limit(1)
        for prec in (dvr3d_b200.DVR3D_PREC_FP64, dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON):
            with pytest.raises(dvr3d_b200.DVR3DError) as e:
                ctx.solve(d, 0, precision=prec)
            assert e.value.code == -5  # DVR3D_ERR_NOCONV
    finally:
        ctx.set_wait_limit(0)
    again = ctx.solve(d, 0)
    np.testing.assert_array_equal(again.eval, ref.eval)
    again_mixed = ctx.solve(d, 0, precision=dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON)
    np.testing.assert_allclose(again_mixed.eval, ref_mixed.eval, rtol=0, atol=1e-12)


def test_batched_inverse_iteration_failure_is_reported(ctx):
    """A block with a non-finite entry has no convergent inverse iteration: the batched
    eigensolver returns DVR3D_ERR_NOCONV; finite blocks in the next call are fine."""
    import ctypes as C

    import torch

    from dvr3d_b200 import _abi

    lib = _abi.load_library()
    rng = np.random.default_rng(3)
    n = [40, 33]
    blocks = []
    for m in n:
        a = rng.standard_normal((m, m))
        blocks.append((a + a.T) / 2)
    bad = [b.copy() for b in blocks]
    bad[1][5, 2] = np.nan
    nb = len(n)
    n_arr = (C.c_int * nb)(*n)
    o_arr = (C.c_longlong * nb)(0, n[0] * n[0])
    w_arr = (C.c_longlong * nb)(0, n[0])
    for mats, expect in ((bad, _abi.DVR3D_ERR_NOCONV), (blocks, 0)):
        flat = np.concatenate([b.ravel(order="F") for b in mats])
        a_dev = torch.tensor(flat, dtype=torch.float64, device="cuda")
        w_dev = torch.zeros(sum(n), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.dvr3d_b200_diag_batched(ctx._h, nb, n_arr, o_arr, w_arr, C.c_void_p(a_dev.data_ptr()),
                                         C.c_void_p(w_dev.data_ptr()), 1)
        assert rc == expect
        if expect == 0:
            w = w_dev.cpu().numpy()
            np.testing.assert_allclose(w[:40], np.linalg.eigvalsh(blocks[0]), rtol=0, atol=1e-12)
            np.testing.assert_allclose(w[40:], np.linalg.eigvalsh(blocks[1]), rtol=0, atol=1e-12)
