"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Tolerance: the plain FP64 path must reproduce the oracle's levels to 1e-6 cm-1
(4.6e-12 Eh); selection counts per block must be identical.
"""
from __future__ import annotations

import numpy as np
import pytest

import dvr3d_b200
from dvr3d_b200 import AUTOCM, configs, parse_deck

pytestmark = pytest.mark.gpu

TOL_CM = 1e-6


def _compare(ctx, oracle_mod, w, kk=None, tol_cm=TOL_CM, check_resid=True):
    # each side reads the deck text with its own reader
    d = parse_deck(w.deck)
    ks = dvr3d_b200.k_blocks(d) if kk is None else [kk]
    assert ks == oracle_mod.k_blocks(w.deck)
    for k in ks:
        ref = oracle_mod.solve(w.deck, k, pes=w.pes, final_mode=1)
        assert ref.status == 0, ref.status
        ctx.set_pes(w.pes)
        got = ctx.solve(d, k, want_resid=check_resid)
        assert got.nham3 == ref.nham3
        np.testing.assert_array_equal(got.iv2, ref.iv2)
        assert len(got.eval) == len(ref.eval)
        err = np.abs(got.eval - ref.eval) * AUTOCM
        assert err.max() <= tol_cm, f"k={k}: max level error {err.max():.3e} cm-1"
        if check_resid:
            assert got.max_resid < 1e-9, got.max_resid
    return got


def test_radau_small_cut(ctx, oracle_mod):
    w = configs.radau_water_like(12, 16, 30000.0, 40, title="radau small")
    _compare(ctx, oracle_mod, w)


def test_radau_small_choosr(ctx, oracle_mod):
    w = configs.radau_water_like(13, 18, 0.0, 30, max3d=150, zcut=False, title="radau choosr")
    _compare(ctx, oracle_mod, w)


def test_radau_odd_parity(ctx, oracle_mod):
    w = configs.radau_water_like(12, 14, 35000.0, 30, title="radau odd")
    d = parse_deck(w.deck)
    txt = w.deck.splitlines()
    card3 = list(txt[2])
    # ipar = 1 (columns 46-50)
    card3[45:50] = list(f"{1:5d}")
    txt[2] = "".join(card3)
    w.deck = "\n".join(txt) + "\n"
    assert parse_deck(w.deck).ipar == 1
    _compare(ctx, oracle_mod, w)


def test_jacobi_theta_last_small(ctx, oracle_mod):
    w = configs.jacobi_h3p_like(10, 12, 16, 45000.0, 40000.0, 40, title="jacobi small")
    _compare(ctx, oracle_mod, w)


def test_jacobi_theta_last_r1_first(ctx, oracle_mod):
    w = configs.jacobi_h3p_like(11, 9, 14, 45000.0, 40000.0, 30, title="jacobi r1 first")
    w.deck = w.deck.replace("ZR2R1=.TRUE.", "ZR2R1=.FALSE.")
    _compare(ctx, oracle_mod, w)


def test_jacobi_theta_first(ctx, oracle_mod):
    w = configs.jacobi_h3p_like(9, 10, 16, 40000.0, 45000.0, 30, title="jacobi theta first")
    w.deck = w.deck.replace("ZTHETA=.FALSE.", "ZTHETA=.TRUE.")
    _compare(ctx, oracle_mod, w)


def test_jacobi_choose(ctx, oracle_mod):
    w = configs.jacobi_h3p_like(10, 10, 12, 50000.0, 0.0, 30, max3d=300, title="jacobi choose")
    w.deck = w.deck.replace("ZCUT=.TRUE.", "ZCUT=.FALSE.")
    _compare(ctx, oracle_mod, w)


def test_jacobi_j1_k_blocks(ctx, oracle_mod):
    """J=1 first step (zrot): k = 0 and 1 blocks with associated-Legendre grids."""
    w = configs.jacobi_h3p_like(9, 10, 14, 45000.0, 40000.0, 20, title="jacobi J1")
    lines = w.deck.splitlines()
    c3 = list(lines[2])
    c3[5:10] = list(f"{1:5d}")     # jrot = 1
    c3[35:40] = list(f"{1:5d}")    # kmin = 1
    lines[2] = "".join(c3)
    w.deck = "\n".join(lines).replace("ZPMIN=.TRUE.", "ZPMIN=.TRUE., ZROT=.TRUE.") + "\n"
    _compare(ctx, oracle_mod, w)


def test_config1_full_size(ctx, oracle_mod):
    got = _compare(ctx, oracle_mod, configs.config1())
    assert got.nham3 > 800


def test_h3_assembly_matches_oracle(ctx, oracle_mod):
    w = configs.radau_water_like(10, 12, 30000.0, 20, title="radau h3")
    d = parse_deck(w.deck)
    ref = oracle_mod.solve(w.deck, 0, pes=w.pes, final_mode=2, want_h3=True)
    ctx.set_pes(w.pes)
    got = ctx.solve(d, 0, want_h3=True)
    n = ref.nham3
    assert got.nham3 == n
    h_ref = np.tril(ref.h3)
    h_got = np.tril(got.h3)
    # basis vectors may differ in sign (eigenvector sign convention): compare magnitudes
    np.testing.assert_allclose(np.diag(h_got), np.diag(h_ref), rtol=0, atol=1e-12)
    np.testing.assert_allclose(np.abs(h_got), np.abs(h_ref), rtol=0, atol=1e-11)
    # and the spectrum is invariant
    np.testing.assert_allclose(np.linalg.eigvalsh(got.h3), np.linalg.eigvalsh(ref.h3 + np.tril(ref.h3, -1).T),
                               rtol=0, atol=1e-11)


def test_pes_grid_table_equals_closed_form(ctx, oracle_mod):
    w = configs.jacobi_h3p_like(8, 9, 12, 45000.0, 40000.0, 20, title="grid pes")
    d = parse_deck(w.deck)
    r1, r2, xa = dvr3d_b200.host_grid(d, 0)
    tab = np.empty((len(xa), len(r2), len(r1)))
    for ia, x in enumerate(xa):
        for i2, b in enumerate(r2):
            for i1, a in enumerate(r1):
                tab[ia, i2, i1] = oracle_mod.pes_morse_sum(w.pes, a, b, x)
    ctx.set_pes(w.pes)
    a = ctx.solve(d, 0)
    ctx.set_pes_grid(tab)
    b = ctx.solve(d, 0)
    np.testing.assert_allclose(b.eval, a.eval, rtol=0, atol=1e-13)
    ref = oracle_mod.solve(w.deck, 0, vgrid=tab, final_mode=1)
    np.testing.assert_allclose(b.eval, ref.eval, rtol=0, atol=TOL_CM / AUTOCM)
    ctx.set_pes(w.pes)


def test_errors_are_codes_not_exits(ctx):
    w = configs.radau_water_like(12, 16, 45000.0, 40, max3d=50, title="overflow")
    d = parse_deck(w.deck)
    ctx.set_pes(w.pes)
    with pytest.raises(dvr3d_b200.DVR3DError) as e:
        ctx.solve(d, 0)
    assert e.value.code == -3  # DVR3D_ERR_CORE_MAX3D
    # context still usable afterwards
    ok = configs.radau_water_like(10, 12, 30000.0, 20, title="after error")
    ctx.solve(parse_deck(ok.deck), 0)


# ---------------------------------------------------------------- iterative (shift-invert Krylov) path
TOL_MIXED_CM = 1e-3  # bar of the iterative path against the plain FP64 GPU path


def _mixed_vs_dense(ctx, w, expect_fallback=False):
    d = parse_deck(w.deck)
    ctx.set_pes(w.pes)
    a = ctx.solve(d, 0)
    b = ctx.solve(d, 0, precision=dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON, want_resid=True)
    assert b.nham3 == a.nham3 and len(b.eval) == len(a.eval)
    assert b.fallback == int(expect_fallback)
    err = np.abs(b.eval - a.eval) * AUTOCM
    assert err.max() <= TOL_MIXED_CM, f"max level error {err.max():.3e} cm-1"
    assert b.max_resid < 1e-5
    if not expect_fallback:
        assert b.iterations > 0
    return a, b, err


def test_mixed_small_basis_falls_back_to_dense(ctx):
    """config 1 (N=924, 200 levels): the Krylov space would exceed the basis -> dense FP64."""
    _mixed_vs_dense(ctx, configs.config1(), expect_fallback=True)


def test_mixed_jacobi_medium_many_levels(ctx):
    _, b, err = _mixed_vs_dense(ctx, configs.jacobi_h3p_like(20, 20, 32, 50000.0, 45000.0, 300, title="jacobi medium"))
    assert b.nham3 > 4000


def test_mixed_radau_config2(ctx):
    _mixed_vs_dense(ctx, configs.config2())


def test_mixed_config4_500_levels(ctx):
    a, b, err = _mixed_vs_dense(ctx, configs.config4())
    assert b.nham3 > 12000 and len(b.eval) == 500


# ---------------------------------------------------------------- full-size workloads vs the oracle
# tests/golden/config{2,4}_oracle.npz: the oracle's N, per-block selection counts and levels of
# the benchmark's workloads (made by tests/golden/make_config_fixtures.py: the oracle needs
# minutes at these sizes). Plain FP64 path: identical counts, levels within 1e-6 cm-1;
# the chosen (iterative) form: within 1e-3 cm-1.
def _fixture(k):
    from pathlib import Path

    f = np.load(Path(__file__).resolve().parent / "golden" / f"config{k}_oracle.npz")
    return {q: f[q] for q in f.files}


@pytest.mark.parametrize("k", [2, 4])
def test_full_size_workload_matches_oracle_fixture(ctx, k):
    fx = _fixture(k)
    w = {2: configs.config2, 4: configs.config4}[k]()
    assert str(fx["deck"]) == w.deck and np.array_equal(fx["pes"], w.pes)
    d = parse_deck(w.deck)
    ctx.set_pes(w.pes)
    nlev = len(fx["levels"])
    plain = ctx.solve(d, 0, nlevels=nlev)
    assert plain.nham3 == int(fx["nham3"])
    np.testing.assert_array_equal(plain.iv2, fx["iv2"])
    err = np.abs(plain.eval - fx["levels"]) * AUTOCM
    assert err.max() <= TOL_CM, f"plain path: max level error {err.max():.3e} cm-1"
    mixed = ctx.solve(d, 0, nlevels=nlev, precision=dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON)
    np.testing.assert_array_equal(mixed.iv2, fx["iv2"])
    err_m = np.abs(mixed.eval - fx["levels"]) * AUTOCM
    assert err_m.max() <= TOL_MIXED_CM, f"chosen form: max level error {err_m.max():.3e} cm-1"
