"""Config 5: Jacobi J = 2 (k = 0, 1, 2 blocks), H/C/N masses, N ~ 20500 per k block, the
lowest 1000 levels of each block (dvr3d_b200/configs.py:config5).

* Against the oracle's fixture of the same workload (tests/golden/config5_oracle.npz, made by
  make_config_fixtures.py): per k block identical selection counts and N, the plain FP64
  path within 1e-6 cm-1 and the chosen (shift-invert) form within 1e-3 cm-1.
* The learned Davidson preconditioner trained on k = 0 (learned_precond = 2) and reused for
  k = 1 and 2 (learned_precond = 1): the same levels as without it, no more H3 products.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import dvr3d_b200
from dvr3d_b200 import AUTOCM, configs, parse_deck

pytestmark = pytest.mark.gpu

FIX = Path(__file__).resolve().parent / "golden" / "config5_oracle.npz"


@pytest.fixture(scope="module")
def cfg5():
    f = np.load(FIX)
    w = configs.config5()
    assert str(f["deck"]) == w.deck and np.array_equal(f["pes"], w.pes)
    return w, {k: f[k] for k in f.files}


@pytest.mark.parametrize("k", [0, 1, 2])
def test_config5_k_block_matches_oracle(ctx, cfg5, k):
    w, fx = cfg5
    d = parse_deck(w.deck)
    assert dvr3d_b200.k_blocks(d) == [0, 1, 2]
    ctx.set_pes(w.pes)
    plain = ctx.solve(d, k)
    assert plain.nham3 == int(fx[f"nham3_k{k}"]) > 20000
    np.testing.assert_array_equal(plain.iv2, fx[f"iv2_k{k}"])
    lv = fx[f"levels_k{k}"]
    assert len(plain.eval) == len(lv) == 1000
    err = np.abs(plain.eval - lv).max() * AUTOCM
    assert err <= 1e-6, f"plain path, k={k}: {err:.3e} cm-1"
    mixed = ctx.solve(d, k, precision=dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON)
    assert mixed.extra["path"] == dvr3d_b200.DVR3D_PATH_SHIFT_INVERT and mixed.fallback == 0
    err_m = np.abs(mixed.eval - lv).max() * AUTOCM
    assert err_m <= 1e-3, f"chosen form, k={k}: {err_m:.3e} cm-1"


def test_config5_preconditioner_trained_on_k0_reused_for_k1_k2(ctx, cfg5):
    w, fx = cfg5
    d = parse_deck(w.deck)
    ctx.set_pes(w.pes)
    M = dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON
    nl = 24
    trained = ctx.solve(d, 0, precision=M, nlevels=nl, learned_precond=2)
    assert trained.extra["lp_pairs"] > 0 and trained.extra["path"] == dvr3d_b200.DVR3D_PATH_DAVIDSON
    assert trained.extra["lp_loss_last"] <= trained.extra["lp_loss_first"]
    for k in (1, 2):
        base = ctx.solve(d, k, precision=M, nlevels=nl, learned_precond=0)
        reuse = ctx.solve(d, k, precision=M, nlevels=nl, learned_precond=1)
        assert reuse.fallback == 0 and base.fallback == 0
        assert reuse.extra["matvecs"] <= base.extra["matvecs"]
        lv = fx[f"levels_k{k}"][:nl]
        assert np.abs(reuse.eval - lv).max() * AUTOCM <= 1e-3
        assert np.abs(base.eval - lv).max() * AUTOCM <= 1e-3


def test_config5_split_form_k1_against_oracle(ctx, cfg5):
    """The split-BF16 form (BF16x3 assembly and products, FP64 residual correction) on the
    N ~ 20500 block k = 1: the lowest 24 levels within 1e-3 cm-1 of the oracle."""
    w, fx = cfg5
    d = parse_deck(w.deck)
    ctx.set_pes(w.pes)
    r = ctx.solve(d, 1, precision=dvr3d_b200.DVR3D_PREC_SPLIT_BF16, nlevels=24)
    assert r.fallback == 0 and r.extra["low_matvecs"] > 0
    assert np.abs(r.eval - fx["levels_k1"][:24]).max() * AUTOCM <= 1e-3
