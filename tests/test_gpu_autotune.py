"""The autotuned split-K of the Krylov triangular products (chosen by timing the candidates on
the first solve of a shape in a context): the levels do not depend on the choice, and the
fixed rule (DVR3D_NO_AUTOTUNE=1) gives the same levels to rounding."""
from __future__ import annotations

import numpy as np
import pytest

import dvr3d_b200
from dvr3d_b200 import AUTOCM, configs, parse_deck

pytestmark = pytest.mark.gpu


def test_autotuned_split_keeps_levels(ctx, monkeypatch):
    w = configs.jacobi_h3p_like(16, 16, 30, 50000.0, 45000.0, 120, title="autotune")
    d = parse_deck(w.deck)
    ctx.set_pes(w.pes)
    M = dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON
    plain = ctx.solve(d, 0)
    tuned = ctx.solve(d, 0, precision=M)
    again = ctx.solve(d, 0, precision=M)
    assert tuned.extra["path"] == dvr3d_b200.DVR3D_PATH_SHIFT_INVERT
    monkeypatch.setenv("DVR3D_NO_AUTOTUNE", "1")
    rule = dvr3d_b200.Context(0)
    try:
        rule.set_pes(w.pes)
        fixed = rule.solve(d, 0, precision=M)
    finally:
        rule.close()
    for r in (tuned, again, fixed):
        assert np.abs(r.eval - plain.eval).max() * AUTOCM <= 1e-6
    assert np.abs(tuned.eval - fixed.eval).max() * AUTOCM <= 1e-7


def test_krylov_steps_replayed_as_a_graph_give_the_same_levels(ctx, monkeypatch):
    """The Krylov block steps between two checks run as one captured CUDA graph, replayed by
    later solves of the same shape: the levels equal those of the step-by-step launches."""
    w = configs.jacobi_h3p_like(16, 16, 30, 50000.0, 45000.0, 120, title="graph")
    d = parse_deck(w.deck)
    ctx.set_pes(w.pes)
    M = dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON
    first = ctx.solve(d, 0, precision=M)   # captures (unless an earlier solve of this shape did)
    replay = ctx.solve(d, 0, precision=M)  # replays
    again = ctx.solve(d, 0, precision=M)
    assert first.extra["path"] == dvr3d_b200.DVR3D_PATH_SHIFT_INVERT
    np.testing.assert_array_equal(first.eval, replay.eval)
    np.testing.assert_array_equal(again.eval, replay.eval)
    assert replay.extra["launches"] == again.extra["launches"]
    monkeypatch.setenv("DVR3D_NO_GRAPH", "1")
    direct = ctx.solve(d, 0, precision=M)
    np.testing.assert_array_equal(direct.eval, replay.eval)


def test_learned_preconditioner_beyond_32_levels(ctx):
    """The channel-block preconditioner with its learned correction in a Davidson solve of 64
    levels (split-BF16 form): trained on one solve, applied to the next, same levels, no more
    products than the untrained correction."""
    w = configs.radau_water_like(18, 30, 32000.0, 64, title="lp64")
    d = parse_deck(w.deck)
    ctx.set_pes(w.pes)
    S = dvr3d_b200.DVR3D_PREC_SPLIT_BF16
    plain = ctx.solve(d, 0, nlevels=64)
    trained = ctx.solve(d, 0, precision=S, nlevels=64, learned_precond=2)
    assert trained.extra["lp_pairs"] > 0 and trained.extra["lp_loss_last"] <= trained.extra["lp_loss_first"]
    base = ctx.solve(d, 0, precision=S, nlevels=64, learned_precond=0)
    reuse = ctx.solve(d, 0, precision=S, nlevels=64, learned_precond=1)
    for r in (trained, base, reuse):
        assert r.fallback == 0 and r.extra["path"] == dvr3d_b200.DVR3D_PATH_DAVIDSON
        assert np.abs(r.eval - plain.eval).max() * AUTOCM <= 1e-3
    assert reuse.extra["matvecs"] <= base.extra["matvecs"]


def test_band_bisection_agrees_with_the_bulge_chase(ctx, monkeypatch):
    """The projected band of the shift-invert Rayleigh-Ritz step solved two independent ways:
    the bulge chase to tridiagonal form (default) and Sturm-count bisection with inverse
    iteration on band LDL^T factors (DVR3D_BAND_EIG=bisect, no reduction). Same levels to
    rounding; both within 1e-6 cm-1 of the plain FP64 path."""
    w = configs.jacobi_h3p_like(16, 16, 30, 50000.0, 45000.0, 120, title="band eig")
    d = parse_deck(w.deck)
    ctx.set_pes(w.pes)
    M = dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON
    plain = ctx.solve(d, 0)
    chase = ctx.solve(d, 0, precision=M)
    monkeypatch.setenv("DVR3D_BAND_EIG", "bisect")
    bis = ctx.solve(d, 0, precision=M)
    assert bis.extra["path"] == dvr3d_b200.DVR3D_PATH_SHIFT_INVERT and bis.fallback == 0
    assert np.abs(bis.eval - chase.eval).max() * AUTOCM <= 1e-7
    for r in (chase, bis):
        assert np.abs(r.eval - plain.eval).max() * AUTOCM <= 1e-6
