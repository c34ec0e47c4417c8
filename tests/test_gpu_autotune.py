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
