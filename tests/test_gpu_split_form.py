"""The split-BF16 form (DVR3D_PREC_SPLIT_BF16): contracted-Hamiltonian assembly and H3 V as
BF16x3 tensor-core products with FP32 accumulation, FP64 Rayleigh-Ritz and residual norms,
and the FP64 residual correction through the matrix-free operator of the contracted basis.

* The split matrix the products use (hi + lo) against the FP64-assembled H3 of the plain path.
* Every level against the FP64 oracle: a small Radau case computed by the oracle here, and the
  300 levels of the N ~ 4000 Radau workload against its committed oracle fixture
  (tests/golden/config2_oracle.npz), within 1e-3 cm-1; the tensor-core products must have
  done part of the work (low_matvecs > 0) and the levels come from the Davidson path.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import dvr3d_b200
from dvr3d_b200 import AUTOCM, configs, parse_deck

pytestmark = pytest.mark.gpu

S = dvr3d_b200.DVR3D_PREC_SPLIT_BF16
TOL_CM = 1e-3
FIX2 = Path(__file__).resolve().parent / "golden" / "config2_oracle.npz"


def test_split_assembly_matches_fp64_assembly(ctx):
    w = configs.radau_water_like(14, 20, 30000.0, 30, title="split assembly")
    d = parse_deck(w.deck)
    ctx.set_pes(w.pes)
    plain = ctx.solve(d, 0, want_h3=True)
    split = ctx.solve(d, 0, precision=S, want_h3=True)
    assert split.nham3 == plain.nham3
    h64, hs = plain.h3, split.h3
    # BF16x3 products (relative 2^-16 of |C|^T |C|) and the split storage (2^-17 of |H|)
    rel = np.linalg.norm(hs - h64) / np.linalg.norm(h64)
    assert 0.0 < rel <= 2.0 ** -13, rel
    assert np.abs(hs - hs.T).max() == 0.0


def test_split_form_small_radau_against_oracle(ctx, oracle_mod):
    w = configs.radau_water_like(16, 24, 35000.0, 40, title="split small")
    ctx.set_pes(w.pes)
    got = ctx.solve(parse_deck(w.deck), 0, precision=S)
    ref = oracle_mod.solve(w.deck, 0, pes=w.pes, final_mode=1)
    assert ref.status == 0 and got.nham3 == ref.nham3
    np.testing.assert_array_equal(got.iv2, ref.iv2)
    assert got.fallback == 0 and got.extra["path"] == dvr3d_b200.DVR3D_PATH_DAVIDSON
    assert got.extra["low_matvecs"] > 0 and got.extra["low_iterations"] > 0
    err = np.abs(got.eval - ref.eval[:len(got.eval)]).max() * AUTOCM
    assert err <= TOL_CM, f"{err:.3e} cm-1"


def test_split_form_300_levels_against_oracle_fixture(ctx):
    f = np.load(FIX2)
    w = configs.config2()
    assert str(f["deck"]) == w.deck and np.array_equal(f["pes"], w.pes)
    ctx.set_pes(w.pes)
    got = ctx.solve(parse_deck(w.deck), 0, precision=S)
    assert got.nham3 == int(f["nham3"])
    np.testing.assert_array_equal(got.iv2, f["iv2"])
    lv = f["levels"]
    assert len(got.eval) == len(lv) == 300
    assert got.fallback == 0 and got.extra["low_matvecs"] > 0
    err = np.abs(got.eval - lv) * AUTOCM
    assert err.max() <= TOL_CM, f"max {err.max():.3e} cm-1 at level {int(err.argmax())}"
