"""Independent problems solved as one batched workload (dvr3d_b200_solve_batch).

The reference's fitting driver runs DVR3DRJZ once per trial surface
(SFIT_DVR3D/H2S/dvr3d_sfit.f90:746-832). The batch entry point takes many J=0 Radau decks
with their own surfaces and runs the 2D stage of all of them together (one launch per
eigensolver phase over every problem's blocks), then each problem's assembly and final
eigensolve. Each problem must give what the oracle gives for it alone (levels within
1e-6 cm-1, identical per-angle selection counts), and what solve_block gives for it alone.
"""
from __future__ import annotations

import numpy as np
import pytest

from dvr3d_b200 import AUTOCM, configs, parse_deck

pytestmark = pytest.mark.gpu

TOL_CM = 1e-6


def _small_batch(n: int, seed: int):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        npnt = int(rng.integers(10, 17))
        nalf = int(rng.integers(14, 29))
        zcut = bool(i % 2)
        emax2 = float(rng.uniform(25000.0, 35000.0)) if zcut else 0.0
        w = configs.radau_water_like(npnt, nalf, emax2, 20, re=float(rng.uniform(1.7, 1.9)),
                                     de=float(rng.uniform(0.15, 0.25)), kb=float(rng.uniform(0.05, 0.12)),
                                     max3d=int(rng.integers(150, 400)) if not zcut else 20000, zcut=zcut,
                                     title=f"batch {i}")
        out.append(w)
    return out


def test_batch_matches_oracle_per_problem(ctx, oracle_mod):
    ws = _small_batch(6, 11)
    got = ctx.solve_batch([parse_deck(w.deck) for w in ws], np.array([w.pes for w in ws]))
    for w, g in zip(ws, got):
        ref = oracle_mod.solve(w.deck, 0, pes=w.pes, final_mode=1)
        assert ref.status == 0
        assert g.nham3 == ref.nham3
        np.testing.assert_array_equal(g.iv2, ref.iv2)
        err = np.abs(g.eval - ref.eval).max() * AUTOCM
        assert err <= TOL_CM, f"{w.name}: {err:.3e} cm-1"


def test_batch_of_64_equals_problem_by_problem(ctx):
    """The 64-problem workload: the batched run equals solving the problems one at a time."""
    ws = configs.config3()
    decks = [parse_deck(w.deck) for w in ws]
    got = ctx.solve_batch(decks, np.array([w.pes for w in ws]))
    for w, d, g in zip(ws, decks, got):
        ctx.set_pes(w.pes)
        one = ctx.solve(d, 0)
        assert g.nham3 == one.nham3
        np.testing.assert_array_equal(g.iv2, one.iv2)
        assert np.abs(g.eval - one.eval).max() * AUTOCM <= 1e-7


def test_batch_chosen_form_within_bar_of_plain(ctx):
    """The iterative final solve per problem (Davidson / shift-invert) inside the batch: every
    level within 1e-3 cm-1 of the plain FP64 batch."""
    import dvr3d_b200

    ws = configs.config3(nprob=12)
    decks = [parse_deck(w.deck) for w in ws]
    pes = np.array([w.pes for w in ws])
    plain = ctx.solve_batch(decks, pes)
    mixed = ctx.solve_batch(decks, pes, precision=dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON)
    for a, b in zip(plain, mixed):
        np.testing.assert_array_equal(a.iv2, b.iv2)
        assert np.abs(a.eval - b.eval).max() * AUTOCM <= 1e-3
