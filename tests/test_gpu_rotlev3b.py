"""The second variational step for J > 0 (the reference's ROTLEV3B, dvr3d_b200_rotlev3b) on
wavefunction files the first step writes (dvr3d_b200_run_deck_wave, Radau, bisector embedding,
ZROT, ZTRAN): the lowest levels of the Coriolis-coupled Hamiltonian against the oracle's
restatement of ROTLEV3B reading the same file, within 1e-6 cm-1; e parity (k = 0..J, with the
k, k+2 blocks for J = 2), f parity (k = 1..J) and the basis selection by energy (IBASS).
"""
from __future__ import annotations

import numpy as np
import pytest

import dvr3d_b200
from dvr3d_b200 import AUTOCM, configs

pytestmark = pytest.mark.gpu

TOL_CM = 1e-6


def _first_step(jrot: int, kmin: int, neval: int = 40, zlin: bool = True):
    w = configs.radau_water_like(12, 16, 30000.0, neval, title=f"rot J{jrot} kmin{kmin}")
    lines = w.deck.splitlines()
    c3 = list(lines[2])
    c3[5:10] = list(f"{jrot:5d}")
    c3[35:40] = list(f"{kmin:5d}")
    lines[2] = "".join(c3)
    # ZLIN: testiv drops the functions left at theta = 0 instead of stopping (k >= 2 blocks)
    flags = ", ZROT=.TRUE., ZTRAN=.TRUE." + (", ZLIN=.TRUE." if zlin else "")
    w.deck = "\n".join(lines).replace("ZPMIN=.TRUE.", "ZPMIN=.TRUE." + flags) + "\n"
    return w


def _rot_deck(nvib: int, neval: int, kmin: int, ibass: int = 0, ezero: float | None = None) -> str:
    card = "".join(f"{v:5d}" for v in (nvib, neval, kmin, ibass, 0, 0))
    text = " &PRT zdcore=.true. /\n" + card + "\n ROTLEV3B test\n"
    if ezero is not None:
        text += f"{ezero:20.6f}\n"
    return text


CASES = [
    dict(jrot=1, kmin=1, nvib=30, neval=20),
    dict(jrot=2, kmin=1, nvib=25, neval=20),
    dict(jrot=2, kmin=0, nvib=25, neval=15),
    dict(jrot=2, kmin=1, nvib=30, neval=20, ibass=55),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_rotlev3b_matches_oracle(ctx, oracle_mod, tmp_path, case):
    w = _first_step(case["jrot"], case["kmin"])
    ctx.set_pes(w.pes)
    path = tmp_path / "fort.26"
    ctx.run_deck(w.deck, wave_path=str(path))
    deck = _rot_deck(case["nvib"], case["neval"], case["kmin"], case.get("ibass", 0), ezero=4500.0)
    got, table = ctx.rotlev3b(deck, str(path))
    ref = oracle_mod.rotlev3b(deck, str(path))
    assert len(got) == len(ref) == case["neval"]
    err = np.abs(got - ref) * AUTOCM
    assert err.max() <= TOL_CM, f"{err.max():.3e} cm-1"
    assert f"lowest{case['neval']:4d} eigenvalues in Hartrees" in table
    assert "relative to ezero" in table
    # the Coriolis coupling mixes the k blocks: the levels are not the vibrational ones
    assert np.all(np.diff(got) >= -1e-12)


def test_rotlev3b_rejects_a_file_of_the_other_parity(ctx, tmp_path):
    w = _first_step(1, 1)
    ctx.set_pes(w.pes)
    path = tmp_path / "fort.26"
    ctx.run_deck(w.deck, wave_path=str(path))
    with pytest.raises(dvr3d_b200.DVR3DError):
        ctx.rotlev3b(_rot_deck(20, 10, 0), str(path))
