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


def _pair_deck(nvib: int, neval: int, neval2: int) -> str:
    card = "".join(f"{v:5d}" for v in (nvib, neval, 2, 0, neval2, 0))
    return " &PRT zdcore=.true., ztran=.true. /\n" + card + "\n ROTLEV3B KMIN = 2\n" + f"{4500.0:20.6f}\n"


def _kmin2_first_step(jrot: int, ipar: int):
    w = _first_step(jrot, 2)
    lines = w.deck.splitlines()
    c3 = list(lines[2])
    c3[45:50] = list(f"{ipar:5d}")
    lines[2] = "".join(c3)
    w.deck = "\n".join(lines) + "\n"
    return w


def _records(path) -> list[bytes]:
    import struct

    data = open(path, "rb").read()
    out, pos = [], 0
    while pos < len(data):
        (n,) = struct.unpack_from("<i", data, pos)
        out.append(data[pos + 4:pos + 4 + n])
        pos += 8 + n
    return out


@pytest.mark.parametrize("jrot,ipar", [(2, 0), (2, 1), (3, 0), (1, 0)])
def test_rotlev3b_kmin2_both_passes_match_oracle(ctx, oracle_mod, tmp_path, jrot, ipar):
    """KMIN = 2: one first-step file with the e blocks k = 0..J and the f-type k = 1 block after
    them; ROTLEV3B's two passes (e, then f with that block in place of the e-type k = 1) against
    the oracle's restatement, levels within 1e-6 cm-1; the two vector files (dstore, and dstore1
    for J = 1) against the oracle's, each level up to its sign."""
    w = _kmin2_first_step(jrot, ipar)
    d = dvr3d_b200.parse_deck(w.deck)
    assert dvr3d_b200.k_blocks(d) == list(range(0, jrot + 2))
    ctx.set_pes(w.pes)
    path = tmp_path / "fort.26"
    ctx.run_deck(w.deck, wave_path=str(path))
    deck = _pair_deck(25, 15, 12)
    le, lf, table = ctx.rotlev3b_pair(deck, str(path), str(tmp_path / "g.8"), str(tmp_path / "g.9"))
    re_, rf = oracle_mod.rotlev3b_pair(deck, str(path), str(tmp_path / "r.8"), str(tmp_path / "r.9"))
    assert len(le) == len(re_) == 15 and len(lf) == len(rf) > 0
    assert np.abs(le - re_).max() * AUTOCM <= TOL_CM
    assert np.abs(lf - rf).max() * AUTOCM <= TOL_CM
    assert "e parity" in table and "f parity" in table
    for a, b in (("g.8", "r.8"), ("g.9", "r.9")):
        g, r = _records(tmp_path / a), _records(tmp_path / b)
        assert len(g) == len(r)
        hg, hr = np.frombuffer(g[0], "<i4"), np.frombuffer(r[0], "<i4")
        np.testing.assert_array_equal(hg, hr)
        for x, y in zip(g[1:], r[1:]):
            assert len(x) == len(y)
        if jrot == 1 and a == "g.9":  # dstore1: the block's own records, copied
            assert g == r
            continue
        nval = int(hg[7])
        lab = np.frombuffer(g[3], "<i4")
        np.testing.assert_array_equal(lab, np.frombuffer(r[3], "<i4"))
        nblk = (len(lab) - 1) // 3
        nk = lab[1 + 2 * nblk:]
        G = np.vstack([np.frombuffer(g[7 + k], "<f8").reshape(nval, nk[k]).T for k in range(nblk)])
        R = np.vstack([np.frombuffer(r[7 + k], "<f8").reshape(nval, nk[k]).T for k in range(nblk)])
        s = np.sign(np.einsum("ij,ij->j", G, R))
        np.testing.assert_allclose(G * s, R, rtol=0, atol=1e-9)


def test_kmin2_chain_to_dipole3(ctx, oracle_mod, tmp_path):
    """The reference's water chain, on a model surface: J = 2 first steps of both radial parities
    with KMIN = 2, ROTLEV3B's two passes on each, DIPOLE3 between the e set of the even run and
    the f set of the odd run (same J, same parity label), product against oracle."""
    import math

    def dipsa(q1, q2, cost):
        th = math.acos(max(-1.0, min(1.0, cost)))
        return (0.38 * (q1 - q2) * math.sin(th / 2), (0.73 + 0.2 * (q1 + q2 - 3.62)) * math.cos(th / 2))

    files = {}
    for ipar in (0, 1):
        w = _kmin2_first_step(2, ipar)
        ctx.set_pes(w.pes)
        p = tmp_path / f"p{ipar}.26"
        ctx.run_deck(w.deck, wave_path=str(p))
        ctx.rotlev3b_pair(_pair_deck(25, 12, 12), str(p), str(tmp_path / f"p{ipar}.8"), str(tmp_path / f"p{ipar}.9"))
        files[ipar] = (tmp_path / f"p{ipar}.8", tmp_path / f"p{ipar}.9")
    deck = " &PRT zstart=.true. /\n chain\n" + "".join(f"{v:5d}" for v in (40, 10, 10, 0, 0)) + f"\n{4500.0:20.6f}\n"
    ket, bra = str(files[0][0]), str(files[1][1])
    got = ctx.dipole3(deck, ket, bra, dipsa=dipsa)
    ref = oracle_mod.dipole3(deck, ket, bra, dipsa=dipsa)
    assert got["nblocks"] == ref["nblocks"] == 5 and (got["j1"], got["j2"]) == (2, 2)
    scale = max(np.abs(ref["tz"]).max(), np.abs(ref["tx"]).max())
    assert scale > 1e-4
    for key in ("tz", "tx"):
        np.testing.assert_allclose(got[key], ref[key], rtol=0, atol=1e-10 * scale)
