"""ROTLEV3 (z along r1 or r2) pinned to the reference's own printed H3+ Jacobi J = 1 example.

``tests/golden/h3p_jacobi_j1.npz`` (make_h3p_pes_fixture.py) holds the J = 1 first-step deck
(``H3+Jacobi/jobs/dvrJ1.job`` with the rotational masses and the ZX term of the printed run), the
potential on the grid of each k block, the printed per-block counts and 400 levels of each block
(``H3+Jacobi/results/result.H3p.J1even.dvr``), ROTLEV3's deck (``H3+Jacobi/jobs/rot.job``: NVIB =
400, NEVAL = 40, KMIN = 2, IBASS = 700) and its two printed sets of 40 levels
(``result.H3p.J1even.rot``): the e set of the k = 0, 1 Hamiltonian and the J = 1 f set.

* CPU: the oracle's first step reproduces both blocks' printed counts and levels to their 12
  digits; on a wavefunction file written from those oracle solves (jacobi_wave.py), the oracle's
  ROTLEV3 reproduces both printed sets of levels to their 12 digits, and its vector files have
  the layout DIPOLE3 reads.
* GPU: the product's first step (per-block PES tables, ZX) writes the file, the product's ROTLEV3
  on it reproduces the printed sets, agrees with the oracle's ROTLEV3 on the same file, and its
  vector files match the oracle's (levels, headers, the vectors up to each level's sign).
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np
import pytest

from jacobi_wave import write_jacobi_wave

AUTOCM = 2.19474624e5
FIX = Path(__file__).resolve().parent / "golden" / "h3p_jacobi_j1.npz"


@pytest.fixture(scope="module")
def j1():
    f = np.load(FIX)
    return {k: f[k] for k in f.files}


def printed_tolerance(levels: np.ndarray) -> np.ndarray:
    """Half a unit of the 12th printed digit of 0.ddddddddddddD+ee, plus 2e-13 Eh."""
    exp10 = np.floor(np.log10(np.abs(levels))) + 1
    return 0.5 * 10.0 ** (exp10 - 12) + 2e-13


def records(path) -> list[bytes]:
    data = Path(path).read_bytes()
    out, pos = [], 0
    while pos < len(data):
        (n,) = struct.unpack_from("<i", data, pos)
        out.append(data[pos + 4:pos + 4 + n])
        pos += 8 + n
    return out


def test_fixture_is_the_printed_run(j1):
    assert [len(j1[f"levels{k}"]) for k in (0, 1)] == [400, 400]
    assert [int(j1[f"counts{k}"].sum()) for k in (0, 1)] == [2000, 2000]
    assert len(j1["rot_e"]) == len(j1["rot_f"]) == 40
    # the printed J = 1 f set is the first step's k = 1 block (dstore1)
    np.testing.assert_array_equal(j1["rot_f"], j1["levels1"][:40])
    assert abs(j1["rot_e"][0] - 0.201679780627e-01) < 1e-16


@pytest.mark.parametrize("k", [0, 1])
def test_oracle_reproduces_printed_j1_blocks(oracle_mod, j1, k):
    r = oracle_mod.solve(str(j1["deck"]), k, vgrid=j1[f"v{k}"], final_mode=1)
    assert r.status == 0 and r.nham3 == int(j1[f"nham3_{k}"])
    np.testing.assert_array_equal(r.iv2, j1[f"counts{k}"])
    lv = j1[f"levels{k}"]
    err = np.abs(r.eval[:len(lv)] - lv)
    assert np.all(err <= printed_tolerance(lv)), f"max {err.max() * AUTOCM:.3e} cm-1"


@pytest.fixture(scope="module")
def oracle_wave(oracle_mod, j1, tmp_path_factory):
    d = tmp_path_factory.mktemp("rl3")
    path = d / "fort.26"
    write_jacobi_wave(path, oracle_mod, str(j1["deck"]), {0: j1["v0"], 1: j1["v1"]})
    return d, path


def test_oracle_rotlev3_reproduces_printed_sets(oracle_mod, j1, oracle_wave):
    d, wave = oracle_wave
    e, f = oracle_mod.rotlev3(str(j1["rot_deck"]), str(wave), str(d / "fort.8"), str(d / "fort.9"))
    for got, want in ((e, j1["rot_e"]), (f, j1["rot_f"])):
        assert len(got) == len(want) == 40
        err = np.abs(got - want)
        assert np.all(err <= printed_tolerance(want)), f"max {err.max() * AUTOCM:.3e} cm-1"
    # the e vectors (dstore): header, labels, levels, one record per k block of nkbas x nval
    rec = records(d / "fort.8")
    h = struct.unpack("<8i", rec[0])
    assert h == (2, 0, 18, 20, 21, 1, 1, 40)
    lab = np.frombuffer(rec[3], "<i4")
    # NEND as printed (15120); lmin: the first even l of k = 0 and k = 1
    assert lab[0] == lab[5] + lab[6] == 15120 and list(lab[1:3]) == [0, 2]
    assert list(lab[3:5]) == [18, 18] and lab[5] == 18 * 420
    assert len(rec) == 8 + 2 and struct.unpack("<i", rec[6]) == (40,)
    np.testing.assert_array_equal(np.frombuffer(rec[7], "<f8"), e)
    G = np.vstack([np.frombuffer(rec[8 + k], "<f8").reshape(40, lab[5 + k]).T for k in range(2)])
    # orthonormal in the FBR basis: the back transform is orthogonal on the kept functions
    np.testing.assert_allclose(G.T @ G, np.eye(40), atol=1e-10)
    # the J = 1 f set (dstore1): a one-block file with the k = 1 block's first 40 levels
    rec2 = records(d / "fort.9")
    assert struct.unpack("<8i", rec2[0]) == (2, 0, 18, 20, 21, 1, 0, 40)
    np.testing.assert_array_equal(np.frombuffer(rec2[10], "<f8"), f)
    assert len(rec2) == 11 + 40


def test_oracle_rotlev3_kmin_variants(oracle_mod, j1, oracle_wave, tmp_path):
    """KMIN = 1 gives the e set alone, KMIN = 0 (J = 1) the f set alone, written to KVEC2."""
    d, wave = oracle_wave
    deck = str(j1["rot_deck"])
    e1, f1 = oracle_mod.rotlev3(deck.replace("  400   40  2  700", "  400   40  1  700"), str(wave))
    e2, _ = oracle_mod.rotlev3(deck, str(wave))
    np.testing.assert_allclose(e1, e2, rtol=0, atol=1e-14)
    assert len(f1) == 0
    f0, _ = oracle_mod.rotlev3(deck.replace("  400   40  2  700", "  400   40  0  700"), str(wave),
                               kvec2_path=str(tmp_path / "f.9"))
    assert np.all(np.abs(f0 - j1["rot_f"]) <= printed_tolerance(j1["rot_f"]))
    assert (tmp_path / "f.9").exists()
