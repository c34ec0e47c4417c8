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


# ------------------------------------------------------------------------------------- GPU
def _sign_aligned_records(got: list[np.ndarray], ref: list[np.ndarray], cols: list[np.ndarray], nval: int):
    """Each record's entries multiplied by the sign of their level's column (cols: the level of
    every entry), the sign chosen over all blocks to align got with ref."""
    dots = np.zeros(nval)
    for g, r, c in zip(got, ref, cols):
        np.add.at(dots, c, g * r)
    s = np.where(dots < 0, -1.0, 1.0)
    return [g * s[c] for g, c in zip(got, cols)]


def compare_vector_files(got_path, ref_path, atol=1e-9):
    """Two dstore files: identical header and label records, levels to 1e-12, every vector
    entry to atol after aligning each level's sign. The block records are the first nkbas nval
    elements of an MBASS-leading array, as the reference writes them."""
    g, r = records(got_path), records(ref_path)
    assert len(g) == len(r)
    for i in (0, 1, 3, 6):
        assert g[i] == r[i], f"record {i}"
    for i in (2, 4, 5, 7):
        np.testing.assert_allclose(np.frombuffer(g[i], "<f8"), np.frombuffer(r[i], "<f8"), rtol=0, atol=1e-12)
    h = struct.unpack("<8i", g[0])
    mbass, nval = h[2] * h[3] * h[4], h[7]
    gv = [np.frombuffer(x, "<f8") for x in g[8:]]
    rv = [np.frombuffer(x, "<f8") for x in r[8:]]
    cols = [np.arange(len(x)) // mbass for x in gv]
    for a, b in zip(_sign_aligned_records(gv, rv, cols, nval), rv):
        np.testing.assert_allclose(a, b, rtol=0, atol=atol)


@pytest.fixture(scope="module")
def h3p_chain(ctx, j1, tmp_path_factory):
    """The product's J = 1 first step of the example (each k block on its own PES table), then
    the product's ROTLEV3 with the example's deck (KMIN = 2)."""
    d = tmp_path_factory.mktemp("rl3gpu")
    ctx.set_pes_grid_k(0, j1["v0"])
    ctx.set_pes_grid_k(1, j1["v1"])
    try:
        ctx.run_deck(str(j1["deck"]), wave_path=str(d / "fort.26"))
    finally:
        ctx.set_pes_grid_k(0, [])
        ctx.set_pes_grid_k(1, [])
    e, f, text = ctx.rotlev3(str(j1["rot_deck"]), str(d / "fort.26"), str(d / "fort.8"), str(d / "fort.9"))
    # the J = 0 first step of the example (its own fixture's table), the ket of the dipole run
    j0 = np.load(Path(__file__).resolve().parent / "golden" / "h3p_jacobi_j0.npz")
    ctx.set_pes_grid(j0["v"])
    ctx.run_deck(str(j0["deck"]), wave_path=str(d / "j0.26"))
    return d, e, f, text


@pytest.mark.gpu
def test_product_j1_first_step_reproduces_printed_blocks(j1, h3p_chain):
    d = h3p_chain[0]
    rec = records(d / "fort.26")
    # the k blocks from record 6: xalf, kz line, pleg, meval, levels, meval vectors
    pos = 6
    for k in (0, 1):
        assert struct.unpack("<4i", rec[pos + 1])[0] == k
        (meval,) = struct.unpack("<i", rec[pos + 3])
        lv = np.frombuffer(rec[pos + 4], "<f8")
        want = j1[f"levels{k}"]
        assert meval == 400
        err = np.abs(lv[:400] - want)
        assert np.all(err <= printed_tolerance(want)), f"k={k} max {err.max() * AUTOCM:.3e} cm-1"
        pos += 5 + meval


@pytest.mark.gpu
def test_product_rotlev3_reproduces_printed_sets(oracle_mod, j1, h3p_chain):
    d, e, f, text = h3p_chain
    for got, want in ((e, j1["rot_e"]), (f, j1["rot_f"])):
        assert len(got) == len(want) == 40
        err = np.abs(got - want)
        assert np.all(err <= printed_tolerance(want)), f"max {err.max() * AUTOCM:.3e} cm-1"
    assert "LOWEST  40 EIGENVALUES IN HARTREES" in text
    # the oracle's ROTLEV3 on the product's file: the same levels and vector files
    re_, rf = oracle_mod.rotlev3(str(j1["rot_deck"]), str(d / "fort.26"), str(d / "ref.8"), str(d / "ref.9"))
    np.testing.assert_allclose(e, re_, rtol=0, atol=1e-12)
    np.testing.assert_array_equal(f, rf)
    compare_vector_files(d / "fort.8", d / "ref.8")
    assert (d / "fort.9").read_bytes() == (d / "ref.9").read_bytes()


def _jacobi_deck(jrot: int, kmin: int, ipar: int, idia: int, flags: dict, neval: int = 60) -> tuple[str, list]:
    from dvr3d_b200 import configs

    masses = (1.007825, 12.0, 14.003074) if idia == 1 else configs.H3P_MASSES
    ur1, ur2 = configs.reduced_masses(masses, 1)
    re1, de1, we1 = (2.18, 0.30, 0.0095) if idia == 1 else (1.65, 0.17, 0.0125)
    re2, de2, we2 = (3.19, 0.20, 0.0150) if idia == 1 else (1.43, 0.12, 0.0110)
    b1, b2 = configs.morse_beta(we1, ur1, de1), configs.morse_beta(we2, ur2, de2)
    fl = {"ZCUT": False, "ZTHETA": True, "ZR2R1": False, "ZROT": True, "ZTRAN": True}
    fl.update(flags)
    deck = configs.deck_text(title=f"rotlev3 J{jrot} idia{idia}", npnt2=10, jrot=jrot, neval=neval, nalf=16,
                             max2d=400, max3d=300, idia=idia, kmin=kmin, npnt1=9, ipar=ipar, masses=masses,
                             emax1=60000.0, emax2=50000.0, morse1=(re1, de1, we1), morse2=(re2, de2, we2),
                             flags=fl)
    pes = configs.pes_row(de1, b1, re1, de2, b2, re2, kb=0.05 if idia == 1 else 0.0, c0=1.0 if idia == 1 else 0.0,
                          c1=0.01, c2=-0.015)
    return deck, pes


def _rot_deck(nvib: int, neval: int, kmin: int, ibass: int = 0, neval2: int = 0) -> str:
    return (" &PRT ztran=.true., zdcore=.true. /\n" + "".join(f"{v:5d}" for v in (nvib, neval, kmin, ibass, neval2))
            + "\n ROTLEV3 test\n" + f"{0.0:20.6f}\n")


# (jrot, first-step kmin, ipar, idia, flags, ROTLEV3 kmin, ibass)
JCASES = [
    (2, 1, 0, 1, {"ZEMBED": True}, 2, 0),               # heteronuclear, z along r2, e and f sets
    (2, 1, 1, 2, {"ZEMBED": False}, 1, 70),             # homonuclear odd, z along r1, energy selection
    (3, 1, 0, 2, {"ZEMBED": False}, 2, 0),             # J = 3: four k blocks, e and f sets
    (2, 0, 0, 1, {"ZEMBED": True}, 0, 0),               # f parity alone (k = 1, 2)
    (1, 1, 0, 1, {"ZEMBED": False, "ZX": True}, 2, 0),  # J = 1: e set, then the k = 1 block (dstore1)
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", JCASES, ids=lambda c: f"J{c[0]}k{c[1]}p{c[2]}d{c[3]}r{c[5]}")
def test_product_rotlev3_matches_oracle(ctx, oracle_mod, case, tmp_path):
    jrot, kmin0, ipar, idia, flags, kmin, ibass = case
    deck, pes = _jacobi_deck(jrot, kmin0, ipar, idia, flags)
    ctx.set_pes(pes)
    wave = tmp_path / "fort.26"
    ctx.run_deck(deck, wave_path=str(wave))
    rd = _rot_deck(40, 25, kmin, ibass, 20)
    e, f, _ = ctx.rotlev3(rd, str(wave), str(tmp_path / "g.8"), str(tmp_path / "g.9"))
    re_, rf = oracle_mod.rotlev3(rd, str(wave), str(tmp_path / "r.8"), str(tmp_path / "r.9"))
    assert len(e) == len(re_) > 0 and len(f) == len(rf)
    np.testing.assert_allclose(e, re_, rtol=0, atol=1e-12)
    np.testing.assert_allclose(f, rf, rtol=0, atol=1e-12)
    if kmin == 2:
        assert len(f) > 0
    if kmin != 0 or jrot != 1:
        compare_vector_files(tmp_path / "g.8", tmp_path / "r.8")
    if kmin == 2 and jrot > 1:
        compare_vector_files(tmp_path / "g.9", tmp_path / "r.9")
    elif (kmin == 2 and jrot == 1) or (kmin == 0 and jrot == 1):
        assert (tmp_path / "g.9").read_bytes() == (tmp_path / "r.9").read_bytes()


def jacobi_dipd(r1: float, r2: float, xcos: float, nu: int) -> float:
    """A smooth dipole plug-in in Jacobi coordinates (z along r1): z component even in cos,
    x component odd with sin theta."""
    if nu == 0:
        return 0.4 * (r2 - 1.5) * xcos + 0.05 * (r1 - 1.65) * (3.0 * xcos * xcos - 1.0)
    return 0.3 * (r2 - 1.5) * np.sqrt(max(0.0, 1.0 - xcos * xcos)) * (1.0 + 0.1 * xcos)


@pytest.mark.gpu
def test_product_dipole3_jacobi_matches_oracle(ctx, oracle_mod, h3p_chain, tmp_path):
    """DIPOLE3 on the example's J = 0 first-step file (ket) and the J = 1 e vectors of ROTLEV3
    (bra), as the reference's H3+ dipole job pairs them (NPOT = 80, 8 and 8 levels): the
    product against the oracle's restatement on the same files."""
    d = h3p_chain[0]
    deck = " &PRT zprint=.false., zstart=.true. /\n Dipole Transitions for H3+\n   80    8    8    0    0\n 4361.60387517\n"
    got = ctx.dipole3(deck, str(d / "j0.26"), str(d / "fort.8"), dipd=jacobi_dipd, tra_path=str(tmp_path / "g.13"))
    ref = oracle_mod.dipole3(deck, str(d / "j0.26"), str(d / "fort.8"), dipd=jacobi_dipd,
                             tra_path=str(tmp_path / "r.13"))
    assert (got["j1"], got["j2"]) == (ref["j1"], ref["j2"]) == (0, 1)
    np.testing.assert_array_equal(got["e1"], ref["e1"])
    np.testing.assert_array_equal(got["e2"], ref["e2"])
    scale = max(np.abs(ref["tz"]).max(), np.abs(ref["tx"]).max())
    assert scale > 1e-4
    for key in ("tz", "tx"):
        np.testing.assert_allclose(got[key], ref[key], rtol=0, atol=1e-10 * scale)
    np.testing.assert_allclose(got["sint"], ref["sint"], rtol=1e-9, atol=1e-18)
