"""Transition moments (the reference's DIPOLE3, dvr3d_b200_dipole3) and the ROTLEV3B vectors they
read (ZTRAN, dvr3d_b200_rotlev3b_trans), on chains built by the product: a J = 0 first-step
wavefunction file (Radau, even radial parity); J = 1 e-parity (first step with ZROT, odd radial
parity, then ROTLEV3B with ZTRAN) and f-parity (the first-step file of its one k block) sets;
J = 2 e and f sets from ROTLEV3B.

* the ROTLEV3B vector file against the oracle's restatement of dstore on the same first-step
  file: identical header records, levels to 1e-12 Eh, every transformed vector to 1e-9 (each
  level up to its sign, which the eigensolvers choose freely);
* DIPOLE3 on those files against the oracle's restatement reading the same files, with the
  reference's own DIPD transform around a model DIPSA surface and with a DIPD plug-in: the z
  and x transition moments, S(f-i) (invariant under the vectors' signs) and the printed table,
  both orders of ket and bra; the ITRA records of outpt.
"""
from __future__ import annotations

import math
import struct

import numpy as np
import pytest

import dvr3d_b200
from dvr3d_b200 import configs

pytestmark = pytest.mark.gpu


def _deck(jrot: int, kmin: int, ipar: int, neval: int = 40):
    w = configs.radau_water_like(12, 16, 30000.0, neval, title=f"dip J{jrot} p{ipar}")
    lines = w.deck.splitlines()
    c3 = list(lines[2])
    c3[5:10] = list(f"{jrot:5d}")
    c3[35:40] = list(f"{kmin:5d}")
    c3[45:50] = list(f"{ipar:5d}")
    lines[2] = "".join(c3)
    flags = ", ZTRAN=.TRUE." + (", ZROT=.TRUE., ZLIN=.TRUE." if jrot else "")
    w.deck = "\n".join(lines).replace("ZPMIN=.TRUE.", "ZPMIN=.TRUE." + flags) + "\n"
    return w


def _rot_deck(nvib: int, neval: int, kmin: int) -> str:
    card = "".join(f"{v:5d}" for v in (nvib, neval, kmin, 0, 0, 0))
    return " &PRT zdcore=.true., ztran=.true. /\n" + card + "\n ROTLEV3B vectors for DIPOLE3\n" + f"{4500.0:20.6f}\n"


def _dip_deck(npot: int, nv1: int, nv2: int, ezero: float = 4500.0, extra: str = "") -> str:
    return (f" &PRT zprint=.false.{extra} /\n DIPOLE3 test\n" + "".join(f"{v:5d}" for v in (npot, nv1, nv2, 0, 0))
            + f"\n{ezero:20.6f}\n")


def _records(path) -> list[bytes]:
    data = open(path, "rb").read()
    out, pos = [], 0
    while pos < len(data):
        (n,) = struct.unpack_from("<i", data, pos)
        out.append(data[pos + 4:pos + 4 + n])
        pos += 8 + n
    return out


def model_dipsa(q1: float, q2: float, cost: float):
    """A smooth bond-frame dipole of an AB2 molecule: along the bisector (dipy) symmetric in the
    two bonds, perpendicular (dipx) antisymmetric."""
    th = math.acos(max(-1.0, min(1.0, cost)))
    c, s = math.cos(th / 2), math.sin(th / 2)
    dy = (0.73 + 0.21 * (q1 + q2 - 3.62) - 0.05 * (q1 - q2) ** 2) * c * (1.0 + 0.1 * cost)
    dx = (0.38 - 0.04 * (q1 + q2 - 3.62)) * (q1 - q2) * s
    return dx, dy


def model_dipd(r1: float, r2: float, xcos: float, nu: int) -> float:
    """A DIPD plug-in in Radau coordinates, bisector frame: z symmetric, x antisymmetric under
    r1 <-> r2."""
    if nu == 0:
        return (0.6 + 0.15 * (r1 + r2 - 3.6)) * math.sqrt((1 + xcos) / 2) * (1.0 - 0.2 * xcos)
    return 0.35 * (r1 - r2) * math.sqrt((1 - xcos) / 2) * (1.0 + 0.1 * (r1 + r2 - 3.6))


@pytest.fixture(scope="module")
def chain(ctx, tmp_path_factory):
    """First-step files and ROTLEV3B vector files: J = 0 (even); J = 1 e (odd, k = 0, 1); J = 1
    e (even) and f (even, k = 1: the first-step file itself; an odd J = 1 f run has no room in
    MAX3D2, insize :335-342); J = 2 e (even, k = 0..2) and f (k = 1, 2)."""
    d = tmp_path_factory.mktemp("dip")
    runs = {"j0.26": (0, 0, 0), "j1.26": (1, 1, 1), "j1e0.26": (1, 1, 0), "j1f.26": (1, 0, 0), "j2e.26": (2, 1, 0),
            "j2f.26": (2, 0, 0)}
    for name, (j, kmin, ipar) in runs.items():
        w = _deck(j, kmin, ipar)
        ctx.set_pes(w.pes)
        ctx.run_deck(w.deck, wave_path=str(d / name))
    lv, table = ctx.rotlev3b_trans(_rot_deck(30, 20, 1), str(d / "j1.26"), str(d / "j1.8"))
    ctx.rotlev3b_trans(_rot_deck(30, 20, 1), str(d / "j1e0.26"), str(d / "j1e0.8"))
    ctx.rotlev3b_trans(_rot_deck(30, 20, 1), str(d / "j2e.26"), str(d / "j2e.8"))
    ctx.rotlev3b_trans(_rot_deck(30, 20, 0), str(d / "j2f.26"), str(d / "j2f.8"))
    return d, lv, table


def _sign_aligned(got: np.ndarray, ref: np.ndarray) -> np.ndarray:
    """got (nkbas x nval) per level multiplied by the sign that aligns it with ref."""
    s = np.sign(np.einsum("ij,ij->j", got, ref))
    s[s == 0] = 1.0
    return got * s


def test_rotlev3b_vectors_match_oracle(chain, oracle_mod):
    d, lv, _ = chain
    ref_lv = oracle_mod.rotlev3b_trans(_rot_deck(30, 20, 1), str(d / "j1.26"), str(d / "j1_ref.8"))
    np.testing.assert_allclose(lv, ref_lv, rtol=0, atol=1e-12)
    got, ref = _records(d / "j1.8"), _records(d / "j1_ref.8")
    assert len(got) == len(ref)
    for i in (0, 1, 3, 5):  # header, flags, labels, nval
        assert got[i] == ref[i], f"record {i}"
    for i in (2, 4, 6):  # Morse constants, r, levels
        np.testing.assert_allclose(np.frombuffer(got[i], "<f8"), np.frombuffer(ref[i], "<f8"), rtol=0, atol=1e-12)
    h = np.frombuffer(got[0], "<i4")
    nval = int(h[7])
    lab = np.frombuffer(got[3], "<i4")
    nblk = (len(lab) - 1) // 3
    nkbas = lab[1 + 2 * nblk:]
    assert lab[0] == nkbas.sum() and nblk == 2
    # the vectors, block by block, aligned per level over the whole basis
    g = [np.frombuffer(got[7 + k], "<f8").reshape(nval, nkbas[k]).T for k in range(nblk)]
    r = [np.frombuffer(ref[7 + k], "<f8").reshape(nval, nkbas[k]).T for k in range(nblk)]
    G, R = np.vstack(g), np.vstack(r)
    np.testing.assert_allclose(_sign_aligned(G, R), R, rtol=0, atol=1e-9)
    # normalised in the FBR basis: the transform is orthogonal
    np.testing.assert_allclose(np.einsum("ij,ij->j", G, G), 1.0, atol=1e-9)


# (ket, bra, plug-in, k -> k' blocks): J = 0 <-> 1 both ways, J = 1 e <-> f (the f set is a
# single first-step block: DIPOLE3 skips the nu = +1 blocks of a one-block bra, :928) and
# J = 2 e <-> f, the five blocks of the reference's water example.
CASES = [
    ("j0.26", "j1.8", "dipsa", 2),
    ("j1.8", "j0.26", "dipsa", 2),
    ("j0.26", "j1.8", "dipd", 2),
    ("j1e0.8", "j1f.26", "dipsa", 1),
    ("j2e.8", "j2f.8", "dipsa", 5),
    ("j2f.8", "j2e.8", "dipd", 5),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{c[1]}-{c[2]}")
def test_dipole3_matches_oracle(ctx, oracle_mod, chain, case, tmp_path):
    d, _, _ = chain
    ket, bra = d / case[0], d / case[1]
    kw = dict(dipsa=model_dipsa) if case[2] == "dipsa" else dict(dipd=model_dipd)
    deck = _dip_deck(24, 10, 8, extra=", zstart=.true.")
    got = ctx.dipole3(deck, str(ket), str(bra), tra_path=str(tmp_path / "g.13"), **kw)
    ref = oracle_mod.dipole3(deck, str(ket), str(bra), tra_path=str(tmp_path / "r.13"), **kw)
    assert (got["neval1"], got["neval2"]) == (ref["neval1"], ref["neval2"]) == (10, 8)
    assert (got["j1"], got["j2"]) == (ref["j1"], ref["j2"])
    assert got["nblocks"] == ref["nblocks"] == case[3]
    np.testing.assert_array_equal(got["e1"], ref["e1"])
    np.testing.assert_array_equal(got["e2"], ref["e2"])
    scale = max(np.abs(ref["tz"]).max(), np.abs(ref["tx"]).max())
    assert scale > 1e-4
    for key in ("tz", "tx"):
        np.testing.assert_allclose(got[key], ref[key], rtol=0, atol=1e-10 * scale)
    np.testing.assert_allclose(got["sint"], ref["sint"], rtol=1e-9, atol=1e-18)
    # the printed table: same rows, same numbers
    rows_g = [ln.split() for ln in got["text"].splitlines() if ln[:8].strip() and ln.split()[0].isdigit()]
    rows_r = [ln.split() for ln in ref["text"].splitlines() if ln[:8].strip() and ln.split()[0].isdigit()]
    assert len(rows_g) == len(rows_r) == 80
    for a, b in zip(rows_g, rows_r):
        assert a[:2] == b[:2]
        np.testing.assert_allclose([float(x) for x in a[2:]], [float(x) for x in b[2:]], rtol=1e-7, atol=1e-9)
    # the ITRA records: header, energies, S(f-i) per bra state
    rg, rr = _records(tmp_path / "g.13"), _records(tmp_path / "r.13")
    assert len(rg) == len(rr) == 3 + 8
    assert rg[0] == rr[0]
    for a, b in zip(rg[1:], rr[1:]):
        np.testing.assert_allclose(np.frombuffer(a, "<f8"), np.frombuffer(b, "<f8"), rtol=1e-9, atol=1e-18)


def test_dipole3_selection_rules_and_limits(ctx, chain):
    d, _, _ = chain
    with pytest.raises(dvr3d_b200.DVR3DError):  # J = 0 -> 0
        ctx.dipole3(_dip_deck(24, 5, 5), str(d / "j0.26"), str(d / "j0.26"), dipsa=model_dipsa)
    with pytest.raises(ValueError):
        ctx.dipole3(_dip_deck(24, 5, 5), str(d / "j0.26"), str(d / "j1.8"))
    # NBLOCK = 1 stops after the first k -> k' block
    one = ctx.dipole3(_dip_deck(24, 4, 4, extra=", nblock=1"), str(d / "j0.26"), str(d / "j1.8"), dipsa=model_dipsa)
    assert one["nblocks"] == 1 and np.abs(one["tx"]).max() == 0.0 and np.abs(one["tz"]).max() > 0.0
