"""The wavefunction file (unit IWAVE, fort.26) written by dvr3d_b200_run_deck_wave.

The reference writes it when the deck sets ZTRAN; ROTLEV3, ROTLEV3B and DIPOLE3 read it.
A small reader here splits the file into its sequential unformatted records (4-byte length
before and after each) and checks, record by record, what DVR3DRJZ writes:
  * setcon's header (:1176-1184): sizes, flags, masses, g1/g2, radial basis constants;
  * ccmain's records (:820-845): the basis sizes (one k block) or the r**(-2) term (several),
    the radial grids;
  * per k block (:972-976): the angular grid, (kz, maxleg, nidvr, lincr), pleg * walf;
  * Radau: testiv's angle count and selection (:3446-3448);
  * the levels and one record of amplitudes per level from trans (Jacobi, psi(idvr, npnt1,
    npnt2)) or transr (Radau, wvfunc(nbass)).
Grids and levels are compared with the oracle; the amplitudes with the oracle's restatement
of trans / transr, level by level up to the sign of each eigenvector (levels closer than
1e-7 Eh to a neighbour are compared through their subspace).
"""
from __future__ import annotations

import struct

import numpy as np
import pytest

from dvr3d_b200 import configs

pytestmark = pytest.mark.gpu

AMP_TOL = 1e-8  # amplitudes are O(0.1); the eigenvectors agree to ~1e-10 / gap


def read_records(path) -> list[bytes]:
    data = open(path, "rb").read()
    recs, pos = [], 0
    while pos < len(data):
        (n,) = struct.unpack_from("<i", data, pos)
        body = data[pos + 4:pos + 4 + n]
        (m,) = struct.unpack_from("<i", data, pos + 4 + n)
        assert m == n and len(body) == n
        recs.append(body)
        pos += 8 + n
    return recs


def ints(b):
    return list(struct.unpack(f"<{len(b) // 4}i", b))


def dbls(b):
    return np.frombuffer(b, dtype="<f8")


def _ztran(deck: str) -> str:
    return deck.replace("ZPMIN=.TRUE.", "ZPMIN=.TRUE., ZTRAN=.TRUE.")


def _compare_amplitudes(got: np.ndarray, ref: np.ndarray, ev: np.ndarray):
    assert got.shape == ref.shape
    n = len(ev)
    gap = np.full(n, np.inf)
    gap[1:] = np.minimum(gap[1:], np.diff(ev))
    gap[:-1] = np.minimum(gap[:-1], np.diff(ev))
    for lv in range(n):
        if gap[lv] > 1e-7:
            d = min(np.abs(got[lv] - ref[lv]).max(), np.abs(got[lv] + ref[lv]).max())
            assert d <= AMP_TOL, f"level {lv}: amplitude difference {d:.3e}"
    # every record is a unit vector and the records are orthogonal (the DVR grid is orthonormal)
    np.testing.assert_allclose(got @ got.T, np.eye(n), rtol=0, atol=1e-10)


def _check_block(recs, i, oracle_mod, w, k, radau: bool):
    """Records of one k block starting at index i; returns the index after them."""
    d = oracle_mod.parse_deck(w.deck)
    q = oracle_mod.quadrature(d, k)
    s = oracle_mod.sizes(d, k)
    idvr = s["idvr"]
    np.testing.assert_array_equal(dbls(recs[i]), np.array(q.xalf[:idvr]))
    kz, maxleg, nidvr, lincr = ints(recs[i + 1])
    assert kz == s["kz"] and nidvr == s["nidvr"] and lincr == s["lincr"] and maxleg == d.nalf - 1
    pl = dbls(recs[i + 2])
    assert pl.size == (maxleg + 1) * nidvr and np.all(np.isfinite(pl))
    i += 3
    ref = oracle_mod.solve(w.deck, k, pes=w.pes, final_mode=1, want_psi=True)
    assert ref.status == 0
    if radau:
        iang, nbass = ints(recs[i])
        assert iang == int(np.count_nonzero(ref.iv2)) and nbass == iang * s["max2d"]
        assert ints(recs[i + 1]) == list(ref.iv2)
        i += 2
    (meval,) = ints(recs[i])
    ev = dbls(recs[i + 1])
    assert meval == len(ref.eval)
    np.testing.assert_allclose(ev, ref.eval, rtol=0, atol=1e-6 / 2.19474624e5)
    i += 2
    psi = np.array([dbls(recs[i + lv]) for lv in range(meval)])
    _compare_amplitudes(psi, ref.psi, ref.eval)
    return i + meval


def _check_header(recs, oracle_mod, w, radau: bool):
    d = oracle_mod.parse_deck(w.deck)
    q = oracle_mod.quadrature(d, oracle_mod.k_blocks(d)[0])
    s = oracle_mod.sizes(d, 0)
    h = ints(recs[0])
    assert h[0] == d.idia and h[2] == s["idvr"] and h[3] == s["npnt1"]
    assert h[4] == (s["npnt1"] if radau else s["npnt2"]) and h[5] == abs(d.jrot) and h[7] == d.neval
    flags = recs[1]
    assert len(flags) == 3 * 4 + 5 * 8 + 2 * 4
    xm = struct.unpack_from("<3d", flags, 12)
    g1, g2 = struct.unpack_from("<2d", flags, 36)
    assert list(xm) == list(d.xmass) and g1 == q.g1 and g2 == q.g2
    rad = dbls(recs[2])
    want = [d.re1, d.diss1, d.we1] + ([d.re1, d.diss1, d.we1] if radau else [d.re2, d.diss2, d.we2])
    assert list(rad) == want
    return d, q, s


@pytest.mark.parametrize("variant", ["theta_last", "theta_first"])
def test_jacobi_j0_wavefunction_file(ctx, oracle_mod, tmp_path, variant):
    w = configs.jacobi_h3p_like(8, 9, 12, 45000.0, 40000.0, 10, title="wave jacobi")
    if variant == "theta_first":
        w.deck = w.deck.replace("ZTHETA=.FALSE.", "ZTHETA=.TRUE.").replace("ZR2R1=.TRUE.", "ZR2R1=.FALSE.")
    w.deck = _ztran(w.deck)
    ctx.set_pes(w.pes)
    path = tmp_path / "fort.26"
    ctx.run_deck(w.deck, wave_path=str(path))
    recs = read_records(path)
    d, q, s = _check_header(recs, oracle_mod, w, radau=False)
    mbass, jstart, nang, mbass2 = ints(recs[3])
    assert mbass == mbass2 == s["idvr"] * s["npnt1"] * s["npnt2"]
    np.testing.assert_array_equal(dbls(recs[4]), np.array(q.r1[:s["npnt1"]]))
    np.testing.assert_array_equal(dbls(recs[5]), np.array(q.r2[:s["npnt2"]]))
    end = _check_block(recs, 6, oracle_mod, w, 0, radau=False)
    assert end == len(recs)


def test_radau_j0_wavefunction_file(ctx, oracle_mod, tmp_path):
    w = configs.radau_water_like(10, 12, 30000.0, 10, title="wave radau")
    w.deck = _ztran(w.deck)
    ctx.set_pes(w.pes)
    path = tmp_path / "fort.26"
    ctx.run_deck(w.deck, wave_path=str(path))
    recs = read_records(path)
    d, q, s = _check_header(recs, oracle_mod, w, radau=True)
    mbass = ints(recs[3])[0]
    assert mbass == s["idvr"] * s["max2d"]
    np.testing.assert_array_equal(dbls(recs[4]), np.array(q.r1[:s["npnt1"]]))
    end = _check_block(recs, 5, oracle_mod, w, 0, radau=True)
    assert end == len(recs)


def test_jacobi_j1_wavefunction_file_two_k_blocks(ctx, oracle_mod, tmp_path):
    w = configs.jacobi_h3p_like(8, 9, 12, 45000.0, 40000.0, 8, title="wave J1")
    lines = w.deck.splitlines()
    c3 = list(lines[2])
    c3[5:10] = list(f"{1:5d}")   # jrot = 1
    c3[35:40] = list(f"{1:5d}")  # kmin = 1
    lines[2] = "".join(c3)
    w.deck = _ztran("\n".join(lines).replace("ZPMIN=.TRUE.", "ZPMIN=.TRUE., ZROT=.TRUE.") + "\n")
    ctx.set_pes(w.pes)
    path = tmp_path / "fort.26"
    ctx.run_deck(w.deck, wave_path=str(path))
    recs = read_records(path)
    d, q, s = _check_header(recs, oracle_mod, w, radau=False)
    ks = oracle_mod.k_blocks(d)
    assert len(ks) == 2
    # several k blocks: the r**(-2) term for ROTLEV3 in place of the basis sizes (:824-833)
    r2m2 = dbls(recs[3])
    r2 = np.array(q.r2[:s["npnt2"]])
    np.testing.assert_allclose(r2m2, 0.5 / (r2 * r2 * q.urr2), rtol=1e-15, atol=0)
    np.testing.assert_array_equal(dbls(recs[4]), np.array(q.r1[:s["npnt1"]]))
    np.testing.assert_array_equal(dbls(recs[5]), r2)
    i = 6
    for k in ks:
        i = _check_block(recs, i, oracle_mod, w, k, radau=False)
    assert i == len(recs)


def test_j2_wave_run_after_back_transforms(ctx, tmp_path):
    """A J = 2 Radau job (k = 0, 1, 2; NPNT = 21, NALF = 40, 2D blocks of 231 and 210) with the
    wavefunction file, run repeatedly: each k block follows the previous block's back-transform
    GEMMs. The batched inverse iteration must not read stale shared memory: its LU leaves the
    last row's superdiagonals to be set explicitly (the back substitution multiplies them by
    zero, and a NaN left there by an earlier kernel poisoned a vector)."""
    w = configs.radau_water_like(21, 40, 40000.0, 200, title="J2 wave")
    lines = w.deck.splitlines()
    c3 = list(lines[2])
    c3[5:10] = list(f"{2:5d}")
    c3[35:40] = list(f"{1:5d}")
    lines[2] = "".join(c3)
    w.deck = "\n".join(lines).replace("ZPMIN=.TRUE.", "ZPMIN=.TRUE., ZROT=.TRUE., ZTRAN=.TRUE., ZLIN=.TRUE.") + "\n"
    ctx.set_pes(w.pes)
    texts = [ctx.run_deck(w.deck, wave_path=str(tmp_path / f"w{t}.26"))[0] for t in range(3)]
    assert texts[0] == texts[1] == texts[2]
    assert "lowest 200 eigenvalues" in texts[0].lower()
    recs = [read_records(tmp_path / f"w{t}.26") for t in range(3)]
    assert [len(r) for r in recs] == [len(recs[0])] * 3
    assert [len(x) for x in recs[2]] == [len(x) for x in recs[0]]
