"""Radau coordinates with the z axis perpendicular to the molecular plane (ZPERP = T: mkmain
:3934-4034 and z_blc2d1 :4038-4127 instead of nfmain / blc2d1; Gauss-Jacobi angular rule with
alpha = beta = sqrt((J(J+1) - k^2)/2), gaujac :4190-4263; Jacobi-polynomial L matrix, lmatrx
:1870-1903; KMIN carries the Q symmetry, k runs from 0 and the parity stays fixed, insize
:255-261 and ccmain :857-866, :989-998).

Every k block of each deck against the oracle: identical per-angle selection counts and N,
levels within 1e-6 cm-1 (the plain FP64 path), and the same error where the oracle stops
(testiv's theta = 0 test).
"""
from __future__ import annotations

import numpy as np
import pytest

import dvr3d_b200
from dvr3d_b200 import AUTOCM, configs, parse_deck

pytestmark = pytest.mark.gpu

TOL_CM = 1e-6


def _zperp_deck(jrot: int, kmin: int, ipar: int, *, zcut: bool = True, zlin: bool = False, nalf: int = 16,
                npnt: int = 12, emax2: float = 30000.0, neval: int = 20):
    w = configs.radau_water_like(npnt, nalf, emax2, neval, zcut=zcut, max3d=400 if not zcut else 20000,
                                 title=f"zperp J{jrot} q{kmin} p{ipar}")
    lines = w.deck.splitlines()
    c3 = list(lines[2])
    c3[5:10] = list(f"{jrot:5d}")
    c3[35:40] = list(f"{kmin:5d}")
    c3[45:50] = list(f"{ipar:5d}")
    lines[2] = "".join(c3)
    extra = ", ZPERP=.TRUE."
    if jrot:
        extra += ", ZROT=.TRUE."
    if zlin:
        extra += ", ZLIN=.TRUE."
    w.deck = "\n".join(lines).replace("ZPMIN=.TRUE.", "ZPMIN=.TRUE." + extra) + "\n"
    return w


CASES = [
    dict(jrot=0, kmin=0, ipar=0),
    dict(jrot=0, kmin=0, ipar=1),
    dict(jrot=0, kmin=0, ipar=0, zcut=False),
    dict(jrot=1, kmin=0, ipar=0, zlin=True),
    dict(jrot=1, kmin=1, ipar=1, zlin=True),
    dict(jrot=2, kmin=0, ipar=0, zlin=True, nalf=14),
    dict(jrot=1, kmin=0, ipar=0),  # no zlin: testiv may stop on theta = 0 amplitude
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_zperp_blocks_match_oracle(ctx, oracle_mod, case):
    w = _zperp_deck(**case)
    d = parse_deck(w.deck)
    ks = dvr3d_b200.k_blocks(d)
    assert ks == oracle_mod.k_blocks(w.deck)
    assert ks == list(range(0, case["jrot"] + 1))
    ctx.set_pes(w.pes)
    for k in ks:
        ref = oracle_mod.solve(w.deck, k, pes=w.pes, final_mode=1)
        if ref.status != 0:
            with pytest.raises(dvr3d_b200.DVR3DError) as e:
                ctx.solve(d, k)
            assert e.value.code == ref.status
            continue
        got = ctx.solve(d, k, want_resid=True)
        assert got.nham3 == ref.nham3 and got.kz == k and got.ipar == case["ipar"]
        np.testing.assert_array_equal(got.iv2, ref.iv2)
        n = min(len(got.eval), len(ref.eval))
        err = np.abs(got.eval[:n] - ref.eval[:n]) * AUTOCM
        assert err.max() <= TOL_CM, f"k={k}: {err.max():.3e} cm-1"
        assert got.max_resid < 1e-9


def test_zperp_wavefunction_file_angular_records(ctx, oracle_mod, tmp_path):
    """The per-k angular records of the wavefunction file in the z-perp embedding: the
    Gauss-Jacobi points and the Jacobi polynomials times the square-rooted weights (:955-976)."""
    import struct

    w = _zperp_deck(0, 0, 0)
    w.deck = w.deck.replace("ZPERP=.TRUE.", "ZPERP=.TRUE., ZTRAN=.TRUE.")
    ctx.set_pes(w.pes)
    path = tmp_path / "fort.26"
    ctx.run_deck(w.deck, wave_path=str(path))
    data = open(path, "rb").read()
    recs, pos = [], 0
    while pos < len(data):
        (n,) = struct.unpack_from("<i", data, pos)
        recs.append(data[pos + 4:pos + 4 + n])
        pos += 8 + n
    q = oracle_mod.quadrature(oracle_mod.parse_deck(w.deck), 0)
    xa = np.frombuffer(recs[5], dtype="<f8")
    np.testing.assert_array_equal(xa, np.array(q.xalf[:len(xa)]))
    kz, maxleg, nidvr, lincr = struct.unpack("<4i", recs[6])
    assert kz == 0 and nidvr == len(xa) and maxleg == len(xa) - 1
    pl = np.frombuffer(recs[7], dtype="<f8").reshape(nidvr, maxleg + 1)
    # normalised Jacobi polynomials (alpha = beta = 0: Legendre) times sqrt(w): orthonormal, to
    # the ~1e-11 of the reference's gammln series in the weights and norms
    np.testing.assert_allclose(pl @ pl.T, np.eye(nidvr), rtol=0, atol=1e-10)
