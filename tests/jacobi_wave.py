"""A first-step ZTRAN wavefunction file (unit IWAVE) for Jacobi coordinates written from the
oracle's own block solves, for testing the second step (ROTLEV3) and DIPOLE3 on the CPU.

The records follow the reference's writes with ZTRAN (and ZROT for J > 0)
(source/dvr3drjz_segmented.f90): the header (:1178-1180: IDIA, IPAR, IDVR, NPNT1, NPNT2, JROT,
KMIN, NEVAL, NLIM; the logical flags with the masses and g1, g2; the Morse constants), the
r^-2 term of the embedding axis (:822-833; for J = 0 the block's basis size, first l and number
of l instead, :835-840), r1 and r2 (:843-844), then per k block its angular
points, (kz, maxleg, nidvr, lincr), the Legendre functions times the DVR weights (:972-976),
the number of levels, the levels and one amplitude record per level (trans :3733-3841).
Test infrastructure: nothing in the product imports it.
"""
from __future__ import annotations

import struct

import numpy as np


def _rec(f, payload: bytes) -> None:
    f.write(struct.pack("<i", len(payload)))
    f.write(payload)
    f.write(struct.pack("<i", len(payload)))


def write_jacobi_wave(path, oracle_mod, deck_text: str, vgrids: dict[int, np.ndarray]) -> dict:
    """Solve every k block of the deck with the oracle (vgrids[k]: the potential on block k's
    grid) and write the file. Returns {k: OracleResult}."""
    d = oracle_mod.parse_deck(deck_text)
    if d.idia not in (1, 2):
        raise ValueError("a Jacobi deck")
    # J = 0: one block, z along r2 and KMIN = 0 whatever the deck says (insize :242-246)
    kmin = d.kmin if d.jrot > 0 else 0
    kd = 0 if (kmin >= 1 or d.jrot == 0) else 1
    ku = d.jrot
    res, quads = {}, {}
    for k in range(kd, ku + 1):
        quads[k] = oracle_mod.quadrature(d, k)
        r = oracle_mod.solve(deck_text, k, vgrid=vgrids[k], final_mode=1, want_psi=True)
        if r.status != 0 or r.psi is None:
            raise RuntimeError(f"oracle block k={k} failed ({r.status})")
        res[k] = r
    q0 = quads[kd]
    n1, n2 = q0.npnt1, q0.npnt2
    r1, r2 = np.array(q0.r1[:n1]), np.array(q0.r2[:n2])
    idvr = q0.nidvr
    zembed = bool(d.zembed) or d.jrot == 0
    with open(path, "wb") as f:
        nlim = (n2 if zembed else n1) if d.jrot > 0 else 0
        _rec(f, struct.pack("<9i", d.idia, d.ipar, idvr, n1, n2, d.jrot, kmin, d.neval, nlim))
        _rec(f, struct.pack("<3i", -1 if zembed else 0, -1, -1) + np.array(d.xmass[:3], "<f8").tobytes()
             + struct.pack("<2d", q0.g1, q0.g2) + struct.pack("<2i", 0 if d.jrot > 0 else -1, -1))
        _rec(f, np.array([d.re1, d.diss1, d.we1, d.re2, d.diss2, d.we2], "<f8").tobytes())
        if d.jrot > 0:  # the r^-2 term of the embedding axis
            rm2 = 0.5 / (r2 * r2 * q0.urr2) if zembed else 0.5 / (r1 * r1 * q0.urr1)
            _rec(f, rm2.astype("<f8").tobytes())
        else:  # one block: its basis size, first l, number of l (:835-840)
            jdia = max(1, d.idia)
            jstart = kmin + (1 if kmin % jdia != d.ipar else 0)
            nang = (res[kd].maxleg - jstart) // jdia + 1
            mbass = idvr * n1 * n2
            _rec(f, struct.pack("<4i", mbass, jstart, nang, mbass))
        _rec(f, r1.astype("<f8").tobytes())
        _rec(f, r2.astype("<f8").tobytes())
        for k in range(kd, ku + 1):
            q, r = quads[k], res[k]
            _rec(f, np.array(q.xalf[:q.nidvr], "<f8").tobytes())
            _rec(f, struct.pack("<4i", k, r.maxleg, r.nidvr, r.lincr))
            _rec(f, r.pleg_walf.astype("<f8").tobytes())
            meval = r.psi.shape[0]
            _rec(f, struct.pack("<i", meval))
            _rec(f, r.eval[:meval].astype("<f8").tobytes())
            for lv in r.psi:
                _rec(f, lv.astype("<f8").tobytes())
    return res
