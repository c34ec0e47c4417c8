"""Known answers for DIPOLE3 from the reference's own printed runs (water, H3+ Jacobi, HCN;
``tests/golden/dipole3_kat.json``, extracted by make_goldens.py), on the CPU:

* lagpt's angular rule (jacobi :1311-1368 with alf = bta = 0) of the oracle: every printed
  point (f23.15) and weight (d25.12) and the printed computed sum of the weights;
* threej (:1778-1823) of the oracle against Racah's formula in exact rational arithmetic;
* spect's arithmetic (:1825-1954) on every printed row: the frequency from the two energies,
  the transition dipole |tz + tx|, S(f-i) and the Einstein A coefficient with the (2j+1) of the
  upper state, from the printed moments -- with the energies the run printed (a.u., d24.12),
  the deck's EZERO and the reference's constants;
* the decks' NPOT, NV1, NV2 against what the runs printed (NPOT made even, the table's size).
"""
from __future__ import annotations

import json
import math
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

KAT = json.loads((Path(__file__).resolve().parent / "golden" / "dipole3_kat.json").read_text())["cases"]
AUTOCM, DETOSEC = 2.19474624e5, 3.136186e-07


def _half_unit(v: float, digits: int) -> float:
    """Half a unit of the last printed digit of 0.d..dD+ee with `digits` digits."""
    if v == 0.0:
        return 0.5 * 10.0 ** (-digits)
    return 0.5 * 10.0 ** (math.floor(math.log10(abs(v))) + 1 - digits)


@pytest.mark.parametrize("name", sorted(KAT))
def test_angular_rule_matches_printed(oracle_mod, name):
    q = KAT[name]["quadrature"]
    x, w, cs, ts = oracle_mod.dipole_quadrature(q["npnt"])
    assert len(q["x"]) == len(x) == q["npnt"] // 2
    np.testing.assert_allclose(x, q["x"], rtol=0, atol=5.1e-16)
    for got, want in zip(w, q["w"]):
        assert abs(got - want) <= _half_unit(want, 12) + 1e-17
    assert abs(cs - q["computed_sum"]) <= _half_unit(q["computed_sum"], 15) + 1e-16
    assert ts == q["exact_sum"] == 1.0


def _threej_exact(j1, j2, j3, m1, m2, m3) -> float:
    """Racah's closed form, in rational arithmetic under the square root."""
    if m1 + m2 + m3 != 0 or not (abs(j1 - j2) <= j3 <= j1 + j2) or any(abs(m) > j for m, j in ((m1, j1), (m2, j2), (m3, j3))):
        return 0.0
    f = math.factorial
    tri = Fraction(f(j1 + j2 - j3) * f(j1 - j2 + j3) * f(-j1 + j2 + j3), f(j1 + j2 + j3 + 1))
    pre = tri * f(j1 + m1) * f(j1 - m1) * f(j2 + m2) * f(j2 - m2) * f(j3 + m3) * f(j3 - m3)
    s = Fraction(0)
    for k in range(0, j1 + j2 + j3 + 1):
        den = [k, j1 + j2 - j3 - k, j1 - m1 - k, j2 + m2 - k, j3 - j2 + m1 + k, j3 - j1 - m2 + k]
        if min(den) < 0:
            continue
        s += Fraction((-1) ** k, math.prod(f(d) for d in den))
    return (-1) ** (j1 - j2 - m3) * math.sqrt(pre) * float(s)


def test_threej_exact(oracle_mod):
    n = 0
    for j1 in range(0, 6):
        for j3 in range(max(0, j1 - 1), j1 + 2):
            for m1 in range(-j1, j1 + 1):
                for m2 in (-1, 0, 1):
                    m3 = -m1 - m2
                    if abs(m3) > j3:
                        continue
                    want = _threej_exact(j1, 1, j3, m1, m2, m3)
                    got = oracle_mod.threej(j1, 1, j3, m1, m2, m3)
                    assert abs(got - want) <= 1e-14, (j1, j3, m1, m2, got, want)
                    n += 1
    assert n > 100


def _deck_ezero(deck: str) -> float:
    lines = [ln for ln in deck.splitlines()]
    i = next(k for k, ln in enumerate(lines) if "/" in ln)
    return float(lines[i + 3][:20].replace("D", "E").replace("d", "e"))


@pytest.mark.parametrize("name", sorted(KAT))
def test_spect_arithmetic_on_printed_rows(name):
    c = KAT[name]
    j1, j2 = c["j1"], c["j2"]
    ez = _deck_ezero(c["deck"])
    assert abs(ez - c["ezero"]) <= _half_unit(c["ezero"], 8)
    e1 = np.array(c["e_ket"]) * AUTOCM - ez
    e2 = np.array(c["e_bra"]) * AUTOCM - ez
    checked = 0
    for ie1, ie2, xe1, xe2, dd, tzd, txd, t, sxd, a in c["rows"]:
        if ie1 <= len(e1):
            assert abs(e1[ie1 - 1] - xe1) <= 1e-6
        if ie2 <= len(e2):
            assert abs(e2[ie2 - 1] - xe2) <= 1e-6
        assert abs((xe2 - xe1) - dd) <= 2e-6
        # |tzd + txd| from the printed (rounded) moments
        tol_t = 1e-8 * max(abs(tzd), abs(txd)) + 1e-15
        assert abs(abs(tzd + txd) - t) <= tol_t
        assert abs(t * t - sxd) <= 2 * t * tol_t + 1e-8 * sxd + 1e-30
        jup = j2 if dd > 0 else j1
        want_a = sxd * abs(dd) ** 3 * DETOSEC / (2 * jup + 1)
        # dd is printed to 1e-6 cm-1: relative 3e-6/|dd| in dd^3
        assert abs(want_a - a) <= a * (1e-7 + 4e-6 / abs(dd)) + 1e-30
        checked += 1
    assert checked == len(c["rows"]) > 0


@pytest.mark.parametrize("name", sorted(KAT))
def test_deck_cards(oracle_mod, name):
    deck = KAT[name]["deck"]
    lines = deck.splitlines()
    i = next(k for k, ln in enumerate(lines) if "/" in ln)
    card = lines[i + 2]
    npot = int(card[0:5])
    q = KAT[name]["quadrature"]
    # lagpt prints NPOT made even
    assert q["npnt"] == npot + npot % 2
    rows = KAT[name]["rows"]
    n1 = max(r[0] for r in rows)
    n2 = max(r[1] for r in rows)
    nv1, nv2 = int(card[5:10]), int(card[10:15])
    assert (n1, n2) == (nv1, nv2)
