"""DIPOLE3 pinned to the transition moments the reference printed for its H3+ Jacobi example.

The chain of the example: the J = 0 odd first step (``H3+Jacobi/jobs/dvrJ0.job``), the J = 1
first step and ROTLEV3 (KMIN = 2, e set to unit KVEC), then DIPOLE3 (``dip.job``: NPOT = 80, the
lowest 8 x 8 states) with the example's dipole surface (``H3+Jacobi/source/dip_h3p.f``). Its
printed table (``H3+Jacobi/results/result.H3p.dip``; the 64 rows in
``tests/golden/dipole3_kat.json``) gives per pair of states the two energies, the z and x
transition moments, |t|, S(f-i) and the Einstein A coefficient. The surface is tabulated at the
points DIPOLE3 evaluates it (``h3p_jacobi_dip.npz``, make_h3p_pes_fixture.py) and given as the
DIPD plug-in; the potentials are the first-step fixtures'. The printed run's J = 1 vectors come
from the J = 1 job as shipped (``dvrJ1.job``: no ZX, the vibrational masses on both cards) --
its bra energies are that chain's ROTLEV3 levels to 1e-8 cm-1 -- so the chain here runs that
deck, not the one that reproduces the printed J = 1 first-step and ROTLEV3 outputs.

* CPU: the oracle's whole chain (first steps written by jacobi_wave.py, its ROTLEV3 and its
  DIPOLE3) reproduces every printed row.
* GPU: the product's chain (first steps with ZTRAN, ROTLEV3, DIPOLE3 through the C ABI) does too.

The moments' signs follow the phases of the two states, which the eigensolvers choose freely, so
the rows are compared through |tz|, |tx|, t = |tz + tx| (tz and tx of a row share the phase) and
the quantities built from t.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from jacobi_wave import write_jacobi_wave

GOLD = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def fix():
    j0 = np.load(GOLD / "h3p_jacobi_j0.npz")
    j1 = np.load(GOLD / "h3p_jacobi_j1.npz")
    dip = np.load(GOLD / "h3p_jacobi_dip.npz")
    kat = json.loads((GOLD / "dipole3_kat.json").read_text())["cases"]["h3p_jacobi_dip"]
    return {"j0": {k: j0[k] for k in j0.files}, "j1": {k: j1[k] for k in j1.files},
            "dip": {k: dip[k] for k in dip.files}, "rows": kat["rows"]}


class TabulatedDipole:
    """DIPD(r1, r2, xcos, nu) from the table: the nearest tabulated point, which must lie within
    1e-10 of the requested one (every miss is recorded, and the test then fails)."""

    def __init__(self, dip: dict):
        self.t, self.r1, self.r2, self.xc = dip["table"], dip["r1"], dip["r2"], dip["xcos"]
        self.misses = []
        self.calls = 0

    @staticmethod
    def _near(grid, v):
        i = int(np.argmin(np.abs(grid - v)))
        return i, abs(grid[i] - v)

    def __call__(self, r1, r2, xcos, nu):
        self.calls += 1
        i1, d1 = self._near(self.r1, r1)
        i2, d2 = self._near(self.r2, r2)
        ix, dx = self._near(self.xc, xcos)
        if max(d1, d2, dx) > 1e-10 or nu not in (0, 1):
            self.misses.append((r1, r2, xcos, nu))
            return 0.0
        return float(self.t[nu, ix, i2, i1])


def table_rows(text: str) -> list[list[float]]:
    rows = []
    for ln in text.splitlines():
        f = ln.split()
        if len(f) == 10 and f[0].isdigit() and f[1].isdigit():
            rows.append([float(x) for x in f])
    return rows


def half_unit(v: float) -> float:
    """Half a unit of the last digit of v printed as es15.8."""
    return 0.5e-8 * 10.0 ** np.floor(np.log10(abs(v))) if v != 0.0 else 0.5e-8


def check_rows(got: list[list[float]], printed: list[list[float]]) -> float:
    """Every printed row against the computed one, both rounded to the printed digits: the
    energies (f14.6), |tz|, |tx| and t within one unit of their last es15.8 digit plus 3e-10 of
    the row's largest moment; S(f-i) and A through t.
    Returns the largest moment error relative to the row's largest moment."""
    assert len(got) == len(printed) == 64
    worst = 0.0
    for g, p in zip(got, printed):
        assert g[:2] == p[:2]
        np.testing.assert_allclose(g[2:5], p[2:5], rtol=0, atol=1.5e-6)  # cm-1, f14.6
        scale = max(abs(p[5]), abs(p[6]))
        for a, b in ((abs(g[5]), abs(p[5])), (abs(g[6]), abs(p[6])), (g[7], p[7])):
            err = abs(a - b)
            # both numbers are rounded to the printed digits: one unit of the last one apart at most
            assert err <= 2 * half_unit(b) + 3e-10 * scale, (p[:2], a, b)
            worst = max(worst, err / scale)
        tol_t = 2 * half_unit(p[7]) + 3e-10 * scale
        assert abs(g[8] - p[8]) <= 2 * p[7] * tol_t + tol_t * tol_t + half_unit(p[8]) + 1e-30
        assert abs(g[9] - p[9]) <= p[9] * (2 * tol_t / max(p[7], 1e-300) + 1e-7) + half_unit(p[9]) + 1e-30
    return worst


def test_fixture_shapes(fix):
    d = fix["dip"]
    assert d["table"].shape == (2, 80, 21, 20)
    assert "  80   08   08" in str(d["deck"])


@pytest.fixture(scope="module")
def oracle_chain(oracle_mod, fix, tmp_path_factory):
    d = tmp_path_factory.mktemp("dipj")
    write_jacobi_wave(d / "j0.26", oracle_mod, str(fix["j0"]["deck"]), {0: fix["j0"]["v"]})
    j1 = fix["j1"]
    write_jacobi_wave(d / "j1.26", oracle_mod, str(fix["dip"]["deck_j1"]), {0: j1["v0"], 1: j1["v1"]})
    oracle_mod.rotlev3(str(j1["rot_deck"]), str(d / "j1.26"), str(d / "j1.8"), str(d / "j1.9"))
    return d


def test_oracle_chain_reproduces_printed_moments(oracle_mod, fix, oracle_chain, tmp_path):
    d = oracle_chain
    dipd = TabulatedDipole(fix["dip"])
    r = oracle_mod.dipole3(str(fix["dip"]["deck"]), str(d / "j0.26"), str(d / "j1.8"), dipd=dipd,
                           tra_path=str(tmp_path / "o.13"))
    assert dipd.calls > 0 and not dipd.misses, dipd.misses[:3]
    assert (r["j1"], r["j2"]) == (0, 1)
    worst = check_rows(table_rows(r["text"]), fix["rows"])
    assert worst < 1e-8


@pytest.mark.gpu
def test_product_chain_reproduces_printed_moments(ctx, fix, tmp_path):
    j0, j1 = fix["j0"], fix["j1"]
    ctx.set_pes_grid(j0["v"])
    ctx.run_deck(str(j0["deck"]), wave_path=str(tmp_path / "j0.26"))
    ctx.set_pes_grid_k(0, j1["v0"])
    ctx.set_pes_grid_k(1, j1["v1"])
    try:
        ctx.run_deck(str(fix["dip"]["deck_j1"]), wave_path=str(tmp_path / "j1.26"))
    finally:
        ctx.set_pes_grid_k(0, [])
        ctx.set_pes_grid_k(1, [])
    ctx.rotlev3(str(j1["rot_deck"]), str(tmp_path / "j1.26"), str(tmp_path / "j1.8"), str(tmp_path / "j1.9"))
    dipd = TabulatedDipole(fix["dip"])
    r = ctx.dipole3(str(fix["dip"]["deck"]), str(tmp_path / "j0.26"), str(tmp_path / "j1.8"), dipd=dipd,
                    tra_path=str(tmp_path / "g.13"))
    assert dipd.calls > 0 and not dipd.misses, dipd.misses[:3]
    worst = check_rows(table_rows(r["text"]), fix["rows"])
    assert worst < 1e-8
