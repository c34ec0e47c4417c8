"""Seeded synthetic workloads (job decks + potential parameters).

The reference ships no benchmark inputs for these sizes, so each workload is a DVR3DRJZ
job deck in the reference's card format plus the parameters of the DVR3D_PES_MORSE_SUM
potential family:

    V = D1 (1-exp(-a1 (r1-re1)))^2 + D2 (1-exp(-a2 (r2-re2)))^2
        + kb (cos t - c0)^2 + c12 (r1-re1)(r2-re2) + sum_l cl P_l(cos t)

The Morse range parameters a1, a2 of the surface are not given by the workload
descriptions; they are set to the Morse basis exponent of the same coordinate,
beta = we sqrt(mu / (2 De)) (setcon :1123), so basis and surface share one Morse shape.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

AMTOAU = 1.8228883e03
AUTOCM = 2.19474624e5


@dataclass
class Workload:
    name: str
    deck: str
    pes: np.ndarray
    nlevels: int
    notes: dict = field(default_factory=dict)


def _f20(*vals) -> str:
    return "".join(f"{v:20.10f}" for v in vals)


def deck_text(*, title: str, npnt2: int, jrot: int, neval: int, nalf: int, max2d: int, max3d: int,
              idia: int, kmin: int, npnt1: int, ipar: int, masses, emax1: float, emax2: float,
              morse1, morse2, flags: dict | None = None, max3d2: int = 0) -> str:
    fl = {"ZPMIN": True}
    fl.update(flags or {})
    nl = " &PRT " + ", ".join(f"{k}=.{'TRUE' if v else 'FALSE'}." for k, v in fl.items()) + ", /"
    card3 = "".join(f"{v:5d}" for v in (npnt2, jrot, neval, nalf, max2d, max3d, idia, kmin, npnt1, ipar, max3d2))
    lines = [nl, f"{3:5d}", card3, title[:72], "", _f20(*masses), _f20(*masses),
             _f20(emax1, emax2), _f20(*morse1), _f20(*morse2)]
    return "\n".join(lines) + "\n"


def reduced_masses(masses, idia: int):
    m1, m2, m3 = masses
    if idia >= 1:
        g1, g2 = m2 / (m2 + m3), 0.0
    else:
        a = math.sqrt(m3 / (m1 + m2 + m3))
        b = m2 / (m1 + m2)
        g1 = 1.0 - a / (a + b - a * b)
        g2 = 1.0 - a / (1.0 - b + a * b)
    ur1 = AMTOAU / (g2 * g2 / m1 + 1.0 / m2 + (1.0 - g2) ** 2 / m3)
    ur2 = AMTOAU / (1.0 / m1 + g1 * g1 / m2 + (1.0 - g1) ** 2 / m3)
    return ur1, ur2


def morse_beta(we: float, mu: float, de: float) -> float:
    return we * math.sqrt(0.5 * mu / de)


def pes_row(D1, a1, re1, D2, a2, re2, kb=0.0, c0=0.0, c12=0.0, c1=0.0, c2=0.0, c3=0.0, c4=0.0) -> np.ndarray:
    return np.array([D1, a1, re1, D2, a2, re2, kb, c0, c12, c1, c2, c3, c4], dtype=np.float64)


# ------------------------------------------------------------------ Radau family (1-3)
H2O_MASSES = (1.007825, 1.007825, 15.994915)


def radau_water_like(npnt: int, nalf: int, emax2_cm: float, neval: int, *, re=1.81, de=0.20, we=0.0172,
                     kb=0.08, max3d=20000, zcut=True, title="Radau synthetic water-like") -> Workload:
    ur1, _ = reduced_masses(H2O_MASSES, -2)
    beta = morse_beta(we, ur1, de)
    deck = deck_text(title=title, npnt2=npnt, jrot=0, neval=neval, nalf=nalf, max2d=0, max3d=max3d,
                     idia=-2, kmin=0, npnt1=0, ipar=0, masses=H2O_MASSES, emax1=0.0, emax2=emax2_cm,
                     morse1=(re, de, we), morse2=(0.0, 0.0, 0.0), flags={"ZCUT": zcut})
    pes = pes_row(de, beta, re, de, beta, re, kb=kb, c0=-0.2504, c12=0.01)
    return Workload(title, deck, pes, neval, {"beta": beta})


def config1() -> Workload:
    """Radau idia=-2, J=0, NPNT=21, NALF=40, 2D cut-off 40000 cm-1, lowest 200 levels."""
    return radau_water_like(21, 40, 40000.0, 200, title="cfg1 Radau NPNT=21 NALF=40")


def config2() -> Workload:
    """Same family at NPNT=30, NALF=64; 2D cut-off chosen for a final basis of ~4000."""
    return radau_water_like(30, 64, 62000.0, 300, title="cfg2 Radau NPNT=30 NALF=64")


def config3(seed: int = 2024, nprob: int = 64) -> list[Workload]:
    """64 independent Radau J=0 problems with seeded sizes and surfaces."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nprob):
        npnt = int(rng.integers(16, 33))
        nalf = int(rng.integers(24, 65))
        re = float(rng.uniform(1.7, 1.9))
        de = float(rng.uniform(0.15, 0.25))
        kb = float(rng.uniform(0.05, 0.12))
        max3d = int(rng.integers(800, 3001))
        w = radau_water_like(npnt, nalf, 0.0, 100, re=re, de=de, kb=kb, max3d=max3d, zcut=False,
                             title=f"cfg3 problem {i}")
        out.append(w)
    return out


# ------------------------------------------------------------------ Jacobi family (4, 5)
H3P_MASSES = (1.007276, 1.007276, 1.007276)


def jacobi_h3p_like(npnt1: int, npnt2: int, nalf: int, emax1_cm: float, emax2_cm: float, neval: int, *,
                    seed: int = 7, max2d: int = 4000, max3d: int = 40000, title="Jacobi synthetic") -> Workload:
    """Jacobi coordinates, three equal masses; r1 = diatom bond, r2 = atom-diatom distance."""
    rng = np.random.default_rng(seed)
    c1, c2 = (float(x) for x in rng.uniform(-0.02, 0.02, size=2))
    ur1, ur2 = reduced_masses(H3P_MASSES, 1)
    re1, de1, we1 = 1.65, 0.17, 0.0125
    re2, de2, we2 = 1.43, 0.12, 0.0110
    b1, b2 = morse_beta(we1, ur1, de1), morse_beta(we2, ur2, de2)
    deck = deck_text(title=title, npnt2=npnt2, jrot=0, neval=neval, nalf=nalf, max2d=max2d, max3d=max3d,
                     idia=1, kmin=0, npnt1=npnt1, ipar=0, masses=H3P_MASSES, emax1=emax1_cm,
                     emax2=emax2_cm, morse1=(re1, de1, we1), morse2=(re2, de2, we2),
                     flags={"ZCUT": True, "ZTHETA": False, "ZR2R1": True})
    pes = pes_row(de1, b1, re1, de2, b2, re2, c1=c1, c2=c2)
    return Workload(title, deck, pes, neval, {"c1": c1, "c2": c2, "beta1": b1, "beta2": b2})


# cut-offs of the headline workload, fixed once against the oracle's 1D/2D stages
CFG4_EMAX1 = 50000.0
CFG4_EMAX2 = 40000.0


def config4(emax1: float = CFG4_EMAX1, emax2: float = CFG4_EMAX2) -> Workload:
    """Jacobi, equal masses 1.007276 u, NPNT1=NPNT2=40, NALF=80, lowest 500 levels."""
    return jacobi_h3p_like(40, 40, 80, emax1, emax2, 500, title="cfg4 Jacobi NPNT=40/40 NALF=80")


HCN_MASSES = (1.007825, 12.0, 14.003074)


# cut-offs of the J=2 workload, fixed once against the oracle's 1D/2D stages (N ~ 20500 per k)
CFG5_EMAX1 = 65000.0
CFG5_EMAX2 = 64000.0


def config5(emax1: float = CFG5_EMAX1, emax2: float = CFG5_EMAX2) -> Workload:
    """Jacobi, H/C/N masses, J=2 with k = 0, 1, 2 blocks, NPNT1=50, NPNT2=30, NALF=100."""
    ur1, ur2 = reduced_masses(HCN_MASSES, 1)
    re1, de1, we1 = 2.18, 0.30, 0.0095
    re2, de2, we2 = 3.19, 0.20, 0.0150
    b1, b2 = morse_beta(we1, ur1, de1), morse_beta(we2, ur2, de2)
    deck = deck_text(title="cfg5 Jacobi HCN-like J=2", npnt2=30, jrot=2, neval=1000, nalf=100, max2d=1500,
                     max3d=40000, idia=1, kmin=1, npnt1=50, ipar=0, masses=HCN_MASSES, emax1=emax1,
                     emax2=emax2, morse1=(re1, de1, we1), morse2=(re2, de2, we2),
                     flags={"ZCUT": True, "ZTHETA": False, "ZR2R1": False, "ZEMBED": False, "ZROT": True,
                            "ZLIN": True})
    pes = pes_row(de1, b1, re1, de2, b2, re2, kb=0.05, c0=1.0)
    return Workload("cfg5", deck, pes, 1000)
