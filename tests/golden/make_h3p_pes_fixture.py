"""Golden fixture for the PES-dependent stages: the reference's H3+ Jacobi J=0 example.

The reference ships one run whose levels depend on everything downstream of the potential:
H3+ in Jacobi coordinates, J = 0 (``H3+Jacobi/jobs/dvrJ0.job``), with its printed per-block
selection counts and 400 levels (``H3+Jacobi/results/result.H3p.J0.dvr:148-168`` and
``:174-502``). Its potential is the reference's POTV plug-in ``H3+Jacobi/source/pot_h3p.f90``
(Polyansky, Prosmiti, Klopper and Tennyson, Mol. Phys. 98, 261 (2000), fit 2).

This script, run once in a checkout that has the reference, writes ``h3p_jacobi_j0.npz``:

* ``deck``: the job deck text;
* ``v``: the potential on the DVR grid of the run, in the layout of DVR3D_PES_GRID
  (v[(ic*npnt2 + i2)*npnt1 + i1] = V(r1[i1], r2[i2], xalf[ic])), the grid taken from the
  oracle's quadrature (itself pinned to the printed points by test_oracle_kat.py);
* ``levels``: the 400 printed levels (Eh), ``counts``: the printed per-block counts,
  ``nham3``: the printed basis size.

The potential is evaluated by a restatement, written here, of the functional form of
pot_h3p.f90 (POTV: the switch between the many-body-expansion surface POTV1 and the
Morse-coordinate fit POTS through SOTV / POTV11; RJ; VLIM; VLIM1). Its coefficient tables
(the DATA statements and CA(i) assignments) are not copied: they are read from the
reference file each time the script runs. Nothing at test time reads the reference.

It also writes ``h3p_jacobi_j1.npz``, the J = 1 run of the same example (main_j1), and
``h3p_jacobi_dip.npz``, its dipole surface dip_h3p.f tabulated at the points of its DIPOLE3 job
(main_dip; the functional form restated here, its coefficients read from the reference file).

Run from the repository root:  python tests/golden/make_h3p_pes_fixture.py /path/to/reference
"""
from __future__ import annotations

import itertools
import math
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

DECK = "H3+Jacobi/jobs/dvrJ0.job"
RESULT = "H3+Jacobi/results/result.H3p.J0.dvr"
PES = "H3+Jacobi/source/pot_h3p.f90"


# --------------------------------------------------------------------------- Fortran data
def _num(tok: str) -> float:
    return float(tok.strip().replace("D", "E").replace("d", "e"))


def _units(src: str) -> dict[str, str]:
    """Program units of a free-form Fortran file (comments stripped, '&' continuations joined),
    keyed by upper-case name."""
    lines = []
    for raw in src.splitlines():
        code = raw.split("!", 1)[0].rstrip()
        lines.append(code)
    joined, cur = [], ""
    for ln in lines:
        s = ln.strip()
        if cur:
            s = s[1:] if s.startswith("&") else s
            cur += " " + s
        else:
            cur = s
        if cur.endswith("&"):
            cur = cur[:-1]
            continue
        joined.append(cur)
        cur = ""
    units, name = {}, None
    for ln in joined:
        m = re.match(r"(?i)\s*(?:double\s+precision\s+)?(subroutine|function|block\s+data)\s+(\w+)", ln)
        if m:
            name = m.group(2).upper()
            units[name] = ""
        if name:
            units[name] += ln + "\n"
    return units


def _data(unit: str) -> dict[str, list[float]]:
    """Values of the DATA statements of one program unit (repeat counts r*v expanded)."""
    out: dict[str, list[float]] = {}
    for stmt in re.findall(r"(?im)^\s*data\s+(.*)$", unit):
        for names, vals in re.findall(r"([\w\s,()]+?)\s*/([^/]*)/", stmt):
            vs = []
            for tok in vals.split(","):
                tok = tok.strip()
                if not tok:
                    continue
                if "*" in tok:
                    r, v = tok.split("*")
                    vs += [_num(v)] * int(r)
                else:
                    vs.append(_num(tok))
            names = [n.strip().upper() for n in names.split(",") if n.strip()]
            if len(names) == 1 and len(vs) > 1:
                out[names[0]] = vs
            else:
                for n, v in zip(names, vs):
                    out[n] = [v]
    return out


def read_coefficients(path: Path) -> dict:
    u = _units(path.read_text())
    top, v1, v11, pots, blk = (u["POTV"], u["POTV1"], u["POTV11"], u["POTS"], u["POT_POINTS"])
    c = {"potv": _data(top), "potv1": _data(v1), "potv11": _data(v11), "pots": _data(pots), "cv": _data(blk)["CV"]}
    # POTV1 overwrites its DATA values of CA with assignments CA(i) = ... before use; their
    # literals carry no D exponent, so Fortran stores them as default (single precision) reals
    ca = list(c["potv1"]["CA"])
    for i, v in re.findall(r"(?i)\bCA\(\s*(\d+)\s*\)\s*=\s*([-+]?[\d.]+(?:[dDeE][-+]?\d+)?)", v1):
        single = not re.search(r"[dD]", v)
        ca[int(i) - 1] = float(np.float32(_num(v))) if single else _num(v)
    c["ca"] = ca
    return c


# --------------------------------------------------------------------------- the surface
# Exponent patterns of the permutation-symmetric polynomial terms of the three-body parts of
# POTV1: term i is the sum over the distinct permutations of pattern i applied to (P1,P2,P3).
SYM_PATTERNS = [
    (1, 0, 0), (2, 0, 0), (1, 1, 0), (3, 0, 0), (2, 1, 0), (1, 1, 1), (4, 0, 0), (3, 1, 0), (2, 2, 0),
    (2, 1, 1), (5, 0, 0), (4, 1, 0), (3, 2, 0), (3, 1, 1), (2, 2, 1), (6, 0, 0), (5, 1, 0), (4, 2, 0),
    (3, 3, 0), (4, 1, 1), (3, 2, 1), (2, 2, 2), (7, 0, 0), (5, 2, 0), (6, 1, 0), (5, 1, 1), (4, 3, 0),
    (4, 2, 1), (3, 3, 1), (3, 2, 2),
]


def sym_poly(coef, p) -> float:
    s = 1.0
    for c, pat in zip(coef, SYM_PATTERNS):
        t = 0.0
        for e in set(itertools.permutations(pat)):
            t += p[0] ** e[0] * p[1] ** e[1] * p[2] ** e[2]
        s += c * t
    return s


BOHR_ANG = 0.52917706  # bohr -> angstrom of POTV1 / POTV11
EV = 0.036749          # eV -> hartree of POTV1 / POTV11
CM_PER_EH = 219474.6354


def vlim(r1, r2, xcos):
    """Long-range H+ + H2 term (hartree, bohr)."""
    rho = r1 - 1.39990951
    a0 = 2.6091 + (2.246 + (0.3181 - 0.1194 * rho) * rho) * rho
    a2 = 0.60735 + (1.3586 + (0.5573 - 0.3170 * rho) * rho) * rho
    q2 = 0.45886 + (0.53223 + (0.03234 - 0.091474 * rho) * rho) * rho
    p2 = 1.5 * xcos * xcos - 0.5
    return -(a0 + a2 * p2) / r2 ** 4 + q2 * p2 / r2 ** 3


def vlim1(r):
    """Long-range H + H2+ term (hartree, bohr)."""
    return -4.5 / r ** 4 - 15.0 / r ** 6


def _bond_lengths(q1, q2, q3):
    r3 = math.sqrt(q2 * q2 + (0.5 * q1) ** 2 + q1 * q2 * q3)
    r2 = math.sqrt(q2 * q2 + (0.5 * q1) ** 2 - q1 * q2 * q3)
    return [q1, r2, r3]


def _shortest_bond_jacobi(R):
    """Jacobi (r, R, cos) about the shortest bond, as the symmetrisation of POTV1 forms it."""
    dmin = min(R)
    q11 = math.sqrt((R[2] ** 2 + R[1] ** 2) * 0.5 - R[0] ** 2 / 4.0)
    q12 = math.sqrt((R[0] ** 2 + R[2] ** 2) * 0.5 - R[1] ** 2 / 4.0)
    q13 = math.sqrt((R[1] ** 2 + R[0] ** 2) * 0.5 - R[2] ** 2 / 4.0)
    if R[0] == dmin:
        q1, q2, other = R[0], q11, R[2]
    elif R[1] == dmin:
        q1, q2, other = R[1], q12, R[0]
    else:
        q1, q2, other = R[2], q13, R[1]
    q3 = (other ** 2 - q1 ** 2 / 4.0 - q2 ** 2) / (q1 * q2)
    return q1, q2, q3


def potv1(c, r, big_r, xcos):
    """Many-body-expansion surface with long-range switching (hartree)."""
    d = c["potv1"]
    dea, re1, a1, a2, a3 = (d[k][0] for k in ("DEA", "RE1", "A1", "A2", "A3"))
    deb, re2, a4, a5, a6 = (d[k][0] for k in ("DEB", "RE2", "A4", "A5", "A6"))
    v0a, r0a, g1a = (d[k][0] for k in ("V0A", "R0A", "G1A"))
    v0b, r0b, g1b = (d[k][0] for k in ("V0B", "R0B", "G1B"))
    v0, r0, g1 = (d[k][0] for k in ("V0", "R0", "G1"))
    dpi = d["DPI"][0]
    R = _bond_lengths(r * BOHR_ANG, big_r * BOHR_ANG, xcos)
    vaa2 = vbb2 = 0.0
    for x in R:
        pa, pb = x - re1, x - re2
        vaa2 += (1.0 + pa * (a1 + pa * (a2 + pa * a3))) * (-dea * math.exp(-a1 * pa))
        vbb2 += (1.0 + pb * (a4 + pb * (a5 + pb * a6))) * (-deb * math.exp(-a4 * pb))
    pa = [x - r0a for x in R]
    pb = [x - r0b for x in R]
    p = [x - r0 for x in R]
    t1a = t1b = t1 = 1.0
    for i in range(3):
        t1a *= 1.0 - math.tanh(0.5 * g1a * pa[i])
        t1b *= 1.0 - math.tanh(0.5 * g1b * pb[i])
        t1 *= 1.0 - math.tanh(0.5 * g1 * p[i])
    vaa3 = sym_poly(c["ca"], pa) * v0a * t1a
    vbb3 = sym_poly(d["CB"], pb) * v0b * t1b
    vab = sym_poly(d["C"], p) * v0 * t1
    q1, q2, q3 = _shortest_bond_jacobi(R)
    x1, x2, x3 = q1 / BOHR_ANG, q2 / BOHR_ANG, q3
    rlim, rmax = 4.5 * BOHR_ANG, 10.0 * BOHR_ANG
    if abs(q2) > rlim:
        sf1 = math.cos(0.5 * dpi * (q2 - rlim) / (rmax - rlim)) ** 2
        vpth = vlim(x1, x2, x3) / EV
        vaa3 = (1.0 - sf1) * vpth + sf1 * vaa3
        if q2 > rmax:
            vaa3 = vpth
    rlim1, rmax1 = 5.0 * BOHR_ANG, 11.0 * BOHR_ANG
    if abs(q1) > rlim1:
        vpth1 = vlim1(x1) / EV
        sf1 = math.cos(0.5 * dpi * (q1 - rlim1) / (rmax1 - rlim1)) ** 2
        vbb3 = (1.0 - sf1) * vpth1 + sf1 * vbb3
        if q1 > rmax1:
            vbb3 = vpth1
    vaa, vbb = vaa2 + vaa3, vbb2 + vbb3
    v = 0.5 * (vaa + vbb - math.sqrt((vaa - vbb) ** 2 + 4.0 * vab ** 2))
    return (v + 9.342357355) * EV


def pots(c, p1, p2, p3):
    """Morse-coordinate symmetric-stretch / bend fit (cm-1) of three bond lengths (bohr)."""
    d = c["pots"]
    re_, bet = d["RE"][0], d["BET"][0]
    nv, nfmax = int(d["NV"][0]), int(d["NFMAX"][0])
    fac = bet / re_
    dr = [p1 - re_, p2 - re_, p3 - re_]
    y = [(1.0 - math.exp(-fac * x)) / bet for x in dr]
    sa = (y[0] + y[1] + y[2]) / math.sqrt(3.0)
    sx1 = (2.0 * dr[2] - dr[0] - dr[1]) / (math.sqrt(2.0) * math.sqrt(3.0))
    sy1 = (dr[1] - dr[0]) / math.sqrt(2.0)
    se1 = math.sqrt(sx1 * sx1 + sy1 * sy1)
    phi = math.acos(sx1 / se1)
    ft = [1.0]
    for order in range(1, nfmax + 1):
        for n in range(order, -1, -1):
            for k in range(0, order - n + 1, 3):
                m = order - k - n
                if m % 2:
                    continue
                ft.append(sa ** n * se1 ** (m + k) * math.cos(k * phi))
    return sum(cv * f for cv, f in zip(c["cv"][:nv], ft[:nv]))


def sotv_scattering(c, r1, r2, xcos, g1):
    """SOTV for scattering coordinates (g2 = 0): bond lengths, then POTS (cm-1)."""
    xx, yy = r1 * g1, r1 * (1.0 - g1)
    tiny = 9.0e-15
    if r2 == 0.0 or xcos >= 1.0 - tiny:
        q1, q2 = abs(xx - r2), yy + r2
    elif xcos <= tiny - 1.0:
        q1, q2 = xx + r2, abs(yy + r2)
    else:
        q1 = math.sqrt(xx * xx + r2 * r2 - 2.0 * xx * r2 * xcos)
        q2 = math.sqrt(yy * yy + r2 * r2 + 2.0 * yy * r2 * xcos)
    return pots(c, q1, q2, r1)


def potv11(c, r, big_r, xcos, v22):
    """Fit surface v22 (hartree) joined to the H+ + H2 asymptote at large R (hartree)."""
    d = c["potv11"]
    dea, re1, a1, a2, a3 = (d[k][0] for k in ("DEA", "RE1", "A1", "A2", "A3"))
    dpi = d["DPI"][0]
    R = _bond_lengths(r * BOHR_ANG, big_r * BOHR_ANG, xcos)
    q1, q2, q3 = _shortest_bond_jacobi(R)
    # the diatom of the asymptote is the shortest bond (POTV11 moves it into R(1))
    x1, x2, x3 = q1 / BOHR_ANG, q2 / BOHR_ANG, q3
    rlim, rmax = 4.0 * BOHR_ANG, 7.0 * BOHR_ANG
    vaa3 = v22
    if abs(q2) > rlim:
        sf1 = math.cos(0.5 * dpi * (q2 - rlim) / (rmax - rlim)) ** 2
        pa = q1 - re1
        vaa2 = (1.0 + pa * (a1 + pa * (a2 + pa * a3))) * (-dea * math.exp(-a1 * pa))
        deconst = (37170.0 + 38180.0) / CM_PER_EH / EV
        vpth = (deconst + vaa2 + vlim(x1, x2, x3) / EV) * EV
        vaa3 = (1.0 - sf1) * vpth + sf1 * v22
        if q2 > rmax:
            vaa3 = vpth
    return vaa3


def potv(c, r1, r2, xcos, g1):
    """POTV(V, R1, R2, XCOS) of pot_h3p.f90 for scattering (Jacobi) coordinates, g2 = 0."""
    d = c["potv"]
    ediss, esp, m, ga1 = d["EDISS"][0], d["ESP"][0], int(d["M"][0]), d["GA1"][0]
    e0 = 0.5 * (ediss + esp)
    ga0 = 1.14877995 / (e0 - esp)
    v2 = sotv_scattering(c, r1, r2, xcos, g1)
    v1 = potv1(c, r1, r2, xcos)  # RJ leaves Jacobi coordinates unchanged
    v2 = potv11(c, r1, r2, xcos, v2 / CM_PER_EH)
    de = v1 - e0
    ga = ga0 + ga1 * de ** m
    ff = 0.5 * (1.0 + math.tanh(ga * de))
    ff1 = 0.5 * (1.0 + math.tanh(-ga * de))
    return ff * v1 + ff1 * v2


# --------------------------------------------------------------------------- printed output
def printed(text: str):
    counts = [int(x) for x in re.findall(r"npntc =\s*\d+, no\. of eigenvectors =\s*(\d+)", text)]
    nham3 = int(re.search(r"(\d+) eigenvalues selected from", text).group(1))
    i = text.index("eigenvalues in hartrees:")
    j = text.index("eigenvalues in wavenumbers:")
    levels = [_num(t) for t in re.findall(r"[-+]?\d\.\d+D[-+]\d+", text[i:j])]
    return counts, nham3, np.array(levels)


def main(ref_root: str) -> None:
    ref = Path(ref_root)
    from oracle import oracle

    deck = (ref / DECK).read_text()
    counts, nham3, levels = printed((ref / RESULT).read_text())
    coef = read_coefficients(ref / PES)
    d = oracle.parse_deck(deck)
    q = oracle.quadrature(d, 0)
    n1, n2, na = q.npnt1, q.npnt2, q.nidvr
    r1, r2, xa = np.array(q.r1[:n1]), np.array(q.r2[:n2]), np.array(q.xalf[:na])
    g1 = q.g1
    v = np.empty((na, n2, n1))
    for ia, x in enumerate(xa):
        for i2, b in enumerate(r2):
            for i1, a in enumerate(r1):
                v[ia, i2, i1] = potv(coef, a, b, x, g1)
    np.savez_compressed(HERE / "h3p_jacobi_j0.npz", deck=np.array(deck), v=v.ravel(), levels=levels,
                        counts=np.array(counts, dtype=np.int32), nham3=np.array(nham3),
                        r1=r1, r2=r2, xalf=xa)
    print(f"grid {na} x {n2} x {n1}, V in [{v.min():.6f}, {v.max():.6f}] Eh, "
          f"{len(levels)} printed levels, N = {nham3}, {len(counts)} blocks")


DECK_J1 = "H3+Jacobi/jobs/dvrJ1.job"
RESULT_J1 = "H3+Jacobi/results/result.H3p.J1even.dvr"
ROT_J1 = "H3+Jacobi/jobs/rot.job"
ROT_RESULT_J1 = "H3+Jacobi/results/result.H3p.J1even.rot"


def printed_j1(text: str):
    """Per k block of the J = 1 run: the printed counts, basis size and 400 levels."""
    out = []
    starts = [m.start() for m in re.finditer(r"point Gauss-associated Legendre integration with k =", text)]
    for a, b in zip(starts, starts[1:] + [len(text)]):
        out.append(printed(text[a:b]))
    return out


def printed_rot(text: str):
    """ROTLEV3's two printed lists of levels in hartrees (the e set, then the J = 1 f set)."""
    sets = []
    for m in re.finditer(r"LOWEST\s+(\d+) EIGENVALUES IN HARTREES", text):
        n = int(m.group(1))
        vals = re.findall(r"[-+]?\d\.\d+D[-+]\d+", text[m.end():])[:n]
        sets.append(np.array([_num(v) for v in vals]))
    return sets


def j1_deck(job: str, job_j0: str) -> str:
    """The J = 1 job deck as the printed run used it. The printed output (a June 2010 build) gives
    the rotational masses as 1.007276 u -- the J = 0 deck's second mass card, 1.007276470 --
    where the job file holds 1.0075372 twice, and its k = 1 levels carry mkham1's extra term for
    unequal vibrational and rotational masses, which the current source applies only with
    ZX = .TRUE. (:571-577, :2166-2171). So: the J = 0 deck's rotational-mass card, and ZX on.
    With these the oracle reproduces both blocks' 400 printed levels to their 12 digits."""
    lines = job.splitlines()
    lines_j0 = job_j0.splitlines()
    lines[7] = lines_j0[7]
    lines[1] = lines[1].replace("ztran=.true.,", "ztran=.true., zx=.true.,")
    assert "zx=.true." in lines[1]
    return "\n".join(lines) + "\n"


def main_j1(ref_root: str) -> None:
    """``h3p_jacobi_j1.npz``: the J = 1 (even, KMIN = 1) first step of the same example with the
    potential on the grid of each k block (k = 0, 1: each has its own associated Legendre points),
    its printed counts and levels per block, and ROTLEV3's deck (rot.job, KMIN = 2) with the two
    printed sets of levels (``result.H3p.J1even.rot``)."""
    ref = Path(ref_root)
    from oracle import oracle

    deck = j1_deck((ref / DECK_J1).read_text(), (ref / DECK).read_text())
    blocks = printed_j1((ref / RESULT_J1).read_text())
    rot = printed_rot((ref / ROT_RESULT_J1).read_text())
    coef = read_coefficients(ref / PES)
    d = oracle.parse_deck(deck)
    out = {"deck": np.array(deck), "rot_deck": np.array((ref / ROT_J1).read_text()),
           "rot_e": rot[0], "rot_f": rot[1]}
    for k in (0, 1):
        q = oracle.quadrature(d, k)
        n1, n2, na = q.npnt1, q.npnt2, q.nidvr
        r1, r2, xa = np.array(q.r1[:n1]), np.array(q.r2[:n2]), np.array(q.xalf[:na])
        v = np.empty((na, n2, n1))
        for ia, x in enumerate(xa):
            for i2, b in enumerate(r2):
                for i1, a in enumerate(r1):
                    v[ia, i2, i1] = potv(coef, a, b, x, q.g1)
        counts, nham3, levels = blocks[k]
        out.update({f"v{k}": v.ravel(), f"xalf{k}": xa, f"levels{k}": levels,
                    f"counts{k}": np.array(counts, dtype=np.int32), f"nham3_{k}": np.array(nham3)})
    np.savez_compressed(HERE / "h3p_jacobi_j1.npz", **out)
    print(f"J=1: {len(blocks)} blocks, {[len(b[2]) for b in blocks]} levels, ROTLEV3 sets {[len(r) for r in rot]}")


DIP = "H3+Jacobi/source/dip_h3p.f"
DIP_JOB = "H3+Jacobi/jobs/dip.job"


def read_dipole(path: Path) -> dict:
    """BETA, RE and the seven D coefficients of DIPD's DATA statements (dip_h3p.f :15-17), taken
    at the precision of the DOUBLE PRECISION variables they initialise: the printed moments of
    the example's dipole run agree with these to the printed digits, while the same literals
    rounded to single precision first leave 2e-8 relative differences (the printing build's
    compiler converted DATA constants to the variables' type from their text)."""
    src = path.read_text()
    unit = src[:src.upper().index("SUBROUTINE DIPD0")]
    out = {}
    for stmt in re.findall(r"(?im)^\s+DATA\s+(.*(?:\n\s+\d(.*))*)", unit):
        text = re.sub(r"\n\s+\d", "", stmt[0])
        for name, vals in re.findall(r"(\w+)\s*/([^/]*)/", text):
            toks = [t.strip() for t in vals.split(",") if t.strip()]
            out[name.upper()] = [_num(t) for t in toks]
    return {"BETA": out["BETA"][0], "RE": out["RE"][0], "D": out["D"]}


def h3p_dipd(c: dict, r1: float, r2: float, xcos: float, nu: int, g1: float, xmass, zembed: bool) -> float:
    """DIPD of dip_h3p.f (the surface of Roeshe et al., J. Chem. Phys. 101, 2231 (1994)) in
    scattering coordinates: symmetry coordinates of the Morse-type bond displacements, the
    z and x components of the body-fixed dipole, and the component nu in the embedding of the
    wavefunctions (z along r2 if ZEMBED, else along r1)."""
    beta, re_, d = c["BETA"], c["RE"], c["D"]
    sr2, sr3 = math.sqrt(2.0), math.sqrt(3.0)
    sr6 = sr2 * sr3
    a, b = r1 * g1, r1 - r1 * g1
    bonds = (r1, math.sqrt(r2 * r2 + a * a - 2.0 * a * r2 * xcos), math.sqrt(r2 * r2 + b * b + 2.0 * b * r2 * xcos))
    disp = [(1.0 - math.exp(-beta * (q / re_ - 1.0))) / beta for q in bonds]
    sa = sum(disp) / sr3
    sz = (2.0 * disp[0] - disp[1] - disp[2]) / sr6
    sx = (disp[2] - disp[1]) / sr2
    se2 = sz * sz + sx * sx
    fz = [sz, sz * sa, sz * sa * sa, sz * sa * sa * sa, sz * sz - sx * sx, (sz * sz - sx * sx) * sa, se2 * sz]
    fx = [sx, sx * sa, sx * sa * sa, sx * sa * sa * sa, -2.0 * sz * sx, -2.0 * sz * sx * sa, se2 * sx]
    dipz = sum(di * f for di, f in zip(d, fz)) * r2 * sr2 / sr3 - (r2 * xmass[0] / sum(xmass) - r2 / 3.0)
    dipx = sum(di * f for di, f in zip(d, fx)) * r1 / sr2
    xsin = math.sqrt(1.0 - xcos * xcos)
    if zembed:
        return dipz + xcos * dipx if nu == 0 else dipx * xsin
    return -(dipx + xcos * dipz) if nu == 0 else dipz * xsin


def main_dip(ref_root: str) -> None:
    """``h3p_jacobi_dip.npz``: the example's dipole job (dip.job: NPOT = 80, 8 x 8 levels between
    the J = 0 odd run and the J = 1 e set of ROTLEV3), the J = 1 job deck that run's vectors came
    from, and its DIPD evaluated, both components, at
    every radial grid point pair and at the +-x of DIPOLE3's 80-point Gauss-Legendre rule (the
    points DIPOLE3 calls it at), with the ket file's masses, g1 and embedding."""
    ref = Path(ref_root)
    from oracle import oracle

    c = read_dipole(ref / DIP)
    deck = (ref / DECK).read_text()
    d = oracle.parse_deck(deck)
    q = oracle.quadrature(d, 0)
    r1, r2 = np.array(q.r1[:q.npnt1]), np.array(q.r2[:q.npnt2])
    x, _, _, _ = oracle.dipole_quadrature(80)
    xs = np.concatenate([np.asarray(x), -np.asarray(x)])
    xmass = list(d.xmass[:3])
    tab = np.empty((2, len(xs), len(r2), len(r1)))
    for nu in (0, 1):
        for ix, xc in enumerate(xs):
            for i2, b in enumerate(r2):
                for i1, a in enumerate(r1):
                    tab[nu, ix, i2, i1] = h3p_dipd(c, a, b, xc, nu, q.g1, xmass, bool(d.zembed))
    # the J = 1 vectors of the printed dipole run come from the J = 1 job as shipped (both mass
    # cards 1.0075372, no ZX): its bra energies are that run's ROTLEV3 e set to 1e-8 cm-1, unlike
    # the printed first-step and ROTLEV3 outputs of the J = 1 example (j1_deck)
    np.savez_compressed(HERE / "h3p_jacobi_dip.npz", deck=np.array((ref / DIP_JOB).read_text()), table=tab,
                        r1=r1, r2=r2, xcos=xs, deck_j1=np.array((ref / DECK_J1).read_text()))
    print(f"dipole table {tab.shape}, |mu| <= {np.abs(tab).max():.4f} a.u.")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    main(root)
    main_j1(root)
    main_dip(root)
