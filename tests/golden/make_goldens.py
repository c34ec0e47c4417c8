"""Extract the PES-independent known-answer data of the reference's example runs.

Reads the job decks and printed outputs shipped with the reference (ExoMol/dvr3d) and
writes ``quadrature_kat.json`` next to this script: for each example the deck text and,
per k block, the printed Gauss-Laguerre points / r values / check sums (lagpt :1315-1361),
Gauss-(associated) Legendre points / weights / check sums (ccmain :932-938) and, for the
z-perpendicular embedding, Gauss-Jacobi points / weights (ccmain :956-960); and the
Gauss-associated Legendre rules ROTLEV3B prints (rotlev3b_segmented.f90 :752-757).
It also writes ``dipole3_kat.json``: for each DIPOLE3 example (dipole3_segmented.f90) the
deck, the printed angular rule, the ket / bra energies, spect's header and every printed
row of its transition table.

The printed Laguerre "weights" column of these outputs comes from a later build of the
program (outputs say "version of June 2010", the source "March 2002") that prints a
different weight normalisation, so only points, r values and point sums are kept for the
radial quadrature; the angular weights and sums are those of the source's routine.

Run from the repository root:  python tests/golden/make_goldens.py /path/to/reference
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent

CASES = {
    "water_J0": ("water/jobs/dvr0.job", "water/results/result-0.water.dvr"),
    "h3p_jacobi_J0": ("H3+Jacobi/jobs/dvrJ0.job", "H3+Jacobi/results/result.H3p.J0.dvr"),
    "hcn_J2": ("HCN/jobs/dvr.job", "HCN/results/result.HCN.dvr"),
    "h3p_radau_zperp_J0": ("H3+Radau/jobs/dvr_J0.job", "H3+Radau/results/result.H3p_J0.dvr"),
    "h3p_radau_zperp_J1_ipar0": ("H3+Radau/jobs/dvr_J1_0.job", "H3+Radau/results/result.H3p_J1_0.dvr"),
    "h3p_radau_zperp_J1_ipar1": ("H3+Radau/jobs/dvr_J1_1.job", "H3+Radau/results/result.H3p_J1_1.dvr"),
}

FNUM = r"[-+]?\d*\.\d+(?:[DdEe][-+]?\d+)?"


def fnum(s: str) -> float:
    return float(s.replace("D", "E").replace("d", "e"))


def parse_output(text: str) -> dict:
    lines = text.splitlines()
    lag = []
    leg = []
    jac = []
    i = 0
    while i < len(lines):
        ln = lines[i]
        m = re.search(r"(\d+) POINT GAUSS-LAGUERRE INTEGRATION", ln, re.I)
        if m:
            npt = int(m.group(1))
            which = "r1" if "R1" in lines[i + 1].upper() else "r2"
            pts = []
            j = i + 2
            while len(pts) < npt:
                t = lines[j].split()
                if len(t) == 3:
                    try:
                        pts.append((fnum(t[0]), fnum(t[2])))
                    except ValueError:
                        pass
                j += 1
            # sums: "COMPUTED SUM OF POINTS x & WEIGHTS y" then "EXACT ..."
            while "SUM OF POINTS" not in lines[j].upper():
                j += 1
            comp = re.findall(FNUM, lines[j])
            exact = re.findall(FNUM, lines[j + 1])
            lag.append({"coord": which, "n": npt, "y": [p[0] for p in pts], "r": [p[1] for p in pts],
                        "sum_points": fnum(comp[0]), "exact_sum_points": fnum(exact[0])})
            i = j + 2
            continue
        m = re.search(r"(\d+) point Gauss-associated Legendre integration with k =\s*(\d+)", ln)
        if m:
            nang, k = int(m.group(1)), int(m.group(2))
            xs, ws = [], []
            j = i + 1
            while not lines[j].strip().startswith("Computed sum of weights"):
                t = lines[j].split()
                if len(t) == 2:
                    try:
                        xs.append(fnum(t[0]))
                        ws.append(fnum(t[1]))
                    except ValueError:
                        pass
                j += 1
            comp = fnum(re.findall(FNUM, lines[j])[0])
            exact = fnum(re.findall(FNUM, lines[j + 1])[0])
            leg.append({"nang": nang, "k": k, "x": xs, "w": ws, "computed_sum": comp, "exact_sum": exact})
            i = j + 2
            continue
        # z-perp embedding: gaujac points and weights (ccmain :956-960), no check sums
        m = re.search(r"(\d+) point Gauss-Jacobi integration with alpha = beta =\s*(" + FNUM + ")", ln)
        if m:
            nang, alf = int(m.group(1)), float(m.group(2))
            xs, ws = [], []
            j = i + 1
            while len(xs) < (nang + 1) // 2 and j < len(lines):
                t = lines[j].split()
                if len(t) == 2:
                    try:
                        xs.append(fnum(t[0]))
                        ws.append(fnum(t[1]))
                    except ValueError:
                        pass
                j += 1
            jac.append({"nang": nang, "alpha_printed": alf, "x": xs, "w": ws})
            i = j
            continue
        i += 1
    return {"laguerre": lag, "legendre": leg, "gauss_jacobi": jac}


# ROTLEV3B runs: its own Gauss-associated Legendre rule (jacobi :941-1007), printed by angin1
# (:752-757) for each k of a Coriolis block pair.
ROT_CASES = {
    "water_rot_even": "water/results/result-even.water.rot",
    "water_rot_odd": "water/results/result-odd.water.rot",
}


def parse_rot_output(text: str) -> list:
    lines = text.splitlines()
    out = []
    i = 0
    while i < len(lines):
        m = re.search(r"(\d+) point gauss-associated legendre integration with k =\s*(\d+)", lines[i])
        if m:
            npnt, k = int(m.group(1)), int(m.group(2))
            xs, ws = [], []
            j = i + 1
            while "computed sum of weights" not in lines[j]:
                t = lines[j].split()
                if len(t) == 2:
                    try:
                        xs.append(fnum(t[0]))
                        ws.append(fnum(t[1]))
                    except ValueError:
                        pass
                j += 1
            comp = fnum(re.findall(FNUM, lines[j])[0])
            exact = fnum(re.findall(FNUM, lines[j + 1])[0])
            out.append({"npnt": npnt, "k": k, "x": xs, "w": ws, "computed_sum": comp, "exact_sum": exact})
            i = j + 2
            continue
        i += 1
    return out


# DIPOLE3 runs: lagpt's Gauss-Legendre rule (jacobi :1311-1368, printed :1199-1206), spect's
# header (:1881-1890) and its table of transitions (:1929-1948), with the ket and bra energies
# dmain prints (:802-815).
DIP_CASES = {
    "water_dip": ("water/jobs/dip.job", "water/results/result.water.dip"),
    "h3p_jacobi_dip": ("H3+Jacobi/jobs/dip.job", "H3+Jacobi/results/result.H3p.dip"),
    "hcn_dip": ("HCN/jobs/dip.job", "HCN/results/result.HCN.dip"),
}


def parse_dip_output(text: str) -> dict:
    lines = text.splitlines()
    out = {"quadrature": parse_rot_output(text)[0]}
    for ln in lines:
        m = re.search(r"j1=\s*(-?\d+)\s+kmin1=\s*(-?\d+)\s+j2=\s*(-?\d+)\s+kmin2=\s*(-?\d+)\s+idia=\s*(-?\d+)"
                      r"\s+ipar1=\s*(-?\d+)\s+ipar2=\s*(-?\d+)", ln)
        if m:
            out.update(zip(("j1", "kmin1", "j2", "kmin2", "idia", "ipar1", "ipar2"), map(int, m.groups())))
        m = re.search(r"ground zero =\s*(\S+) cm-1", ln)
        if m:
            out["ezero"] = fnum(m.group(1))
    for side in ("ket", "bra"):
        i = next(k for k, ln in enumerate(lines) if f"First 10 energies for the {side} in a.u." in ln)
        vals, j = [], i + 1
        while len(vals) < 10 and j < len(lines):
            toks = lines[j].split()
            if toks and not all(re.fullmatch(FNUM, t) for t in toks):
                break
            vals += [fnum(t) for t in toks]
            j += 1
        out[f"e_{side}"] = vals
    rows = []
    head = next(k for k, ln in enumerate(lines) if ln.lstrip().startswith("ie1 ie2"))
    for ln in lines[head + 1:]:
        toks = ln.split()
        if len(toks) == 10 and toks[0].isdigit() and toks[1].isdigit():
            rows.append([int(toks[0]), int(toks[1])] + [float(t) for t in toks[2:]])
    out["rows"] = rows
    return out


def main(ref: str) -> None:
    root = Path(ref)
    out = {"source": "ExoMol/dvr3d example decks and printed outputs", "cases": {}}
    for name, (job, res) in CASES.items():
        deck = (root / job).read_text()
        data = parse_output((root / res).read_text())
        data["deck"] = deck
        data["deck_file"] = job
        data["output_file"] = res
        out["cases"][name] = data
    out["rot_cases"] = {name: {"output_file": res, "legendre": parse_rot_output((root / res).read_text())}
                        for name, res in ROT_CASES.items()}
    (HERE / "quadrature_kat.json").write_text(json.dumps(out, indent=1))
    print("wrote", HERE / "quadrature_kat.json")
    dip = {"source": "ExoMol/dvr3d DIPOLE3 example decks and printed outputs", "cases": {}}
    for name, (job, res) in DIP_CASES.items():
        data = parse_dip_output((root / res).read_text())
        data["deck"] = (root / job).read_text()
        data["deck_file"] = job
        data["output_file"] = res
        dip["cases"][name] = data
    (HERE / "dipole3_kat.json").write_text(json.dumps(dip, indent=1))
    print("wrote", HERE / "dipole3_kat.json")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
