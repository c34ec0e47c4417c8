"""Run one solve of a named workload (for profiler captures such as ncu).

    python -m dvr3d_b200.profile_case --case jacobi24 [--precision fp64|mixed] [--repeat 1]

Cases: cfg1, cfg2, cfg4 (the benchmark workload), jacobi24 (Jacobi, NPNT1=NPNT2=24,
NALF=40, EMAX1/EMAX2 = 50000/45000 cm-1, N=5724: a capture-sized case that still spills
the 126 MB L2).
"""
from __future__ import annotations

import argparse
import json

from . import DVR3D_PREC_FP64, DVR3D_PREC_MIXED_DAVIDSON, Context, configs, parse_deck


def workload(name: str):
    if name == "cfg1":
        return configs.config1()
    if name == "cfg2":
        return configs.config2()
    if name == "cfg4":
        return configs.config4()
    if name == "jacobi24":
        return configs.jacobi_h3p_like(24, 24, 40, 50000.0, 45000.0, 200, title="jacobi24")
    raise SystemExit(f"unknown case {name}")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="jacobi24")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--repeat", type=int, default=1)
    a = ap.parse_args()
    w = workload(a.case)
    prec = DVR3D_PREC_FP64 if a.precision == "fp64" else DVR3D_PREC_MIXED_DAVIDSON
    with Context(0) as ctx:
        ctx.set_pes(w.pes)
        d = parse_deck(w.deck)
        for _ in range(a.repeat):
            r = ctx.solve(d, 0, precision=prec, nlevels=w.nlevels)
        print(json.dumps({"case": a.case, "N": r.nham3, "levels": len(r.eval), "stage_ms": list(r.stage_ms),
                          **r.extra}))


if __name__ == "__main__":
    main()
