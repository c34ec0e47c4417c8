"""Oracle fixtures for the benchmark workloads at full size (configs 2 and 4).

The benchmark's workloads (dvr3d_b200/configs.py: config 2, Radau NPNT=30 NALF=64, N=3984;
config 4, Jacobi NPNT1=NPNT2=40 NALF=80, N=12202; config 5, Jacobi J=2 with k = 0, 1, 2,
N ~ 20500 per k) are too large for the oracle inside a test run, so this script runs the
oracle once on the CPU and writes ``config<k>_oracle.npz``: the basis size N, the per-block
selection counts and the lowest levels (Eh), per k block for config 5. The final
eigensolve is LAPACK dsyevd, the divide-and-conquer variant the reference keeps beside its
dsyev call (source/dvr3drjz_segmented.f90:2612-2636); on the 2000-dimensional H3+ example
the two agree to 5e-10 cm-1.

Run from the repository root:  python tests/golden/make_config_fixtures.py [2] [4] [5]
(config 4 takes minutes, config 5 about half an hour: the oracle's assembly loops and dsyevd).
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def _configs():
    # the workload definitions are plain Python; loading them does not load the product library
    import importlib.util

    spec = importlib.util.spec_from_file_location("workloads", ROOT / "dvr3d_b200" / "configs.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["workloads"] = mod
    spec.loader.exec_module(mod)
    return mod


def make(k: int) -> None:
    from oracle import oracle

    cf = _configs()
    w = {2: cf.config2, 4: cf.config4, 5: cf.config5}[k]()
    if k == 5:
        # J = 2: one solve per k block (k = 0, 1, 2), the lowest 1000 levels of each
        out = {"deck": np.array(w.deck), "pes": w.pes}
        for kk in oracle.k_blocks(w.deck):
            t0 = time.time()
            r = oracle.solve(w.deck, kk, pes=w.pes, final_mode=1)
            if r.status != 0:
                raise RuntimeError(f"oracle failed on config 5, k={kk}: {r.status}")
            out[f"nham3_k{kk}"] = np.array(r.nham3)
            out[f"iv2_k{kk}"] = r.iv2.astype(np.int32)
            out[f"levels_k{kk}"] = r.eval
            print(f"config 5 k={kk}: N={r.nham3}, {len(r.eval)} levels, {time.time() - t0:.1f} s", flush=True)
        np.savez_compressed(HERE / "config5_oracle.npz", **out)
        return
    t0 = time.time()
    r = oracle.solve(w.deck, 0, pes=w.pes, final_mode=1)
    if r.status != 0:
        raise RuntimeError(f"oracle failed on config {k}: {r.status}")
    np.savez_compressed(HERE / f"config{k}_oracle.npz", deck=np.array(w.deck), pes=w.pes, nham3=np.array(r.nham3),
                        iv2=r.iv2.astype(np.int32), levels=r.eval, stage_s=r.stage_s)
    print(f"config {k}: N={r.nham3}, {len(r.eval)} levels, {time.time() - t0:.1f} s "
          f"(stages {np.round(r.stage_s, 2).tolist()})")


if __name__ == "__main__":
    for a in (sys.argv[1:] or ["2", "4"]):
        make(int(a))
