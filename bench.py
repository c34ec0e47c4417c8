"""Benchmark of the DVR3DRJZ hot path on B200: solves/s for the lowest 500 levels at N~12k.

Workload (one "step" = one complete J=0 solve through the C ABI): the Jacobi-coordinate
problem with three equal masses 1.007276 u, NPNT1 = NPNT2 = 40 Morse DVR points, NALF = 80
Legendre points, cut-offs EMAX1 = 50000 / EMAX2 = 40000 cm-1 (final basis N = 12202),
seeded synthetic Morse + P1/P2 surface (dvr3d_b200/configs.py:config4), lowest 500 levels.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision mixed|fp64|split]

Multi-GPU: one process per GPU (torchrun), each rank solves its own replica of the
workload (the path has no exchange step); value = solves of all ranks / max elapsed.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "solves/s, lowest 500 levels at N~12k, <=1e-3 cm^-1 vs plain FP64 GPU path"
UNIT = "solves/s"
WORKLOAD = "Jacobi J=0, masses 3x1.007276 u, NPNT1=NPNT2=40, NALF=80, EMAX1/EMAX2=50000/40000 cm-1, N=12202, lowest 500 levels"


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows: list[list[str]] = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)

            def rd():
                for line in self.proc.stdout:
                    self.rows.append([x.strip() for x in line.split(",")])

            self.thread = threading.Thread(target=rd, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) < 9:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def _fp64_peak(dev: int) -> float:
    import torch

    a = torch.randn(8192, 8192, dtype=torch.float64, device=f"cuda:{dev}")
    b = torch.randn(8192, 8192, dtype=torch.float64, device=f"cuda:{dev}")
    best = 1e30
    for _ in range(6):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize(dev)
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * 8192 ** 3 / (best / 1000.0) / 1e12


def _workloads():
    """The workload definitions (dvr3d_b200/configs.py: deck text + surface parameters) loaded
    as a plain module, so the CPU arms use the same inputs without importing the product
    package or loading its library."""
    import importlib.util

    name = "dvr3d_workloads"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, ROOT / "dvr3d_b200" / "configs.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def _blas_threads() -> int:
    try:
        from threadpoolctl import threadpool_info

        return int(max([i.get("num_threads", 1) for i in threadpool_info()
                        if i.get("internal_api") == "openblas"] or [1]))
    except Exception:
        return os.cpu_count() or 1


def _fixture_check(levels) -> float | None:
    """Largest difference (cm-1) between CPU levels and the committed oracle fixture."""
    p = ROOT / "tests" / "golden" / "config4_oracle.npz"
    if not p.exists() or levels is None:
        return None
    ref = np.load(p)["levels"]
    n = min(len(ref), len(levels))
    return float(np.abs(np.asarray(levels[:n]) - ref[:n]).max() * 2.19474624e5)


def cpu_baseline_sample(budget_s: float = 15.0) -> dict:
    """The reference's CPU implementation (the oracle) on a bounded sample of the workload,
    about 25 s of CPU work, scaled to one solve. The oracle's stepwise solve of the workload
    runs its units in order: every 1D and 2D block, the selection, the back-transformation
    rows and then assembly block rows until `budget_s` of assembly time is spent, all measured.
    Two parts are scaled: the assembly rows not run, by their exact multiply-add counts (row
    b: iv2[b] * sum_{b' <= b} iv2[b'] * P), and the final diagonalisation, LAPACK dsyevd timed
    at n = 3000 on a seeded symmetric matrix times (N / 3000)^3. The fully measured solve is
    the reference arm's (bench.py --impl reference)."""
    from oracle import oracle

    w = _workloads().config4()
    t_wall = time.perf_counter()
    s = oracle.Session(w.deck, 0, pes=w.pes, final_mode=1)
    d = oracle.parse_deck(w.deck)
    sz = oracle.sizes(d, 0)
    nb = sz["npntc"]
    P = sz["npnta"] * sz["npntb"]
    t_pre = 0.0
    for _ in range(3 * nb + 1):  # 1D, 2D, selection, back-transformation rows
        t = time.perf_counter()
        s.step(1)
        t_pre += time.perf_counter() - t
    iv2, _n2d = s.counts()
    row_macs = iv2.astype(float) * np.cumsum(iv2).astype(float) * P
    t_asm, rows = 0.0, 0
    while rows < nb and t_asm < budget_s:
        t = time.perf_counter()
        s.step(1)
        t_asm += time.perf_counter() - t
        rows += 1
    s.finish()  # abandoned
    done_macs = row_macs[:rows].sum()
    t_asm_full = t_asm * (row_macs.sum() / done_macs) if done_macs > 0 else float("nan")
    nham3 = int(iv2.sum())
    n_s = 3000
    t_diag_s = oracle.time_dsyev(n_s, 1, 1)
    t_diag = t_diag_s * (nham3 / n_s) ** 3
    t_full = t_pre + t_asm_full + t_diag
    thr = _blas_threads()
    return {"value": 1.0 / t_full, "unit": UNIT, "cores": thr, "kind": "port",
            "sample": (f"oracle stepwise solve of the workload (N={nham3}): 1D/2D stage, selection and "
                       f"back-transformation measured ({t_pre:.1f} s); {rows}/{nb} assembly block rows measured "
                       f"({t_asm:.1f} s), the rest scaled by exact multiply-add counts ({t_asm_full:.1f} s); "
                       f"dsyevd at n={n_s} {t_diag_s:.2f} s x (N/{n_s})^3 = {t_diag:.1f} s; "
                       f"{t_full:.0f} s a solve; sample wall {time.perf_counter() - t_wall:.1f} s; "
                       f"restated loops 1 thread, LAPACK {thr} threads")}


def run_reference(args, rank: int, world: int) -> int:
    """The reference's CPU implementation of the path (the oracle: DVR3DRJZ restated routine
    by routine, LAPACK from OpenBLAS) on the benchmark's own workload, config 4 at full size.

    One complete solve takes minutes on the CPU, so the K timed steps together make exactly
    one complete solve: the solve runs on the oracle's worker thread in units of work (per
    block of the 1D and 2D stages, the selection, per block row of the assembly, the final
    diagonalisation), and step i runs units [U i / K, U (i+1) / K). Nothing is scaled: the
    timed region is one real solve, value = 1 / its wall time. The W warm-up steps run the
    first W / K of another solve, which is then abandoned. The final diagonalisation is
    LAPACK dsyevd (all eigenpairs, divide and conquer, OpenBLAS threads), the variant the
    reference keeps beside its dsyev call; its own dsyev with lwork = 3 N would be slower.
    """
    if rank != 0:
        return 0
    from oracle import oracle

    w = _workloads().config4()
    warm = oracle.Session(w.deck, 0, pes=w.pes, final_mode=1)
    U = warm.units
    K = max(1, args.steps)
    bounds = [U * i // K for i in range(K + 1)]
    for q in range(args.warmup):
        warm.step(max(1, bounds[min(q + 1, K)] - bounds[min(q, K)]))
    warm.finish()  # abandoned
    sess = oracle.Session(w.deck, 0, pes=w.pes, final_mode=1)
    times = []
    for i in range(K):
        t = time.perf_counter()
        sess.step(bounds[i + 1] - bounds[i])
        times.append(time.perf_counter() - t)
    left = sess.step(0)
    res = sess.finish()
    total = float(np.sum(times))
    ok = res is not None and left == 0
    v = 1.0 / total if ok else 0.0
    thr = _blas_threads()
    sample = (f"one complete solve of the workload split over the {K} timed steps ({U} units of work: "
              f"1D and 2D blocks, selection, assembly block rows, final dsyevd; {U // K}-{-(-U // K)} units a step); "
              f"{total:.1f} s wall; restated loops 1 thread, LAPACK {thr} threads")
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * total / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Morse + Legendre surface)",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "arm": "CPU oracle: restated DVR3DRJZ + LAPACK (oracle/)",
                       "nham3": None if res is None else int(res.nham3),
                       "levels": None if res is None else int(len(res.eval)),
                       "max_level_diff_vs_fixture_cm": None if res is None else _fixture_check(res.eval),
                       "step_s": [round(x, 3) for x in times]},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": thr, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0 if ok else 1


def run_batch64(args) -> int:
    """64 independent J=0 Radau problems (configs.config3: seeded sizes and surfaces, the
    lowest 100 levels of each) per step through dvr3d_b200_solve_batch, reported in
    problems/s; the same problems solved one solve_block call at a time are timed beside it."""
    import torch

    import dvr3d_b200
    from dvr3d_b200 import configs, parse_deck

    dev = 0
    torch.cuda.set_device(dev)
    ctx = dvr3d_b200.Context(dev)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    ws = configs.config3()
    decks = [parse_deck(w.deck) for w in ws]
    pes = np.array([w.pes for w in ws])

    def timed(fn, k):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / k

    prec = dvr3d_b200.DVR3D_PREC_FP64 if args.precision == "fp64" else dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON

    def one_by_one():
        for w, d in zip(ws, decks):
            ctx.set_pes(w.pes)
            ctx.solve(d, 0, precision=prec)

    def batched():
        return ctx.solve_batch(decks, pes, precision=prec)

    # every level of every problem against the plain FP64 path solved problem by problem
    ref = ctx.solve_batch(decks, pes)
    got = batched()
    err = max(float(np.abs(g.eval - r.eval).max()) for g, r in zip(got, ref)) * dvr3d_b200.AUTOCM
    if err > 1e-3:
        print(json.dumps({"error": "batched levels outside 1e-3 cm-1 of the plain FP64 path", "max_err_cm": err}))
        return 1

    for _ in range(args.warmup):
        batched()
    with ClockSampler(dev) as clk:
        ms = timed(batched, args.steps)
    one_by_one()
    ms1 = timed(one_by_one, min(args.steps, 2))
    res = batched()
    line = {"metric": "problems/s, 64 independent J=0 Radau problems, lowest 100 levels each", "value": 64000.0 / ms,
            "unit": "problems/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded sizes and Morse + bend surfaces)",
            "config": {"workload": "64 Radau problems, NPNT U{16..32}, NALF U{24..64}, final H 800-3000, 100 levels",
                       "path": "fp64-dense" if prec == dvr3d_b200.DVR3D_PREC_FP64 else "mixed (Davidson / shift-invert)",
                       "max_level_err_vs_plain_cm": err,
                       "sizes": [int(r.nham3) for r in res],
                       "one_by_one": {"ms_per_step": ms1, "problems_per_s": 64000.0 / ms1}},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def _dipole_model(q1: float, q2: float, cost: float):
    """Bond-frame dipole of an AB2 molecule (a.u.) for the DIPOLE3 workload: bisector component
    symmetric in the two bonds, perpendicular one antisymmetric."""
    import math

    th = math.acos(max(-1.0, min(1.0, cost)))
    c, s = math.cos(th / 2), math.sin(th / 2)
    dy = (0.73 + 0.21 * (q1 + q2 - 3.62) - 0.05 * (q1 - q2) ** 2) * c * (1.0 + 0.1 * cost)
    dx = (0.38 - 0.04 * (q1 + q2 - 3.62)) * (q1 - q2) * s
    return dx, dy


def run_dipole(args) -> int:
    """Transition moments J = 2 e <-> J = 2 f (the reference's water example chain, at its sizes
    and with all states): first steps (Radau, NPNT = 21, NALF = 40, EMAX2 = 40000 cm-1, ZROT,
    ZTRAN), ROTLEV3B with ZTRAN (NVIB = 150, NEVAL = 200) for each parity -- not timed -- then
    per step one DIPOLE3 run (NPOT = 60, all 200 x 200 states, five k -> k' blocks) through
    dvr3d_b200_dipole3 with the files on disk and a Python DIPSA plug-in. Reported: runs/s end
    to end, the device time and flop rate of its GEMMs, and the oracle's restatement of DIPOLE3
    (the reference's rank-1 updates) on the same files on the host's cores."""
    import tempfile

    import torch

    import dvr3d_b200
    from dvr3d_b200 import configs

    dev = 0
    torch.cuda.set_device(dev)
    ctx = dvr3d_b200.Context(dev)
    tmp = tempfile.TemporaryDirectory()
    d = Path(tmp.name)

    def first_step(jrot, kmin, ipar, name):
        w = configs.radau_water_like(21, 40, 40000.0, 200, title=f"dipole bench J{jrot} kmin{kmin}")
        lines = w.deck.splitlines()
        c3 = list(lines[2])
        c3[5:10] = list(f"{jrot:5d}")
        c3[35:40] = list(f"{kmin:5d}")
        c3[45:50] = list(f"{ipar:5d}")
        lines[2] = "".join(c3)
        w.deck = "\n".join(lines).replace("ZPMIN=.TRUE.", "ZPMIN=.TRUE., ZROT=.TRUE., ZTRAN=.TRUE., ZLIN=.TRUE.") + "\n"
        ctx.set_pes(w.pes)
        ctx.run_deck(w.deck, wave_path=str(d / name))

    def rot_deck(kmin):
        return (" &PRT zdcore=.true., ztran=.true. /\n" + "".join(f"{v:5d}" for v in (150, 200, kmin, 0, 0, 0))
                + "\n ROTLEV3B for DIPOLE3\n" + f"{4500.0:20.6f}\n")

    first_step(2, 1, 0, "e.26")
    first_step(2, 0, 0, "f.26")
    ctx.rotlev3b_trans(rot_deck(1), str(d / "e.26"), str(d / "e.8"))
    ctx.rotlev3b_trans(rot_deck(0), str(d / "f.26"), str(d / "f.8"))
    deck = " &PRT zstart=.true. /\n DIPOLE3 bench\n" + "".join(f"{v:5d}" for v in (60, 200, 200, 0, 0)) + f"\n{4500.0:20.6f}\n"
    ket, bra = str(d / "e.8"), str(d / "f.8")
    run = lambda: ctx.dipole3(deck, ket, bra, dipsa=_dipole_model, tra_path=str(d / "g.13"), cap=256)  # noqa: E731
    for _ in range(max(1, args.warmup)):
        got = run()
    walls, devs = [], []
    with ClockSampler(dev) as clk:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            got = run()
            walls.append(time.perf_counter() - t0)
            devs.append(got["dev_ms"])
    wall = float(np.median(walls))
    dev_ms = float(np.median(devs))
    # the oracle on the same files: parity and the host baseline
    from oracle import oracle as O

    t0 = time.perf_counter()
    ref = O.dipole3(deck, ket, bra, dipsa=_dipole_model, tra_path=str(d / "r.13"), cap=256)
    cpu_s = time.perf_counter() - t0
    scale = max(np.abs(ref["tz"]).max(), np.abs(ref["tx"]).max())
    err = max(np.abs(got["tz"] - ref["tz"]).max(), np.abs(got["tx"] - ref["tx"]).max()) / scale
    peak = _fp64_peak(dev)
    achieved = got["flops"] / (dev_ms * 1e-3) / 1e12
    line = {"metric": "DIPOLE3 runs/s, J=2 e<->f, 200 x 200 states, NPOT=60", "value": 1.0 / wall, "unit": "runs/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Morse + bend surface, model bond dipole)",
            "config": {"workload": "Radau J=2 e/f first steps NPNT=21 NALF=40 EMAX2=40000, ROTLEV3B NVIB=150 NEVAL=200, "
                                   "DIPOLE3 NPOT=60 NV1=NV2=200 (5 k->k' blocks)",
                       "device_ms": dev_ms, "gflop": got["flops"] / 1e9, "blocks": got["nblocks"],
                       "max_rel_err_vs_oracle": float(err)},
            "roofline": {"bound": "fp64 tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak},
            "cpu_baseline": {"value": 1.0 / cpu_s, "unit": "runs/s", "cores": 1, "kind": "port",
                             "sample": "the oracle's DIPOLE3 restatement (rank-1 updates as loops) on the same files, one run"},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    ctx.close()
    tmp.cleanup()
    return 0 if err < 1e-9 else 1


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="auto", choices=["auto", "fp64", "mixed", "split"],
                    help="mixed (default): the chosen form; fp64: the plain path; split (--profile-solve "
                         "only): the split-BF16 tensor-core form")
    ap.add_argument("--levels", type=int, default=500, help="--profile-solve: levels of the solve")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-solve", action="store_true",
                    help="one solve of the workload and nothing else (for ncu captures of its kernels)")
    ap.add_argument("--profile-ozaki", action="store_true",
                    help="one int8-sliced FP64 product of the top-level Cholesky-inverse shape at the "
                         "workload's size (6058 x 6144 x 6144, triangular transposed second operand) and "
                         "nothing else (for ncu captures of oz_gemm_kernel)")
    ap.add_argument("--workload", default="cfg4", choices=["cfg4", "batch64", "dipole"],
                    help="cfg4: the headline solve; batch64: 64 independent Radau problems per step; "
                         "dipole: DIPOLE3 transition moments J=2 e<->f")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "batch64" and args.impl == "ours":
        return run_batch64(args)
    if args.workload == "dipole" and args.impl == "ours":
        return run_dipole(args)
    if args.profile_solve:
        # one solve of the workload and nothing else. The chosen form: the 1D/2D stage,
        # assembly, the Cholesky-inverse (764 GEMM launches at this size, counting the start
        # block's Cholesky-QR), then the Krylov steps. --precision fp64: the plain path (one
        # dense_panel_kernel launch per 32-column panel of the reduction).
        import dvr3d_b200
        from dvr3d_b200 import configs, parse_deck

        ctx = dvr3d_b200.Context(0)
        w = configs.config4()
        ctx.set_pes(w.pes)
        prec = {"fp64": dvr3d_b200.DVR3D_PREC_FP64, "split": dvr3d_b200.DVR3D_PREC_SPLIT_BF16}.get(
            args.precision, dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON)
        r = ctx.solve(parse_deck(w.deck), 0, precision=prec, nlevels=args.levels)
        print(json.dumps({"profile_solve": WORKLOAD, "nham3": r.nham3, "stage_ms": list(r.stage_ms)}), flush=True)
        ctx.close()
        return 0
    if args.profile_ozaki:
        # L21 = A21 inv(L11)^T of the first split of the N = 12202 factorisation (n1 = 6144,
        # n2 = 6058): A21 dense, inv(L11) lower triangular, through dvr3d_b200_ozaki_gemm
        import dvr3d_b200

        rng = np.random.default_rng(1)
        n1, n2 = 6144, 6058
        a21 = np.asfortranarray(rng.standard_normal((n2, n1)))
        l11 = np.asfortranarray(np.tril(rng.standard_normal((n1, n1))))
        with dvr3d_b200.Context(0) as ctx:
            c = ctx.ozaki_gemm(a21, l11, tb=True, tri_b=2)
        print(json.dumps({"profile_ozaki": [n2, n1, n1], "checksum": float(np.abs(c).sum())}), flush=True)
        return 0
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.precision == "split":
        print(json.dumps({"error": "--precision split is a --profile-solve mode (the headline arms are mixed and fp64)"}))
        return 2

    import torch

    import dvr3d_b200
    from dvr3d_b200 import configs, parse_deck

    dist = None
    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = local
    torch.cuda.set_device(dev)
    ctx = dvr3d_b200.Context(dev)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    w = configs.config4()
    deck = parse_deck(w.deck)
    ctx.set_pes(w.pes)
    mixed = args.precision in ("auto", "mixed")
    prec = dvr3d_b200.DVR3D_PREC_MIXED_DAVIDSON if mixed else dvr3d_b200.DVR3D_PREC_FP64
    prec_name = "shift-invert-krylov" if mixed else "fp64-dense"
    # the accuracy bar of the metric: every level within 1e-3 cm-1 of the plain FP64 GPU path
    # (checked once, outside the timed region, together with the plain path's own speed)
    check = {}
    ref = None
    if mixed:
        ref = ctx.solve(deck, 0, precision=dvr3d_b200.DVR3D_PREC_FP64, nlevels=500)
        got = ctx.solve(deck, 0, precision=prec, nlevels=500)
        err = np.abs(got.eval - ref.eval) * dvr3d_b200.AUTOCM
        check = {"max_level_err_cm": float(err.max()), "levels_checked": int(len(err)),
                 "fallback": int(got.fallback)}
        fx = ROOT / "tests" / "golden" / "config4_oracle.npz"
        if fx.exists():  # and both against the CPU oracle's levels of the same workload
            lv = np.load(fx)["levels"]
            check["max_level_err_vs_oracle_cm"] = float(np.abs(got.eval - lv[:len(got.eval)]).max() * dvr3d_b200.AUTOCM)
            check["plain_max_level_err_vs_oracle_cm"] = float(np.abs(ref.eval - lv[:len(ref.eval)]).max()
                                                              * dvr3d_b200.AUTOCM)
        if not (err.max() <= 1e-3 and len(err) == 500):
            print(json.dumps({"error": "mixed path outside 1e-3 cm-1 of the plain FP64 path", **check}), flush=True)
            return 1

    def step():
        return ctx.solve(deck, 0, precision=prec, nlevels=500)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    results = []
    walls = []
    with ClockSampler(dev) as clk:
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        e0.record(stream)
        for _ in range(args.steps):
            t = time.perf_counter()
            results.append(step())
            walls.append(time.perf_counter() - t)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
    ms = e0.elapsed_time(e1)
    wall_s = float(np.sum(walls))
    if mixed:
        # the plain FP64 GPU path as a second arm of the same run: same stream, CUDA events,
        # one untimed warm-up solve (above), then min(K, 3) timed solves
        kp = min(args.steps, 3)
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        p0.record(stream)
        for _ in range(kp):
            ctx.solve(deck, 0, precision=dvr3d_b200.DVR3D_PREC_FP64, nlevels=500)
        p1.record(stream)
        torch.cuda.synchronize(dev)
        plain_ms = p0.elapsed_time(p1) / kp
        check["plain_fp64"] = {"ms_per_step": plain_ms, "steps": kp, "warmup": 1,
                               "speedup_of_chosen_form": plain_ms / (ms / args.steps)}
    if dist:
        t = torch.tensor([ms, wall_s], device=f"cuda:{dev}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, wall_s = float(t[0]), float(t[1])
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0
    total = args.steps * world
    value = total / (ms / 1000.0)
    e2e = total / wall_s
    hbm, bf16, src = _peaks()
    prof = results
    if mixed:
        # the dominant kernel family's launches, each timed by its own CUDA event pair, on one
        # more solve of the same workload right after the timed region (per-launch events are
        # off in the timed solves: recording and reading them costs host time between solves)
        os.environ["DVR3D_GEMM_EVENTS"] = "1"
        prof = [step()]
        os.environ.pop("DVR3D_GEMM_EVENTS")
        torch.cuda.synchronize(dev)
    nprof = len(prof)
    dom_ms = sum(r.extra["dom_ms"] for r in prof)
    dom_bytes = sum(r.extra["dom_bytes"] for r in prof)
    dom_flops = sum(r.extra["dom_flops"] for r in prof)
    dom_launch = sum(r.extra["dom_launches"] for r in prof)
    kern = results[0].extra["dom_kernel"]
    if dom_flops > 0:
        # tensor-bound FP64 GEMM: against cuBLAS DGEMM measured here (no FP64 figure is in
        # MEASURED_PEAKS.json)
        fp64_peak = _fp64_peak(dev)
        achieved = dom_flops / (dom_ms / 1000.0) / 1e12 if dom_ms > 0 else None
        # DRAM bytes per launch from the ncu capture of the family's most frequent large launch,
        # the Krylov triangular product (profiles/traffic.json, profiles/gemm_pipe_kernel_*.md)
        traffic, traffic_note = None, None
        tp = ROOT / "profiles" / "traffic.json"
        if tp.exists():
            ent = json.loads(tp.read_text()).get("gemm_pipe_kernel")
            if ent:
                traffic = ent["dram_bytes_per_launch"]
                traffic_note = ent["launch"]
        roof = {"bound": "tensor", "kernel": kern, "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": (achieved / fp64_peak) if achieved else None, "traffic": traffic,
                "traffic_launch": traffic_note,
                "peak_source": "measured in this run: cuBLAS DGEMM (torch.matmul float64) 8192^3, best of 5",
                "alg_flops_per_step": dom_flops / nprof, "launches": dom_launch / nprof,
                "note": "achieved = algorithmic flops of the DMMA GEMM launches of a solve (Cholesky-inverse, "
                        "Krylov steps, Ritz vectors, H3 X; per launch from M, N, K and its triangular structure) "
                        "/ the sum of their durations, each launch timed by a CUDA event pair on the solve's stream "
                        "(one solve after the timed region)",
                "share_of_step": (dom_ms / nprof) / (ms / args.steps) if ms > 0 else None}
    else:
        achieved = dom_bytes / (dom_ms / 1000.0) / 1e9 if dom_ms > 0 else None
        traffic = None
        tp = ROOT / "profiles" / "traffic.json"
        if tp.exists() and dom_launch:
            tj = json.loads(tp.read_text())
            ent = tj.get(kern)
            if ent:
                traffic = ent["bytes_per_alg_byte"] * dom_bytes / dom_launch
        roof = {"bound": "hbm", "kernel": kern, "achieved": achieved, "peak": hbm,
                "unit": "GB/s", "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else "fallback",
                "alg_bytes_per_launch": dom_bytes / max(dom_launch, 1), "launches": dom_launch / args.steps,
                "share_of_step": dom_ms / ms if ms > 0 else None}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Morse + Legendre surface)",
            "config": {"workload": WORKLOAD, "path": prec_name, "nham3": results[0].nham3,
                       "levels": len(results[0].eval), "l2": "inputs larger than L2 (H3 = 1.19 GB FP64)",
                       "parallelism": f"replicas x{world}", **check},
            "e2e": {"value": e2e, "unit": UNIT,
                    "h2d_bytes_per_step": int(np.mean([r.extra["h2d_bytes"] for r in results])),
                    "d2h_bytes_per_step": int(np.mean([r.extra["d2h_bytes"] for r in results]))},
            "roofline": roof,
            "gpu_launches": int(sum(r.extra["launches"] for r in results)),
            "clocks": clk.summary(),
            "stage_ms": {k: float(np.mean([r.stage_ms[i] for r in results])) for i, k in
                         enumerate(["host_setup", "blocks_1d2d_select", "assembly", "final_eigensolve",
                                    "device_total", "call_total"])}}
    if world == 1 and not args.no_cpu_baseline:
        try:
            cb = cpu_baseline_sample()
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as ex:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "port",
                                    "sample": f"failed: {ex}"}
    print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
