"""Energy accuracy of the mixed-precision walker step against the complex128 one.

    python -m safire_b200.accuracy --steps 2000 --walkers 1024 [--exchange-split 3,1]

Runs the same synthetic workload (M=200, N=50+50, Nc=1600, dt=0.005) twice from the same seeds,
once with every contraction in complex128 and once in mixed precision (3xTF32 tensor-core
contractions, FP64 determinants, weights and energy sums), and prints one JSON line with the
mixed-estimator energy of each run (mean over the measurements after equilibration, with a
blocking error bar), the mean and largest per-measurement difference, and the difference of the
two estimates.  Both runs draw the same auxiliary fields (device Philox, same seed) and the same
comb uniforms, so the two trajectories see identical noise and their energies differ only by the
arithmetic.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch

from . import afqmc as A
from .driver import RunParams, Simulation
from .synth import make_workload


def blocked_error(x, nblocks=10):
    """Standard error of the mean from nblocks contiguous blocks (serial correlation)."""
    x = np.asarray(x, dtype=np.float64)
    if x.size < 2 * nblocks:
        return float(np.std(x, ddof=1) / math.sqrt(max(x.size - 1, 1))) if x.size > 1 else 0.0
    b = np.array_split(x, nblocks)
    m = np.array([v.mean() for v in b])
    return float(m.std(ddof=1) / math.sqrt(nblocks))


def run(precision, steps, walkers, equil, seed, exchange_split=3, workload="cfg2", lscale=0.5):
    wl = make_workload(workload, lscale=lscale)
    rp = RunParams(equilibration_steps=equil, seed=seed)
    sim = Simulation.from_workload(wl, W=walkers, precision=precision, rp=rp)
    if precision == A.PREC_MIXED and exchange_split != 3:
        sim.ham.set_exchange_split(exchange_split)
    t0 = time.time()
    for _ in range(steps):
        sim.step()
    torch.cuda.synchronize()
    return sim.energies, time.time() - t0


def lockstep(steps, walkers, equil, seed, workload, lscale, exchange_split=3, mixed_ops=7,
             restart_every=0, measure_every=10, split_format=0, taylor_mode=1):
    """Correlated sampling: the complex128 and the mixed run advance side by side with the same
    fields, the same Eshift and the same population-control decisions (the comb of the complex128
    run's weights applied to both walker sets), so the paired energies differ only through the
    arithmetic of the mixed step.

    restart_every > 0 restarts both runs from the trial every that many steps (both walker sets
    back at the trial, Eshift re-seeded, equilibration run again): the benchmark system's total
    weight collapses some 130-200 steps after the walkers leave the trial, so its paired
    comparison runs in windows shorter than that.  Measurements come every measure_every steps
    once a window is past its equilibration.  Returns the two measurement series, the total
    weights at the combs, the per-component differences and the window of every measurement."""
    from .population import WalkerRows, exchange_walkers
    wl = make_workload(workload, lscale=lscale)
    sims = []
    for prec in (A.PREC_FP64, A.PREC_MIXED):
        rp = RunParams(equilibration_steps=equil, seed=seed, population_control_interval=0)
        sim = Simulation.from_workload(wl, W=walkers, precision=prec, rp=rp)
        if prec == A.PREC_MIXED and exchange_split != 3:
            sim.ham.set_exchange_split(exchange_split)
        if prec == A.PREC_MIXED and mixed_ops != 7:  # 8 (vHS alone) only for attribution
            sim.ham.set_mixed_ops(mixed_ops)
        if prec == A.PREC_MIXED and split_format:
            sim.ham.set_split_format(split_format)
        if prec == A.PREC_MIXED and taylor_mode != 1:
            sim.ham.set_taylor_fused(taylor_mode)
        sims.append(sim)
    s64, smx = sims
    rng = A.HostRandomGenerator(A.split_seed(seed, 0, 0))
    e64, emx, weights, comp, window = [], [], [], [], []
    win, k = 0, 0  # window index, step within the window
    for _ in range(steps):
        if restart_every and k == restart_every:
            for sim in sims:
                sim.restart()
            win, k = win + 1, 0
        smx.Eshift = s64.Eshift
        for sim in sims:
            sim.step(measure=False)  # propagation, orthogonalisation, Eshift update
        if k % 10 == 0:
            w = np.abs(s64.wset.getProperty(0))
            weights.append(float(w.sum()))
            off = A.comb(rng, w, walkers)
            for sim in sims:
                exchange_walkers(WalkerRows(sim.wset), off, [walkers], 0)
                sim.wset.normalize_weights()
                sim._g_ready = False
        if k >= equil and k % measure_every == 0:
            a, sa, _ = s64.measure()
            b, sb, _ = smx.measure()
            e64.append(a)
            emx.append(b)
            window.append(win)
            # per-component difference of the weighted averages (E1, EXX, EJ)
            comp.append([((sb[i] / sb[3]) - (sa[i] / sa[3])).real for i in range(3)])
        k += 1
    torch.cuda.synchronize()
    return np.array(e64), np.array(emx), weights, np.array(comp), np.array(window)


def window_error(x, window):
    """Standard error of the mean of x from its per-window means (restarted windows are
    independent); falls back to blocking for a single window."""
    x, window = np.asarray(x, dtype=np.float64), np.asarray(window)
    ids = np.unique(window)
    if ids.size < 2:
        return blocked_error(x)
    m = np.array([x[window == i].mean() for i in ids])
    return float(m.std(ddof=1) / math.sqrt(ids.size))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--walkers", type=int, default=1024)
    ap.add_argument("--equil", type=int, default=100)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--exchange-split", default="3",
                    help="comma-separated TF32 products per exchange product (3 and/or 1)")
    ap.add_argument("--workload", default="cfg2", choices=["cfg1", "cfg2"])
    ap.add_argument("--lscale", type=float, default=0.5,
                    help="Cholesky-vector scale of the synthetic Hamiltonian (0.5: benchmark)")
    ap.add_argument("--lockstep", action="store_true",
                    help="correlated sampling: shared fields, Eshift and comb decisions")
    ap.add_argument("--restart-every", type=int, default=0,
                    help="lockstep: restart both runs from the trial every this many steps "
                         "(0: never)")
    ap.add_argument("--measure-every", type=int, default=10,
                    help="lockstep: steps between measurements")
    ap.add_argument("--split-format", type=int, default=0, choices=[0, 1, 2],
                    help="lockstep: operand format of the mixed split (0 auto, 1 TF32, 2 FP16)")
    ap.add_argument("--taylor-mode", default="1",
                    help="lockstep: comma-separated Taylor propagation modes of the mixed run "
                         "(afqmc_ham_set_taylor_fused; 1 the default)")
    ap.add_argument("--mixed-ops", default="7",
                    help="comma-separated masks of the operations run in mixed precision "
                         "(1 vbias, 2 vHS + propagation, 4 energy, 8 vHS alone)")
    args = ap.parse_args(argv)
    if args.lockstep:
        outs = []
        runs = [(int(x), int(m), int(t)) for x in args.exchange_split.split(",")
                for m in args.mixed_ops.split(",") for t in args.taylor_mode.split(",")]
        for split, mops, tmode in runs:
            t0 = time.time()
            e64, emx, wsum, comp, win = lockstep(args.steps, args.walkers, args.equil,
                                                 args.seed, args.workload, args.lscale, split,
                                                 mops, args.restart_every, args.measure_every,
                                                 args.split_format, tmode)
            d = emx - e64
            out = {
                "mode": "lockstep", "workload": args.workload, "lscale": args.lscale,
                "steps": args.steps, "walkers": args.walkers, "equilibration_steps": args.equil,
                "restart_every": args.restart_every, "measure_every": args.measure_every,
                "windows": int(np.unique(win).size) if win.size else 0,
                "exchange_split": split, "mixed_ops": mops, "split_format": args.split_format,
                "taylor_mode": tmode,
                "measurements": int(d.size),
                "E_fp64": float(e64.mean()), "E_fp64_err": window_error(e64, win),
                "E_mixed": float(emx.mean()), "E_mixed_err": window_error(emx, win),
                "dE_estimate_mHa": 1e3 * float(d.mean()),
                "dE_estimate_err_mHa": 1e3 * window_error(d, win),
                "dE_max_abs_mHa": 1e3 * float(np.abs(d).max()),
                "dE_components_mHa": {k: 1e3 * float(comp[:, i].mean())
                                      for i, k in enumerate(("E1", "EXX", "EJ"))},
                "dE_components_err_mHa": {k: 1e3 * window_error(comp[:, i], win)
                                          for i, k in enumerate(("E1", "EXX", "EJ"))},
                "total_weight_min_max": [min(wsum), max(wsum)],
                "wall_s": time.time() - t0,
            }
            print(json.dumps(out), flush=True)
            outs.append(out)
        return outs
    e64, t64 = run(A.PREC_FP64, args.steps, args.walkers, args.equil, args.seed,
                   workload=args.workload, lscale=args.lscale)
    s64 = np.array([e for _, e in e64])
    outs = []
    for split in (int(x) for x in args.exchange_split.split(",")):
        emx, tmx = run(A.PREC_MIXED, args.steps, args.walkers, args.equil, args.seed, split,
                       workload=args.workload, lscale=args.lscale)
        smx = np.array([e for _, e in emx])
        n = min(s64.size, smx.size)
        d = smx[:n] - s64[:n]
        out = {
            "workload": args.workload, "steps": args.steps, "walkers": args.walkers,
            "equilibration_steps": args.equil, "exchange_split": split,
            "measurements": int(n),
            "E_fp64": float(s64.mean()), "E_fp64_err": blocked_error(s64),
            "E_mixed": float(smx.mean()), "E_mixed_err": blocked_error(smx),
            "dE_estimate_mHa": 1e3 * float(smx.mean() - s64.mean()),
            "dE_mean_abs_mHa": 1e3 * float(np.abs(d).mean()) if n else None,
            "dE_max_abs_mHa": 1e3 * float(np.abs(d).max()) if n else None,
            "wall_s": {"fp64": t64, "mixed": tmx},
        }
        print(json.dumps(out), flush=True)
        outs.append(out)
    return outs


if __name__ == "__main__":
    main()
