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


def run(precision, steps, walkers, equil, seed, exchange_split=3, workload="cfg2"):
    wl = make_workload(workload)
    rp = RunParams(equilibration_steps=equil, seed=seed)
    sim = Simulation.from_workload(wl, W=walkers, precision=precision, rp=rp)
    if precision == A.PREC_MIXED and exchange_split != 3:
        sim.ham.set_exchange_split(exchange_split)
    t0 = time.time()
    for _ in range(steps):
        sim.step()
    torch.cuda.synchronize()
    return sim.energies, time.time() - t0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--walkers", type=int, default=1024)
    ap.add_argument("--equil", type=int, default=100)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--exchange-split", default="3",
                    help="comma-separated TF32 products per exchange product (3 and/or 1)")
    ap.add_argument("--workload", default="cfg2", choices=["cfg1", "cfg2"])
    args = ap.parse_args(argv)
    e64, t64 = run(A.PREC_FP64, args.steps, args.walkers, args.equil, args.seed,
                   workload=args.workload)
    s64 = np.array([e for _, e in e64])
    outs = []
    for split in (int(x) for x in args.exchange_split.split(",")):
        emx, tmx = run(A.PREC_MIXED, args.steps, args.walkers, args.equil, args.seed, split,
                       workload=args.workload)
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
