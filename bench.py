#!/usr/bin/env python
"""Walker-steps/s of the batched phaseless AFQMC walker step on B200.

Workload: M=200 orbitals, N_up=N_dn=50 (CLOSED walkers), N_chol=1600 (decay 0.995^n), 1024 walkers
per GPU, dt=0.005, Taylor order 6, seeded synthetic Hamiltonian and RHF trial (no public input:
the reference reads pyscf-generated HDF5 files that are not available here).

One bench "step" is one block of the reference's production loop (run_afqmc.cpp:69-113) at its
cadence: 10 propagation steps, QR re-orthogonalisation every 5, comb population control every 10
and one mixed-estimator energy measurement every 10.  value = walker-steps/s over all ranks
(= W * 10 * K * N_gpus / max-over-ranks device time).

The default run times the mixed-precision path (3xTF32 tensor-core contractions, FP64
determinants, weights and energy sums) and then the complex128 path on the same inputs
(`fp64` in the JSON line, with the mixed / FP64 ratio).  `--workload phmsd` times the
particle-hole multi-determinant system instead (COLLINEAR M=120, N=30+30, N_chol=960, reference
+ 4095 determinants, 512 walkers, complex128).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
                  [--workload nomsd|phmsd] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BLOCK = 10  # AFQMC steps per bench step


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--workload", default="nomsd", choices=["nomsd", "phmsd", "control-variate"],
                    help="nomsd: the single-determinant M=200 system (the metric's workload); "
                         "phmsd: the particle-hole multi-determinant system; control-variate: "
                         "the learned exchange estimator's cost at equal error bar")
    ap.add_argument("--cv-epochs", type=int, default=30)
    ap.add_argument("--cv-fraction", type=float, default=1.0 / 8,
                    help="walkers (or draws) evaluated exactly per measurement")
    ap.add_argument("--cv-sampling", default="weight", choices=["uniform", "weight"])
    ap.add_argument("--cv-lowrank", type=int, default=-1,
                    help="leading Cholesky vectors of the low-fidelity exchange base (0: none, "
                         "-1: Nc / 16)")
    ap.add_argument("--cv-system", default="cfg2", choices=["cfg1", "cfg2"],
                    help="control-variate workload: cfg2 = M=200 N=50+50 Nc=1600, cfg1 = M=32 "
                         "N=8+8 Nc=128")
    ap.add_argument("--no-fp64-compare", action="store_true",
                    help="skip timing the complex128 path beside the mixed one")
    ap.add_argument("--walkers", type=int, default=1024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--exchange-split", type=int, default=3, choices=[1, 3],
                    help="TF32 products per real product in the mixed exchange contraction")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch every kernel of a step eagerly instead of replaying the step's "
                         "CUDA graph")
    ap.add_argument("--taylor-mode", type=int, default=1, choices=[0, 1, 2, 3],
                    help="mixed Taylor propagation: 0 per-term GEMMs, 1 fused (auto), 2 / 3 fused "
                         "with one / two walkers in flight per CTA")
    return ap.parse_args()


def metric_name():
    return "walker-steps/s at M=200, 1024 walkers: mixed vs FP64 on B200 at |dE|<0.5 mHa"


# ------------------------------------------------------------------------------------------
# CPU leg: the oracle (restatement of the reference CPU path) on the host cores
# ------------------------------------------------------------------------------------------
def cpu_sample(wl, n_walkers, n_blocks=1):
    """Time the oracle on n_walkers walkers of the workload; returns (walker-steps/s, seconds,
    description).  One block = 10 propagations + 2 orthogonalisations + 1 energy measurement."""
    import numpy as np
    from oracle import afqmc as O
    oham = O.Real3IndexFactorization(wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij, wl.E0,
                                     wl.PsiT)
    owfn = O.NOMSD(oham, wl.PsiT)
    prop = O.Propagator(owfn, O.PropagatorParams(dt=wl.dt))
    ws = O.WalkerSet.from_trial(owfn, n_walkers)
    E, ov = owfn.Energy(ws.SA, ws.SB)
    ws.props[:, O.OVLP] = ov
    ws.props[:, O.PSEUDO_ELOC] = E.sum(axis=1)
    Eshift = float(np.mean(E.sum(axis=1)).real)
    rng = O.HostRandomGenerator(O.split_seed(0, 0, 1))
    wrng = O.HostRandomGenerator(O.split_seed(0, 0, 0))
    t0 = time.perf_counter()
    for b in range(n_blocks):
        for s in range(BLOCK):
            u = rng.sample_uniform(n_walkers * wl.Nc).reshape(n_walkers, wl.Nc)
            prop.propagate(ws, Eshift, u)
            if s % 5 == 0:
                prop.orthogonalize(ws)
            if s == 0:
                O.population_control_single_rank(wrng, ws)
        O.energy_measure(owfn, ws)
    dt = time.perf_counter() - t0
    ws_s = n_walkers * BLOCK * n_blocks / dt
    desc = (f"oracle (numpy/scipy, OpenBLAS) on {n_walkers} walkers x {BLOCK * n_blocks} steps "
            f"of the same workload, incl. orthogonalisation, comb and one energy measurement per "
            f"{BLOCK} steps")
    return ws_s, dt, desc


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload == "control-variate":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the learned control variate has no reference counterpart"}), flush=True)
        return 0
    if args.workload == "phmsd":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the oracle's PHMSD energy is a per-determinant Python loop; no CPU "
                          "timing of the 4096-determinant system"}), flush=True)
        return 0
    cores = host_cores()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    os.environ.setdefault("OPENBLAS_NUM_THREADS", str(cores))
    from safire_b200.synth import make_workload
    wl = make_workload("cfg2")
    n_walkers = 16
    for _ in range(args.warmup):
        cpu_sample(wl, n_walkers, 0)
    tot_ws, tot_t = 0.0, 0.0
    for _ in range(args.steps):
        v, t, desc = cpu_sample(wl, n_walkers, 1)
        tot_ws += n_walkers * BLOCK
        tot_t += t
    value = tot_ws / tot_t
    line = {
        "impl": "reference", "metric": metric_name(), "value": value, "unit": "walker-steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * tot_t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": "M=200 N=50+50 Nc=1600 W=1024 dt=0.005 (sampled on 16 walkers)",
                   "parallelism": "host threads"},
        "cpu_baseline": {"value": value, "unit": "walker-steps/s", "cores": cores, "kind": "port",
                         "sample": desc},
        "e2e": {"value": value, "unit": "walker-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------
# GPU leg
# ------------------------------------------------------------------------------------------
class ClockSampler:
    def __init__(self, device_index):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None
        self.dev = device_index

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.strip().split(",") for r in self.file.read().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
                for k, n in enumerate(names):
                    if r[3 + k].strip().lower() in ("active", "1"):
                        reasons.add(n)
            except Exception:
                continue
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def fp64_peak_tflops(torch):
    """Dense FP64 throughput of cuBLAS DGEMM on this GPU (the FP64 roofline denominator)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(4):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1000)
    del a, b
    return 2 * n ** 3 / best / 1e12


def tf32_peak_tflops(torch):
    """Dense TF32 tensor-core throughput of cuBLAS (FP32 GEMM with TF32 allowed) on this GPU."""
    n = 8192
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    a = torch.randn(n, n, dtype=torch.float32, device="cuda")
    b = torch.randn(n, n, dtype=torch.float32, device="cuda")
    for _ in range(3):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1000)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    return 2 * n ** 3 / best / 1e12


def _timed_blocks(sim, steps, warmup, world, local, clocks=None):
    """Warm up, then time `steps` blocks of BLOCK steps with CUDA events on the current stream,
    barriers on both sides; returns (max-over-ranks ms, our kernel launches, clock summary)."""
    import torch
    import torch.distributed as dist
    from safire_b200 import capi

    def barrier():
        if world > 1:
            dist.barrier()

    def block():
        for _ in range(BLOCK):
            sim.step()

    for _ in range(warmup):
        block()
    torch.cuda.synchronize()
    barrier()
    launches0 = capi.lib().afqmc_kernel_launches()
    graph_k0 = sim.graph.kernels_replayed() if sim.graph is not None else 0
    if clocks is not None:
        clocks.start()
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        block()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop() if clocks is not None else None
    launches = capi.lib().afqmc_kernel_launches() - launches0
    if sim.graph is not None:  # kernels the step graph replayed inside the timed region
        launches += sim.graph.kernels_replayed() - graph_k0
    t_ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([t_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_ms = float(t.item())
    return t_ms, int(launches), clk


def _phases(sim):
    """Per-phase device time of one step and of one energy measurement and orthogonalisation
    (outside the timed region)."""
    import torch
    stream = torch.cuda.current_stream()
    sim.prop.set_timing(True)
    sim.prop.Propagate(sim.wset, sim.Eshift)
    sim._g_ready = False  # that step did not leave the density matrix for the next one
    phases = sim.prop.timings()
    sim.prop.set_timing(False)
    torch.cuda.synchronize()
    for name, fn in (("energy_measurement", sim.measure),
                     ("orthogonalize", lambda: sim.prop.Orthogonalize(sim.wset))):
        m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        fn()
        m1.record(stream)
        torch.cuda.synchronize()
        phases[name] = m0.elapsed_time(m1)
    return phases


def _e2e(sim, W, Nc, steps, world, prec):
    """The same blocks through the public API with host uniforms copied in from pinned memory
    and the weights + energy estimate read back every block."""
    import torch
    import torch.distributed as dist
    from safire_b200 import afqmc as A
    stream = torch.cuda.current_stream()
    host_u = torch.rand((BLOCK, W, Nc), dtype=torch.float64).pin_memory()
    dev_u = torch.empty((BLOCK, W, Nc), dtype=torch.float64, device="cuda")
    host_w = torch.empty((W,), dtype=torch.complex128).pin_memory()
    host_e = torch.empty((4,), dtype=torch.complex128).pin_memory()

    def block_e2e():
        dev_u.copy_(host_u, non_blocking=True)
        for s in range(BLOCK):
            sim.step(dev_u[s], measure=False)
        E, _ = sim.wfn.Energy(sim.wset, set_properties=False, precision=prec)
        sums = A.energy_sums(sim.wset, E)
        if world > 1:
            dist.all_reduce(sums)
        host_e.copy_(sums, non_blocking=True)
        host_w.copy_(sim.wset.properties()[:, 0], non_blocking=True)

    block_e2e()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k0.record(stream)
    for _ in range(steps):
        block_e2e()
    k1.record(stream)
    torch.cuda.synchronize()
    te = k0.elapsed_time(k1)
    if world > 1:
        t = torch.tensor([te], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        te = float(t.item())
    return {"value": W * world * BLOCK * steps / (te / 1000), "unit": "walker-steps/s",
            "h2d_bytes_per_step": int(host_u.numel() * 8),
            "d2h_bytes_per_step": int((host_w.numel() + host_e.numel()) * 16)}


def _init_dist():
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def run_ours(args):
    if args.workload == "phmsd":
        return run_phmsd(args)
    if args.workload == "control-variate":
        return run_control_variate(args)
    import torch
    import torch.distributed as dist

    from safire_b200 import afqmc as A
    from safire_b200.driver import RunParams, Simulation
    from safire_b200.synth import make_workload

    world, rank, local = _init_dist()
    prec = A.PREC_MIXED if args.precision == "mixed" else A.PREC_FP64
    W = args.walkers
    wl = make_workload("cfg2")
    rp = RunParams(equilibration_steps=0, seed=0)
    sim = Simulation.from_workload(wl, W=W, precision=prec, rp=rp)
    sim.use_graph = not args.no_graph
    if prec == A.PREC_MIXED and args.exchange_split != 3:
        sim.ham.set_exchange_split(args.exchange_split)
    tuned = None
    if prec == A.PREC_MIXED and args.taylor_mode != 1:
        sim.ham.set_taylor_fused(args.taylor_mode)
    elif prec == A.PREC_MIXED:
        # the library's autotuner times each Taylor variant on these walkers (state restored)
        best, ms = sim.autotune()
        tuned = {"taylor_mode": best, "step_ms": ms}

    t_ms, launches, clk = _timed_blocks(sim, args.steps, args.warmup, world, local,
                                        ClockSampler(local))
    value = W * world * BLOCK * args.steps / (t_ms / 1000)
    phases = _phases(sim)

    # roofline of the dominant contraction: the kernel with the largest share of a block
    M, N, Nc = wl.M, wl.nup, wl.Nc
    peaks = measured_peaks()
    if prec == A.PREC_FP64:
        # flops the FP64 kernels execute (real trial: Lnak, L and P1 are real)
        flops = {"vHS": 4.0 * M * M * Nc * W, "vbias": 4.0 * N * M * Nc * W,
                 "propagate": W * (2 * 4.0 * M * M * N + 6 * 8.0 * M * M * N),
                 "energy_measurement": W * (4.0 * N * N * M * Nc + 8.0 * N * N * Nc)}
        peak = fp64_peak_tflops(torch)
        peak_src = "cuBLAS DGEMM 8192^3 measured in this run (dense FP64; no FP64 entry in " \
                   "MEASURED_PEAKS.json)"
    else:
        # TF32 MMA flops of the split products (x3 for 3xTF32, unpadded tile extents)
        sp = 3.0
        ex = float(args.exchange_split)
        flops = {"vHS": sp * 4.0 * M * M * Nc * W, "vbias": sp * 4.0 * N * M * Nc * W,
                 "propagate": sp * W * (2 * 4.0 * M * M * N + 6 * 8.0 * M * M * N),
                 "energy_measurement": ex * W * 4.0 * N * N * M * Nc}
        if peaks.get("bf16_tflops"):
            peak = peaks["bf16_tflops"] / 2
            peak_src = "of measured: MEASURED_PEAKS.json bf16_tflops / 2 (dense TF32 runs at " \
                       "half the BF16 tensor rate)"
        else:
            peak = tf32_peak_tflops(torch)
            peak_src = "cuBLAS TF32 GEMM 8192^3 measured in this run"
    block_share = {k: (phases[k] * (1 if k == "energy_measurement" else BLOCK)) for k in flops}
    top = max(block_share, key=block_share.get)
    achieved = flops[top] / (phases[top] / 1000) / 1e12
    roofline = {"kernel": top, "bound": "tensor", "achieved": achieved,
                "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                "peak_source": peak_src, "flops_per_launch": flops[top],
                "block_share_ms": block_share}
    if top == "energy_measurement" and prec == A.PREC_MIXED:
        # the dominant kernel on its own: the fused exchange contraction (with its G split and
        # the final sums), timed with CUDA events on the launching stream
        G, _ = sim.wfn.MixedDensityMatrix(sim.wset)
        E = torch.empty((W, 3), dtype=torch.complex128, device=G.device)
        sim.ham.energy(E, G, addH1=False, precision=prec)
        stream = torch.cuda.current_stream()
        x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 5
        x0.record(stream)
        for _ in range(reps):
            sim.ham.energy(E, G, addH1=False, precision=prec)
        x1.record(stream)
        torch.cuda.synchronize()
        t_x = x0.elapsed_time(x1) / reps
        del G, E
        # DRAM bytes per launch from the ncu capture at 128 walkers (155.7 MB read + 10.1 MB
        # written = Lnak planes once + G planes and the per-(walker, vector) sums), scaled to W:
        # 2 Lnak planes + W x (4 G planes + 2 complex outputs per Cholesky vector)
        traffic = 2 * Nc * N * M * 4 + W * (4 * N * M * 4 + 2 * Nc * 16)
        roofline.update({"kernel": "exchange_tc_kernel<3> (fused EXX/EJ contraction)",
                         "achieved": flops[top] / (t_x / 1000) / 1e12,
                         "frac": flops[top] / (t_x / 1000) / 1e12 / peak,
                         "launch_ms": t_x, "traffic": traffic,
                         "traffic_source": "ncu capture at 128 walkers, scaled by walkers"})

    # the synthetic system's total weight collapses after ~200 steps: restart from the trial
    sim.restart()
    e2e = None if args.no_e2e else _e2e(sim, W, Nc, args.steps, world, prec)

    # the plain complex128 path on the same inputs, timed the same way: the mixed-vs-FP64 ratio
    fp64 = None
    if prec == A.PREC_MIXED and not args.no_fp64_compare:
        err_flag = int(sim.ham.device_error_flag())
        del sim
        torch.cuda.empty_cache()
        ref = Simulation.from_workload(wl, W=W, precision=A.PREC_FP64, rp=rp)
        ref.use_graph = not args.no_graph
        t64, _, _ = _timed_blocks(ref, args.steps, args.warmup, world, local)
        v64 = W * world * BLOCK * args.steps / (t64 / 1000)
        fp64 = {"value": v64, "ms_per_step": t64 / args.steps, "mixed_over_fp64": value / v64}
        sim = ref
    else:
        err_flag = int(sim.ham.device_error_flag())

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = host_cores()
        os.environ.setdefault("OPENBLAS_NUM_THREADS", str(cores))
        v, t, desc = cpu_sample(wl, 16, 1)
        cpu = {"value": v, "unit": "walker-steps/s", "cores": cores, "kind": "port", "sample": desc}

    if rank == 0:
        line = {
            "metric": metric_name(), "value": value, "unit": "walker-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c128" if prec == A.PREC_FP64 else
                     ("c128+tf32x3" if args.exchange_split == 3 else "c128+tf32x3 (exchange tf32)"),
            "data": "synthetic",
            "config": {"workload": "M=200 N=50+50 Nc=1600 W=1024/GPU dt=0.005 taylor=6, "
                                   "block of 10 steps (ortho/5, comb/10, energy/10)",
                       "precision": args.precision, "global_walkers": W * world,
                       "exchange_split": args.exchange_split if prec == A.PREC_MIXED else None,
                       "taylor_mode": (tuned["taylor_mode"] if tuned else args.taylor_mode)
                                      if prec == A.PREC_MIXED else None,
                       "autotune": tuned,
                       "step_graph": not args.no_graph,
                       "parallelism": f"walker dp{world}",
                       "l2": "inputs larger than L2 (V 655 MB, Likn 512 MB per step)"},
            "fp64": fp64,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches, "clocks": clk, "phases_ms": phases,
            "device_error_flag": err_flag,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_control_variate(args):
    """The learned exchange control variate on the M=200 workload (mixed precision): pairs from
    the exact kernel over the first steps train the MLP on top of the exchange over the leading
    Nc / 16 Cholesky vectors; afterwards every measurement is timed both ways (all-exact vs the
    base + network on all walkers + exact exchange on 1/8 weight-proportional draws), and the cost
    ratio at equal statistical error bar is reported with the estimator's spread."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from safire_b200 import afqmc as A
    from safire_b200.driver import RunParams, Simulation
    from safire_b200.mlp import ExchangeControlVariate, lowrank_hamiltonian
    from safire_b200.synth import make_workload

    world, rank, local = _init_dist()
    W = args.walkers
    wl = make_workload(args.cv_system)
    if args.cv_system == "cfg2":
        # training pairs from the first 150 steps at a fixed Eshift (one set every step): on this
        # synthetic system the reference algorithm's total weight collapses after
        # a few hundred steps, so a 500-step equilibration cannot run
        equil, every, eq_steps = 150, 1, 0
    else:
        # the M=32 system equilibrates: 500 steps with the Eshift update, a pair set every 10
        equil, every, eq_steps = 500, 10, 500
    sim = Simulation.from_workload(wl, W=W, precision=A.PREC_MIXED,
                                   rp=RunParams(equilibration_steps=eq_steps, seed=0))
    sim.use_graph = not args.no_graph
    lowrank = None
    if args.cv_lowrank < 0:
        args.cv_lowrank = wl.Nc // 16
    if args.cv_lowrank:
        lowrank = lowrank_hamiltonian((wl.walker_type, wl.M, wl.nup, wl.ndn, wl.Likn, wl.hij,
                                       wl.E0, wl.PsiT), args.cv_lowrank)
    cv = ExchangeControlVariate(sim, hidden=512, fraction=args.cv_fraction, seed=0,
                                sampling=args.cv_sampling, lowrank=lowrank)
    for step in range(equil):
        sim.step(measure=False)
        if step % every == 0:
            cv.collect()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = cv.fit(epochs=args.cv_epochs, batch=1024, lr=1e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0

    stream = torch.cuda.current_stream()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return r, e0.elapsed_time(e1)

    exact_e, mf_e, t_ex, t_mf = [], [], [], []
    for m in range(args.steps + args.warmup):
        for _ in range(BLOCK):
            sim.step(measure=False)
        (e_exact, _, _), te = timed(sim.measure)
        (e_mf, _), tm = timed(cv.measure)
        if m >= args.warmup:
            exact_e.append(e_exact)
            mf_e.append(e_mf)
            t_ex.append(te)
            t_mf.append(tm)
    # the Coulomb term the estimator takes from the force bias against the energy kernel's
    _, o = cv.measure(exact=True)
    ej_gap = (o["ej_from_vbias"] - o["ej_exact"]).real
    exact_e, mf_e = np.array(exact_e), np.array(mf_e)
    diff = mf_e - exact_e
    s_qmc = float(np.std(exact_e, ddof=1))
    s_sub = float(np.std(diff, ddof=1))
    factor = (s_qmc ** 2 + s_sub ** 2) / s_qmc ** 2  # measurements needed for equal error bar
    tex, tmf = float(np.median(t_ex)), float(np.median(t_mf))
    value = tex / (tmf * factor)
    if rank == 0:
        line = {
            "metric": "energy-measurement cost reduction at equal statistical error bar, "
                      f"learned exchange control variate (M={wl.M}, {W} walkers, mixed)",
            "value": value, "unit": "x (all-exact cost / control-variate cost)",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 MLP (fp32 accumulate) + c128/tf32x3 exact exchange",
            "data": "synthetic",
            "config": {"workload": f"M={wl.M} N={wl.nup}+{wl.ndn} Nc={wl.Nc} W={W} "
                                   f"dt={wl.dt}; MLP {cv.mlp.D}-512-512-1 GELU trained on pairs "
                                   f"from the first {equil} steps (one set per {every} steps"
                                   f"{', fixed Eshift' if eq_steps == 0 else ''}); exact "
                                   f"exchange on {args.cv_fraction:.3g} of the walkers "
                                   f"({args.cv_sampling} draws) per measurement; "
                                   + (f"network on top of the exchange over the leading "
                                      f"{args.cv_lowrank} Cholesky vectors; "
                                      if args.cv_lowrank else "")
                                   + "one measurement per 10-step block",
                       "training_samples": int(sum(x.shape[0] for x in cv.X)),
                       "epochs": args.cv_epochs, "train_seconds": t_train,
                       "loss_first_last": [hist[0], hist[-1]]},
            "measurement_ms": {"all_exact": tex, "control_variate": tmf},
            "sigma": {"qmc_between_measurements": s_qmc, "subsampling": s_sub,
                      "measurements_factor_for_equal_error": factor},
            "bias": {"mean_mf_minus_exact": float(diff.mean()),
                     "standard_error": float(s_sub / np.sqrt(diff.size)),
                     "ej_from_vbias_minus_energy_kernel": float(ej_gap)},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_phmsd(args):
    """The multi-determinant workload: COLLINEAR M=120, N=30+30, Nc=960, reference + 4095
    particle-hole determinants, 512 walkers per GPU; FP64 (the PHMSD kernels run in complex128)."""
    import torch
    import torch.distributed as dist

    from safire_b200 import afqmc as A
    from safire_b200.driver import RunParams, Simulation
    from safire_b200.synth import make_phmsd_workload

    world, rank, local = _init_dist()
    W = args.walkers if args.walkers != 1024 else 512
    wl, trial = make_phmsd_workload(W=W)
    rp = RunParams(equilibration_steps=0, seed=0)
    sim = Simulation.from_workload(wl, W=W, rp=rp, trial=trial)
    sim.use_graph = False
    t_ms, launches, clk = _timed_blocks(sim, args.steps, args.warmup, world, local,
                                        ClockSampler(local))
    value = W * world * BLOCK * args.steps / (t_ms / 1000)
    phases = _phases(sim)
    # the excited-determinant energy tables, per (walker, Cholesky index) and spin: the table
    # products Y = t[:, r] QQ0^T (nel x nv x nel), U = t[holes, r] t (nh x nact x nel),
    # Z = t[holes, r] Y (nh x nv x nel), then 3 n^3 + 6 n^2 + 3 n complex MACs per n-hole
    # determinant (the closed-form sums of excited_terms); 8 flops per complex MAC
    macs = 0.0
    for s in (0, 1):
        nel = trial.nup if s == 0 else trial.ndn
        nact = trial.orbmat[s].shape[0]
        nv = nact - nel
        nh = len({int(h) for n, e in trial.exc[s].items() for h in e[:, :n].ravel()})
        macs += nel * nv * nel + nh * nact * nel + nh * nv * nel
        macs += sum(len(e) * (3 * n ** 3 + 6 * n ** 2 + 3 * n) for n, e in trial.exc[s].items())
    flops = 8.0 * W * wl.Nc * macs
    fp64 = fp64_peak_tflops(torch)
    achieved = flops / (phases["energy_measurement"] / 1000) / 1e12
    roofline = {"kernel": "energy_measurement (excited_energy_tables_kernel ~80%)",
                "bound": "fp64", "achieved": achieved, "peak": fp64, "unit": "TFLOP/s",
                "frac": achieved / fp64, "traffic": None, "flops_per_launch": flops,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run"}
    e2e = None if args.no_e2e else _e2e(sim, W, wl.Nc, args.steps, world, A.PREC_FP64)
    if rank == 0:
        line = {
            "metric": "walker-steps/s, PHMSD trial (M=120, 30+30 electrons, 4096 determinants, "
                      "512 walkers) on B200",
            "value": value, "unit": "walker-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": f"PHMSD M=120 N=30+30 Nc=960 W={W}/GPU dt=0.005 taylor=6, "
                                   "reference + 4095 determinants (20 occ / 40 virt window), "
                                   "block of 10 steps (ortho/5, comb/10, energy/10)",
                       "precision": "fp64", "global_walkers": W * world,
                       "parallelism": f"walker dp{world}"},
            "roofline": roofline, "cpu_baseline": None, "e2e": e2e,
            "gpu_launches": launches, "clocks": clk, "phases_ms": phases,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
