"""Walker-propagation benchmark (MPSQMC2::Walk hot path) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference] [--workload snake8x8]

Default workload snake8x8 (the full chosen configuration): the open 8x8 Heisenberg lattice on the
snake path, D_T = 256 DMRG ground-state trial, 4096 walkers of D_W = 64 (the trial compressed),
dtau = 0.005, Marsaglia(4) grid.  One walker-step = propagation over all 112 couplings, local
energy, statistics and threshold branching.  The timed arm is the walker-batched mixed-precision
sweep on the tcgen05 tensor cores (TF32 x3, FP32-accurate products; FP64 walkers, weights,
overlaps, energies and population control); the plain FP64 sweep on the same configuration is
timed beside it for the ratio.  Prints one JSON line (rank 0).

Timing: W untimed steps, then K steps in one engine call; device time from CUDA events recorded on
the engine's stream around those K steps (the walker population, 14 GB, exceeds L2 so no flush
is needed).  Multi-GPU: independent replicas (one population per rank), max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "walker-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--workload", default="snake8x8", choices=["chain64", "snake6x6", "snake6x6_dmrg", "snake8x8",
                                                                "snake8x8_dmrg", "snake8x8_random"],
                    help="snake8x8: the 8x8 lattice with its D_T = 256 DMRG trial (default line); chain64: the "
                         "L = 64 chain; snake6x6: the 6x6 lattice with uneven walkers; *_dmrg: D_T = 64 "
                         "DMRG trials; snake8x8_random: the 8x8 shapes with a random trial")
    ap.add_argument("--fp64-steps", type=int, default=2,
                    help="steps of the plain FP64 sweep timed beside a mixed-precision main arm (its "
                         "throughput for the ratio); 0: skip")
    ap.add_argument("--walkers", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--sweep", default="auto", choices=["auto", "nearest", "general"],
                    help="walker-step kernel (auto: the general sweep)")
    ap.add_argument("--vn", type=int, default=0, metavar="STEPS",
                    help="after the timed steps, walk STEPS more and report the variance-normalised "
                         "throughput (blocking error of the mixed energy; first 20%% discarded)")
    ap.add_argument("--workspace", default="auto", choices=["auto", "global"],
                    help="matrix work buffers: shared memory when they fit (auto) or global scratch")
    ap.add_argument("--precision", default=None, choices=["fp64", "tf32x3", "tf32", "tf32x3_tc", "tf32_tc", "bf16_tc"],
                    help="walker-step contractions: FP64 tensor cores, or FP32 buffers on TF32 tensor cores "
                         "(three passes / one pass; *_tc: the walker-batched sweep on tcgen05); weights, "
                         "overlaps, energies stay FP64.  Default: tf32x3_tc on snake8x8, fp64 otherwise")
    ap.add_argument("--proposal", default="grid", choices=["grid", "learned"],
                    help="auxiliary-field proposal: the exact grid PDF, or the learned network (trained online "
                         "on the grid walk for --train-steps steps first; exact-ratio reweighting)")
    ap.add_argument("--train-steps", type=int, default=100)
    ap.add_argument("--proposal-mix", type=int, default=None, metavar="ALPHA",
                    help="learned proposal: thousandths of the exact PDF in the defensive mixture it draws "
                         "from (default: the engine's, 100)")
    ap.add_argument("--canon", type=int, default=None, metavar="K",
                    help="QR-free sweep, left-normalise every K steps (0: Householder QR per site; "
                         "default: the engine's, 16)")
    ap.add_argument("--vn-compare", type=int, default=None, metavar="STEPS",
                    help="variance-normalised throughput (the headline metric) of the plain FP64 grid walk "
                         "and of the --vn-arms variants, STEPS steps each after their timed steps, from the "
                         "same start and random stream; ratios against the plain walk (default off: the FP64 "
                         "arm's steps at config 5 take 20 s each; the default line reports the throughput "
                         "ratio of the same walk in fp64_arm)")
    ap.add_argument("--sharded", action="store_true",
                    help="N>1: one walk split over the ranks (global population control and walker "
                         "balancing, mpsqmc_b200.population; NCCL, records in device buffers) instead of N "
                         "independent replicas")
    ap.add_argument("--gain-steps", type=int, default=3, metavar="STEPS",
                    help="untimed grid steps after the timed ones that measure the proposal gain bound")
    ap.add_argument("--tiles", default="autotune", choices=["autotune", "default"],
                    help="tcgen05 sweep: tile choices picked by mpsqmc_autotune for this bond profile (untimed "
                         "set-up, remembered for the process) or the built-in defaults")
    ap.add_argument("--vn-arms", default="tf32x3/grid,tf32x3/learned",
                    help="precision/proposal variants compared with the plain FP64 grid walk")
    a = ap.parse_args()
    if a.precision is None:
        a.precision = "tf32x3_tc" if a.workload == "snake8x8" else "fp64"
    return a


PRECISIONS = {"fp64": 0, "tf32": 1, "tf32x3": 2, "tf32x3_tc": 3, "tf32_tc": 4, "bf16_tc": 5}


def configure(eng, args, sweep, plain=False):
    """Kernel and method options of a bench engine; plain: the FP64 grid walk (the VN yardstick)."""
    from mpsqmc_b200.capi import (OPT_CANONICAL_INTERVAL, OPT_PRECISION, OPT_PROPOSAL_MIX, OPT_SWEEP,
                                  OPT_WORKSPACE, WORKSPACE_GLOBAL)
    eng.set_option(OPT_SWEEP, sweep)
    if args.proposal_mix is not None:
        eng.set_option(OPT_PROPOSAL_MIX, args.proposal_mix)
    if args.workspace == "global":
        eng.set_option(OPT_WORKSPACE, WORKSPACE_GLOBAL)
    if args.canon is not None:
        eng.set_option(OPT_CANONICAL_INTERVAL, args.canon)
    if not plain:
        eng.set_option(OPT_PRECISION, PRECISIONS[args.precision])


def train_proposal(make, args, sweep, seed):
    """Online training of the learned proposal (untimed set-up) on a separate engine that walks
    the grid walk from the start, so that the walk using the network starts where the other
    variants start (the same imaginary time in every compared window).  Returns (network
    parameters, what the training did), or (None, None) for the grid proposal."""
    from mpsqmc_b200.capi import OPT_PROPOSAL_TRAINING
    if args.proposal != "learned":
        return None, None
    eng = make()
    configure(eng, args, sweep)
    eng.set_rng(seed + 1, 0)
    eng.set_option(OPT_PROPOSAL_TRAINING, 1)
    t0 = time.perf_counter()
    st = eng.walk(args.train_steps)
    dt = time.perf_counter() - t0
    ps = eng.proposal_stats()
    params = eng.proposal_params()
    eng.close()
    return params, {"steps": args.train_steps, "pairs": int(sum(s["n_walkers"] for s in st)),
                    "adam_steps": ps["updates"], "final_kl": ps["loss"], "seconds": dt,
                    "walk": "a separate engine from the same start"}


def use_proposal(eng, params):
    """The walk samples from the trained network (exact-ratio weights)."""
    from mpsqmc_b200.capi import OPT_PROPOSAL, PROPOSAL_LEARNED
    if params is not None:
        eng.proposal_params(params)
        eng.set_option(OPT_PROPOSAL, PROPOSAL_LEARNED)


def dist_setup(n, nccl=False):
    """One process per GPU.  nccl: the split walk's data plane (global sums and walker records
    in device buffers over NCCL); otherwise gloo, which only carries the replicas' barriers and
    timing aggregation."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        if nccl:
            import torch
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=timedelta(seconds=120))
        pg = dist
    return rank, world, local, pg


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def aggregate_ranks(pg, t_ms, k_ms, walker_steps):
    """Whole-job figures over the ranks: the slowest rank's times (max) and the walker-steps of all
    ranks (sum).  pg is torch.distributed (any backend) or None for one rank."""
    if pg is None:
        return t_ms, k_ms, float(walker_steps)
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    tt = torch.tensor([t_ms, k_ms, float(walker_steps)], dtype=torch.float64, device=dev)
    mx = tt.clone()
    pg.all_reduce(mx, op=pg.ReduceOp.MAX)
    sm = tt.clone()
    pg.all_reduce(sm, op=pg.ReduceOp.SUM)
    return float(mx[0].item()), float(mx[1].item()), float(sm[2].item())


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    return json.load(open(p)) if os.path.exists(p) else {}


def fp64_peak_tflops():
    """cuBLAS DGEMM 8192^3, best of 5 (CUDA events): the FP64 denominator (none is pre-measured)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c = a @ b
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c = a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def tf32_peak_tflops(dtype="float32"):
    """cuBLAS GEMM 8192^3, best of 5 (CUDA events): FP32 with TF32 tensor cores allowed (the
    denominator of the TF32 sweeps) or bfloat16 (that of the BF16 sweep)."""
    import torch
    keep = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    n = 8192
    dt = getattr(torch, dtype)
    a = torch.randn(n, n, dtype=torch.float32, device="cuda").to(dt)
    b = torch.randn(n, n, dtype=torch.float32, device="cuda").to(dt)
    c = a @ b
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        c = a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    torch.backends.cuda.matmul.allow_tf32 = keep
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def reference_cpu(wl, sample_walkers=None, steps=1, threads=None, max_couplings=None):
    """The reference's own classes (oracle/_ref/ref_harness, built from the reference sources) timed on
    this host: propagation of `sample_walkers` walkers for `steps` steps, energy excluded (the
    reference's H*Psi_T MPS does not fit at these sizes).  max_couplings: time only the first k
    couplings of each step and extrapolate to all of them (the reference's cost per coupling is
    16 full-chain InnerProducts and one LeftNormalize whatever the coupling, so the rate scales)."""
    from oracle import pyoracle as po
    if not po.harness_available():
        return None
    threads = threads or os.cpu_count()
    sample_walkers = sample_walkers or threads
    trial = wl.trial() if callable(getattr(wl, "trial", None)) else wl.trial
    env = {"OMP_NUM_THREADS": str(threads)}
    if hasattr(wl, "W"):
        env["MPSQMC_REF_LATTICE"] = f"snake:{wl.W}x{wl.H}"
    if max_couplings:
        env["MPSQMC_REF_MAX_COUPLINGS"] = str(max_couplings)
    DW = wl.DW if hasattr(wl, "DW") else max(wl.Ds)
    with tempfile.TemporaryDirectory() as t:
        path = os.path.join(t, "trial.mps")
        po.write_mps(path, po.MPS(trial.dims, trial.data))
        out = po.run_harness("propagate", path, DW, sample_walkers, wl.dtau, steps, env_extra=env)
    r = json.loads(out.strip().splitlines()[-1])
    part = (f", {r['couplings_timed']} of {r['couplings']} couplings timed per step and the rate "
            f"extrapolated to all" if r.get("couplings_timed", 0) < r.get("couplings", 0) else "")
    r["sample"] = (f"{sample_walkers} walkers x {steps} step(s) of {wl.name}, propagation only "
                   f"(reference classes, per-coupling trial terms, no energy{part})")
    r["cores"] = threads
    return r


def lattice_population(wl):
    """Walkers of a 2D workload as SetupWalkers makes them (MPSQMC2.cpp:404-409): copies of the trial
    compressed to D_W (CompressState + setOverlap), on the host when D_W < D_T; with uneven targets
    that include D_T, on the device (compress_walkers).  Returns (slot bond profile, host population
    or None, device targets or None)."""
    from mpsqmc_b200 import problem as pb
    trial = wl.trial()
    if max(wl.Ds) >= wl.DT:
        return trial.dims, None, wl.targets()
    w = pb.compress(trial, max(wl.Ds))
    return w.dims, w.data, None


def main():
    args = parse()
    rank, world, local, pg = dist_setup(args.gpus, nccl=args.sharded and args.impl == "mine")
    from mpsqmc_b200 import workloads

    lattice = args.workload != "chain64"
    if lattice:
        wl = getattr(workloads, args.workload)(Nw=args.walkers) if args.walkers else getattr(workloads, args.workload)()
        te = wl.trial_energy()
        cfg = {"workload": f"{wl.name}: {wl.W}x{wl.H} open Heisenberg lattice on the snake path (L={wl.L}, "
                           f"{len(wl.couplings()[0])} couplings), D_T={wl.DT}, D_W in {wl.Ds}, {wl.Nw} walkers/GPU, "
                           f"dtau={wl.dtau}, Marsaglia(4) grid; "
                           + (f"trial: DMRG ground state at D_T={wl.DT} (E={te:.10f})" if wl.trial_file
                              else "seeded random left-normalised trial of the D_T shape")
                           + "; walkers = the trial compressed to D_W",
               "walkers_per_gpu": wl.Nw, "L": wl.L, "D_T": wl.DT, "D_W": wl.Ds, "dtau": wl.dtau,
               "l2": f"population ({wl.Nw * 8 * 2 * sum(int(a) * int(b) for a, b in zip(workloads.pb.virtual_dims(wl.L, max(wl.Ds))[:-1], workloads.pb.virtual_dims(wl.L, max(wl.Ds))[1:])) / 1e9:.1f} GB) larger than L2 (126 MB); no flush"}
    else:
        wl = workloads.chain64(Nw=args.walkers or 2048)
        cfg = {"workload": f"{wl.name}: L={wl.L} Heisenberg chain, D_T={wl.DT}, D_W={wl.DW}, {wl.Nw} walkers/GPU, "
                           f"dtau={wl.dtau}, Marsaglia(4) grid",
               "walkers_per_gpu": wl.Nw, "L": wl.L, "D_T": wl.DT, "D_W": wl.DW, "dtau": wl.dtau,
               "l2": f"population ({wl.Nw * wl.walker.data.size * 8 / 1e9:.2f} GB) larger than L2 (126 MB); no flush"}
    cfg.update({"parallelism": f"{'split walk' if args.sharded else 'replicas'} x{world}", "sweep": args.sweep,
                "workspace": args.workspace, "precision": args.precision, "proposal": args.proposal,
                "proposal_mix": args.proposal_mix if args.proposal_mix is not None else 100,
                "canonical_interval": args.canon if args.canon is not None else 16})
    # the reference CPU sample: all couplings of chain64; two of the lattices' (extrapolated)
    ref_couplings = 2 if lattice else None
    ref_walkers = min(os.cpu_count() or 1, 16)

    if args.impl == "reference":
        if rank != 0:
            return
        r = reference_cpu(wl, sample_walkers=ref_walkers, steps=max(1, args.steps), threads=ref_walkers,
                          max_couplings=ref_couplings)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_harness not built"}))
            return
        v = r["walker_steps_per_s"]
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "walker-steps/s", "n_gpus": 0,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f64",
                "data": "synthetic", "config": cfg,
                "cpu_baseline": {"value": v, "unit": "walker-steps/s", "cores": r["cores"], "kind": "reference",
                                 "sample": r["sample"]},
                "e2e": {"value": v, "unit": "walker-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    torch.cuda.set_device(local)
    from mpsqmc_b200 import Engine

    sweep = {"auto": 0, "nearest": 1, "general": 2}[args.sweep]
    seed = wl.seed + 7919 * rank
    if lattice:
        from mpsqmc_b200 import problem as pb
        ci, cj, cJ = wl.couplings()
        trial = wl.trial()
        U, S, VT = pb.trotter_tables(1.0, wl.dtau)
        wdims, w0, targets = lattice_population(wl)
        N = wl.Nw
        inputs = dict(L=wl.L, ci=ci, cj=cj, cJ=cJ, h=0.0, dtau=wl.dtau, trial_dims=trial.dims, trial=trial.data,
                      Jvals=[1.0], U=U, S=S, VT=VT, grid=pb.grid_marsaglia(4, 4), Ndesired=N,
                      capacity=max(1000, 2 * N), walker_dims=wdims)
        if w0 is not None:
            # the population in pinned host memory (the device upload and the e2e arm read it)
            walkers = torch.empty((N, w0.size), dtype=torch.float64, pin_memory=True).numpy()
            walkers[:] = w0[None, :]
        else:
            walkers = None
            args.no_e2e = True
    else:
        inputs = wl.inputs()
        walkers = wl.walkers()
        N = walkers.shape[0]

    def make():
        e = Engine(device=local, **inputs)
        if walkers is not None:
            e.set_walkers(walkers, np.ones(N), None, np.zeros(N), normalize=True)
        else:
            e.set_walkers(np.tile(inputs["trial"], (N, 1)), np.ones(N), normalize=False)
            e.compress_walkers(targets, normalize=True)
        return e

    def timed_arm(precision, steps, warmup, proposal="grid", params=None):
        """One engine walking `warmup` untimed then `steps` timed steps from the common start and
        random stream; returns (engine, stats, timing)."""
        a = argparse.Namespace(**vars(args))
        a.precision, a.proposal = precision, proposal
        e = make()
        configure(e, a, sweep, plain=(precision == "fp64"))
        e.set_rng(seed, 0)
        use_proposal(e, params)
        if precision.endswith("_tc") and args.tiles == "autotune":
            e.autotune(steps=1)  # restores population, random stream and step count
        e.walk(warmup)
        torch.cuda.synchronize()
        return e, a

    params, training = train_proposal(make, args, sweep, seed)
    eng, _ = timed_arm(args.precision, args.steps, args.warmup, args.proposal, params)
    if args.precision.endswith("_tc"):
        from mpsqmc_b200.capi import OPT_TC_KC, OPT_TC_SPLIT_OUT, OPT_TC_STACK_TN, OPT_TC_STAGES, OPT_TC_WIDE_TN
        cfg["tiles"] = {"split_out": eng.get_option(OPT_TC_SPLIT_OUT), "kc_trial": eng.get_option(OPT_TC_KC),
                        "stack_tn": eng.get_option(OPT_TC_STACK_TN),
                        "wide_tn": eng.get_option(OPT_TC_WIDE_TN), "max_stages": eng.get_option(OPT_TC_STAGES),
                        "chosen_by": ("mpsqmc_autotune: coordinate search over the tile choices on up to 1024 "
                                      "walkers of this bond profile" if args.tiles == "autotune" else "defaults")}
    if pg is not None:
        pg.barrier()
    rw = None
    if args.sharded and pg is not None:
        from mpsqmc_b200.population import RankWalk
        # walker records and the five sums in device buffers, moved by NCCL into the receiver's HBM
        rw = RankWalk(eng, pg, [N] * world, device=f"cuda:{local}")
    with ClockSampler(local) as clk:
        if rw is None:
            stats = eng.walk(args.steps)
            torch.cuda.synchronize()
            tim = eng.last_timing()
        else:
            # split walk: every step ends in a host exchange, so the device time is the host time
            # between synchronised ends (max over ranks below)
            t0 = time.perf_counter()
            stats = [rw.step() for _ in range(args.steps)]
            torch.cuda.synchronize()
            wall = (time.perf_counter() - t0) * 1e3
            tim = {"total_ms": wall, "step_kernel_ms": wall, "launches": eng.last_timing()["launches"] * args.steps}
    if pg is not None:
        pg.barrier()
    ws_done = sum(s["n_walkers"] for s in stats)
    t_ms = tim["total_ms"]
    k_ms = tim["step_kernel_ms"]
    t_ms, k_ms, ws_all = aggregate_ranks(pg, t_ms, k_ms, ws_done)
    value = ws_all / (t_ms * 1e-3)

    # roofline of the dominant work (the walker step): canonical FP64-equivalent work / its device
    # time, averaged over the walkers' own bond dims
    cpl = list(zip(inputs["ci"], inputs["cj"]))
    dims_now = eng.get_walker_dims()
    rows, counts = np.unique(dims_now, axis=0, return_counts=True)
    flops_ws = float(sum(c * workloads.algorithmic_flops_per_walker_step(inputs["trial_dims"], r, cpl)
                         for r, c in zip(rows, counts)) / counts.sum())
    achieved = flops_ws * ws_done / (k_ms * 1e-3) / 1e12
    mixed = args.precision != "fp64"
    tc = args.precision.endswith("_tc")
    passes = 1 if args.precision in ("tf32", "tf32_tc", "bf16_tc") else 3
    E_last = {"E_P_last": stats[-1]["E_P"], "E_T_last": stats[-1]["E_T"], "walkers_last": stats[-1]["n_after"],
              "E_P_mean": float(np.mean([s["E_P"] for s in stats]))}

    # what any auxiliary-field proposal could gain over the grid PDF on this walk (untimed steps
    # after the timed ones): N sum w^2 / (sum w)^2 of the propagated weights
    gain = None
    if args.gain_steps > 0 and rw is None and args.proposal == "grid" and not (args.vn or args.vn_compare):
        from mpsqmc_b200 import analysis
        ws_g = []
        for _ in range(args.gain_steps):
            eng.walk(1)
            ws_g.append(eng.last_step_walkers()["weight"])
        gain = {"value": analysis.proposal_gain_bound(ws_g), "steps": args.gain_steps,
                "definition": "mean over steps of N sum w^2 / (sum w)^2 of the walkers' weights after "
                              "propagation: the largest factor by which any proposal (learned or look-ahead) "
                              "could lower the variance of the weighted mean energy"}

    vn = None
    vn_steps = max(args.vn, args.vn_compare or 0)
    if vn_steps > 0 and rw is None:
        from mpsqmc_b200 import analysis
        e_ref = wl.trial_energy() if lattice else None
        e_src = f"DMRG D={wl.DT} energy of the trial (a variational upper bound)" if e_ref is not None else None

        def vn_of(e, throughput):
            more = e.walk(vn_steps)
            r = analysis.variance_normalised(throughput, [x["E_P"] for x in more], [x["n_walkers"] for x in more])
            r["throughput_per_gpu"] = throughput
            if e_ref is not None:
                r["E_ref"] = e_ref
                r["E_ref_source"] = e_src
            return r

        this = vn_of(eng, value / max(world, 1))
        this["arm"] = f"{args.precision}/{args.proposal}"
        vn = this
        if args.vn_compare:
            eng.close()
            arms = {this["arm"]: this}
            named = [x if "/" in x else x + "/grid" for x in args.vn_arms.split(",") if x]
            for name in ["fp64/grid"] + named:
                if name in arms:
                    continue
                prec, prop = name.split("/")
                p_arm, tr = train_proposal(make, argparse.Namespace(**{**vars(args), "precision": prec,
                                                                          "proposal": prop}), sweep, seed)
                e, _ = timed_arm(prec, args.steps, args.warmup, prop, p_arm)
                st = e.walk(args.steps)
                t = e.last_timing()
                r = vn_of(e, sum(x["n_walkers"] for x in st) / (t["total_ms"] * 1e-3))
                if tr:
                    r["proposal_training"] = tr
                e.close()
                arms[name] = r
            plain = arms["fp64/grid"]
            vn = {"plain_fp64_grid": plain, "vn_ratio_vs_plain_fp64": {}, "throughput_ratio_vs_plain_fp64": {},
                  "E_mean_diff_vs_plain_per_site": {}}
            for name, r in arms.items():
                if name == "fp64/grid":
                    continue
                vn[name] = r
                vn["vn_ratio_vs_plain_fp64"][name] = r["vn"] / plain["vn"] if plain["vn"] else None
                vn["throughput_ratio_vs_plain_fp64"][name] = r["throughput_per_gpu"] / plain["throughput_per_gpu"]
                vn["E_mean_diff_vs_plain_per_site"][name] = abs(r["E_mean"] - plain["E_mean"]) / wl.L
            eng = None
    if eng is not None:
        eng.close()

    # the plain FP64 sweep on the same configuration, timed beside a mixed-precision main arm
    fp64_arm = None
    if mixed and args.fp64_steps > 0 and vn is None:
        e, _ = timed_arm("fp64", args.fp64_steps, 1)
        st = e.walk(args.fp64_steps)
        t = e.last_timing()
        e.close()
        t_f, _, ws_f = aggregate_ranks(pg, t["total_ms"], t["step_kernel_ms"], sum(x["n_walkers"] for x in st))
        v_f = ws_f / (t_f * 1e-3)
        fp64_arm = {"value": v_f, "unit": "walker-steps/s", "steps": args.fp64_steps, "warmup": 1,
                    "ms_per_step": t_f / args.fp64_steps, "E_P_mean": float(np.mean([x["E_P"] for x in st])),
                    "throughput_ratio_mixed_vs_fp64": value / v_f,
                    "note": "same configuration, start and random stream; the mixed arm's products are "
                            "FP32-accurate, so it follows the FP64 trajectory and the energy variance per "
                            "walker-step is the same: the throughput ratio is the variance-normalised ratio "
                            "(measured over long walks in profiles/)"}

    peak = None
    if rank == 0:
        peak = (tf32_peak_tflops("bfloat16") if args.precision == "bf16_tc" else tf32_peak_tflops()) if mixed \
            else fp64_peak_tflops()

    # end to end through the public API: host population -> device, K steps (stats read back each
    # step), population -> host; host wall clock.
    e2e = None
    if not args.no_e2e and walkers is not None:
        eng2, _ = timed_arm(args.precision, args.steps, args.warmup, args.proposal, params)
        # the population in pinned host memory (both directions), as a serving caller would keep it
        host_w = walkers if lattice else torch.empty(walkers.shape, dtype=torch.float64, pin_memory=True).numpy()
        if not lattice:
            host_w[:] = walkers
        back_w = torch.empty((max(N + N // 2, 64), eng2.walker_size), dtype=torch.float64, pin_memory=True).numpy()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng2.set_walkers(host_w, np.ones(N), None, np.zeros(N), normalize=True)
        eng2.set_rng(seed, 0)
        st2 = eng2.walk(args.steps)
        back = eng2.get_walkers(out=back_w)
        t1 = time.perf_counter()
        ws2 = sum(s["n_walkers"] for s in st2)
        nbytes = host_w.nbytes
        t_e2e, _, ws2_all = aggregate_ranks(pg, (t1 - t0) * 1e3, 0.0, ws2)
        e2e = {"value": ws2_all / (t_e2e * 1e-3), "unit": "walker-steps/s",
               "h2d_bytes_per_step": int(nbytes / args.steps),
               "d2h_bytes_per_step": int(back[0].nbytes / args.steps + 72)}
        eng2.close()

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        r = reference_cpu(wl, sample_walkers=ref_walkers, steps=1, threads=ref_walkers, max_couplings=ref_couplings)
        if r is not None:
            cpu = {"value": r["walker_steps_per_s"], "unit": "walker-steps/s", "cores": r["cores"],
                   "kind": "reference", "sample": r["sample"]}

    if rank == 0:
        prof_traffic = None
        kname = "walker_step_kernel" if args.sweep == "nearest" else (
            "tc_gemm_kernel" if tc else ("walker_step_mixed_kernel" if mixed else "walker_step_general_kernel"))
        tp = os.path.join(ROOT, "profiles", f"{kname}_{wl.name}_traffic.json")
        if os.path.exists(tp):
            prof_traffic = json.load(open(tp)).get("bytes_per_step_per_walker")
            if prof_traffic is not None:
                prof_traffic = prof_traffic * N  # one step processes every walker once
        line = {
            "metric": METRIC, "value": value, "unit": "walker-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if not mixed else f"{args.precision}+f64", "data": "synthetic",
            "config": cfg,
            "energy": E_last,
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if peak else None, "traffic": prof_traffic,
                         "kernel": kname, "flops_per_walker_step": flops_ws,
                         "timed": ("the whole walker-step sweep (all its launches) on the engine's stream"
                                   if tc else "the walker-step kernel on the engine's stream"),
                         **({"passes": passes, "executed_frac": passes * achieved / peak if peak else None}
                            if mixed else {}),
                         "peak_source": ("cuBLAS %s GEMM 8192^3 measured in this run (%s tensor path; the "
                                         "canonical flops count each product once)"
                                         % (("BF16", "BF16") if args.precision == "bf16_tc" else ("TF32", "TF32")))
                         if mixed else
                                        "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor path)"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": tim["launches"],
            **({"fp64_arm": fp64_arm} if fp64_arm is not None else {}),
            **({"variance_normalised": vn} if vn is not None else {}),
            **({"proposal_training": training} if training else {}),
            **({"proposal_gain_bound": gain} if gain is not None else {}),
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
