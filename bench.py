"""Walker-propagation benchmark (MPSQMC2::Walk hot path) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference] [--workload chain64]

Workload chain64 (the L=64 chain configuration): D_T=64 trial, 2048 walkers of D_W=32 (trial
compressed + N(0,1e-3) noise), dtau=0.01, one walker-step = propagation over all 63 couplings,
local energy, statistics and threshold branching.  Prints one JSON line (rank 0).

Timing: W untimed steps, then K steps in one engine call; device time from CUDA events recorded on
the engine's stream around those K steps (the walker population, 1.8 GB, exceeds L2 so no flush
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
    ap.add_argument("--workload", default="chain64", choices=["chain64", "snake6x6", "snake6x6_dmrg", "snake8x8",
                                                               "snake8x8_dmrg"],
                    help="chain64: the L=64 chain (default line); snake6x6 / snake8x8: the 2D lattices "
                         "(walkers compressed on the device; no CPU baseline or e2e); *_dmrg: with "
                         "their DMRG ground-state trials")
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
    ap.add_argument("--precision", default="fp64", choices=["fp64", "tf32x3", "tf32", "tf32x3_tc", "tf32_tc"],
                    help="walker-step contractions: FP64 tensor cores, or FP32 buffers on TF32 tensor cores "
                         "(three passes / one pass; *_tc: the walker-batched sweep on tcgen05); weights, "
                         "overlaps, energies stay FP64")
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
                         "same start and random stream; ratios against the plain walk (default: 300 on the "
                         "default chain64 run, else off)")
    ap.add_argument("--sharded", action="store_true",
                    help="N>1: one walk split over the ranks (global population control and walker "
                         "balancing, mpsqmc_b200.population) instead of N independent replicas")
    ap.add_argument("--vn-arms", default="tf32x3/grid,tf32x3/learned",
                    help="precision/proposal variants compared with the plain FP64 grid walk")
    return ap.parse_args()


PRECISIONS = {"fp64": 0, "tf32": 1, "tf32x3": 2, "tf32x3_tc": 3, "tf32_tc": 4}


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


def dist_setup(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
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
    tt = torch.tensor([t_ms, k_ms, float(walker_steps)], dtype=torch.float64)
    mx = tt.clone()
    pg.all_reduce(mx, op=pg.ReduceOp.MAX)
    sm = tt.clone()
    pg.all_reduce(sm, op=pg.ReduceOp.SUM)
    return float(mx[0]), float(mx[1]), float(sm[2])


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


def tf32_peak_tflops():
    """cuBLAS FP32 GEMM 8192^3 with TF32 tensor cores allowed, best of 5 (CUDA events): the
    denominator of the mixed-precision sweep."""
    import torch
    keep = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    n = 8192
    a = torch.randn(n, n, dtype=torch.float32, device="cuda")
    b = torch.randn(n, n, dtype=torch.float32, device="cuda")
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


def reference_cpu(wl, sample_walkers=None, steps=1, threads=None):
    """The reference's own classes (oracle/_ref/ref_harness, built from the reference sources) timed on
    this host: propagation of `sample_walkers` walkers for `steps` steps, energy excluded (the
    reference's H*Psi_T MPS does not fit at L=64, D_T=64)."""
    from oracle import pyoracle as po
    if not po.harness_available():
        return None
    threads = threads or os.cpu_count()
    sample_walkers = sample_walkers or threads
    with tempfile.TemporaryDirectory() as t:
        path = os.path.join(t, "trial.mps")
        po.write_mps(path, po.MPS(wl.trial.dims, wl.trial.data))
        out = po.run_harness("propagate", path, wl.DW, sample_walkers, wl.dtau, steps,
                             env_extra={"OMP_NUM_THREADS": str(threads)})
    r = json.loads(out.strip().splitlines()[-1])
    r["sample"] = (f"{sample_walkers} walkers x {steps} step(s) of {wl.name}, propagation only "
                   f"(reference classes, per-coupling trial terms, no energy)")
    r["cores"] = threads
    return r


def lattice_engine(wl, device):
    """Engine for a 2D lattice workload.  Walkers start as copies of the trial compressed
    (CompressState + setOverlap, as SetupWalkers does): on the device to uneven targets in one
    population when D_T is among them, else one walker compressed on the host and replicated
    (slots of the D_W layout)."""
    from mpsqmc_b200 import Engine
    from mpsqmc_b200 import problem as pb
    ci, cj, cJ = wl.couplings()
    trial = wl.trial()
    U, S, VT = pb.trotter_tables(1.0, wl.dtau)
    common = dict(L=wl.L, ci=ci, cj=cj, cJ=cJ, h=0.0, dtau=wl.dtau, trial_dims=trial.dims, trial=trial.data,
                  Jvals=[1.0], U=U, S=S, VT=VT, grid=pb.grid_marsaglia(4, 4), Ndesired=wl.Nw, device=device)
    N = wl.Nw
    if max(wl.Ds) >= wl.DT:
        eng = Engine(capacity=max(1000, 3 * N), walker_dims=trial.dims, **common)
        eng.set_walkers(np.tile(trial.data, (N, 1)), np.ones(N), normalize=False)
        eng.compress_walkers(wl.targets(), normalize=True)
        dims = trial.dims
    else:
        # one walker compressed on the host (the engine's slots hold walkers up to D = 128)
        w = pb.compress(trial, max(wl.Ds))
        dims, w0 = w.dims, w.data
        eng = Engine(capacity=max(1000, 3 * N), walker_dims=dims, **common)
        eng.set_walkers(np.tile(w0, (N, 1)), np.ones(N), normalize=True)
    inputs = dict(common, walker_dims=dims)
    return eng, inputs


def main():
    args = parse()
    rank, world, local, pg = dist_setup(args.gpus)
    from mpsqmc_b200 import workloads

    lattice = args.workload != "chain64"
    if lattice:
        wl = getattr(workloads, args.workload)(Nw=args.walkers) if args.walkers else getattr(workloads, args.workload)()
        cfg = {"workload": f"{wl.name}: {wl.W}x{wl.H} open Heisenberg lattice on the snake path (L={wl.L}, "
                           f"{len(wl.couplings()[0])} couplings), D_T={wl.DT}, D_W in {wl.Ds}, {wl.Nw} walkers/GPU, "
                           f"dtau={wl.dtau}, Marsaglia(4) grid, FP64; "
                           + (f"trial: DMRG ground state at D_T={wl.DT} (E={wl.trial_energy():.10f})"
                              if wl.trial_file else "seeded random left-normalised trial of the D_T shape")
                           + ", walkers = trial compressed on the device",
               "walkers_per_gpu": wl.Nw, "L": wl.L, "D_T": wl.DT, "D_W": wl.Ds, "dtau": wl.dtau,
               "parallelism": f"{'split walk' if args.sharded else 'replicas'} x{world}", "sweep": args.sweep,
               "workspace": args.workspace, "precision": args.precision, "proposal": args.proposal,
               "proposal_mix": args.proposal_mix if args.proposal_mix is not None else 100,
               "canonical_interval": args.canon if args.canon is not None else 16}
    else:
        wl = workloads.chain64(Nw=args.walkers or 2048)
        cfg = {"workload": f"{wl.name}: L={wl.L} Heisenberg chain, D_T={wl.DT}, D_W={wl.DW}, {wl.Nw} walkers/GPU, "
                           f"dtau={wl.dtau}, Marsaglia(4) grid, FP64",
               "walkers_per_gpu": wl.Nw, "L": wl.L, "D_T": wl.DT, "D_W": wl.DW, "dtau": wl.dtau,
               "l2": f"population ({wl.Nw * wl.walker.data.size * 8 / 1e9:.2f} GB) larger than L2 (126 MB); no flush",
               "parallelism": f"{'split walk' if args.sharded else 'replicas'} x{world}", "sweep": args.sweep,
               "workspace": args.workspace, "precision": args.precision, "proposal": args.proposal,
               "proposal_mix": args.proposal_mix if args.proposal_mix is not None else 100,
               "canonical_interval": args.canon if args.canon is not None else 16}

    if args.impl == "reference":
        if rank != 0:
            return
        if lattice:
            print(json.dumps({"impl": "reference", "unavailable": "the reference classes need nC*16 trial copies "
                              "and H*Psi_T per thread at this size; only chain64 has a CPU arm"}))
            return
        r = reference_cpu(wl, steps=1)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_harness not built"}))
            return
        total_t = 0.0
        ws = 0
        for _ in range(max(1, args.steps)):
            rr = reference_cpu(wl, steps=1)
            total_t += rr["seconds"]
            ws += rr["walker_steps"]
        v = ws / total_t
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
        eng, inputs = lattice_engine(wl, local)
        walkers = None
        N = wl.Nw
        args.no_e2e = True
        args.no_cpu_baseline = True

        def make():
            return lattice_engine(wl, local)[0]
    else:
        inputs = wl.inputs()
        walkers = wl.walkers()
        N = walkers.shape[0]

        def make():
            e = Engine(device=local, **inputs)
            e.set_walkers(walkers, np.ones(N), None, np.zeros(N), normalize=True)
            return e

        eng = make()
    configure(eng, args, sweep)
    eng.set_rng(seed, 0)
    params, training = train_proposal(make, args, sweep, seed)
    use_proposal(eng, params)
    eng.walk(args.warmup)
    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    rw = None
    if args.sharded and pg is not None:
        from mpsqmc_b200.population import RankWalk
        rw = RankWalk(eng, pg, [N] * world, device="cpu")
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

    vn = None
    vn_compare = args.vn_compare
    if rw is not None:
        vn_compare = 0
    if vn_compare is None:
        vn_compare = 300 if (not lattice and args.precision == "fp64" and args.proposal == "grid"
                             and args.walkers is None and args.steps >= 5) else 0
    vn_steps = max(args.vn, vn_compare)
    if vn_steps > 0:
        from mpsqmc_b200 import analysis
        e_ref, e_src = None, None
        if not lattice:
            e_ref = float(np.load(os.path.join(ROOT, "mpsqmc_b200", "data", "trial_L64D64.npz"))["energy"])
            e_src = "DMRG D=64 energy of the trial (mpsqmc_b200/data)"
        elif wl.trial_energy() is not None:
            e_ref = wl.trial_energy()
            e_src = f"DMRG D={wl.DT} energy of the trial (mpsqmc_b200/data; a variational upper bound)"

        def vn_of(e, throughput):
            more = e.walk(vn_steps)
            r = analysis.variance_normalised(throughput, [x["E_P"] for x in more], [x["n_walkers"] for x in more])
            r["throughput_per_gpu"] = throughput
            if e_ref is not None:
                r["E_ref"] = e_ref
                r["E_ref_source"] = e_src
                r["abs_err_per_site"] = abs(r["E_mean"] - e_ref) / wl.L
            return r

        def arm(precision, proposal):
            """A variant from the same start and random stream: set-up (training for the learned
            proposal), warm-up, timed steps for its throughput, then the VN steps."""
            a = argparse.Namespace(**vars(args))
            a.precision, a.proposal = precision, proposal
            e = make()
            configure(e, a, sweep, plain=(precision == "fp64"))
            e.set_rng(seed, 0)
            p_arm, tr = train_proposal(make, a, sweep, seed)
            use_proposal(e, p_arm)
            e.walk(args.warmup)
            st = e.walk(args.steps)
            t = e.last_timing()
            thr = sum(x["n_walkers"] for x in st) / (t["total_ms"] * 1e-3)
            r = vn_of(e, thr)
            if tr:
                r["proposal_training"] = tr
            e.close()
            return r

        this = vn_of(eng, value / max(world, 1))
        this["arm"] = f"{args.precision}/{args.proposal}"
        vn = this
        if vn_compare > 0:
            plain = this if (args.precision, args.proposal) == ("fp64", "grid") else arm("fp64", "grid")
            vn = {"plain_fp64_grid": plain, "vn_ratio_vs_plain_fp64": {}, "throughput_ratio_vs_plain_fp64": {}}
            arms = [this["arm"]] if this is not plain else []
            named = [x if "/" in x else x + "/grid" for x in args.vn_arms.split(",") if x]
            arms += [x for x in named if x not in arms and x != "fp64/grid"]
            for name in arms:
                r = this if name == this["arm"] else arm(*name.split("/"))
                vn[name] = r
                vn["vn_ratio_vs_plain_fp64"][name] = r["vn"] / plain["vn"] if plain["vn"] else None
                vn["throughput_ratio_vs_plain_fp64"][name] = r["throughput_per_gpu"] / plain["throughput_per_gpu"]

    # roofline of the dominant kernel (the walker-step kernel): canonical FP64 work / kernel time,
    # averaged over the walkers' own bond dims
    cpl = list(zip(inputs["ci"], inputs["cj"]))
    dims_now = eng.get_walker_dims()
    rows, counts = np.unique(dims_now, axis=0, return_counts=True)
    flops_ws = float(sum(c * workloads.algorithmic_flops_per_walker_step(inputs["trial_dims"], r, cpl)
                         for r, c in zip(rows, counts)) / counts.sum())
    achieved = flops_ws * ws_done / (k_ms * 1e-3) / 1e12
    mixed = args.precision != "fp64"
    peak = (tf32_peak_tflops() if mixed else fp64_peak_tflops()) if rank == 0 else None

    # end to end through the public API: host population -> device, K steps (stats read back each
    # step), population -> host; host wall clock.
    e2e = None
    if not args.no_e2e:
        eng2 = Engine(device=local, **inputs)
        configure(eng2, args, sweep)
        use_proposal(eng2, params)  # the trained network, as the timed engine walks with it
        # the population in pinned host memory (both directions), as a serving caller would keep it
        host_w = torch.empty(walkers.shape, dtype=torch.float64, pin_memory=True).numpy()
        host_w[:] = walkers
        back_w = torch.empty((eng2.capacity, eng2.walker_size), dtype=torch.float64, pin_memory=True).numpy()
        # untimed warm-up on this engine, as for the device-timed steps (step graphs captured, kernels
        # loaded); the timed run then starts again from the host population
        eng2.set_walkers(host_w, np.ones(N), None, np.zeros(N), normalize=True)
        eng2.set_rng(wl.seed + 7919 * rank, 0)
        eng2.walk(args.warmup)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eng2.set_walkers(host_w, np.ones(N), None, np.zeros(N), normalize=True)
        eng2.set_rng(wl.seed + 7919 * rank, 0)
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
        r = reference_cpu(wl, steps=1)
        if r is not None:
            cpu = {"value": r["walker_steps_per_s"], "unit": "walker-steps/s", "cores": r["cores"],
                   "kind": "reference", "sample": r["sample"]}

    if rank == 0:
        prof_traffic = None
        kname = "walker_step_kernel" if args.sweep == "nearest" else (
            "walker_step_mixed_kernel" if mixed else "walker_step_general_kernel")
        tp = os.path.join(ROOT, "profiles", f"{kname}_traffic.json")
        if os.path.exists(tp) and not lattice and N == 2048:
            prof_traffic = json.load(open(tp)).get("bytes_per_launch")
        line = {
            "metric": METRIC, "value": value, "unit": "walker-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if not mixed else f"{args.precision}+f64", "data": "synthetic",
            "config": cfg,
            "energy": {"E_P_last": stats[-1]["E_P"], "E_T_last": stats[-1]["E_T"], "walkers_last": stats[-1]["n_after"]},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if peak else None, "traffic": prof_traffic,
                         "kernel": kname, "flops_per_walker_step": flops_ws,
                         "peak_source": ("cuBLAS TF32 GEMM 8192^3 measured in this run (TF32 tensor path; the "
                                         "canonical flops count each product once)") if mixed else
                                        "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor path)"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": tim["launches"],
            **({"variance_normalised": vn} if vn is not None else {}),
            **({"proposal_training": training} if training else {}),
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    eng.close()
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
