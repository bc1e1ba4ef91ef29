"""Walks split over ranks: one engine per rank and GPU, global population control and walker
balancing, over torch.distributed (NCCL between GPUs; gloo works for host-only tests).

This is the reference's MPI path through MPSQMC2::Walk (MPSQMC2.cpp:465-511 with
USE_MPI_IN_MPSQMC):
  1. every rank propagates its walkers (mpsqmc_step_propagate);
  2. the five per-rank sums are summed over the ranks (MPSQMC2.cpp:475, 716-731: Allreduce);
  3. every rank runs its population control with the global scaling (mpsqmc_step_control);
  4. MPSQMC2::PopulationBalancing (MPSQMC2.cpp:778-934) moves walkers from ranks above their
     share of the population to ranks below it: `balance_plan` restates its rounds, and the
     walkers travel as records (mpsqmc_export_walkers / mpsqmc_import_walkers) by
     point-to-point sends.
"""
from __future__ import annotations

import numpy as np

THRESHOLD_START = 0.1   # MPSQMC2.cpp:782: rebalance when a rank deviates by more than 10%
THRESHOLD_STOP = 0.03   # MPSQMC2.cpp:783: until every rank is within 3%


def _order_desc(values):
    """Indices by descending value; equal values keep their rank order (the reference's bubble
    sort swaps only on strict <, MPSQMC2.cpp:760-776)."""
    return sorted(range(len(values)), key=lambda k: (-values[k], k))


def balance_plan(counts, desired, start=THRESHOLD_START, stop=THRESHOLD_STOP, max_rounds=64):
    """Transfer rounds of MPSQMC2::PopulationBalancing (MPSQMC2.cpp:778-934).

    counts: walkers per rank now; desired: NDesiredWalkersPerRank.  Each rank's target is its
    desired count scaled by (total current / total desired); its offset is counts - target.  If any
    rank deviates by more than `start` (relative to its target), rounds run until all are within
    `stop`: ranks sorted by offset, the k-th largest surplus sends int(min(surplus, -deficit))
    walkers to the k-th largest deficit, for k < size/2.  Returns a list of rounds, each a list of
    (sender, receiver, amount)."""
    counts = [int(x) for x in counts]
    desired = [float(x) for x in desired]
    size = len(counts)
    frac_scaling = sum(counts) / sum(desired)
    target = [d * frac_scaling for d in desired]

    def offsets():
        return [counts[r] - target[r] for r in range(size)]

    off = offsets()
    if not any(abs(off[r]) / target[r] > start for r in range(size) if target[r] > 0):
        return []
    rounds = []
    while len(rounds) < max_rounds:
        order = _order_desc(off)
        moves = []
        for k in range(size // 2):
            snd, rcv = order[k], order[size - 1 - k]
            if off[snd] > 0.0 and off[rcv] < 0.0:
                amount = int(min(off[snd], -off[rcv]))
                if amount > 0:
                    moves.append((snd, rcv, amount))
                    counts[snd] -= amount
                    counts[rcv] += amount
        rounds.append(moves)
        off = offsets()
        if not any(abs(off[r]) / target[r] > stop for r in range(size) if target[r] > 0) or not moves:
            break
    return rounds


class RankWalk:
    """One rank's share of a walk split over ranks.

    engine: this rank's engine (mpsqmc_b200.Engine, or any object with step_propagate,
    step_control, record_size, export_walkers, import_walkers and n_walkers); dist: a
    torch.distributed module with an initialised process group; desired: walkers wanted per rank.
    Record buffers live on `device`: a CUDA device for NCCL, or "cpu" for gloo, in which case they
    are pinned when CUDA is present (the engine's kernels write and read them in place)."""

    def __init__(self, engine, dist, desired, device):
        import torch
        self.torch, self.engine, self.dist = torch, engine, dist
        self.rank, self.size = dist.get_rank(), dist.get_world_size()
        self.desired = [int(x) for x in desired]
        self.device = device
        self.pin = str(device) == "cpu" and torch.cuda.is_available()
        self.rec = engine.record_size()

    def _allreduce(self, v):
        t = self.torch.tensor(np.asarray(v, dtype=np.float64), device=self.device)
        self.dist.all_reduce(t)
        return t.cpu().numpy()

    def step(self):
        """One step on every rank: propagation, the global sums, population control, balancing.
        Returns this rank's statistics (global E_P, E_T, scaling, fluctuation metric) and the
        balancing rounds that ran."""
        local = self.engine.step_propagate()
        total = self._allreduce(local)
        stats = self.engine.step_control(total, sum(self.desired))
        rounds = self.balance()
        stats["rounds"] = rounds
        return stats

    def balance(self):
        counts = self._allreduce([self.engine.n_walkers if r == self.rank else 0 for r in range(self.size)])
        rounds = balance_plan([int(round(x)) for x in counts], self.desired)
        torch = self.torch
        for moves in rounds:
            for snd, rcv, amount in moves:
                if self.rank == snd:
                    buf = torch.empty(amount * self.rec, dtype=torch.float64, device=self.device, pin_memory=self.pin)
                    self.engine.export_walkers(amount, buf.data_ptr())
                    self.dist.send(buf, dst=rcv)
                elif self.rank == rcv:
                    buf = torch.empty(amount * self.rec, dtype=torch.float64, device=self.device, pin_memory=self.pin)
                    self.dist.recv(buf, src=snd)
                    if buf.is_cuda:  # the engine reads the buffer on its own stream
                        torch.cuda.current_stream().synchronize()
                    self.engine.import_walkers(amount, buf.data_ptr())
            self.dist.barrier()
        return rounds
