"""Walks split over ranks, host side: the balancing plan of MPSQMC2::PopulationBalancing and the
per-step protocol (sums over ranks, population control, walker transfers) on gloo ranks with a
host-only stand-in for the engine."""
import ctypes
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT
from mpsqmc_b200.population import balance_plan


def test_no_plan_within_ten_percent():
    assert balance_plan([105, 96, 99], [100, 100, 100]) == []


def test_two_ranks_even_out():
    assert balance_plan([150, 50], [100, 100]) == [[(0, 1, 50)]]


def test_pairs_largest_surplus_with_largest_deficit():
    # offsets +30, -30, +10, -10 from a target of 100: (0 -> 1, 30) and (2 -> 3, 10) in one round
    assert balance_plan([130, 70, 110, 90], [100] * 4) == [[(0, 1, 30), (2, 3, 10)]]


def test_uneven_desired_shares_and_conservation():
    counts, desired = [300, 20, 90, 190], [100, 50, 150, 100]
    rounds = balance_plan(counts, desired)
    assert rounds
    c = list(counts)
    for moves in rounds:
        for s, r, a in moves:
            assert a > 0 and c[s] - a >= 0
            c[s] -= a
            c[r] += a
    assert sum(c) == sum(counts)
    scale = sum(counts) / sum(desired)
    # within the stop threshold, up to the integer truncation of each move
    assert all(abs(c[k] - desired[k] * scale) <= max(0.03 * desired[k] * scale, 1.0) + len(rounds) for k in range(4))


class FakeEngine:
    """Host stand-in with the engine's split-walk interface: walkers are rows of records whose
    first entries are weight, overlap, energy history, then an id; energies are fixed per id."""

    REC = 8

    def __init__(self, rank, n, seed):
        rng = np.random.default_rng(seed)
        self.w = np.zeros((n, self.REC))
        self.w[:, 0] = rng.uniform(0.5, 1.5, n)
        self.w[:, 1] = 1.0
        self.w[:, 3] = 1000 * rank + np.arange(n)
        self.step_no = 0

    def energy(self, rows):
        return -1.0 - 1e-3 * (rows[:, 3] % 17)

    @property
    def n_walkers(self):
        return self.w.shape[0]

    def record_size(self):
        return self.REC

    def step_propagate(self):
        self.step_no += 1
        e = self.energy(self.w)
        self.w[:, 2] += e
        eh = self.w[:, 2] / self.step_no
        return np.array([self.w[:, 0].sum(), (self.w[:, 0] * e).sum(), eh.sum(), (eh * eh).sum(), len(e)])

    def step_control(self, g, ndesired):
        scaling = ndesired / g[0]
        out = dict(E_P=g[1] / g[0], scaling=scaling, n_walkers=self.n_walkers)
        # population control with the global scaling: int(w s + 0.5) copies of weight 1
        s = self.w[:, 0] * scaling
        copies = np.floor(s + 0.5).astype(int)
        self.w = np.repeat(self.w, copies, axis=0)
        self.w[:, 0] = 1.0
        out["n_after"] = self.n_walkers
        return out

    def export_walkers(self, k, ptr):
        buf = np.ctypeslib.as_array((ctypes.c_double * (k * self.REC)).from_address(ptr))
        buf[:] = self.w[-k:].ravel()
        self.w = self.w[:-k]

    def import_walkers(self, k, ptr):
        buf = np.ctypeslib.as_array((ctypes.c_double * (k * self.REC)).from_address(ptr))
        self.w = np.concatenate([self.w, buf.reshape(k, self.REC).copy()])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from datetime import timedelta
    from mpsqmc_b200.population import RankWalk
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    # uneven start: rank 0 holds many walkers of high weight, the others few of low weight
    n = [60, 12, 20][rank]
    eng = FakeEngine(rank, n, seed=rank)
    if rank == 0:
        eng.w[:, 0] *= 2.0
    rw = RankWalk(eng, dist, desired=[40, 40, 40], device="cpu")
    res = []
    for _ in range(3):
        before = eng.w[:, 3].copy()
        st = rw.step()
        res.append(dict(E_P=st["E_P"], scaling=st["scaling"], n=eng.n_walkers, rounds=st["rounds"],
                        ids_after=sorted(eng.w[:, 3].tolist()), ids_before=sorted(before.tolist())))
    out[rank] = res
    dist.barrier()
    dist.destroy_process_group()


def test_three_gloo_ranks_share_statistics_and_balance():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 3, port, out)) for r in range(3)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = [out[r] for r in range(3)]
    for step in range(3):
        eps = [res[r][step]["E_P"] for r in range(3)]
        assert eps[0] == eps[1] == eps[2]                     # one global E_P
        assert len({res[r][step]["scaling"] for r in range(3)}) == 1
        counts = [res[r][step]["n"] for r in range(3)]
        total = sum(counts)
        assert all(abs(c - total / 3) <= 0.03 * total / 3 + 2 for c in counts), counts
    # the first step had to move walkers off rank 0; every walker is on exactly one rank
    assert res[0][0]["rounds"]
    for step in range(3):
        ids = sorted(sum((res[r][step]["ids_after"] for r in range(3)), []))
        assert len(ids) == sum(res[r][step]["n"] for r in range(3))
