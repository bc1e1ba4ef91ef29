"""Named walker-propagation workloads (the run configurations the bench and tests use).

chain64   L=64 open Heisenberg chain, J=1, h=0, D_T=64 trial (compact-MPO DMRG, E=-28.1754248083),
          walkers = trial compressed to D_W=32 plus i.i.d. N(0, 1e-3) noise per element, dtau=0.01,
          2048 walkers, Marsaglia(4) grid (240 points).
chain16   L=16 chain, D_T=D_W=16 trial from the reference's DMRG, 128 walkers, dtau=0.01.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

from . import problem as pb

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


@dataclass
class Workload:
    name: str
    L: int
    DT: int
    DW: int
    Nw: int
    dtau: float
    trial: pb.MPS
    walker: pb.MPS              # the walker every copy starts from (before noise)
    noise: float = 0.0
    seed: int = 20131015
    J: float = 1.0
    h: float = 0.0
    extra: dict = field(default_factory=dict)

    def inputs(self):
        ci, cj, cJ = pb.chain(self.L, self.J)
        U, S, VT = pb.trotter_tables(self.J, self.dtau)
        return dict(L=self.L, ci=ci, cj=cj, cJ=cJ, h=self.h, dtau=self.dtau, trial_dims=self.trial.dims,
                    trial=self.trial.data, Jvals=[self.J], U=U, S=S, VT=VT, grid=pb.grid_marsaglia(4, 4),
                    Ndesired=self.Nw, capacity=max(1000, 3 * self.Nw), walker_dims=self.walker.dims)

    def walkers(self, n=None):
        n = self.Nw if n is None else n
        rng = np.random.default_rng(self.seed)
        base = self.walker.data
        w = np.tile(base, (n, 1))
        if self.noise > 0:
            w = w + rng.normal(0.0, self.noise, size=w.shape)
        return w


def load_trial_L64D64() -> pb.MPS:
    z = np.load(os.path.join(DATA, "trial_L64D64.npz"))
    return pb.MPS(z["dims"].astype(np.int32), z["data"])


def chain64(Nw: int = 2048, DW: int = 32) -> Workload:
    trial = load_trial_L64D64()
    walker = pb.compress(trial, DW)
    return Workload("chain64", 64, 64, DW, Nw, 0.01, trial, walker, noise=1e-3)


def chain16(trial: pb.MPS, Nw: int = 128) -> Workload:
    return Workload("chain16", 16, 16, 16, Nw, 0.01, trial, trial.copy())


def site_flops(a_l, a_r, b_l, b_r, d=2):
    """Canonical transfer-step cost T = 2d min(b_l a_r (a_l + b_r), a_l b_r (b_l + a_r))."""
    return 2 * d * min(b_l * a_r * (a_l + b_r), a_l * b_r * (b_l + a_r))


def algorithmic_flops_per_walker_step(aT, bW, couplings, d=2, mpo_nnz_bulk=8):
    """Algorithmic FP work of one walker-step of the nearest-neighbour walk (canonical count):
    per coupling (i, j), g = j - i: (5g + 4 + r_c) T_i + 16 closures of 2 a b + QR of the two
    touched walker sites (4 m n^2 - 4/3 n^3 + 2 d n^3, m = d b_l, n = b_r); per step L T for the
    right-environment sweep and sum_k nnz(W_k) T_k for the local energy."""
    aT, bW = list(aT), list(bW)
    L = len(aT) - 1
    T = [site_flops(aT[k], aT[k + 1], bW[k], bW[k + 1], d) for k in range(L)]

    def qr(k):
        m, n = d * bW[k], bW[k + 1]
        return 4 * m * n * n - (4.0 / 3.0) * n ** 3 + 2 * d * n ** 3

    f = 0.0
    for (i, j) in couplings:
        g = j - i
        f += (5 * g + 4) * T[i]
        f += 16 * 2 * aT[i + 1] * bW[i + 1]
        f += qr(i) + qr(j)
    f += sum(T)
    for k in range(L):
        nnz = mpo_nnz_bulk if 0 < k < L - 1 else 4
        f += nnz * T[k]
    return f
