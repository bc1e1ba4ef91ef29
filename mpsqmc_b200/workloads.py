"""Named walker-propagation workloads (the run configurations the bench and tests use).

chain64   L=64 open Heisenberg chain, J=1, h=0, D_T=64 trial (compact-MPO DMRG, E=-28.1754248083),
          walkers = trial compressed to D_W=32 plus i.i.d. N(0, 1e-3) noise per element, dtau=0.01,
          2048 walkers, Marsaglia(4) grid (240 points).
chain16   L=16 chain, D_T=D_W=16 trial from the reference's DMRG, 128 walkers, dtau=0.01.
snake6x6  open 6x6 lattice on the snake path with a seeded random trial of the D_T = 128 bond
          profile (throughput: the work per walker-step does not depend on the trial).
snake8x8  the open 8x8 lattice with its D_T = 256 DMRG ground-state trial (made on the GPU),
          D_W = 64, 4096 walkers, dtau = 0.005; snake8x8_random the same shapes with a random trial.
snake6x6_dmrg   the open 6x6 lattice with its ground-state trial from the compact-MPO DMRG at
          D_T = 64 (mpsqmc_b200/data, made by data/make_trials.py), walkers of D_W in {16, 32, 64}.
snake8x8_dmrg   the open 8x8 lattice with its DMRG ground-state trial at D_T = 64, walkers of D_W
          in {32, 64}.
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


def mpo_nnz(L, couplings, h=0.0):
    """Nonzero operator entries of each site's compact MPO for H = sum J S_i.S_j - h sum S^z:
    done -> done, identity -> identity, the field, 3 per coupling closed on the site, 3 per
    channel carried through it and 3 for the channel it opens.  8 per bulk site of the
    nearest-neighbour chain."""
    last = {}
    for (i, j) in couplings:
        last[i] = max(last.get(i, -1), j)
    nnz = []
    for k in range(L):
        n = (1 if k > 0 else 0) + (1 if k < L - 1 else 0) + (1 if h != 0.0 else 0)
        for i, lj in last.items():
            if i < k <= lj:
                if (i, k) in couplings:
                    n += 3
                if lj > k:
                    n += 3
        if last.get(k, -1) > k:
            n += 3
        nnz.append(n)
    return nnz


def algorithmic_flops_per_walker_step(aT, bW, couplings, d=2, h=0.0):
    """Algorithmic FP work of one walker-step (canonical count): per coupling (i, j), g = j - i:
    (5g + 4 + r_c) T_i, with r_c the right environments an earlier coupling of the step invalidated
    (sites beyond j changed since they were built); 16 closures of 2 a b; QR of the two touched
    walker sites (4 m n^2 - 4/3 n^3 + 2 d n^3, m = d b_l, n = b_r); per step L T for the
    right-environment sweep and sum_k nnz(W_k) T_k for the local energy."""
    aT, bW = list(aT), list(bW)
    L = len(aT) - 1
    T = [site_flops(aT[k], aT[k + 1], bW[k], bW[k + 1], d) for k in range(L)]

    def qr(k):
        m, n = d * bW[k], bW[k + 1]
        return 4 * m * n * n - (4.0 / 3.0) * n ** 3 + 2 * d * n ** 3

    couplings = [tuple(int(x) for x in c) for c in couplings]
    f = 0.0
    valid_from = 1  # right environments R[k], k >= valid_from, describe the current walker
    for (i, j) in couplings:
        g = j - i
        r_c = max(0, valid_from - (j + 1))
        f += (5 * g + 4 + r_c) * T[i]
        f += 16 * 2 * aT[i + 1] * bW[i + 1]
        f += qr(i) + qr(j)
        valid_from = j + 1
    f += sum(T)
    cs = set(couplings)
    for k, n in enumerate(mpo_nnz(L, cs, h)):
        f += n * T[k]
    return f


@dataclass
class LatticeWorkload:
    """A 2D open W x H Heisenberg lattice on the snake path with a D_T trial and walkers made on
    the device by CompressState to per-walker bond dimensions (the 2D configurations)."""
    name: str
    W: int
    H: int
    DT: int
    Ds: list
    Nw: int
    dtau: float
    seed: int = 20131015
    trial_file: str | None = None  # a DMRG trial in mpsqmc_b200/data (else a random one)

    @property
    def L(self):
        return self.W * self.H

    def has_trial(self):
        """False when the workload names a stored trial that is not present."""
        return not self.trial_file or os.path.exists(os.path.join(DATA, self.trial_file))

    def trial_energy(self):
        """The DMRG energy of the stored trial (a variational upper bound), or None."""
        if not self.trial_file:
            return None
        return float(np.load(os.path.join(DATA, self.trial_file))["energy"])

    def couplings(self):
        return pb.snake(self.W, self.H)

    def targets(self):
        rng = np.random.default_rng(self.seed + 1)
        return rng.choice(np.asarray(self.Ds, dtype=np.int32), size=self.Nw)

    def trial(self):
        if self.trial_file:
            z = np.load(os.path.join(DATA, self.trial_file))
            m = pb.MPS(z["dims"].astype(np.int32), z["data"].astype(np.float64))
            # trials stored in FP32 (26 MB instead of 52 MB at D_T = 256) are left-normalised
            # again in FP64; their energy is stored for that FP64 state
            return pb.left_normalize(m) if z["data"].dtype == np.float32 else m
        rng = np.random.default_rng(self.seed)
        dims = pb.virtual_dims(self.L, self.DT)
        data = rng.normal(size=int(sum(dims[k] * dims[k + 1] * 2 for k in range(self.L))))
        return pb.left_normalize(pb.MPS(dims, data))


def snake6x6(Nw: int = 1024) -> LatticeWorkload:
    """6x6 open lattice, D_T = 128, walkers of D_W drawn uniformly from {16, 32, 64, 128}, dtau 0.005."""
    return LatticeWorkload("snake6x6", 6, 6, 128, [16, 32, 64, 128], Nw, 0.005)


def snake6x6_dmrg(Nw: int = 1024) -> LatticeWorkload:
    """6x6 open lattice with its DMRG ground-state trial (D_T = 64), walkers of D_W drawn from
    {16, 32, 64}, dtau 0.005."""
    return LatticeWorkload("snake6x6_dmrg", 6, 6, 64, [16, 32, 64], Nw, 0.005, trial_file="trial_snake6x6_D64.npz")


def snake8x8_dmrg(Nw: int = 1024) -> LatticeWorkload:
    """8x8 open lattice with its DMRG ground-state trial (D_T = 64), walkers of D_W drawn from
    {32, 64}, dtau 0.005."""
    return LatticeWorkload("snake8x8_dmrg", 8, 8, 64, [32, 64], Nw, 0.005, trial_file="trial_snake8x8_D64.npz")


def snake8x8(Nw: int = 4096) -> LatticeWorkload:
    """The full chosen configuration: 8x8 open lattice, D_T = 256 DMRG ground-state trial (made on
    the GPU, data/make_trials.py snake8x8_256), D_W = 64, 4096 walkers, dtau 0.005."""
    return LatticeWorkload("snake8x8", 8, 8, 256, [64], Nw, 0.005, trial_file="trial_snake8x8_D256.npz")


def snake8x8_random(Nw: int = 4096) -> LatticeWorkload:
    """The 8x8 shapes (D_T = 256, D_W = 64) with a seeded random left-normalised trial."""
    return LatticeWorkload("snake8x8_random", 8, 8, 256, [64], Nw, 0.005)
