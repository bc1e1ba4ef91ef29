"""CUDA engine against the CPU oracle at bond dimensions whose matrix work buffers exceed one
CTA's shared memory (they then live in global scratch): a chain and a 2D snake lattice with
D_T = D_W = 64.  Same trial, walkers, tables, grid and random stream on both sides; FP64
tolerance 1e-10 relative on weights, overlaps and local energies, bit-exact parents."""
import numpy as np
import pytest

from mpsqmc_b200 import Engine
from mpsqmc_b200 import problem as pb
from mpsqmc_b200.capi import OPT_WORKSPACE, WORKSPACE_GLOBAL
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def random_trial(L, D, rng):
    dims = po.virtual_dims(L, D)
    m = po.MPS(dims, rng.normal(size=po.mps_size(dims)))
    return po.left_normalize(m)[0]


@pytest.mark.parametrize("lattice", ["chain:12", "snake:3x4"])
def test_large_bond_walk_matches_oracle(lattice):
    rng = np.random.default_rng(7)
    ci, cj, cJ = pb.lattice(lattice)
    L = int(max(cj)) + 1
    D, N, steps, dtau, seed = 64, 4, 2, 0.05, 12345
    trial = random_trial(L, D, rng)
    walkers = trial.data[None, :] + 0.05 * rng.normal(size=(N, trial.data.size))
    U, S, VT = pb.trotter_tables(1.0, dtau)
    grid = pb.grid_marsaglia(4, 4)
    eng = Engine(L=L, ci=ci, cj=cj, cJ=cJ, h=0.0, dtau=dtau, trial_dims=trial.dims, trial=trial.data, Jvals=[1.0],
                 U=U, S=S, VT=VT, grid=grid, Ndesired=N, capacity=64, walker_dims=trial.dims)
    assert eng.get_option(OPT_WORKSPACE) == WORKSPACE_GLOBAL  # chosen automatically at this size
    eng.set_walkers(walkers, np.ones(N), None, np.zeros(N), normalize=True)
    eng.set_rng(seed, 0)
    res = po.walk(trial, walkers, trial.dims, np.ones(N), np.ones(N), np.zeros(N), ci=ci, cj=cj, cJ=cJ,
                  Jvals=np.array([1.0]), U=U, S=S, VT=VT, grid=grid, dtau=dtau, nsteps=steps, Ndesired=N,
                  capacity=64, seed=seed, skip=0)
    assert res.status == 0
    for s in range(steps):
        st = eng.walk(1)[0]
        lw = eng.last_step_walkers()
        n = res.n[s]
        assert st["n_walkers"] == n
        assert st["E_P"] == pytest.approx(res.EP[s], rel=RTOL)
        np.testing.assert_allclose(lw["weight"], res.weight[s, :n], rtol=RTOL)
        np.testing.assert_allclose(lw["overlap"], res.overlap[s, :n], rtol=RTOL)
        np.testing.assert_allclose(lw["energy"], res.energy[s, :n], rtol=RTOL)
        np.testing.assert_array_equal(lw["parent"], res.parent[s, :len(lw["parent"])])
