"""Walkers of uneven bond dimension in one population (the reference's MPSstate keeps per-walker
VirtualD): the CUDA engine against the CPU oracle, on a chain and a 2D snake lattice, with
branching (copies keep their parent's dims).  FP64 tolerance 1e-10 relative; parents and dims
bit-exact."""
import numpy as np
import pytest

from conftest import load_golden
from mpsqmc_b200 import Engine
from mpsqmc_b200 import problem as pb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def population(trial, Ds, N, rng, noise=1e-2):
    dims, data = [], []
    for w in range(N):
        m = pb.compress(pb.MPS(trial.dims, trial.data), Ds[w % len(Ds)])
        dims.append(np.asarray(m.dims, np.int32))
        data.append(m.data + noise * rng.normal(size=m.data.size))
    return np.stack(dims), data


@pytest.mark.parametrize("case", ["chain", "snake"])
def test_uneven_population_matches_oracle(case):
    rng = np.random.default_rng(3)
    if case == "chain":
        z = load_golden("trials")
        trial = po.MPS(z["L10D8_dims"], z["L10D8_data"])
        ci, cj, cJ = pb.chain(10)
        Ds, N, steps, dtau = [2, 4, 8], 12, 6, 0.3
    else:
        z = load_golden("trials2d")
        trial = po.MPS(z["snake4x4D16_dims"], z["snake4x4D16_data"])
        ci, cj, cJ = pb.snake(4, 4)
        Ds, N, steps, dtau = [4, 8, 16], 9, 4, 0.2
    trial = po.left_normalize(trial)[0]
    dims, data = population(trial, Ds, N, rng)
    U, S, VT = pb.trotter_tables(1.0, dtau)
    grid = pb.grid_marsaglia(4, 4)
    L = trial.L
    eng = Engine(L=L, ci=ci, cj=cj, cJ=cJ, h=0.0, dtau=dtau, trial_dims=trial.dims, trial=trial.data, Jvals=[1.0],
                 U=U, S=S, VT=VT, grid=grid, Ndesired=N, capacity=256, walker_dims=trial.dims)
    eng.set_walkers_dims(dims, data, np.ones(N), normalize=True)
    np.testing.assert_array_equal(eng.get_walker_dims(), dims)
    eng.set_rng(99, 0)
    size = po.mps_size(trial.dims)
    rows = np.zeros((N, size))
    for w in range(N):
        rows[w, :data[w].size] = data[w]
    res = po.walk(trial, rows, trial.dims, np.ones(N), np.ones(N), np.zeros(N), ci=ci, cj=cj, cJ=cJ,
                  Jvals=np.array([1.0]), U=U, S=S, VT=VT, grid=grid, dtau=dtau, nsteps=steps, Ndesired=N,
                  capacity=256, seed=99, skip=0, wdims=dims)
    assert res.status == 0
    branched = False
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
        branched |= not np.array_equal(lw["parent"], np.arange(n))
    assert branched  # the case exercises copies of uneven walkers
    np.testing.assert_array_equal(eng.get_walker_dims(), res.wdims)
    w, wt, ov, eh = eng.get_walkers()
    np.testing.assert_allclose(wt, res.weights, rtol=RTOL)
    for k in range(w.shape[0]):  # same states (the engine's gauge differs)
        d = res.wdims[k]
        n = po.mps_size(d)
        A, B = po.MPS(d, w[k, :n]), po.MPS(d, res.walkers[k, :n])
        f = po.inner_product(A, B) / np.sqrt(po.inner_product(A, A) * po.inner_product(B, B))
        assert f == pytest.approx(1.0, abs=1e-12)
