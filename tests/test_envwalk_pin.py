"""Pin the environment-based oracle step (oracle/envwalk.py) before the large-shape GPU parity
tests trust it: against the reference's own first-step values (tests/golden walk_* fixtures,
written by the reference harness) and against liboracle's literal restatement (16 full-chain
InnerProducts per coupling) on random states with uneven bond dimensions and a field."""
import numpy as np
import pytest

from conftest import WALK_CASES, couplings, load_golden
from mpsqmc_b200 import problem as pb
from oracle import envwalk as ew
from oracle import pyoracle as po

RTOL = 1e-10


def test_mt19937_known_answer():
    g = ew.MT19937(5489)
    for _ in range(9999):
        g.next_u32()
    assert g.next_u32() == 4123659995  # the C++ standard's required 10000th output


@pytest.mark.parametrize("case", WALK_CASES)
def test_envwalk_first_step_matches_reference(case):
    z = load_golden(case)
    meta = z["meta"]
    N, nC = meta["Nw"], meta["nCouplings"]
    ci, cj, cJ = couplings(z)
    h = meta.get("h", 0.0)
    for w in range(N):
        u = z["step001_trace_u"][w * nC:(w + 1) * nC]
        r = ew.step(z["trial_ln_dims"], z["trial_ln_data"], z["walker0_init_dims"], z["walker0_init_data"],
                    z["init_weight"][w], ci=ci, cj=cj, cJ=cJ, Jvals=[1.0], U=z["U"], S=z["S"], VT=z["VT"],
                    grid=z["grid"], dtau=meta["dtau"], u=u, h=h)
        np.testing.assert_array_equal(r["index"], z["step001_trace_index"][w * nC:(w + 1) * nC].astype(int))
        assert r["weight"] == pytest.approx(z["step001_weight"][w], rel=RTOL)
        assert r["overlap"] == pytest.approx(z["step001_overlap"][w], rel=RTOL)
        assert r["energy"] == pytest.approx(z["step001_energy"][w], rel=RTOL)


@pytest.mark.parametrize("lattice,D,h", [("chain:10", 8, 0.0), ("snake:3x3", 8, 0.4), ("snake:3x4", 12, 0.0)])
def test_envwalk_matches_literal_oracle_on_uneven_walkers(lattice, D, h):
    rng = np.random.default_rng(5)
    ci, cj, cJ = pb.lattice(lattice)
    L = int(max(cj)) + 1
    dims = po.virtual_dims(L, D)
    trial = po.left_normalize(po.MPS(dims, rng.normal(size=po.mps_size(dims))))[0]
    dtau, seed = 0.2, 4242
    U, S, VT = pb.trotter_tables(1.0, dtau)
    grid = pb.grid_marsaglia(4, 4)
    Ds = [2, 4, D]
    wdims, rows, raw = [], np.zeros((len(Ds), po.mps_size(dims))), []
    for w, Dw in enumerate(Ds):
        m = pb.compress(pb.MPS(trial.dims, trial.data), Dw)
        data = m.data + 0.05 * rng.normal(size=m.data.size)
        wdims.append(np.asarray(m.dims, np.int32))
        rows[w, :data.size] = data
        raw.append(data)
    wdims = np.stack(wdims)
    N = len(Ds)
    res = po.walk(trial, rows, trial.dims, np.ones(N), np.ones(N), np.zeros(N), ci=ci, cj=cj, cJ=cJ,
                  Jvals=np.array([1.0]), U=U, S=S, VT=VT, grid=grid, dtau=dtau, nsteps=1, Ndesired=N,
                  capacity=16, seed=seed, skip=0, h=h, wdims=wdims, popctl_interval=1000)
    assert res.status == 0
    nC = len(ci)
    uni = ew.uniforms(seed, 0, N * nC)
    for w in range(N):
        # the reference normalises the walker before the step (setOverlap)
        m = po.left_normalize(po.MPS(wdims[w], raw[w].copy()))[0]
        if po.inner_product(trial, m) < 0:
            m = po.change_phase(m)
        r = ew.step(trial.dims, trial.data, wdims[w], m.data, 1.0, ci=ci, cj=cj, cJ=cJ, Jvals=[1.0], U=U, S=S,
                    VT=VT, grid=grid, dtau=dtau, u=uni[w * nC:(w + 1) * nC], h=h)
        assert r["weight"] == pytest.approx(res.weight[0, w], rel=RTOL)
        assert r["overlap"] == pytest.approx(res.overlap[0, w], rel=RTOL)
        assert r["energy"] == pytest.approx(res.energy[0, w], rel=RTOL)
