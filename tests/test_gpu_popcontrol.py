"""Population-control variants of the engine against the CPU oracle: branching every K steps
(weights only rescaled in between) and comb resampling.  The reference has neither (it branches
every step by threshold), so the oracle's restatement of the reference walk, extended by the same
two rules, is the check.  Same inputs as the reference fixture walk_L10D8_DW2_branch (dtau = 0.3,
16 walkers, 8 steps: strong weight spread)."""
import numpy as np
import pytest

from conftest import couplings, load_golden
from mpsqmc_b200 import Engine
from mpsqmc_b200.capi import OPT_POPCONTROL_INTERVAL, OPT_RESAMPLING, RESAMPLE_COMB, RESAMPLE_THRESHOLD
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

RTOL = 1e-10


@pytest.mark.parametrize("interval,mode", [(1, RESAMPLE_COMB), (3, RESAMPLE_THRESHOLD), (2, RESAMPLE_COMB)])
def test_population_control_variants_match_oracle(interval, mode):
    z = load_golden("walk_L10D8_DW2_branch")
    meta = z["meta"]
    L, N, steps = meta["L"], meta["Nw"], meta["steps"]
    ci, cj, cJ = couplings(z)
    eng = Engine(L=L, ci=ci, cj=cj, cJ=cJ, h=0.0, dtau=meta["dtau"], trial_dims=z["trial_ln_dims"],
                 trial=z["trial_ln_data"], Jvals=[1.0], U=z["U"], S=z["S"], VT=z["VT"], grid=z["grid"],
                 Ndesired=N, capacity=1000, walker_dims=z["walker0_init_dims"])
    walkers = np.tile(z["walker0_init_data"], (N, 1))
    eng.set_walkers(walkers, z["init_weight"], z["init_overlap"], np.zeros(N), normalize=False)
    eng.set_rng(meta["seed"], meta["setup_draws"])
    eng.set_option(OPT_POPCONTROL_INTERVAL, interval)
    eng.set_option(OPT_RESAMPLING, mode)
    trial = po.MPS(z["trial_ln_dims"], z["trial_ln_data"])
    res = po.walk(trial, walkers, z["walker0_init_dims"], z["init_weight"], z["init_overlap"], np.zeros(N),
                  ci=ci, cj=cj, cJ=cJ, Jvals=np.array([1.0]), U=z["U"], S=z["S"], VT=z["VT"], grid=z["grid"],
                  dtau=meta["dtau"], nsteps=steps, Ndesired=N, capacity=1000, seed=meta["seed"],
                  skip=meta["setup_draws"], popctl_interval=interval, comb=(mode == RESAMPLE_COMB))
    assert res.status == 0
    total = 0
    for s in range(steps):
        st = eng.walk(1)[0]
        lw = eng.last_step_walkers()
        n = res.n[s]
        assert st["n_walkers"] == n
        assert st["sum_weight"] == pytest.approx(res.sumw[s], rel=RTOL)
        assert st["E_P"] == pytest.approx(res.EP[s], rel=RTOL)
        np.testing.assert_allclose(lw["weight"], res.weight[s, :n], rtol=RTOL)
        np.testing.assert_allclose(lw["energy"], res.energy[s, :n], rtol=RTOL)
        np.testing.assert_array_equal(lw["parent"], res.parent[s, :len(lw["parent"])])
        if (s + 1) % interval:
            np.testing.assert_array_equal(lw["parent"], np.arange(n))  # no population control
        total += st["draws"]
    assert total == res.draws
    _, wt, _, _ = eng.get_walkers()
    np.testing.assert_allclose(wt, res.weights, rtol=RTOL)
