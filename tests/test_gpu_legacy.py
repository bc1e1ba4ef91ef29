"""The MPO-term projector (the reference's MPSQMC::Walk, MPSQMC.cpp:236-440) on the CUDA engine
against the reference's own runs (tests/golden/legacy_*.npz, from oracle/_ref/ref_harness legacy):
chain, chain with field, 3x3 snake lattice.  Per step: walker count, the int weight sum, E_P,
E_T, fluctuation metric; per walker: weight, overlap and local energy after propagation (1e-10
relative), overlaps and energy histories after population control, uniforms consumed (exact);
after the last step the walker tensors element by element (the walkers a term hits are
re-normalised with the reference's Householder conventions, the others are untouched)."""
import numpy as np
import pytest

from conftest import load_golden
from mpsqmc_b200 import Engine
from mpsqmc_b200 import problem as pb
from mpsqmc_b200.capi import OPT_PROJECTOR, PROJECTOR_MPO_TERMS

pytestmark = pytest.mark.gpu

RTOL = 1e-10


@pytest.mark.parametrize("case", ["legacy_L10D8", "legacy_L10D8_field", "legacy_snake3x3_D8"])
def test_mpo_term_projector_matches_reference(case):
    z = load_golden(case)
    meta = z["meta"]
    L, N, dtau = meta["L"], meta["Nw"], meta["dtau"]
    ci, cj, cJ = pb.lattice(meta.get("lattice", f"chain:{L}"))
    U, S, VT = pb.trotter_tables(1.0, dtau)
    dims = z["trial_ln_dims"]
    eng = Engine(L=L, ci=ci, cj=cj, cJ=cJ, h=meta["h"], dtau=dtau, trial_dims=dims, trial=z["trial_ln_data"],
                 Jvals=[1.0], U=U, S=S, VT=VT, grid=pb.grid_marsaglia(4, 4), Ndesired=N,
                 capacity=max(1000, 3 * N), walker_dims=dims)
    # SetupWalkers (MPSQMC.cpp:195-233): trial copies, weight 1, overlap 1, no normalisation
    eng.set_walkers(np.tile(z["trial_ln_data"], (N, 1)), np.ones(N), np.ones(N), np.zeros(N), normalize=False)
    eng.set_option(OPT_PROJECTOR, PROJECTOR_MPO_TERMS)
    eng.set_rng(meta["seed"], meta["setup_draws"])
    assert eng.energy() == pytest.approx(meta["E0"], rel=RTOL)
    total = 0
    for s in range(1, meta["steps"] + 1):
        p = f"step{s:03d}_"
        st = eng.walk(1)[0]
        lw = eng.last_step_walkers()
        n = int(z["stat_n"][s - 1])
        assert st["n_walkers"] == n
        assert st["sum_weight"] == z["stat_sum"][s - 1]  # summed into an int, exactly
        assert st["E_P"] == pytest.approx(z["stat_EP"][s - 1], rel=RTOL)
        assert st["E_T"] == pytest.approx(z["stat_ET"][s - 1], rel=1e-10, abs=1e-10)
        assert abs(st["omega"] - z["stat_omega"][s - 1]) <= 1e-9 * z["stat_EP"][s - 1] ** 2
        np.testing.assert_allclose(lw["weight"], z[p + "weight"], rtol=RTOL)
        np.testing.assert_allclose(lw["overlap"], z[p + "overlap"], rtol=RTOL)
        np.testing.assert_allclose(lw["energy"], z[p + "energy"], rtol=RTOL)
        assert st["draws"] == int(np.sum(z["stat_draws"][s - 1]))
        total += st["draws"]
        _, wt, ov, eh = eng.get_walkers()
        np.testing.assert_allclose(ov, z[p + "newoverlap"], rtol=RTOL)
        np.testing.assert_allclose(eh, z[p + "newehist"], rtol=RTOL, atol=1e-12)
        np.testing.assert_array_equal(wt, np.ones(len(wt)))
    assert eng.rng_draws() == total
    w, _, _, _ = eng.get_walkers()
    last = f"step{meta['steps']:03d}_tensors"
    np.testing.assert_allclose(w, z[last], rtol=0, atol=1e-12)
