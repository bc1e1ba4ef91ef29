"""Walks split over ranks, device side: the split step (mpsqmc_step_propagate / _control) equals
mpsqmc_walk on one rank, walker records survive export and import, and two engines emulating two
ranks on one GPU (sums added by hand, records moved through a device buffer) share one global
E_P and rebalance by the reference's plan."""
import numpy as np
import pytest
import torch

from conftest import couplings, load_golden
from mpsqmc_b200 import Engine
from mpsqmc_b200.population import balance_plan

pytestmark = pytest.mark.gpu


def engine_for(z, n=None, seed_skip=None, walkers=None):
    meta = z["meta"]
    L, N = meta["L"], n or meta["Nw"]
    ci, cj, cJ = couplings(z)
    eng = Engine(L=L, ci=ci, cj=cj, cJ=cJ, h=meta.get("h", 0.0), dtau=meta["dtau"], trial_dims=z["trial_ln_dims"],
                 trial=z["trial_ln_data"], Jvals=[1.0], U=z["U"], S=z["S"], VT=z["VT"], grid=z["grid"],
                 Ndesired=N, capacity=max(1000, 3 * N), walker_dims=z["walker0_init_dims"])
    w = np.tile(z["walker0_init_data"], (N, 1)) if walkers is None else walkers
    eng.set_walkers(w, np.ones(N) if walkers is not None else z["init_weight"][:N],
                    None if walkers is not None else z["init_overlap"][:N], np.zeros(N), normalize=walkers is not None)
    eng.set_rng(meta["seed"], meta["setup_draws"] if seed_skip is None else seed_skip)
    return eng


def test_split_step_equals_walk():
    z = load_golden("walk_L10D8_DW2_branch")
    a, b = engine_for(z), engine_for(z)
    sa = a.walk(4)
    for s in range(4):
        local = b.step_propagate()
        sb = b.step_control(local, z["meta"]["Nw"])
        for k in ("n_walkers", "n_after", "sum_weight", "E_P", "E_T", "omega", "scaling", "draws", "step"):
            assert sb[k] == sa[s][k], (s, k)
    for x, y in zip(a.get_walkers(), b.get_walkers()):
        np.testing.assert_array_equal(x, y)
    assert a.rng_draws() == b.rng_draws()


def test_export_import_round_trip():
    z = load_golden("walk_snake4x4_D16_DW8_branch")
    a, b = engine_for(z), engine_for(z, seed_skip=123)
    a.walk(2)
    b.walk(1)
    b.get_walkers()  # left-normalised now, so the read-back below leaves every tensor as it is
    wa, wta, ova, eha = a.get_walkers()
    nb = b.n_walkers
    k = 5
    buf = torch.empty(k * a.record_size(), dtype=torch.float64, device="cuda")
    a.export_walkers(k, buf.data_ptr())
    b.import_walkers(k, buf.data_ptr())
    assert a.n_walkers == wa.shape[0] - k and b.n_walkers == nb + k
    wb, wtb, ovb, ehb = b.get_walkers()
    np.testing.assert_array_equal(wb[-k:], wa[-k:])
    np.testing.assert_array_equal(wtb[-k:], wta[-k:])
    np.testing.assert_array_equal(ehb[-k:], eha[-k:])
    np.testing.assert_allclose(ovb[-k:], ova[-k:], rtol=1e-14)
    # both populations keep walking
    a.walk(1)
    b.walk(1)
    assert np.all(np.isfinite(b.get_walkers()[1]))


def test_two_engines_share_global_statistics_and_rebalance():
    """Two ranks emulated by two engines on one GPU: the sums of both enter both controls, so
    both report the E_P of the union; the uneven populations are then evened out."""
    z = load_golden("walk_L16D16_DW16")
    rng = np.random.default_rng(3)
    w0 = z["walker0_init_data"]
    counts = [96, 32]
    engines = [engine_for(z, n=n, seed_skip=s, walkers=w0[None, :] + 1e-3 * rng.standard_normal((n, w0.size)))
               for n, s in zip(counts, (0, 10 ** 6))]
    desired = [64, 64]
    for step in range(3):
        local = [e.step_propagate() for e in engines]
        g = local[0] + local[1]
        st = [e.step_control(g, sum(desired)) for e in engines]
        lw = [e.last_step_walkers() for e in engines]
        assert st[0]["E_P"] == st[1]["E_P"] and st[0]["scaling"] == st[1]["scaling"]
        num = sum(float(np.sum(x["weight"] * x["energy"])) for x in lw)
        den = sum(float(np.sum(x["weight"])) for x in lw)
        assert st[0]["E_P"] == pytest.approx(num / den, rel=1e-12)
        assert st[0]["scaling"] == pytest.approx(sum(desired) / den, rel=1e-12)
        # balance
        n = [e.n_walkers for e in engines]
        for moves in balance_plan(n, desired):
            for s, r, k in moves:
                buf = torch.empty(k * engines[s].record_size(), dtype=torch.float64, device="cuda")
                engines[s].export_walkers(k, buf.data_ptr())
                engines[r].import_walkers(k, buf.data_ptr())
        n2 = [e.n_walkers for e in engines]
        assert sum(n2) == sum(n)
        assert abs(n2[0] - n2[1]) <= max(0.06 * sum(n2) / 2, 2), n2
