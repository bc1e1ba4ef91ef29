"""The walk against exact diagonalisation: the projected energy of the L = 16 open Heisenberg
chain (the trial from the compact-MPO DMRG at D = 16, walkers of D_W = 16, dtau 0.01, the
Marsaglia(4) grid) agrees with the Lanczos ground energy of oracle/ed.py within its blocking
error plus 2e-4 (Trotter and population-control bias).
"""
import numpy as np
import pytest

from conftest import couplings, load_golden
from mpsqmc_b200 import Engine, analysis
from oracle import ed

pytestmark = pytest.mark.gpu


def test_projected_energy_matches_exact_diagonalisation_L16():
    z = load_golden("walk_L16D16_DW16")
    meta = z["meta"]
    L, N = meta["L"], 256
    ci, cj, cJ = couplings(z)
    e_exact = ed.ground_energy(L)
    assert e_exact == pytest.approx(-6.9117371455749, abs=1e-9)
    eng = Engine(L=L, ci=ci, cj=cj, cJ=cJ, h=0.0, dtau=meta["dtau"], trial_dims=z["trial_ln_dims"],
                 trial=z["trial_ln_data"], Jvals=[1.0], U=z["U"], S=z["S"], VT=z["VT"], grid=z["grid"],
                 Ndesired=N, capacity=3 * N, walker_dims=z["walker0_init_dims"])
    eng.set_walkers(np.tile(z["walker0_init_data"], (N, 1)), np.ones(N), None, np.zeros(N), normalize=True)
    eng.set_rng(meta["seed"], 0)
    st = eng.walk(240)
    ep = np.array([s["E_P"] for s in st[40:]])
    assert np.all(np.isfinite(ep))
    err = analysis.blocking_error(ep)
    assert abs(ep.mean() - e_exact) < 5.0 * err + 2e-4, (ep.mean(), e_exact, err)
    # the trial itself (D = 16) is within 1e-5 of the ground state, and the walk stays there
    assert abs(meta["E0"] - e_exact) < 1e-5
    eng.close()
