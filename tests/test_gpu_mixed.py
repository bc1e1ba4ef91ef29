"""Mixed-precision walker step (MPSQMC_OPT_PRECISION) against the reference's FP64 trajectories.

The mixed sweep keeps the site tensors, environments and branches in FP32 and forms their
products on the TF32 tensor cores; the closures, PDF, sampling, weights, overlaps, norms,
energies and population control stay FP64.  Its error is stated per mode and checked here:
  - TF32X3 (three TF32 passes, about FP32 accuracy): every per-walker weight, overlap and local
    energy of the first step within 2e-5 relative of the reference's, E_P within 1e-6;
  - TF32 (one pass, 10-bit mantissa operands): E_P of the first step within 2e-3 relative, and the
    median per-walker weight error below 5e-3 (a sampled grid index may flip for a walker whose
    uniform falls within the PDF error of a CDF boundary).
Over longer walks TF32X3 stays on the FP64 trajectory and both modes' mean projected energies agree
with the FP64 walk's.
"""
import numpy as np
import pytest

from conftest import couplings, load_golden
from mpsqmc_b200 import Engine
from mpsqmc_b200.capi import (E_ARG, E_UNSUPPORTED, OPT_PRECISION, PRECISION_FP64, PRECISION_TF32, PRECISION_TF32X3,
                              MpsqmcError)

pytestmark = pytest.mark.gpu

CASES = ["walk_L16D16_DW16", "walk_L10D8_DW4", "walk_snake4x4_D16_DW8_branch", "walk_L10D8_DW4_field",
         "walk_snake3x3_D8_DW4_field"]


def engine_for(z, precision):
    meta = z["meta"]
    L, N = meta["L"], meta["Nw"]
    ci, cj, cJ = couplings(z)
    eng = Engine(L=L, ci=ci, cj=cj, cJ=cJ, h=meta.get("h", 0.0), dtau=meta["dtau"], trial_dims=z["trial_ln_dims"],
                 trial=z["trial_ln_data"], Jvals=[1.0], U=z["U"], S=z["S"], VT=z["VT"], grid=z["grid"],
                 Ndesired=N, capacity=max(1000, 3 * N), walker_dims=z["walker0_init_dims"])
    eng.set_walkers(np.tile(z["walker0_init_data"], (N, 1)), z["init_weight"], z["init_overlap"], np.zeros(N),
                    normalize=False)
    eng.set_rng(meta["seed"], meta["setup_draws"])
    eng.set_option(OPT_PRECISION, precision)
    assert eng.get_option(OPT_PRECISION) == precision
    return eng


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)) / np.abs(np.asarray(b))


@pytest.mark.parametrize("case", CASES)
def test_tf32x3_first_step_matches_reference(case):
    z = load_golden(case)
    eng = engine_for(z, PRECISION_TF32X3)
    st = eng.walk(1)[0]
    lw = eng.last_step_walkers()
    assert st["n_walkers"] == z["stat_n"][0]
    assert st["E_P"] == pytest.approx(z["stat_EP"][0], rel=1e-6)
    for k in ("weight", "overlap", "energy"):
        assert np.max(rel(lw[k], z["step001_" + k])) < 2e-5, k
    np.testing.assert_array_equal(lw["parent"], z["step001_parent"])


@pytest.mark.parametrize("case", CASES)
def test_tf32_first_step_close_to_reference(case):
    z = load_golden(case)
    eng = engine_for(z, PRECISION_TF32)
    st = eng.walk(1)[0]
    lw = eng.last_step_walkers()
    assert st["E_P"] == pytest.approx(z["stat_EP"][0], rel=2e-3)
    assert np.median(rel(lw["weight"], z["step001_weight"])) < 5e-3
    assert np.all(np.isfinite(lw["energy"]))


def test_precision_option_and_trace():
    """Unknown precisions are refused; the per-coupling trace is FP64-only."""
    z = load_golden("walk_L10D8_DW4")
    eng = engine_for(z, PRECISION_TF32)
    with pytest.raises(MpsqmcError) as ei:
        eng.set_option(OPT_PRECISION, 9)
    assert ei.value.code == E_ARG
    assert eng.get_option(OPT_PRECISION) == PRECISION_TF32
    eng.set_trace(True)
    with pytest.raises(MpsqmcError) as ei:
        eng.walk(1)
    assert ei.value.code == E_UNSUPPORTED
    eng.set_trace(False)
    eng.set_option(OPT_PRECISION, PRECISION_FP64)
    eng.walk(1)


def test_tf32x3_walk_follows_fp64_trajectory():
    """Twenty steps of the 4x4 snake (dtau 0.3, heavy branching) from the same start and random
    stream: with about FP32 accuracy no sampled index flips, so the per-step E_P of the TF32X3
    walk stays on the FP64 walk's trajectory."""
    z = load_golden("walk_snake4x4_D16_DW8_branch")
    runs = {}
    for prec in (PRECISION_FP64, PRECISION_TF32X3):
        eng = engine_for(z, prec)
        st = eng.walk(20)
        runs[prec] = np.array([s["E_P"] for s in st])
        w, wt, ov, eh = eng.get_walkers()
        assert np.all(np.isfinite(w)) and np.all(ov > 0)
        eng.close()
    np.testing.assert_allclose(runs[PRECISION_TF32X3], runs[PRECISION_FP64], rtol=1e-5)


@pytest.mark.parametrize("precision", [PRECISION_TF32X3, PRECISION_TF32])
def test_mixed_walk_energy_agrees_with_fp64(precision):
    """Thirty steps of 256 walkers of the L=16 chain (D_T = D_W = 16, dtau 0.01) from the same
    start and random stream: the mean projected energy of the mixed walk agrees with the FP64
    walk's to the mode's accuracy (a TF32 walk may part from the FP64 trajectory once a sampled
    index flips, so the comparison is of means)."""
    z = load_golden("walk_L16D16_DW16")
    meta = z["meta"]
    ci, cj, cJ = couplings(z)
    N = 256
    rng = np.random.default_rng(7)
    w0 = z["walker0_init_data"]
    walkers = w0[None, :] + 1e-3 * rng.standard_normal((N, w0.size))
    means = {}
    for prec in (PRECISION_FP64, precision):
        eng = Engine(L=meta["L"], ci=ci, cj=cj, cJ=cJ, h=0.0, dtau=meta["dtau"], trial_dims=z["trial_ln_dims"],
                     trial=z["trial_ln_data"], Jvals=[1.0], U=z["U"], S=z["S"], VT=z["VT"], grid=z["grid"],
                     Ndesired=N, capacity=3 * N, walker_dims=z["walker0_init_dims"])
        eng.set_walkers(walkers, np.ones(N), None, np.zeros(N), normalize=True)
        eng.set_rng(meta["seed"], 0)
        eng.set_option(OPT_PRECISION, prec)
        st = eng.walk(30)
        means[prec] = float(np.mean([s["E_P"] for s in st]))
        w, wt, ov, eh = eng.get_walkers()
        assert np.all(np.isfinite(w)) and np.all(ov > 0)
        eng.close()
    tol = 1e-6 if precision == PRECISION_TF32X3 else 1e-3
    assert means[precision] == pytest.approx(means[PRECISION_FP64], rel=tol)
