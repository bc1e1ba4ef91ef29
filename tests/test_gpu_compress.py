"""Walker recompression on the device (MPSstate::CompressState, two-site SVD sweeps) against the
reference's own compressed walkers (the walker0_init of the golden walks: SetupWalkers compresses
the left-normalised trial to D_W and calls setOverlap) and against the oracle's restatement for
uneven targets.  States are compared by fidelity (SVD signs are implementation-specific), bond
dims exactly, overlaps to 1e-10."""
import numpy as np
import pytest

from conftest import couplings, load_golden
from mpsqmc_b200 import Engine
from mpsqmc_b200 import problem as pb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def fidelity(a: po.MPS, b: po.MPS) -> float:
    return po.inner_product(a, b) / np.sqrt(po.inner_product(a, a) * po.inner_product(b, b))


def engine(z, trial_dims, trial, N, ci, cj, cJ):
    meta = z["meta"]
    return Engine(L=meta["L"], ci=ci, cj=cj, cJ=cJ, h=0.0, dtau=meta["dtau"], trial_dims=trial_dims, trial=trial,
                  Jvals=[1.0], U=z["U"], S=z["S"], VT=z["VT"], grid=z["grid"], Ndesired=N, capacity=64,
                  walker_dims=trial_dims)


@pytest.mark.parametrize("case", ["walk_L10D8_DW4", "walk_L10D8_DW1_branch", "walk_debug_DW2",
                                  "walk_snake4x4_D16_DW8_branch", "walk_snake3x3_D8_DW4"])
def test_compression_matches_reference_setup(case):
    z = load_golden(case)
    DW = z["meta"]["DW"]
    ci, cj, cJ = couplings(z)
    N = 3
    eng = engine(z, z["trial_ln_dims"], z["trial_ln_data"], N, ci, cj, cJ)
    eng.set_walkers(np.tile(z["trial_ln_data"], (N, 1)), np.ones(N), normalize=False)
    eng.compress_walkers(DW, normalize=True)
    dims = eng.get_walker_dims()
    ref_dims = z["walker0_init_dims"]
    for k in range(N):
        np.testing.assert_array_equal(dims[k], ref_dims)
    w, wt, ov, eh = eng.get_walkers()
    n = po.mps_size(ref_dims)
    ref = po.MPS(ref_dims, z["walker0_init_data"])
    for k in range(N):
        assert fidelity(po.MPS(ref_dims, w[k, :n]), ref) == pytest.approx(1.0, abs=1e-12)
    np.testing.assert_allclose(ov, z["init_overlap"][0], rtol=1e-10)


def test_uneven_targets_match_oracle():
    rng = np.random.default_rng(11)
    z = load_golden("walk_L16D16_DW16")
    trial = po.MPS(z["trial_ln_dims"], z["trial_ln_data"])
    ci, cj, cJ = couplings(z)
    targets = np.array([1, 2, 3, 5, 8, 13, 15, 0, 16], dtype=np.int32)
    N = len(targets)
    walkers = trial.data[None, :] + 0.05 * rng.normal(size=(N, trial.data.size))
    eng = engine(z, trial.dims, trial.data, N, ci, cj, cJ)
    eng.set_walkers(walkers, np.ones(N), normalize=False)
    eng.compress_walkers(targets, normalize=False)
    dims = eng.get_walker_dims()
    w, _, _, _ = eng.get_walkers()
    for k in range(N):
        src = po.MPS(trial.dims, walkers[k])
        if targets[k] <= 0 or targets[k] >= max(trial.dims):
            np.testing.assert_array_equal(dims[k], trial.dims)
            np.testing.assert_array_equal(w[k], walkers[k])
            continue
        ref = po.compress(src, int(targets[k]))
        np.testing.assert_array_equal(dims[k], ref.dims)
        n = po.mps_size(ref.dims)
        got = po.MPS(ref.dims, w[k, :n])
        assert fidelity(got, ref) == pytest.approx(1.0, abs=1e-11)
        # CompressState keeps the norm-weighted projection: <src|got> = <src|ref>
        assert po.inner_product(src, got) == pytest.approx(po.inner_product(src, ref), rel=1e-10)
