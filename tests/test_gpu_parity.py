"""CUDA engine (libmpsqmc_b200.so through its C ABI) against the reference's own trajectories.

Same trial, Trotter tables, grid, initial walkers and random stream as the reference run that
produced the fixture; every quantity of the walk is compared:
  - per-step N, sum of weights, E_P, E_T, fluctuation metric;
  - per-walker weight, overlap and local energy after propagation (relative 1e-10, FP64 mode);
  - per-coupling C_kl, uniform and sampled grid index;
  - branching parents (bit-exact) and the number of uniforms consumed;
  - final walker states (fidelity with the reference tensors; the engine's gauge differs).
"""
import numpy as np
import pytest

from conftest import WALK_CASES, couplings, load_golden
from mpsqmc_b200 import Engine
from mpsqmc_b200 import problem as pb
from mpsqmc_b200.capi import OPT_CANONICAL_INTERVAL, OPT_SWEEP, OPT_WORKSPACE, SWEEP_NEAREST, WORKSPACE_GLOBAL
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def engine_for(z, capacity=None, sweep=None, workspace=None, canon=None):
    meta = z["meta"]
    L, N = meta["L"], meta["Nw"]
    ci, cj, cJ = couplings(z)
    eng = Engine(L=L, ci=ci, cj=cj, cJ=cJ, h=meta.get("h", 0.0), dtau=meta["dtau"], trial_dims=z["trial_ln_dims"],
                 trial=z["trial_ln_data"], Jvals=[1.0], U=z["U"], S=z["S"], VT=z["VT"], grid=z["grid"],
                 Ndesired=N, capacity=capacity or max(1000, 3 * N), walker_dims=z["walker0_init_dims"])
    walkers = np.tile(z["walker0_init_data"], (N, 1))
    eng.set_walkers(walkers, z["init_weight"], z["init_overlap"], np.zeros(N), normalize=False)
    eng.set_rng(meta["seed"], meta["setup_draws"])
    if sweep is not None:
        eng.set_option(OPT_SWEEP, sweep)
    if workspace is not None:
        eng.set_option(OPT_WORKSPACE, workspace)
        assert eng.get_option(OPT_WORKSPACE) == workspace
    if canon is not None:
        eng.set_option(OPT_CANONICAL_INTERVAL, canon)
        assert eng.get_option(OPT_CANONICAL_INTERVAL) == canon
    return eng


def fidelity(dims_a, a, dims_b, b):
    A, B = po.MPS(np.asarray(dims_a, np.int32), a), po.MPS(np.asarray(dims_b, np.int32), b)
    ab = po.inner_product(A, B)
    return ab / np.sqrt(po.inner_product(A, A) * po.inner_product(B, B))


MODES = {"auto": (None, None, None), "qr-per-site": (None, None, 0), "nearest": (SWEEP_NEAREST, None, None),
         "global-ws": (None, WORKSPACE_GLOBAL, None), "nearest-global-ws": (SWEEP_NEAREST, WORKSPACE_GLOBAL, None),
         "qr-free-2": (None, None, 2), "qr-free-global-ws": (None, WORKSPACE_GLOBAL, 3)}


@pytest.mark.parametrize("mode", list(MODES))
@pytest.mark.parametrize("case", WALK_CASES)
def test_walk_matches_reference(case, mode):
    """Every case runs the general sweep (the default); chains also run the nearest-neighbour
    sweep.  "global-ws" keeps the matrix work buffers in global scratch (the placement large bond
    dimensions use) instead of shared memory.  The default general sweep skips the per-site QR and
    left-normalises every 16 steps; "qr-per-site" runs the Householder QR at every site, "qr-free-2"
    ("qr-free-global-ws") left-normalise every 2 (3) steps, so that steps of both kinds are
    compared."""
    z = load_golden(case)
    meta = z["meta"]
    sweep, ws, canon = MODES[mode]
    if sweep == SWEEP_NEAREST and "snake" in case:
        pytest.skip("the nearest-neighbour sweep takes chains only")
    eng = engine_for(z, sweep=sweep, workspace=ws, canon=canon)
    assert eng.energy() == pytest.approx(meta["E0"], rel=RTOL)
    total_draws = 0
    for s in range(1, meta["steps"] + 1):
        p = f"step{s:03d}_"
        eng.set_trace(True)
        st = eng.walk(1)[0]
        lw = eng.last_step_walkers()
        tr = eng.get_trace()
        n = len(z[p + "weight"])
        assert st["n_walkers"] == n == z["stat_n"][s - 1]
        assert st["sum_weight"] == pytest.approx(z["stat_sumw"][s - 1], rel=RTOL)
        assert st["E_P"] == pytest.approx(z["stat_EP"][s - 1], rel=RTOL)
        assert st["E_T"] == pytest.approx(z["stat_ET"][s - 1], rel=1e-8, abs=1e-8)
        assert abs(st["omega"] - z["stat_omega"][s - 1]) <= 1e-9 * z["stat_EP"][s - 1] ** 2
        np.testing.assert_allclose(lw["weight"], z[p + "weight"], rtol=RTOL)
        np.testing.assert_allclose(lw["overlap"], z[p + "overlap"], rtol=RTOL)
        np.testing.assert_allclose(lw["energy"], z[p + "energy"], rtol=RTOL)
        t = tr.reshape(-1, 21)
        np.testing.assert_array_equal(t[:, 17], z[p + "trace_u"])
        np.testing.assert_array_equal(t[:, 18].astype(int), z[p + "trace_index"])
        np.testing.assert_allclose(t[:, :16], z[p + "trace_C"], rtol=0, atol=1e-12)
        np.testing.assert_allclose(t[:, 16], z[p + "trace_pdfnorm"], rtol=RTOL)
        np.testing.assert_array_equal(lw["parent"], z[p + "parent"])
        assert st["draws"] == int(np.sum(z["stat_draws"][s - 1]))
        total_draws += st["draws"]
    assert eng.rng_draws() == total_draws
    w, wt, ov, eh = eng.get_walkers()
    last = f"step{meta['steps']:03d}_"
    ref = z[last + "tensors"][z[last + "parent"]]
    dims = z["walker0_init_dims"]
    for k in range(w.shape[0]):
        assert fidelity(dims, w[k], dims, ref[k]) == pytest.approx(1.0, abs=1e-12)
    np.testing.assert_allclose(wt, z[last + "newweight"], rtol=RTOL)
    np.testing.assert_allclose(eh, z[last + "ehist"][z[last + "parent"]], rtol=RTOL)


def test_set_overlap_is_reference_exact():
    """Walker::setOverlap on device: Householder LeftNormalize element by element, overlap, sign."""
    z = load_golden("mpsops_debug")
    g = load_golden("grids")["marsaglia4"]
    tr = load_golden("trotter")
    trial_dims, trial = z["leftnorm_dims"], z["leftnorm_data"]
    L = len(trial_dims) - 1
    ci, cj, cJ = pb.chain(L)
    eng = Engine(L=L, ci=ci, cj=cj, cJ=cJ, h=0.0, dtau=0.01, trial_dims=trial_dims, trial=trial, Jvals=[1.0],
                 U=tr["dt0.01_J1.0_U"], S=tr["dt0.01_J1.0_S"], VT=tr["dt0.01_J1.0_VT"], grid=g, Ndesired=1,
                 capacity=4, walker_dims=z["other_dims"])
    eng.set_walkers(z["other_data"][None, :], [1.0], normalize=True)
    w, wt, ov, eh = eng.get_walkers()
    ref = z["other_leftnorm_data"].copy()
    sc = z["scalars"]
    ov_ref = sc[5]
    if ov_ref < 0:  # ChangePhase on site 0
        n0 = int(z["other_dims"][0] * z["other_dims"][1] * 2)
        ref[:n0] *= -1
        ov_ref = -ov_ref
    np.testing.assert_allclose(w[0], ref, rtol=0, atol=1e-13)
    assert ov[0] == pytest.approx(ov_ref, rel=1e-12)


def test_local_energy_matches_oracle():
    z = load_golden("walk_L16D16_DW16")
    eng = engine_for(z)
    eng.walk(2)
    w, wt, ov, eh = eng.get_walkers()
    lw_e = eng.energy()
    trial = po.MPS(z["trial_ln_dims"], z["trial_ln_data"])
    ci, cj, cJ = pb.chain(16)
    num = 0.0
    den = 0.0
    for k in range(w.shape[0]):
        phi = po.MPS(z["walker0_init_dims"], w[k])
        e = po.energy_numerator(trial, phi, ci, cj, cJ) / ov[k]
        num += wt[k] * e
        den += wt[k]
    assert lw_e == pytest.approx(num / den, rel=RTOL)


def test_capacity_overflow_is_an_error_not_a_crash():
    from mpsqmc_b200.capi import E_CAPACITY, MpsqmcError
    z = load_golden("walk_L10D8_DW1_branch")
    eng = engine_for(z, capacity=33)
    with pytest.raises(MpsqmcError) as ei:
        eng.walk(8)
    assert ei.value.code == E_CAPACITY


def test_nearest_neighbour_sweep_refuses_long_couplings():
    from mpsqmc_b200.capi import E_UNSUPPORTED, SWEEP_NEAREST, MpsqmcError
    eng = engine_for(load_golden("walk_snake3x3_D8_DW4"))
    with pytest.raises(MpsqmcError) as ei:
        eng.set_option(OPT_SWEEP, SWEEP_NEAREST)
    assert ei.value.code == E_UNSUPPORTED
    assert eng.get_option(OPT_SWEEP) == 0


def test_autotune_restores_population_and_keeps_trajectory():
    """mpsqmc_autotune measures the kernel choices on a copy of the population's state: after it,
    walkers, weights, overlaps, random stream and step count are as before, and the walk follows
    the reference trajectory."""
    from mpsqmc_b200.capi import OPT_SWEEP, OPT_WORKSPACE
    z = load_golden("walk_L10D8_DW2_branch")
    meta = z["meta"]
    eng = engine_for(z)
    before = eng.get_walkers()
    d0 = eng.rng_draws()
    sweep, ws = eng.autotune(steps=2)
    assert eng.get_option(OPT_SWEEP) == sweep and eng.get_option(OPT_WORKSPACE) == ws
    after = eng.get_walkers()
    for a, b in zip(before, after):
        np.testing.assert_array_equal(a, b)
    assert eng.rng_draws() == d0
    for s in range(1, meta["steps"] + 1):
        st = eng.walk(1)[0]
        assert st["step"] == s
        assert st["E_P"] == pytest.approx(z["stat_EP"][s - 1], rel=RTOL)
        np.testing.assert_array_equal(eng.last_step_walkers()["parent"], z[f"step{s:03d}_parent"])
    # the choice is remembered for the same shape
    eng2 = engine_for(z)
    assert eng2.autotune(steps=2) == (sweep, ws)


def test_qr_free_walkers_read_back_left_canonical():
    """After QR-free steps (default interval 16, so the walkers were not left-normalised by the
    walk), mpsqmc_get_walkers returns Walker::setOverlap's state: every site but the last
    left-orthonormal, norm 1, overlaps <Psi_T|phi> > 0 of those tensors."""
    z = load_golden("walk_snake4x4_D16_DW8_branch")
    eng = engine_for(z)
    eng.walk(3)
    w, wt, ov, eh = eng.get_walkers()
    dims = z["walker0_init_dims"]
    trial = po.MPS(z["trial_ln_dims"], z["trial_ln_data"])
    for k in range(w.shape[0]):
        m = po.MPS(np.asarray(dims, np.int32), w[k])
        for s in range(m.L - 1):
            A = m.site(s)  # [sigma, Dr, Dl]: the transposed sigma blocks
            G = sum(A[q] @ A[q].T for q in range(A.shape[0]))
            np.testing.assert_allclose(G, np.eye(G.shape[0]), atol=1e-12)
        assert po.inner_product(m, m) == pytest.approx(1.0, abs=1e-12)
        assert po.inner_product(trial, m) == pytest.approx(ov[k], rel=1e-10)
        assert ov[k] > 0
