"""The walker-batched sweep on the tcgen05 tensor cores (MPSQMC_PRECISION_TF32X3_TC): every
contraction of a step is one batched tcgen05 product over the whole population.

Checked against the reference's own FP64 trajectories (tests/golden) and the FP64 oracle at the
bench shapes, with the tolerances of the TF32X3 mode (FP32-accurate products): per-walker
weight, overlap and local energy of the first step within 2e-5 relative, E_P within 2e-6
(measured 1.1e-6 on the 4x4 lattice: sigma-stacked sums round in another order);
sampled grid indices equal to the reference's.  Over several steps with branching it follows the
TF32X3 persistent sweep's trajectory."""
import numpy as np
import pytest

from conftest import couplings, load_golden
from mpsqmc_b200 import Engine
from mpsqmc_b200.capi import (E_UNSUPPORTED, OPT_PRECISION, OPT_TC_KC, OPT_TC_SPLIT_OUT, OPT_TC_STACK_TN,
                              OPT_TC_STAGES, OPT_TC_WIDE_TN, PRECISION_BF16_TC,
                              PRECISION_TF32_TC, PRECISION_TF32X3, PRECISION_TF32X3_TC, TRACE_STRIDE, MpsqmcError)

pytestmark = pytest.mark.gpu

CASES = ["walk_L16D16_DW16", "walk_L10D8_DW4", "walk_snake4x4_D16_DW8_branch", "walk_L10D8_DW4_field",
         "walk_snake3x3_D8_DW4_field", "walk_snake3x3_D8_DW4"]


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
    return eng


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)) / np.abs(np.asarray(b))


@pytest.mark.parametrize("case", CASES)
def test_tc_first_step_matches_reference(case):
    z = load_golden(case)
    eng = engine_for(z, PRECISION_TF32X3_TC)
    eng.set_trace(True)
    st = eng.walk(1)[0]
    lw = eng.last_step_walkers()
    tr = eng.get_trace()
    nC = z["meta"]["nCouplings"]
    N = z["meta"]["Nw"]
    idx = tr.reshape(N, nC, TRACE_STRIDE)[:, :, 18].astype(int).reshape(-1)
    np.testing.assert_array_equal(idx, z["step001_trace_index"].astype(int))
    assert st["n_walkers"] == z["stat_n"][0]
    assert st["E_P"] == pytest.approx(z["stat_EP"][0], rel=2e-6)
    for k in ("weight", "overlap", "energy"):
        assert np.max(rel(lw[k], z["step001_" + k])) < 2e-5, k
    np.testing.assert_array_equal(lw["parent"], z["step001_parent"])
    eng.close()


@pytest.mark.parametrize("case", ["walk_L16D16_DW16", "walk_snake4x4_D16_DW8_branch"])
def test_tc_follows_the_tf32x3_sweep_over_steps(case):
    z = load_golden(case)
    a = engine_for(z, PRECISION_TF32X3_TC)
    b = engine_for(z, PRECISION_TF32X3)
    sa, sb = a.walk(6), b.walk(6)
    for x, y in zip(sa, sb):
        assert x["n_walkers"] == y["n_walkers"]
        assert x["E_P"] == pytest.approx(y["E_P"], rel=2e-6)
        assert x["sum_weight"] == pytest.approx(y["sum_weight"], rel=2e-5)
    a.close()
    b.close()


def test_tc_one_pass_is_close():
    z = load_golden("walk_L16D16_DW16")
    eng = engine_for(z, PRECISION_TF32_TC)
    st = eng.walk(1)[0]
    assert st["E_P"] == pytest.approx(z["stat_EP"][0], rel=2e-3)
    eng.close()


def test_tc_bf16_pass_is_close():
    """The tcgen05 sweep with one bfloat16 pass per product (MPSQMC_PRECISION_BF16_TC): operands
    carry 8 mantissa bits, so the first step's E_P is checked loosely against the reference
    (5e-2; the FP32-accurate mode is the one held to the reference's trajectory)."""
    z = load_golden("walk_L16D16_DW16")
    eng = engine_for(z, PRECISION_BF16_TC)
    st = eng.walk(1)[0]
    print(f"bf16 E_P {st['E_P']:.8f} vs {z['stat_EP'][0]:.8f}")
    assert st["E_P"] == pytest.approx(z["stat_EP"][0], rel=5e-2)
    eng.close()


def test_tc_rejects_uneven_populations():
    z = load_golden("walk_L10D8_DW4")
    meta = z["meta"]
    L, N = meta["L"], meta["Nw"]
    ci, cj, cJ = couplings(z)
    eng = Engine(L=L, ci=ci, cj=cj, cJ=cJ, h=0.0, dtau=meta["dtau"], trial_dims=z["trial_ln_dims"],
                 trial=z["trial_ln_data"], Jvals=[1.0], U=z["U"], S=z["S"], VT=z["VT"], grid=z["grid"],
                 Ndesired=N, capacity=64, walker_dims=z["trial_ln_dims"])
    eng.set_walkers(np.tile(z["trial_ln_data"], (N, 1)), np.ones(N), normalize=False)
    eng.compress_walkers(np.array([4, 8] * (N // 2) + [4] * (N % 2), dtype=np.int32), normalize=True)
    eng.set_option(OPT_PRECISION, PRECISION_TF32X3_TC)
    with pytest.raises(MpsqmcError) as e:
        eng.walk(1)
    assert e.value.code == E_UNSUPPORTED
    eng.close()


def test_tc_tile_choices_give_the_same_walk():
    """Other tile shapes, ring depths, stage depths in k and split right factors (the autotuner's
    candidates) only regroup the same per-element products (a factor written as TF32 head and tail is split as the
    shared-memory conversion would split it): the step's results agree with the defaults' to FP32
    rounding."""
    z = load_golden("walk_snake4x4_D16_DW8_branch")
    a = engine_for(z, PRECISION_TF32X3_TC)
    b = engine_for(z, PRECISION_TF32X3_TC)
    for opt, v in ((OPT_TC_STACK_TN, 64), (OPT_TC_WIDE_TN, 128), (OPT_TC_STAGES, 2), (OPT_TC_SPLIT_OUT, 31),
                   (OPT_TC_KC, 16)):
        b.set_option(opt, v)
        assert b.get_option(opt) == v
    sa, sb = a.walk(3), b.walk(3)
    for x, y in zip(sa, sb):
        assert x["n_walkers"] == y["n_walkers"]
        assert x["E_P"] == pytest.approx(y["E_P"], rel=1e-6)
    la, lb = a.last_step_walkers(), b.last_step_walkers()
    for k in ("weight", "overlap", "energy"):
        assert np.max(rel(lb[k], la[k])) < 1e-6, k
    with pytest.raises(MpsqmcError):
        b.set_option(OPT_TC_STACK_TN, 96)
    a.close()
    b.close()


def test_tc_autotune_picks_valid_tiles_and_keeps_the_walk():
    z = load_golden("walk_L16D16_DW16")
    a = engine_for(z, PRECISION_TF32X3_TC)
    b = engine_for(z, PRECISION_TF32X3_TC)
    b.autotune(steps=1)  # population, random stream and step count restored afterwards
    assert b.get_option(OPT_TC_STACK_TN) in (64, 128, 256)
    assert b.get_option(OPT_TC_WIDE_TN) in (64, 128, 256)
    assert b.get_option(OPT_TC_STAGES) in (2, 4, 8)
    assert b.get_option(OPT_TC_KC) in (16, 32)
    assert 0 <= b.get_option(OPT_TC_SPLIT_OUT) <= 31
    sa, sb = a.walk(2), b.walk(2)
    for x, y in zip(sa, sb):
        assert x["n_walkers"] == y["n_walkers"]
        assert x["E_P"] == pytest.approx(y["E_P"], rel=1e-6)
    a.close()
    b.close()


@pytest.mark.parametrize("mask", [1, 2, 4, 8, 16])
def test_tc_each_split_class_gives_the_same_step(mask):
    """Each class of right factors stored as TF32 head and tail arrays (right environments and
    closures, left branches, carries, energy, channels) on its own: the step agrees with the
    default (every right factor split in shared memory) to FP32 rounding."""
    z = load_golden("walk_snake4x4_D16_DW8_branch")
    a = engine_for(z, PRECISION_TF32X3_TC)
    b = engine_for(z, PRECISION_TF32X3_TC)
    b.set_option(OPT_TC_SPLIT_OUT, mask)
    sa, sb = a.walk(2), b.walk(2)
    for x, y in zip(sa, sb):
        assert x["n_walkers"] == y["n_walkers"]
        assert x["E_P"] == pytest.approx(y["E_P"], rel=1e-6)
    la, lb = a.last_step_walkers(), b.last_step_walkers()
    for k in ("weight", "overlap", "energy"):
        assert np.max(rel(lb[k], la[k])) < 1e-6, k
    a.close()
    b.close()
