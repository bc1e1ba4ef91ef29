"""The CUDA engine against the FP64 oracle at the shapes the bench measures, so that every
throughput figure belongs to a configuration whose output is checked:

  chain64    L = 64 chain, D_T = 64 DMRG trial, D_W = 32 walkers (compressed trial + noise): the
             default instantiation (general sweep with stored right branches, QR-free), matrix
             work buffers in shared memory;
  snake6x6   6x6 open lattice on the snake path (60 couplings, ranges 1..11), D_T = 128, walkers
             of D_W 16, 32, 64 and 128 in one population (compressed on the device);
  snake8x8   8x8 open lattice (112 couplings, ranges 1..15), D_T = 256 DMRG trial, D_W = 64.

Each case runs one step of a few walkers and compares every walker's weight, overlap and local
energy with oracle/envwalk.py (same trial, walkers, tables and uniforms; the oracle is pinned
to the reference's outputs in tests/test_envwalk_pin.py):
  FP64       1e-10 relative (the reference-parity tolerance);
  TF32X3     2e-5 relative (FP32 work buffers on the TF32 tensor cores, three passes) on the
             chain, 1e-4 on the lattices (small trial-walker overlaps whose FP32 sums cancel);
  TF32X3_TC  the same (the walker-batched sweep on tcgen05, three passes; one bond profile).
"""
import numpy as np
import pytest

from mpsqmc_b200 import Engine, workloads
from mpsqmc_b200 import problem as pb
from mpsqmc_b200.capi import (OPT_PRECISION, OPT_WORKSPACE, PRECISION_FP64, PRECISION_TF32X3, PRECISION_TF32X3_TC,
                              WORKSPACE_AUTO)
from oracle import envwalk as ew

pytestmark = pytest.mark.gpu

TOL = {PRECISION_FP64: 1e-10, PRECISION_TF32X3: 2e-5, PRECISION_TF32X3_TC: 2e-5}
# On the lattices the FP32 sweeps meet 1e-4: the 6x6 trial is random, so trial-walker overlaps
# are ~1e-3 and their FP32 sums cancel (measured 2.7e-5 on the 6x6 overlap)
LATTICE_TOL_FP32 = 1e-4
SEED = 31337


def chain64_case():
    wl = workloads.chain64(Nw=4)
    inputs = wl.inputs()
    eng = Engine(**inputs)
    eng.set_walkers(wl.walkers(), np.ones(4), None, np.zeros(4), normalize=True)
    return eng, inputs


def lattice_case(wl, targets):
    ci, cj, cJ = wl.couplings()
    trial = wl.trial()
    U, S, VT = pb.trotter_tables(1.0, wl.dtau)
    N = len(targets)
    inputs = dict(L=wl.L, ci=ci, cj=cj, cJ=cJ, h=0.0, dtau=wl.dtau, trial_dims=trial.dims, trial=trial.data,
                  Jvals=[1.0], U=U, S=S, VT=VT, grid=pb.grid_marsaglia(4, 4), Ndesired=N, capacity=64)
    if max(targets) >= wl.DT:  # uneven walkers made on the device, as the bench does
        eng = Engine(walker_dims=trial.dims, **inputs)
        eng.set_walkers(np.tile(trial.data, (N, 1)), np.ones(N), normalize=False)
        eng.compress_walkers(np.asarray(targets, np.int32), normalize=True)
    else:
        w = pb.compress(trial, max(targets))
        rng = np.random.default_rng(1)
        eng = Engine(walker_dims=w.dims, **inputs)
        eng.set_walkers(w.data[None, :] + 1e-3 * rng.normal(size=(N, w.data.size)), np.ones(N), normalize=True)
    return eng, dict(inputs, walker_dims=None)


CASES = {
    "chain64": chain64_case,
    "snake6x6": lambda: lattice_case(workloads.snake6x6(Nw=4), [16, 32, 64, 128]),
    "snake8x8": lambda: lattice_case(workloads.snake8x8(Nw=2) if workloads.snake8x8().has_trial()
                                     else workloads.snake8x8_random(Nw=2), [64, 64]),
}


@pytest.mark.parametrize("precision", [PRECISION_FP64, PRECISION_TF32X3, PRECISION_TF32X3_TC],
                         ids=["fp64", "tf32x3", "tf32x3_tc"])
@pytest.mark.parametrize("case", list(CASES))
def test_bench_shape_step_matches_oracle(case, precision):
    if precision == PRECISION_TF32X3_TC and case == "snake6x6":
        pytest.skip("the tcgen05 sweep runs populations of one bond profile (snake6x6 mixes four)")
    eng, inp = CASES[case]()
    if case == "chain64" and precision == PRECISION_FP64:
        assert eng.get_option(OPT_WORKSPACE) == WORKSPACE_AUTO  # work buffers in shared memory
    eng.set_option(OPT_PRECISION, precision)
    eng.set_rng(SEED, 0)
    w0, wt0, _, _ = eng.get_walkers()
    dims = eng.get_walker_dims()
    N = w0.shape[0]
    eng.walk(1)
    lw = eng.last_step_walkers()
    nC = len(inp["ci"])
    uni = ew.uniforms(SEED, 0, N * nC)
    tol = TOL[precision] if (precision == PRECISION_FP64 or case == "chain64") else LATTICE_TOL_FP32
    for w in range(N):
        size = int(np.sum(dims[w][:-1] * dims[w][1:]) * 2)
        r = ew.step(inp["trial_dims"], inp["trial"], dims[w], w0[w, :size], wt0[w], ci=inp["ci"], cj=inp["cj"],
                    cJ=inp["cJ"], Jvals=inp["Jvals"], U=inp["U"], S=inp["S"], VT=inp["VT"], grid=inp["grid"],
                    dtau=inp["dtau"], u=uni[w * nC:(w + 1) * nC])
        for k in ("weight", "overlap", "energy"):
            assert lw[k][w] == pytest.approx(r[k], rel=tol), (case, w, k)
    eng.close()


def test_tc_sweep_follows_the_fp64_walk_at_the_headline_shape():
    """Config 5's shapes (8x8 lattice, D_T = 256 trial, D_W = 64): from the same start and random
    stream, the tcgen05 sweep's population follows the FP64 sweep's step by step and its E_P stays
    within half the energy criterion (1e-4 J per site) of the FP64 value.  The three-pass products
    are FP32-accurate per term; through the 64-site chains of contractions the local energies
    carry about 1e-5 relative rounding (2.8e-5 relative, 1.7e-5 J per site, measured on E_P)."""
    wl = workloads.snake8x8(Nw=64) if workloads.snake8x8().has_trial() else workloads.snake8x8_random(Nw=64)
    ci, cj, cJ = wl.couplings()
    trial = wl.trial()
    U, S, VT = pb.trotter_tables(1.0, wl.dtau)
    N = 64
    inputs = dict(L=wl.L, ci=ci, cj=cj, cJ=cJ, h=0.0, dtau=wl.dtau, trial_dims=trial.dims, trial=trial.data,
                  Jvals=[1.0], U=U, S=S, VT=VT, grid=pb.grid_marsaglia(4, 4), Ndesired=N, capacity=256)
    w = pb.compress(trial, 64)
    rng = np.random.default_rng(3)
    start = w.data[None, :] + 1e-3 * rng.normal(size=(N, w.data.size))
    runs = []
    for precision in (PRECISION_FP64, PRECISION_TF32X3_TC):
        eng = Engine(walker_dims=w.dims, **inputs)
        eng.set_walkers(start, np.ones(N), normalize=True)
        eng.set_option(OPT_PRECISION, precision)
        eng.set_rng(SEED, 0)
        runs.append(eng.walk(4))
        eng.close()
    for step, (x, y) in enumerate(zip(*runs)):
        print(f"step {step}: E_P {x['E_P']:.10f} / {y['E_P']:.10f}, per site {abs(y['E_P'] - x['E_P']) / wl.L:.2e}, "
              f"sum w rel {abs(y['sum_weight'] / x['sum_weight'] - 1):.2e}")
        assert x["n_walkers"] == y["n_walkers"]
        assert abs(y["E_P"] - x["E_P"]) / wl.L < 5e-5
        assert y["sum_weight"] == pytest.approx(x["sum_weight"], rel=1e-4)
