"""Learned auxiliary-field proposal: the device network against the CPU oracle, its online
training, and what it changes in the walk.

The grid PDF P(x) of one coupling is the zero-variance proposal for that coupling's weight
factor: drawing x from P / sum P multiplies the weight by sum P whatever x is.  The learned
proposal q~ reweights by P(x) / q~(x), whose mean over x ~ q~ is again sum P (unbiased) and whose
spread is what q~ loses against P / sum P.  The walk draws from the defensive mixture
q_mix = (1 - alpha) q~ + alpha P / sum P (MPSQMC_OPT_PROPOSAL_MIX), which bounds the factor by
sum P / alpha.  The tests check the forward pass, loss and gradient against oracle/mlp.py, that
online training drives the loss down, that a trained network's weight factors scatter far less
around sum P than an untrained one's, and the mixture's bound.
"""
import numpy as np
import pytest

from conftest import couplings, load_golden
from mpsqmc_b200 import Engine
from mpsqmc_b200.capi import (E_ARG, OPT_CANONICAL_INTERVAL, OPT_PROPOSAL, OPT_PROPOSAL_MIX, OPT_PROPOSAL_TRAINING,
                              PROPOSAL_GRID, PROPOSAL_LEARNED, MpsqmcError)
from oracle import mlp

pytestmark = pytest.mark.gpu


def chain_engine(n_walkers=256, seed_skip=0):
    z = load_golden("walk_L16D16_DW16")
    meta = z["meta"]
    L = meta["L"]
    ci, cj, cJ = couplings(z)
    eng = Engine(L=L, ci=ci, cj=cj, cJ=cJ, h=0.0, dtau=meta["dtau"], trial_dims=z["trial_ln_dims"],
                 trial=z["trial_ln_data"], Jvals=[1.0], U=z["U"], S=z["S"], VT=z["VT"], grid=z["grid"],
                 Ndesired=n_walkers, capacity=3 * n_walkers, walker_dims=z["walker0_init_dims"])
    rng = np.random.default_rng(7)
    w0 = z["walker0_init_data"]
    walkers = w0[None, :] + 1e-3 * rng.standard_normal((n_walkers, w0.size))
    eng.set_walkers(walkers, np.ones(n_walkers), None, np.zeros(n_walkers), normalize=True)
    eng.set_rng(meta["seed"], seed_skip)
    return eng, z


def test_forward_loss_and_gradient_match_oracle():
    eng, z = chain_engine(n_walkers=64)
    G = z["grid"].shape[0]
    theta = mlp.init_params(G, seed=3) + 0.01 * np.random.default_rng(4).standard_normal(mlp.n_params(G))
    eng.proposal_params(theta.astype(np.float32))
    rng = np.random.default_rng(5)
    B = 64
    X = rng.standard_normal((B, mlp.N_IN)).astype(np.float32)
    logits = 2.0 * rng.standard_normal((B, G))
    logits[rng.random((B, G)) < 0.4] = -np.inf  # PDFs with zeros, as max(0, .) leaves them
    P = mlp.softmax(logits).astype(np.float32)
    loss, grad = eng.proposal_loss_grad(X, P)
    ref_loss, ref_grad = mlp.loss_grad(theta.astype(np.float32).astype(np.float64), X, P, G)
    assert loss == pytest.approx(ref_loss, rel=1e-4)
    scale = np.max(np.abs(ref_grad))
    np.testing.assert_allclose(grad, ref_grad, rtol=2e-3, atol=2e-5 * scale)


def weight_factors(eng, steps_before=0):
    """Per-walker weight factor of the first coupling of the next step (trace column 16)."""
    eng.set_trace(True)
    eng.walk(1)
    t = eng.get_trace()
    eng.set_trace(False)
    return t[:, 0, 16]


def test_online_training_lowers_the_loss_and_the_weight_spread():
    # grid walk with online training: one (features, PDF) pair per walker per step, one Adam step
    eng, z = chain_engine()
    eng.set_option(OPT_CANONICAL_INTERVAL, 1)
    eng.set_option(OPT_PROPOSAL_TRAINING, 1)
    losses = []
    for _ in range(60):
        eng.walk(1)
        losses.append(eng.proposal_stats()["loss"])
    assert eng.proposal_stats()["updates"] == 60
    assert losses[-1] < 0.3 * losses[0], (losses[0], losses[-1])
    trained = eng.proposal_params()

    # the same population state and uniforms, first coupling of the next step: grid pnorm vs the
    # learned factors of the trained and of an untrained network
    def factors(params, proposal):
        e, _ = chain_engine()
        e.set_option(OPT_CANONICAL_INTERVAL, 1)
        e.set_option(OPT_PROPOSAL_MIX, 0)  # the network's own proposal
        if params is not None:
            e.proposal_params(params)
        e.set_option(OPT_PROPOSAL, proposal)
        return weight_factors(e)

    pn = factors(None, PROPOSAL_GRID)
    r_trained = factors(trained, PROPOSAL_LEARNED) / pn
    r_untrained = factors(mlp.init_params(z["grid"].shape[0], seed=11).astype(np.float32), PROPOSAL_LEARNED) / pn
    n = len(pn)
    # unbiased: E[P(x) / q~(x)] = sum P
    for r in (r_trained, r_untrained):
        assert abs(np.mean(r) - 1.0) < 4.0 * np.std(r) / np.sqrt(n) + 1e-12
    assert np.std(r_trained) < 0.5 * np.std(r_untrained), (np.std(r_trained), np.std(r_untrained))


def test_defensive_mixture_bounds_the_weight_factor():
    """An untrained network through the default mixture (alpha = 0.1): every factor within
    sum P / alpha, still unbiased; alpha = 1 draws from P itself, so every factor is sum P."""
    def factors(mix):
        e, z = chain_engine()
        e.set_option(OPT_CANONICAL_INTERVAL, 1)
        if mix is not None:
            e.set_option(OPT_PROPOSAL_MIX, mix)
        assert e.get_option(OPT_PROPOSAL_MIX) == (100 if mix is None else mix)
        e.proposal_params(mlp.init_params(z["grid"].shape[0], seed=11).astype(np.float32))
        e.set_option(OPT_PROPOSAL, PROPOSAL_LEARNED)
        return weight_factors(e)

    e, _ = chain_engine()
    e.set_option(OPT_CANONICAL_INTERVAL, 1)
    pn = weight_factors(e)
    for bad in (-1, 1001):
        with pytest.raises(MpsqmcError) as ei:
            e.set_option(OPT_PROPOSAL_MIX, bad)
        assert ei.value.code == E_ARG
    r = factors(None) / pn
    assert np.all(r <= 10.0 * (1 + 1e-12)) and np.all(r > 0)
    assert abs(np.mean(r) - 1.0) < 4.0 * np.std(r) / np.sqrt(len(r)) + 1e-12
    r_net = factors(0) / pn
    assert np.std(r) < np.std(r_net)
    np.testing.assert_allclose(factors(1000), pn, rtol=1e-12)


def test_no_proposal_can_gain_more_than_the_weight_spread_allows():
    """The grid walk's per-step weights bound what ANY proposal could gain in variance of the
    weighted mean energy: at most N / N_eff = N sum w^2 / (sum w)^2 (all weights equal being the
    best case; mpsqmc_b200.analysis.proposal_gain_bound).  The bound is printed and recorded in
    the design notes next to the learned proposal's measured VN ratio, which stays below 1."""
    from mpsqmc_b200 import analysis
    eng, z = chain_engine()
    eng.walk(10)
    ws = []
    for _ in range(40):
        eng.walk(1)
        ws.append(eng.last_step_walkers()["weight"])
    bound = analysis.proposal_gain_bound(ws)
    print(f"proposal gain bound N/N_eff = {bound:.6f}")
    assert 1.0 <= bound < 2.0
    eng.close()
