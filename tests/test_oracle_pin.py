"""The CPU oracle (oracle/mpsqmc_oracle.cpp) against outputs of the reference itself.

Fixtures under tests/golden/ were produced by the reference's own C++ (tests/golden/make_golden.py).
These checks pin the oracle before it is trusted as the checker of the CUDA engine.
"""
import numpy as np
import pytest

from conftest import WALK_CASES, couplings, load_golden
from oracle import pyoracle as po


def test_grid_marsaglia_matches_reference():
    g = load_golden("grids")["marsaglia4"]
    mine = po.grid_marsaglia(4, 4)
    assert mine.shape == g.shape == (240, 4)
    np.testing.assert_allclose(mine, g, rtol=0, atol=1e-15)
    # isotropy: sum_p x x^T = G/dim * I (GridGenerator.cpp:93-102)
    np.testing.assert_allclose(g.T @ g, 60.0 * np.eye(4), atol=1e-12)


def test_grid_simple_matches_reference():
    g = load_golden("grids")["simple4"]
    mine = po.grid_simple(4, 4)
    assert mine.shape == g.shape
    np.testing.assert_allclose(mine, g, rtol=0, atol=1e-15)


@pytest.mark.parametrize("key", ["dt0.01_J1.0", "dt0.005_J1.0", "dt0.01_J0.5", "dt0.3_J1.0", "dt0.5_J1.0"])
def test_trotter_tables_match_reference(key):
    z = load_golden("trotter")
    dt = float(key.split("_")[0][2:])
    J = float(key.split("_")[1][1:])
    U, S, VT = po.trotter(J, dt)
    np.testing.assert_allclose(S, z[key + "_S"], rtol=1e-13, atol=1e-15)

    def recon(U, S, VT):
        return U.reshape(4, 4, order="F") @ np.diag(S) @ VT.reshape(4, 4, order="F")

    np.testing.assert_allclose(recon(U, S, VT), recon(z[key + "_U"], z[key + "_S"], z[key + "_VT"]),
                               atol=1e-14)


def _mps(z, prefix):
    return po.MPS(z[prefix + "_dims"].astype(np.int32), z[prefix + "_data"])


def test_inner_product_and_left_normalize_match_reference():
    z = load_golden("mpsops_debug")
    sc = z["scalars"]
    trial = _mps(z, "trial")
    other = _mps(z, "other")
    assert po.inner_product(trial, trial) == pytest.approx(sc[0], rel=1e-13)
    ln, r = po.left_normalize(trial)
    assert r == pytest.approx(sc[1], rel=1e-13)
    ref_ln = _mps(z, "leftnorm")
    np.testing.assert_array_equal(ln.dims, ref_ln.dims)
    # element by element: same Householder conventions as dgeqrf/dorgqr
    np.testing.assert_allclose(ln.data, ref_ln.data, rtol=0, atol=1e-13)
    assert po.inner_product(trial, other) == pytest.approx(sc[2], rel=1e-12)
    assert po.inner_product(other, trial) == pytest.approx(sc[3], rel=1e-12)
    oln, r2 = po.left_normalize(other)
    assert r2 == pytest.approx(sc[4], rel=1e-12)
    np.testing.assert_allclose(oln.data, _mps(z, "other_leftnorm").data, rtol=0, atol=1e-12)
    assert po.inner_product(ln, oln) == pytest.approx(sc[5], rel=1e-12)


def test_site_operators_match_reference():
    z = load_golden("mpsops_debug")
    ln = _mps(z, "leftnorm")
    tr = load_golden("trotter")
    U, S, VT = tr["dt0.01_J1.0_U"], tr["dt0.01_J1.0_S"], tr["dt0.01_J1.0_VT"]
    g = load_golden("grids")["marsaglia4"]
    got = po.apply_grid_op(ln, 1, 2, S, U, VT, g[37])
    np.testing.assert_allclose(got.data, _mps(z, "gridop_1_2_37").data, rtol=0, atol=1e-14)
    got = po.apply_svd_op(ln, 2, 3, S, U, VT, 1, 3, hc=True)
    np.testing.assert_allclose(got.data, _mps(z, "svdop_2_3_1_3_hc").data, rtol=0, atol=1e-15)
    ph = po.change_phase(ln)
    assert po.inner_product(ph, ln) == pytest.approx(z["scalars"][8], rel=1e-13)


def test_compress_is_the_same_state_as_reference():
    """SVD signs differ between LAPACK and the oracle's Jacobi SVD; the state does not."""
    z = load_golden("mpsops_debug")
    ln = _mps(z, "leftnorm")
    ref = _mps(z, "compressed")
    mine = po.compress(ln, 2)
    np.testing.assert_array_equal(mine.dims, ref.dims)
    f = po.inner_product(mine, ref) / np.sqrt(po.inner_product(mine, mine) * po.inner_product(ref, ref))
    assert abs(f) == pytest.approx(1.0, abs=1e-12)
    assert po.inner_product(ln, mine) == pytest.approx(z["scalars"][6], rel=1e-10)


def _walk_oracle(z, trace=True):
    meta = z["meta"]
    trial = po.MPS(z["trial_ln_dims"], z["trial_ln_data"])
    w0 = po.MPS(z["walker0_init_dims"], z["walker0_init_data"])
    L, N = meta["L"], meta["Nw"]
    ci, cj, cJ = couplings(z)
    walkers = np.tile(w0.data, (N, 1))
    return po.walk(trial, walkers, w0.dims, z["init_weight"], z["init_overlap"], np.zeros(N), ci=ci, cj=cj,
                   cJ=cJ, Jvals=np.array([1.0]), U=z["U"], S=z["S"], VT=z["VT"], grid=z["grid"],
                   dtau=meta["dtau"], nsteps=meta["steps"], Ndesired=N, capacity=max(1000, 3 * N),
                   seed=meta["seed"], skip=meta["setup_draws"], trace=trace, h=meta.get("h", 0.0))


@pytest.mark.parametrize("case", WALK_CASES)
def test_walk_trajectory_matches_reference(case):
    z = load_golden(case)
    meta = z["meta"]
    res = _walk_oracle(z)
    assert res.status == 0
    assert res.E0 == pytest.approx(meta["E0"], rel=1e-12)
    np.testing.assert_array_equal(res.n, z["stat_n"])
    np.testing.assert_allclose(res.sumw, z["stat_sumw"], rtol=1e-12)
    np.testing.assert_allclose(res.EP, z["stat_EP"], rtol=1e-12)
    np.testing.assert_allclose(res.ET, z["stat_ET"], rtol=1e-10, atol=1e-10)
    # the fluctuation metric is a difference of nearly equal sums: absolute scale E^2
    np.testing.assert_allclose(res.omega, z["stat_omega"], rtol=0, atol=1e-9 * np.max(np.abs(z["stat_EP"])) ** 2)
    for s in range(1, meta["steps"] + 1):
        p = f"step{s:03d}_"
        n = len(z[p + "weight"])
        np.testing.assert_allclose(res.weight[s - 1, :n], z[p + "weight"], rtol=1e-12)
        np.testing.assert_allclose(res.overlap[s - 1, :n], z[p + "overlap"], rtol=1e-12)
        np.testing.assert_allclose(res.energy[s - 1, :n], z[p + "energy"], rtol=1e-12)
        np.testing.assert_array_equal(res.parent[s - 1, :len(z[p + "parent"])], z[p + "parent"])
        tr = res.trace[s - 1, :n].reshape(-1, 21)
        np.testing.assert_array_equal(tr[:, 18].astype(int), z[p + "trace_index"])
        np.testing.assert_array_equal(tr[:, 17], z[p + "trace_u"])
        np.testing.assert_allclose(tr[:, :16], z[p + "trace_C"], rtol=0, atol=1e-13)
    last = f"step{meta['steps']:03d}_tensors"
    # walkers after the last branching are copies of pre-branching ones
    par = z[f"step{meta['steps']:03d}_parent"]
    # 5 steps x 24 couplings of QR sweeps accumulate roundoff in the tensors (LAPACK vs the
    # restated Householder): 1e-11 absolute on entries of order 1
    np.testing.assert_allclose(res.walkers, z[last][par], rtol=0, atol=1e-11)
    draws = int(np.sum(z["stat_draws"]))
    assert res.draws == draws


def test_ed_pins_reference_value():
    """main.cpp:153: E_FCI of the L=10 spin-1/2 chain = -4.25803520728288."""
    from oracle import ed
    assert ed.ground_energy(10) == pytest.approx(-4.25803520728288, abs=1e-11)


def test_dmrg_trials_are_variational():
    from oracle import ed
    z = load_golden("trials")
    for L, D in [(8, 4), (10, 8), (16, 16)]:
        e = float(z[f"L{L}D{D}_energy"])
        e0 = ed.ground_energy(L)
        assert e0 <= e + 1e-10
        assert e - e0 < 1e-2


def test_2d_trials_against_ed():
    """Reference DMRG trials of the open 3x3 and 4x4 snake lattices are variational; 4x4 ED is
    the known -9.189207065 of the open 4x4 Heisenberg model."""
    from oracle import ed
    from mpsqmc_b200 import problem as pb
    z = load_golden("trials2d")
    e44 = ed.ground_energy_couplings(16, *pb.snake(4, 4))
    assert e44 == pytest.approx(-9.189207065192948, abs=1e-9)
    for W, H, D in [(3, 3, 8), (4, 4, 16)]:
        e0 = ed.ground_energy_couplings(W * H, *pb.snake(W, H))
        e = float(z[f"snake{W}x{H}D{D}_energy"])
        assert e0 - 1e-10 <= e < e0 + 0.1


def test_snake_couplings_match_reference_list():
    from mpsqmc_b200 import problem as pb
    for case, (W, H) in [("walk_snake3x3_D8_DW4", (3, 3)), ("walk_snake4x4_D16_DW8_branch", (4, 4))]:
        z = load_golden(case)
        ci, cj, cJ = pb.snake(W, H)
        np.testing.assert_array_equal(ci, z["coup_i"])
        np.testing.assert_array_equal(cj, z["coup_j"])
        np.testing.assert_array_equal(cJ, z["coup_J"])


def test_compact_mpo_of_any_couplings():
    """mpsqmc_b200.dmrg.coupling_mpo: on a chain it is the chain MPO; on the 3x3 snake its
    <m|H|m> is the oracle's energy numerator of the same (left-normalised) state."""
    import numpy as np
    from mpsqmc_b200 import dmrg, problem as pb
    from oracle import pyoracle as po
    rng = np.random.default_rng(1)

    def rand_mps(L, D):
        dims = pb.virtual_dims(L, D)
        return pb.MPS(dims, rng.normal(size=int(sum(dims[k] * dims[k + 1] * 2 for k in range(L)))))

    ci, cj, cJ = pb.chain(6)
    m = rand_mps(6, 4)
    assert dmrg.mpo_energy(m, dmrg.coupling_mpo(6, ci, cj, cJ, 0.3)) == pytest.approx(
        dmrg.mpo_energy(m, dmrg.chain_mpo(6, cJ, 0.3)), rel=1e-13)
    ci, cj, cJ = pb.snake(3, 3)
    ln = pb.left_normalize(rand_mps(9, 4))
    e = po.energy_numerator(po.MPS(ln.dims, ln.data), po.MPS(ln.dims, ln.data), ci, cj, cJ)
    assert dmrg.mpo_energy(ln, dmrg.coupling_mpo(9, ci, cj, cJ)) == pytest.approx(e, rel=1e-12)


def test_lattice_dmrg_reaches_ed():
    """Two-site DMRG with the compact MPO of the open 3x3 snake lattice at D = 16 (exact bond
    dimension) reaches the ED ground energy; the 4x4 at D = 16 stays variational and close."""
    from mpsqmc_b200 import dmrg, problem as pb
    from oracle import ed
    c33 = pb.snake(3, 3)
    _, e = dmrg.dmrg(9, 16, couplings=c33)
    assert e == pytest.approx(ed.ground_energy_couplings(9, *c33), abs=1e-9)
    c44 = pb.snake(4, 4)
    m, e = dmrg.dmrg(16, 16, couplings=c44)
    e0 = -9.189207065192948
    assert e0 - 1e-10 <= e < e0 + 0.1
    assert dmrg.mpo_energy(m, dmrg.coupling_mpo(16, *c44)) == pytest.approx(e, rel=1e-9)


@pytest.mark.parametrize("name", ["snake6x6_dmrg", "snake8x8_dmrg"])
def test_stored_lattice_trial_is_the_dmrg_state(name):
    """The lattice workloads' stored trials: left-normalised, bond dims within D_T = 64, and the
    energy under the lattice's compact MPO is the stored DMRG energy (a variational bound)."""
    import numpy as np
    from mpsqmc_b200 import dmrg, workloads
    wl = getattr(workloads, name)()
    m = wl.trial()
    assert m.L == wl.L and int(max(m.dims)) == wl.DT
    e = dmrg.mpo_energy(m, dmrg.coupling_mpo(wl.L, *wl.couplings()))
    assert e == pytest.approx(wl.trial_energy(), rel=1e-9)
    assert -0.62 * wl.L < e < -0.55 * wl.L
    for k in range(m.L - 1):
        A = m.site(k)  # [sigma, Dl, Dr]
        G = sum(A[s].T @ A[s] for s in range(2))
        np.testing.assert_allclose(G, np.eye(G.shape[0]), atol=1e-10)


def test_stored_d256_trial_is_left_normalised():
    """The 8x8 D_T = 256 trial (grown on the GPU by dmrg.dmrg_device, stored in FP32 and
    left-normalised again in FP64 on load): bond profile and left-canonical sites.  Its energy
    under the compact MPO equals the stored one (checked once when it was made: the host
    contraction at D = 256 takes minutes)."""
    import numpy as np
    from mpsqmc_b200 import workloads
    wl = workloads.snake8x8()
    m = wl.trial()
    np.testing.assert_array_equal(m.dims, workloads.pb.virtual_dims(64, 256))
    for k in (0, 7, 8, 31, 56, 62):
        A = m.site(k)
        G = sum(A[s].T @ A[s] for s in range(2))
        np.testing.assert_allclose(G, np.eye(G.shape[0]), atol=1e-10)
    assert -0.62 * wl.L < wl.trial_energy() < -0.61 * wl.L
