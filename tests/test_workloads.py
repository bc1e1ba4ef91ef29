"""The canonical FLOP count behind every roofline figure (mpsqmc_b200/workloads.py): its terms by
hand on small cases, and the chain64 value the bench reports (0.796 GFLOP per walker-step)."""
import numpy as np
import pytest

from mpsqmc_b200 import problem as pb
from mpsqmc_b200 import workloads as wk


def test_transfer_step_cost_takes_the_cheaper_order():
    # T = 2d min(b_l a_r (a_l + b_r), a_l b_r (b_l + a_r))
    assert wk.site_flops(64, 64, 32, 32) == 4 * min(32 * 64 * 96, 64 * 32 * 96)
    assert wk.site_flops(8, 16, 4, 2) == 4 * min(4 * 16 * (8 + 2), 8 * 2 * (4 + 16))


def test_chain_mpo_has_eight_entries_per_bulk_site():
    L = 10
    nnz = wk.mpo_nnz(L, {(k, k + 1) for k in range(L - 1)})
    assert nnz[1:-1] == [8] * (L - 2)
    assert nnz[0] == 4 and nnz[-1] == 4  # identity + opened channel; done + closed channel


def test_nearest_neighbour_chain_has_no_invalidated_environments():
    """On a chain every coupling (i, i+1) finds R[i+2] valid: the count is exactly
    sum_i (9 T_i + 32 a b + QR_i + QR_{i+1}) + sum T + sum nnz T."""
    L, D = 8, 4
    aT = pb.virtual_dims(L, D)
    bW = aT
    cpl = [(k, k + 1) for k in range(L - 1)]
    T = [wk.site_flops(aT[k], aT[k + 1], bW[k], bW[k + 1]) for k in range(L)]

    def qr(k):
        m, n = 2 * bW[k], bW[k + 1]
        return 4 * m * n * n - (4.0 / 3.0) * n ** 3 + 4 * n ** 3

    expect = sum(9 * T[i] + 32 * aT[i + 1] * bW[i + 1] + qr(i) + qr(i + 1) for i, _ in cpl)
    expect += sum(T) + sum(n * t for n, t in zip(wk.mpo_nnz(L, set(cpl)), T))
    assert wk.algorithmic_flops_per_walker_step(aT, bW, cpl) == pytest.approx(expect, rel=1e-14)


def test_long_range_coupling_pays_for_the_middle_sites_and_stale_environments():
    """(0, 3) then (1, 2): the first carries its branches through g - 1 = 2 middle sites; the second
    needs R[3], which the change of site 3 invalidated (r_c = 4 - 3 = 1)."""
    L, D = 5, 2
    aT = pb.virtual_dims(L, D)
    bW = aT
    base = wk.algorithmic_flops_per_walker_step(aT, bW, [])
    T = [wk.site_flops(aT[k], aT[k + 1], bW[k], bW[k + 1]) for k in range(L)]
    both = wk.algorithmic_flops_per_walker_step(aT, bW, [(0, 3), (1, 2)])
    one = wk.algorithmic_flops_per_walker_step(aT, bW, [(0, 3)])
    nnz_both = wk.mpo_nnz(L, {(0, 3), (1, 2)})
    nnz_one = wk.mpo_nnz(L, {(0, 3)})
    energy = lambda nnz: sum(n * t for n, t in zip(nnz, T))  # noqa: E731
    coupling_03 = one - base - energy(nnz_one) + energy(wk.mpo_nnz(L, set()))
    coupling_12 = both - one - energy(nnz_both) + energy(nnz_one)
    q = lambda k: 4 * (2 * bW[k]) * bW[k + 1] ** 2 - (4.0 / 3.0) * bW[k + 1] ** 3 + 4 * bW[k + 1] ** 3  # noqa: E731
    assert coupling_03 == pytest.approx((5 * 3 + 4) * T[0] + 32 * aT[1] * bW[1] + q(0) + q(3), rel=1e-14)
    assert coupling_12 == pytest.approx((5 * 1 + 4 + 1) * T[1] + 32 * aT[2] * bW[2] + q(1) + q(2), rel=1e-14)


def test_chain64_count_is_the_reported_one():
    wl = wk.chain64(Nw=4)
    inp = wl.inputs()
    cpl = list(zip(inp["ci"], inp["cj"]))
    f = wk.algorithmic_flops_per_walker_step(inp["trial_dims"], inp["walker_dims"], cpl)
    assert f == pytest.approx(796283536.0, rel=1e-9)
    assert 0.7e9 < f < 1.0e9  # the rough 0.9 GFLOP per walker-step of the configuration
    assert np.all(np.diff(inp["ci"]) == 1) and np.all(np.asarray(inp["cj"]) - np.asarray(inp["ci"]) == 1)
