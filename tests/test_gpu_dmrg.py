"""The two-site compact-MPO DMRG with its contractions, Lanczos vectors and SVDs on the GPU
(dmrg.dmrg_device; set-up code that makes the D_T = 256 trial of the 8x8 lattice) against exact
diagonalisation (the L = 10 chain of main.cpp:153, the open 3x3 lattice on the snake path) and
against the host solver on the truncated 4x4, and a run grown from a smaller-bond trial."""
import numpy as np
import pytest

from mpsqmc_b200 import dmrg
from mpsqmc_b200 import problem as pb
from oracle import ed

pytestmark = pytest.mark.gpu


def test_device_dmrg_chain_matches_main_cpp_value():
    m, e = dmrg.dmrg_device(10, 32)
    assert e == pytest.approx(-4.25803520728288, abs=1e-9)
    assert dmrg.mpo_energy(m, dmrg.chain_mpo(10, np.ones(9))) == pytest.approx(e, abs=1e-9)


def test_device_dmrg_3x3_matches_ed():
    ci, cj, cJ = pb.snake(3, 3)
    m, e = dmrg.dmrg_device(9, 16, couplings=(ci, cj, cJ))  # D = 16 is exact for L = 9
    assert e == pytest.approx(ed.ground_energy_couplings(9, ci, cj, cJ), abs=1e-8)
    assert dmrg.mpo_energy(m, dmrg.coupling_mpo(9, ci, cj, cJ)) == pytest.approx(e, abs=1e-8)


def test_device_dmrg_4x4_matches_host_dmrg():
    """At D = 16 the 4x4 state is truncated: the device run and the host solver (same sweeps and
    truncation, scipy Lanczos) reach the same variational energy above the ED ground energy."""
    ci, cj, cJ = pb.snake(4, 4)
    _, e_host = dmrg.dmrg(16, 16, couplings=(ci, cj, cJ))
    m, e = dmrg.dmrg_device(16, 16, couplings=(ci, cj, cJ))
    e_ed = ed.ground_energy_couplings(16, ci, cj, cJ)
    assert e_ed - 1e-9 <= e < e_ed + 0.1
    assert e == pytest.approx(e_host, abs=1e-6)
    assert dmrg.mpo_energy(m, dmrg.coupling_mpo(16, ci, cj, cJ)) == pytest.approx(e, abs=1e-8)


def test_device_dmrg_grows_a_stored_trial():
    ci, cj, cJ = pb.snake(4, 4)
    small, e_small = dmrg.dmrg(16, 4, couplings=(ci, cj, cJ), sweeps=2)
    m, e = dmrg.dmrg_device(16, 32, couplings=(ci, cj, cJ), init=small)
    assert max(m.dims) > 4
    e_ed = ed.ground_energy_couplings(16, ci, cj, cJ)
    assert e_ed - 1e-9 <= e < e_small - 1e-3
    assert e < e_ed + 0.02
