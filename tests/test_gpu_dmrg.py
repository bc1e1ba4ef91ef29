"""The two-site compact-MPO DMRG with its contractions, Lanczos vectors and SVDs on the GPU
(dmrg.dmrg_device; set-up code that makes the D_T = 256 trial of the 8x8 lattice) against exact
diagonalisation: the L = 10 chain of main.cpp:153 and open 3x3 / 4x4 lattices on the snake path,
and a run grown from a stored smaller-bond trial."""
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


@pytest.mark.parametrize("W,H,D", [(3, 3, 16), (4, 4, 32)])
def test_device_dmrg_lattice_matches_ed(W, H, D):
    ci, cj, cJ = pb.snake(W, H)
    L = W * H
    m, e = dmrg.dmrg_device(L, D, couplings=(ci, cj, cJ))
    e_ed = ed.ground_energy_couplings(L, ci, cj, cJ)
    assert e == pytest.approx(e_ed, abs=2e-7 * L)
    assert dmrg.mpo_energy(m, dmrg.coupling_mpo(L, ci, cj, cJ)) == pytest.approx(e, abs=1e-9 * L)


def test_device_dmrg_grows_a_stored_trial():
    ci, cj, cJ = pb.snake(4, 4)
    small, e_small = dmrg.dmrg(16, 4, couplings=(ci, cj, cJ), sweeps=2)
    m, e = dmrg.dmrg_device(16, 32, couplings=(ci, cj, cJ), init=small)
    assert max(m.dims) > 4
    assert e < e_small - 1e-3
    assert e == pytest.approx(ed.ground_energy_couplings(16, ci, cj, cJ), abs=1e-5)
