"""The reference-compatible C++ classes (mpsqmc_b200/host) against the reference's own outputs,
and the drop-in check: the reference's main.cpp compiles and links unchanged against them."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, load_golden
from mpsqmc_b200 import build
from oracle import ed
from oracle import pyoracle as po

HOST_INC = os.path.join(ROOT, "mpsqmc_b200", "host", "include")
PKG = os.path.join(ROOT, "mpsqmc_b200")
REF_DIR = po.ref_dir() or ""


def compile_cpp(src: str, out: str) -> str:
    build.build_host()
    cmd = ["g++", "-std=c++17", "-O2", "-I", HOST_INC, src, "-L", PKG, "-lmpsqmc_host", "-lmpsqmc_b200",
           f"-Wl,-rpath,{PKG}", "-o", out]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


@pytest.fixture(scope="module")
def selftest(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("host") / "host_selftest")
    compile_cpp(os.path.join(ROOT, "tests", "cpp", "host_selftest.cpp"), exe)

    def run(*args):
        r = subprocess.run([exe, *map(str, args)], check=True, capture_output=True, text=True,
                           env={**os.environ, "MPSQMC_SEED": "7"})
        return json.loads(r.stdout)
    return run


def test_grids_match_reference(selftest):
    g = load_golden("grids")
    out = selftest("grid")
    np.testing.assert_allclose(np.array(out["marsaglia"]).reshape(-1, 4), g["marsaglia4"], atol=1e-15)
    np.testing.assert_allclose(np.array(out["simple"]).reshape(-1, 4), g["simple4"], atol=1e-15)


@pytest.mark.parametrize("dt,J", [(0.01, 1.0), (0.005, 1.0), (0.01, 0.5)])
def test_trotter_tables_reconstruct_reference(selftest, dt, J):
    z = load_golden("trotter")
    key = f"dt{dt}_J{J}"
    out = selftest("trotter", dt, J)
    np.testing.assert_allclose(out["S"], z[key + "_S"], rtol=1e-13)
    rec = lambda U, S, VT: np.reshape(U, (4, 4), order="F") @ np.diag(S) @ np.reshape(VT, (4, 4), order="F")
    np.testing.assert_allclose(rec(out["U"], out["S"], out["VT"]), rec(z[key + "_U"], z[key + "_S"], z[key + "_VT"]),
                               atol=1e-14)


def test_mps_algebra_matches_reference(selftest):
    z = load_golden("mpsops_debug")
    with tempfile.TemporaryDirectory() as t:
        path = os.path.join(t, "trial.mps")
        po.write_mps(path, po.MPS(z["trial_dims"], z["trial_data"]))
        out = selftest("mpsops", path, 2)
    sc = z["scalars"]
    assert out["scalars"][0] == pytest.approx(sc[0], rel=1e-13)       # InnerProduct
    assert out["scalars"][1] == pytest.approx(sc[1], rel=1e-13)       # LeftNormalize's last R
    np.testing.assert_allclose(out["leftnorm"], z["leftnorm_data"], atol=1e-13)  # same Householder signs
    np.testing.assert_array_equal(out["compressed_dims"], z["compressed_dims"])
    assert out["scalars"][2] == pytest.approx(sc[6], rel=1e-10)       # <ln|compressed>
    assert out["scalars"][4] == pytest.approx(sc[0], rel=1e-12)       # RightNormalize keeps the state


def test_dmrg_reaches_reference_energy(selftest):
    out = selftest("dmrg", 10, 8)
    E, E_mpo, E_comp = out["energies"]
    ref = float(load_golden("trials")["L10D8_energy"])
    assert E == pytest.approx(ref, abs=2e-7)
    assert E >= ed.ground_energy(10) - 1e-10
    assert E_mpo == pytest.approx(E, rel=1e-9)      # ApplyMPO + InnerProduct
    assert E_comp == pytest.approx(E, rel=1e-9)     # after the lossless CompressState


def test_mpo_energy_matches_oracle(selftest):
    z = load_golden("trials")
    with tempfile.TemporaryDirectory() as t:
        path = os.path.join(t, "trial.mps")
        m = po.MPS(z["L16D16_dims"], z["L16D16_data"])
        po.write_mps(path, m)
        out = selftest("energy", path)
    ln, _ = po.left_normalize(m)
    ci, cj, cJ = po.chain_couplings(16)
    e = po.energy_numerator(ln, ln, ci, cj, cJ)
    assert out["energies"][0] == pytest.approx(e, rel=1e-11)
    assert out["energies"][1] == pytest.approx(e, rel=1e-11)
    assert e == pytest.approx(float(z["L16D16_energy"]), rel=1e-11)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_DIR, "main.cpp")), reason="MPSQMC_REF_DIR (the reference tree) not set")
def test_reference_main_links_unchanged(tmp_path):
    """The reference's own main.cpp builds against these headers and libraries without edits."""
    exe = compile_cpp(os.path.join(REF_DIR, "main.cpp"), str(tmp_path / "main_dropin"))
    assert os.path.getsize(exe) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("options", [{}, {"MPSQMC_PRECISION": "tf32x3", "MPSQMC_CANONICAL_INTERVAL": "4"}])
def test_dropin_walk_runs_main_call_sequence(tmp_path, options):
    """main.cpp's call sequence (MPSstate from file, HeisenbergMPO, Marsaglia grid, MPSQMC2::Walk)
    on the GPU engine: console lines and the energy file of the reference, energies of the trial.
    Engine options reach an unchanged caller through the environment."""
    exe = compile_cpp(os.path.join(ROOT, "tests", "cpp", "dropin_walk.cpp"), str(tmp_path / "dropin_walk"))
    z = load_golden("trials")
    po.write_mps(str(tmp_path / "trial.mps"), po.MPS(z["L10D8_dims"], z["L10D8_data"]))
    (tmp_path / "output" / "Heisenberg1D").mkdir(parents=True)
    steps, N = 6, 16
    r = subprocess.run([exe, "trial.mps", "4", str(N), "0.05", str(steps)], cwd=tmp_path, capture_output=True,
                       text=True, env={**os.environ, "MPSQMC_SEED": "20131015", **options}, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "GPU engine unavailable" not in r.stderr and "MPSQMC::Walk" not in r.stderr
    assert "ignoring" not in r.stderr
    meta = load_golden("walk_L10D8_DW4")["meta"]
    E0 = float(r.stdout.split("Energy at start = ")[1].split()[0])
    assert E0 == pytest.approx(meta["E0"], rel=1e-10)    # same trial, same compressed walkers
    lines = (tmp_path / "output" / "Heisenberg1D" / "ener_L10DT8DW4.txt").read_text().splitlines()
    assert lines[0].startswith("#Step")
    rows = [ln.split() for ln in lines[1:]]
    assert [int(x[0]) for x in rows] == list(range(1, steps + 1))
    assert all(int(x[1]) > 0 for x in rows)
    EP = np.array([float(x[2]) for x in rows])
    assert np.all(np.abs(EP - ed.ground_energy(10)) < 5e-3)   # projected energies stay at the ground state
    assert r.stdout.count("        Step = ") == steps
    assert "The min. encountered weight on rank 0 is" in r.stdout


@pytest.mark.gpu
def test_dropin_legacy_projector(tmp_path):
    """MPSQMC (the MPO-term projector class) over the engine: DMRG trial on the host, walk on the
    GPU, the reference's console lines and energies.txt; energies stay at the ground state."""
    exe = compile_cpp(os.path.join(ROOT, "tests", "cpp", "dropin_legacy.cpp"), str(tmp_path / "dropin_legacy"))
    steps = 5
    r = subprocess.run([exe, "10", "8", "32", "0.05", str(steps), "0.0"], cwd=tmp_path, capture_output=True,
                       text=True, env={**os.environ, "MPSQMC_SEED": "11"}, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "GPU engine unavailable" not in r.stderr and "MPSQMC::Walk" not in r.stderr
    lines = (tmp_path / "energies.txt").read_text().splitlines()
    assert lines[0].startswith("#Step") and len(lines) == steps + 1
    EP = np.array([float(x.split()[1]) for x in lines[1:]])
    assert np.all(np.abs(EP - ed.ground_energy(10)) < 5e-3)
    assert r.stdout.count("        Step = ") == steps
