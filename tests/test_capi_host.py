"""Host-side checks that need no GPU: the C-ABI library loads and exports what the header declares,
fails loudly without a device, and the host set-up code reproduces the reference's inputs."""
import os
import re
import tempfile

import numpy as np
import pytest

from conftest import ROOT, load_golden
from mpsqmc_b200 import capi
from mpsqmc_b200 import problem as pb
from oracle import pyoracle as po


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "mpsqmc_gpu.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(mpsqmc_[a-z_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(capi.EXPORTED)
    assert b"sm_100a" in lib.mpsqmc_version()


def test_python_constants_match_the_header():
    """Every integer constant of the binding equals the header's #define of the same name
    (MPSQMC_ prefix), and every option, status and value the header defines is bound."""
    hdr = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "mpsqmc_gpu.h")).read(), flags=re.S)
    defs = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define MPSQMC_(\w+)\s+\(?(-?\d+)\)?\s*$", hdr, re.M)}
    assert "OPT_PROPOSAL_MIX" in defs and defs["E_ARG"] == -1
    skip = {"NOALLOC_MAX_L"}  # a size limit of the allocation-free entry point, checked in its own test
    for name, v in defs.items():
        if name in skip:
            continue
        assert hasattr(capi, name), name
        assert getattr(capi, name) == v, (name, getattr(capi, name), v)


def test_create_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    z = load_golden("walk_L10D8_DW4")
    ci, cj, cJ = pb.chain(10)
    with pytest.raises(capi.MpsqmcError) as ei:
        capi.Engine(L=10, ci=ci, cj=cj, cJ=cJ, h=0.0, dtau=0.05, trial_dims=z["trial_ln_dims"],
                    trial=z["trial_ln_data"], Jvals=[1.0], U=z["U"], S=z["S"], VT=z["VT"], grid=z["grid"],
                    Ndesired=16, capacity=64, walker_dims=z["walker0_init_dims"])
    assert ei.value.code == capi.E_NODEVICE


def test_product_grid_matches_reference():
    g = load_golden("grids")["marsaglia4"]
    np.testing.assert_allclose(pb.grid_marsaglia(4, 4), g, rtol=0, atol=1e-15)


def test_product_trotter_tables_reconstruct_reference_propagator():
    z = load_golden("trotter")
    for dt, J in [(0.01, 1.0), (0.005, 1.0), (0.01, 0.5)]:
        key = f"dt{dt}_J{J}"
        U, S, VT = pb.trotter_tables(J, dt)
        np.testing.assert_allclose(S, z[key + "_S"], rtol=1e-13)
        rec = lambda U, S, VT: U.reshape(4, 4, order="F") @ np.diag(S) @ VT.reshape(4, 4, order="F")
        np.testing.assert_allclose(rec(U, S, VT), rec(z[key + "_U"], z[key + "_S"], z[key + "_VT"]), atol=1e-14)


def test_mps_text_format_round_trip():
    z = load_golden("trials")
    m = pb.MPS(z["L16D16_dims"], z["L16D16_data"])
    with tempfile.TemporaryDirectory() as t:
        path = os.path.join(t, "x.mps")
        pb.write_mps(path, m)
        back = pb.read_mps(path)
    np.testing.assert_array_equal(back.dims, m.dims)
    np.testing.assert_array_equal(back.data, m.data)


def test_product_compress_is_same_state_as_oracle():
    z = load_golden("trials")
    t = pb.MPS(z["L10D8_dims"], z["L10D8_data"])
    mine = pb.compress(t, 4)
    ref = po.compress(po.MPS(t.dims, t.data), 4)
    np.testing.assert_array_equal(mine.dims, ref.dims)
    a, b = po.MPS(mine.dims, mine.data), ref
    f = po.inner_product(a, b) / np.sqrt(po.inner_product(a, a) * po.inner_product(b, b))
    assert abs(f) == pytest.approx(1.0, abs=1e-12)


def test_virtual_dims_profile():
    np.testing.assert_array_equal(pb.virtual_dims(16, 16), load_golden("trials")["L16D16_dims"])
    np.testing.assert_array_equal(pb.virtual_dims(6, 100), [1, 2, 4, 8, 4, 2, 1])
