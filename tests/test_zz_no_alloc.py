"""mpsqmc_local_energy_noalloc: local energies for callers that cannot call cudaMalloc.

Such callers (device memory owned by a framework allocator or a fixed arena, or code that must
not allocate) pass their own device buffers; the entry point's scratch is a static device
array inside the library.  These tests feed it walkers produced by the engine and check the
energies against the engine's own energy entry point (mpsqmc_energy) and the CPU oracle, on two
calls in a row with different populations, so that scratch contents left by the first call
cannot leak into the second; then a field, uneven trial/walker bond dimensions and padded walker
rows, and bond dimensions whose work buffers live in the array instead of shared memory, against
the oracle.  The file is named to be collected last.
"""
import numpy as np
import pytest

from conftest import load_golden
from mpsqmc_b200 import Engine, capi
from mpsqmc_b200 import problem as pb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def _engine(z):
    meta = z["meta"]
    L, N = meta["L"], meta["Nw"]
    ci, cj, cJ = pb.chain(L)
    eng = Engine(L=L, ci=ci, cj=cj, cJ=cJ, h=0.0, dtau=meta["dtau"], trial_dims=z["trial_ln_dims"],
                 trial=z["trial_ln_data"], Jvals=[1.0], U=z["U"], S=z["S"], VT=z["VT"], grid=z["grid"],
                 Ndesired=N, capacity=max(1000, 3 * N), walker_dims=z["walker0_init_dims"])
    eng.set_walkers(np.tile(z["walker0_init_data"], (N, 1)), z["init_weight"], z["init_overlap"],
                    np.zeros(N), normalize=False)
    eng.set_rng(meta["seed"], meta["setup_draws"])
    return eng


def test_noalloc_energy_matches_engine_on_two_calls():
    import torch

    z = load_golden("walk_L16D16_DW16")
    L = z["meta"]["L"]
    ci, cj, cJ = pb.chain(L)
    eng = _engine(z)
    trial_d = torch.tensor(z["trial_ln_data"], dtype=torch.float64, device="cuda")
    for call in range(2):
        eng.walk(1)
        w, wt, ov, eh = eng.get_walkers()
        eng.energy()
        ref = eng.last_step_walkers()["energy"]
        assert len(ref) == w.shape[0]
        walkers_d = torch.tensor(w, dtype=torch.float64, device="cuda")
        ov_d = torch.tensor(ov, dtype=torch.float64, device="cuda")
        out_d = torch.full((w.shape[0],), float("nan"), dtype=torch.float64, device="cuda")
        rc = capi.local_energy_noalloc(L=L, trial_dims=z["trial_ln_dims"], walker_dims=z["walker0_init_dims"],
                                       ci=ci, cj=cj, cJ=cJ, h=0.0, trial_ptr=trial_d.data_ptr(),
                                       walkers_ptr=walkers_d.data_ptr(), walker_stride=w.shape[1],
                                       overlaps_ptr=ov_d.data_ptr(), n_walkers=w.shape[0],
                                       energies_ptr=out_d.data_ptr(), device=0,
                                       stream=torch.cuda.current_stream().cuda_stream)
        assert rc == 0, capi.load().mpsqmc_last_error().decode()
        torch.cuda.synchronize()
        np.testing.assert_allclose(out_d.cpu().numpy(), ref, rtol=RTOL, err_msg=f"call {call + 1}")
        trial = po.MPS(z["trial_ln_dims"], z["trial_ln_data"])
        orc = [po.energy_numerator(trial, po.MPS(z["walker0_init_dims"], w[k]), ci, cj, cJ) / ov[k]
               for k in range(w.shape[0])]
        np.testing.assert_allclose(out_d.cpu().numpy(), orc, rtol=RTOL, err_msg=f"call {call + 1} vs oracle")
    eng.close()


def _random_mps(dims, rng):
    return po.MPS(np.asarray(dims, np.int32), rng.normal(size=po.mps_size(dims)))


@pytest.mark.parametrize("L,DT,DW,h,pad", [(12, 16, 8, 0.3, 37), (12, 64, 64, 0.0, 0)],
                         ids=["field-uneven-padded", "buffers-in-array"])
def test_noalloc_energy_matches_oracle(L, DT, DW, h, pad):
    """A field, trial and walker bond dimensions that differ, walker rows padded beyond one walker;
    and D = 64, whose matrix work buffers do not fit in shared memory and go to the array."""
    import torch

    rng = np.random.default_rng(11)
    ci, cj, cJ = pb.chain(L)
    tdims, wdims = po.virtual_dims(L, DT), po.virtual_dims(L, DW)
    trial = po.left_normalize(_random_mps(tdims, rng))[0]
    size = po.mps_size(wdims)
    stride = size + pad
    trial_d = torch.tensor(trial.data, dtype=torch.float64, device="cuda")
    for call in range(2):
        n = 5 + call
        walkers = [_random_mps(wdims, rng) for _ in range(n)]
        rows = np.zeros((n, stride))
        for k, m in enumerate(walkers):
            rows[k, :size] = m.data
        ov = np.array([po.inner_product(trial, m) for m in walkers])
        orc = np.array([po.energy_numerator(trial, m, ci, cj, cJ, h) for m in walkers]) / ov
        walkers_d = torch.tensor(rows, dtype=torch.float64, device="cuda")
        ov_d = torch.tensor(ov, dtype=torch.float64, device="cuda")
        out_d = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        rc = capi.local_energy_noalloc(L=L, trial_dims=tdims, walker_dims=wdims, ci=ci, cj=cj, cJ=cJ, h=h,
                                       trial_ptr=trial_d.data_ptr(), walkers_ptr=walkers_d.data_ptr(),
                                       walker_stride=stride, overlaps_ptr=ov_d.data_ptr(), n_walkers=n,
                                       energies_ptr=out_d.data_ptr(), device=0,
                                       stream=torch.cuda.current_stream().cuda_stream)
        assert rc == 0, capi.load().mpsqmc_last_error().decode()
        torch.cuda.synchronize()
        np.testing.assert_allclose(out_d.cpu().numpy(), orc, rtol=RTOL, err_msg=f"call {call + 1}")


def test_noalloc_rejects_sizes_beyond_the_static_array():
    # bond dimension 1024: the compact-MPO environments alone (8 x 1024^2 doubles) exceed the array
    for L, D in ((24, 1024), (20, 256)):
        # D = 256: the environments fit, with the matrix work buffers (too large for shared
        # memory, so placed in the array too) they do not
        ci, cj, cJ = pb.chain(L)
        dims = pb.virtual_dims(L, D)
        stride = int(np.sum(dims[:-1] * dims[1:]) * 2)
        rc = capi.local_energy_noalloc(L=L, trial_dims=dims, walker_dims=dims, ci=ci, cj=cj, cJ=cJ, h=0.0,
                                       trial_ptr=None, walkers_ptr=None, walker_stride=stride, overlaps_ptr=None,
                                       n_walkers=0, energies_ptr=None)
        assert rc == capi.E_UNSUPPORTED, (L, D, rc)
        assert b"scratch" in capi.load().mpsqmc_last_error()
