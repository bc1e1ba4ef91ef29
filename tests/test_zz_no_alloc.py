"""mpsqmc_local_energy_noalloc: local energies for callers that cannot call cudaMalloc.

Such callers (device memory owned by a framework allocator or a fixed arena, or code that must
not allocate) pass their own device buffers; the entry point's scratch is a static device
array inside the library.  This test feeds it walkers produced by the engine and checks the
energies against the engine's own energy entry point (mpsqmc_energy), on two calls in a row with
different populations, so that scratch contents left by the first call cannot leak into the
second.  The file is named to be collected last.
"""
import numpy as np
import pytest

from conftest import load_golden
from mpsqmc_b200 import Engine, capi
from mpsqmc_b200 import problem as pb

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
    eng.close()


def test_noalloc_rejects_sizes_beyond_the_static_array():
    L = 16
    big = np.array([1] + [4096] * (L - 1) + [1], dtype=np.int32)
    ci, cj, cJ = pb.chain(L)
    rc = capi.local_energy_noalloc(L=L, trial_dims=big, walker_dims=big, ci=ci, cj=cj, cJ=cJ, h=0.0,
                                   trial_ptr=None, walkers_ptr=None, walker_stride=0, overlaps_ptr=None,
                                   n_walkers=0, energies_ptr=None)
    assert rc != 0
    L = 24  # bond dimension up to 1024: 8 * 1024^2 doubles of scratch per CTA, beyond the array
    ci, cj, cJ = pb.chain(L)
    dims = pb.virtual_dims(L, 1024)
    stride = int(np.sum(dims[:-1] * dims[1:]) * 2)
    rc = capi.local_energy_noalloc(L=L, trial_dims=dims, walker_dims=dims, ci=ci, cj=cj, cJ=cJ, h=0.0,
                                   trial_ptr=None, walkers_ptr=None, walker_stride=stride, overlaps_ptr=None,
                                   n_walkers=0, energies_ptr=None)
    assert rc == capi.E_UNSUPPORTED
    assert b"scratch" in capi.load().mpsqmc_last_error()
