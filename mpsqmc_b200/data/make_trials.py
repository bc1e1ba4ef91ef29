"""Regenerate the stored trial states of the named workloads (mpsqmc_b200/workloads.py).

    python mpsqmc_b200/data/make_trials.py [chain64] [snake6x6] [snake8x8] [snake8x8_256]

chain64:  trial_L64D64.npz, the open L=64 Heisenberg chain at D_T = 64;
snake6x6: trial_snake6x6_D64.npz, the open 6x6 lattice on the snake path at D_T = 64;
snake8x8: trial_snake8x8_D64.npz, the open 8x8 lattice on the snake path at D_T = 64;
snake8x8_256: trial_snake8x8_D256.npz, the open 8x8 lattice at D_T = 256, grown on the GPU
          (dmrg.dmrg_device) from the D_T = 64 trial; stored in FP32 (26 MB instead of 52 MB)
          and left-normalised again in FP64 when loaded (workloads.LatticeWorkload.trial), with
          the energy of that FP64 state beside it.  MPSQMC_TRIAL_OUT=<dir> writes elsewhere.

All others come from the host compact-MPO two-site DMRG (mpsqmc_b200/dmrg.py, seed 7),
left-normalised, in the reference's storage layout, with the DMRG energy beside them.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mpsqmc_b200 import dmrg, problem as pb  # noqa: E402


def make(name: str) -> None:
    t = time.time()
    if name == "chain64":
        m, e = dmrg.dmrg(64, 64)
        out = "trial_L64D64.npz"
    elif name == "snake6x6":
        m, e = dmrg.dmrg(36, 64, couplings=pb.snake(6, 6))
        out = "trial_snake6x6_D64.npz"
    elif name == "snake8x8_256":
        z = np.load(os.path.join(HERE, "trial_snake8x8_D64.npz"))
        init = pb.MPS(z["dims"].astype(np.int32), z["data"])
        m, e = dmrg.dmrg_device(64, 256, couplings=pb.snake(8, 8), init=init, verbose=True)
        m32 = pb.left_normalize(pb.MPS(m.dims, m.data.astype(np.float32).astype(np.float64)))
        e32 = dmrg.mpo_energy(m32, dmrg.coupling_mpo(64, *pb.snake(8, 8)))
        out_dir = os.environ.get("MPSQMC_TRIAL_OUT", HERE)
        out = "trial_snake8x8_D256.npz"
        np.savez(os.path.join(out_dir, out), dims=m.dims, data=m.data.astype(np.float32), energy=e32,
                 dmrg_energy=e)
        print(f"{out}: E = {e:.12f} (DMRG), {e32:.12f} (stored FP32 state) ({time.time() - t:.0f} s)")
        return
    elif name == "snake8x8":
        m, e = dmrg.dmrg(64, 64, couplings=pb.snake(8, 8))
        out = "trial_snake8x8_D64.npz"
    else:
        raise SystemExit(f"unknown trial {name!r}")
    np.savez(os.path.join(HERE, out), dims=m.dims, data=m.data, energy=e)
    print(f"{out}: E = {e:.12f} ({time.time() - t:.0f} s)")


if __name__ == "__main__":
    for n in sys.argv[1:] or ["chain64", "snake6x6", "snake8x8"]:
        make(n)
