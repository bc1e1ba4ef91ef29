"""Generate the golden fixtures under tests/golden/ from the reference itself.

Runs oracle/_ref/ref_harness, which is the reference's own C++ (compiled from the reference
sources by oracle/Makefile with stand-ins for the three Boost pieces it includes), with
OMP_NUM_THREADS=1 and the seed pinned to 20131015, and stores what it prints as compressed .npz
files.  Requires the reference tree (it is read only here, at generation time):

    make -C oracle ref && python tests/golden/make_golden.py

The fixtures are what tests and the GPU parity checks compare against on machines without the
reference tree.
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import pyoracle as po  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
REF_DIR = po.ref_dir()
if REF_DIR is None:
    sys.exit("set MPSQMC_REF_DIR to the reference source tree")
SEED = 20131015


def harness(*args):
    return po.run_harness(*args, env_extra={"OMP_NUM_THREADS": "1", "MPSQMC_REF_SEED": str(SEED)})


def save(name, **arrays):
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **arrays)
    print("wrote", name, sum(np.asarray(v).nbytes for v in arrays.values()), "bytes raw")


def gen_grids():
    with tempfile.TemporaryDirectory() as t:
        harness("grid", "marsaglia", 4, t)
        m = np.load(os.path.join(t, "grid.npy"))
        harness("grid", "simple", 4, t)
        s = np.load(os.path.join(t, "grid.npy"))
    save("grids", marsaglia4=m, simple4=s)


def gen_trotter():
    out = {}
    for dtau, J in [(0.01, 1.0), (0.005, 1.0), (0.01, 0.5), (0.3, 1.0), (0.5, 1.0)]:
        with tempfile.TemporaryDirectory() as t:
            harness("trotter", dtau, J, t)
            key = f"dt{dtau}_J{J}"
            for n in ("U", "S", "VT"):
                out[f"{key}_{n}"] = np.load(os.path.join(t, n + ".npy"))
    save("trotter", **out)


def gen_trials():
    out = {}
    for L, D in [(16, 16), (10, 8), (8, 4)]:
        with tempfile.TemporaryDirectory() as t:
            path = os.path.join(t, "trial.mps")
            info = json.loads(harness("dmrg", L, D, path))
            m = po.read_mps(path)
        out[f"L{L}D{D}_dims"] = m.dims
        out[f"L{L}D{D}_data"] = m.data
        out[f"L{L}D{D}_energy"] = np.array(info["energy"])
    save("trials", **out)
    return out


def gen_mpsops():
    with tempfile.TemporaryDirectory() as t:
        harness("mpsops", os.path.join(REF_DIR, "debug.mps"), 2, t)
        D = po.load_npy_dir(t)
    save("mpsops_debug", **D)


def gen_trials_2d():
    """Reference DMRG trials of open W x H lattices on the snake path."""
    out = {}
    for W, H, D in [(3, 3, 8), (4, 4, 16)]:
        with tempfile.TemporaryDirectory() as t:
            path = os.path.join(t, "trial.mps")
            info = json.loads(po.run_harness("dmrg", W * H, D, path, env_extra={
                "OMP_NUM_THREADS": "1", "MPSQMC_REF_SEED": str(SEED), "MPSQMC_REF_LATTICE": f"snake:{W}x{H}"}))
            m = po.read_mps(path)
        key = f"snake{W}x{H}D{D}"
        out[key + "_dims"] = m.dims
        out[key + "_data"] = m.data
        out[key + "_energy"] = np.array(info["energy"])
    save("trials2d", **out)
    return out


def gen_walk(name, trial: po.MPS, DW, Nw, dtau, steps, tensors=True, field=0.0, lattice=None):
    with tempfile.TemporaryDirectory() as t:
        path = os.path.join(t, "trial.mps")
        po.write_mps(path, trial)
        D = po.harness_walk(path, DW, Nw, dtau, steps, trace=True, tensors=tensors, seed=SEED, field=field,
                            lattice=lattice)
    meta = D.pop("meta")
    keep = {}
    last = f"step{steps:03d}_"
    for k, v in D.items():
        if "_walker" in k and not k.startswith(last):
            continue  # only the last step's tensors are kept
        keep[k] = v
    if tensors:
        n = len(D[last + "weight"])
        keep[last + "tensors"] = np.stack([D[f"{last}walker{w:04d}_data"] for w in range(n)])
        for w in range(n):
            keep.pop(f"{last}walker{w:04d}_data", None)
            keep.pop(f"{last}walker{w:04d}_dims", None)
    keep["meta"] = np.array(json.dumps(meta))
    save(name, **keep)


def gen_legacy(name, L, D, Nw, dtau, steps, field=0.0, lattice=None):
    D_ = po.harness_legacy(L, D, Nw, dtau, steps, seed=SEED, field=field, lattice=lattice)
    meta = D_.pop("meta")
    if lattice:
        meta["lattice"] = lattice
    last = f"step{steps:03d}_"
    n = len(D_[last + "newoverlap"])
    D_[last + "tensors"] = np.stack([D_.pop(f"{last}walker{w:04d}_data") for w in range(n)])
    for w in range(n):
        D_.pop(f"{last}walker{w:04d}_dims", None)
    D_["meta"] = np.array(json.dumps(meta))
    save(name, **D_)


def gen_legacy_all():
    gen_legacy("legacy_L10D8", 10, 8, 16, 0.05, 4)
    gen_legacy("legacy_L10D8_field", 10, 8, 16, 0.05, 3, field=0.4)
    gen_legacy("legacy_snake3x3_D8", 9, 8, 12, 0.1, 3, lattice="snake:3x3")


def main():
    if not po.harness_available():
        po.build(ref=True)
    gen_grids()
    gen_trotter()
    trials = gen_trials()
    gen_mpsops()
    T = lambda L, D: po.MPS(trials[f"L{L}D{D}_dims"], trials[f"L{L}D{D}_data"])
    gen_walk("walk_L16D16_DW16", T(16, 16), 16, 8, 0.01, 3)
    gen_walk("walk_L10D8_DW4", T(10, 8), 4, 16, 0.05, 4)
    gen_walk("walk_L10D8_DW2_branch", T(10, 8), 2, 16, 0.3, 8)
    gen_walk("walk_L10D8_DW1_branch", T(10, 8), 1, 32, 0.5, 8)
    dbg = po.read_mps(os.path.join(REF_DIR, "debug.mps"))
    gen_walk("walk_debug_DW2", dbg, 2, 32, 0.01, 3)
    gen_walk("walk_L10D8_DW4_field", T(10, 8), 4, 16, 0.05, 3, field=0.7)
    gen_2d()
    gen_legacy_all()


def gen_2d():
    z = gen_trials_2d()
    T = lambda k: po.MPS(z[k + "_dims"], z[k + "_data"])
    gen_walk("walk_snake3x3_D8_DW4", T("snake3x3D8"), 4, 16, 0.05, 4, lattice="snake:3x3")
    gen_walk("walk_snake3x3_D8_DW4_field", T("snake3x3D8"), 4, 16, 0.05, 3, field=0.5, lattice="snake:3x3")
    gen_walk("walk_snake4x4_D16_DW8_branch", T("snake4x4D16"), 8, 16, 0.3, 5, lattice="snake:4x4")


if __name__ == "__main__":
    only = sys.argv[1:]
    if only:  # regenerate selected walk fixtures only, e.g. walk_L10D8_DW4_field
        z = np.load(os.path.join(OUT, "trials.npz"))
        T = lambda L, D: po.MPS(z[f"L{L}D{D}_dims"], z[f"L{L}D{D}_data"])
        if "walk_L10D8_DW4_field" in only:
            gen_walk("walk_L10D8_DW4_field", T(10, 8), 4, 16, 0.05, 3, field=0.7)
        if "2d" in only:
            gen_2d()
        if "legacy" in only:
            gen_legacy_all()
    else:
        main()
