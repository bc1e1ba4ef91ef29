"""Test infrastructure: numpy front end of the CPU oracle (oracle/_ref/liboracle.so) and of the
reference-harness binary (oracle/_ref/ref_harness).

Only tests, tests/golden/make_golden.py, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline
leg import this module, and only to check or time against the reference algorithm.  The product
(mpsqmc_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import tempfile
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "liboracle.so")
HARNESS_PATH = os.path.join(HERE, "_ref", "ref_harness")

_lib = None


def ref_dir() -> str | None:
    """The reference source tree named by MPSQMC_REF_DIR, or None when it is unset or absent."""
    d = os.environ.get("MPSQMC_REF_DIR")
    return d if d and os.path.isfile(os.path.join(d, "MPSQMC2.cpp")) else None


def build(ref: bool = False) -> None:
    """Compile the oracle library (and the reference harness when the reference tree exists)."""
    targets = ["oracle"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(ref=False)
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class WalkConfig(C.Structure):
    _fields_ = [
        ("L", C.c_int), ("d", C.c_int), ("nC", C.c_int), ("nJ", C.c_int), ("G", C.c_int),
        ("Ndesired", C.c_int), ("capacity", C.c_int), ("nsteps", C.c_int), ("nthreads", C.c_int),
        ("dtau", C.c_double), ("h", C.c_double), ("seed", C.c_uint), ("skip", C.c_ulonglong),
        ("popctl_interval", C.c_int), ("comb", C.c_int),
    ]


def _declare(l):
    l.orc_mps_size.restype = C.c_long
    l.orc_mps_size.argtypes = [C.c_int, C.c_int, _ip]
    l.orc_inner_product.restype = C.c_double
    l.orc_inner_product.argtypes = [C.c_int, C.c_int, _ip, _dp, _ip, _dp]
    l.orc_left_normalize.restype = C.c_double
    l.orc_left_normalize.argtypes = [C.c_int, C.c_int, _ip, _dp]
    l.orc_change_phase.restype = None
    l.orc_change_phase.argtypes = [C.c_int, C.c_int, _ip, _dp]
    l.orc_apply_grid_op.restype = None
    l.orc_apply_grid_op.argtypes = [C.c_int, C.c_int, _ip, _dp, C.c_int, C.c_int, _dp, _dp, _dp, _dp]
    l.orc_apply_svd_op.restype = None
    l.orc_apply_svd_op.argtypes = [C.c_int, C.c_int, _ip, _dp, C.c_int, C.c_int, _dp, _dp, _dp,
                                   C.c_int, C.c_int, C.c_int]
    l.orc_grid_marsaglia.restype = C.c_int
    l.orc_grid_marsaglia.argtypes = [C.c_int, C.c_int, _dp, C.c_int]
    l.orc_grid_simple.restype = C.c_int
    l.orc_grid_simple.argtypes = [C.c_int, C.c_int, _dp, C.c_int]
    l.orc_trotter.restype = C.c_int
    l.orc_trotter.argtypes = [C.c_int, C.c_double, C.c_double, _dp, _dp, _dp]
    l.orc_local_energy_numerator.restype = C.c_double
    l.orc_local_energy_numerator.argtypes = [C.c_int, C.c_int, _ip, _dp, _ip, _dp, C.c_int, _ip, _ip,
                                             _dp, C.c_double]
    l.orc_compress.restype = C.c_int
    l.orc_compress.argtypes = [C.c_int, C.c_int, _ip, _dp, _dp, C.c_int]
    l.orc_walk.restype = C.c_int
    null_dp = C.c_void_p
    l.orc_walk.argtypes = [C.POINTER(WalkConfig), _ip, _dp, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp, _ip,
                           _dp, _dp, _dp, _dp, C.POINTER(C.c_int), C.POINTER(C.c_double),
                           _dp, _dp, _dp, _dp, _ip, null_dp, null_dp, null_dp, null_dp, null_dp,
                           C.POINTER(C.c_ulonglong)]
    l.orc_walk_dims.restype = C.c_int
    l.orc_walk_dims.argtypes = [C.POINTER(WalkConfig), _ip, _dp, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp, _ip,
                                null_dp, _dp, _dp, _dp, _dp, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                _dp, _dp, _dp, _dp, _ip, null_dp, null_dp, null_dp, null_dp, null_dp,
                                C.POINTER(C.c_ulonglong)]


# --------------------------------------------------------------------------------------------
# MPS helpers (layout of MPStensor.cpp:91-96)
# --------------------------------------------------------------------------------------------
@dataclass
class MPS:
    dims: np.ndarray  # int32, L+1
    data: np.ndarray  # float64, concatenated sites
    d: int = 2

    @property
    def L(self) -> int:
        return len(self.dims) - 1

    def copy(self) -> "MPS":
        return MPS(self.dims.copy(), self.data.copy(), self.d)

    def site(self, s: int) -> np.ndarray:
        """Site s as an array [sigma, col, row] view of the flat storage."""
        off = int(sum(self.dims[t] * self.dims[t + 1] * self.d for t in range(s)))
        dl, dr = int(self.dims[s]), int(self.dims[s + 1])
        return self.data[off:off + dl * dr * self.d].reshape(self.d, dr, dl)


def virtual_dims(L: int, D: int, d: int = 2) -> np.ndarray:
    """Bond profile of MPSstate.cpp:20-28."""
    v = [1] * (L + 1)
    for c in range(1, L):
        v[c] = min(v[c - 1] * d, D)
    v[L] = 1
    for c in range(L - 1, 0, -1):
        v[c] = min(min(v[c + 1] * d, D), v[c])
    return np.asarray(v, dtype=np.int32)


def read_mps(path: str) -> MPS:
    """MPSstate file format (writer MPSstate.cpp:661-686, reader 92-128)."""
    toks = open(path).read().split()
    L, _D, d = int(toks[0]), int(toks[1]), int(toks[2])
    p = 3
    dims = np.zeros(L + 1, dtype=np.int32)
    for _ in range(L + 1):
        i, v = int(toks[p]), int(toks[p + 1])
        dims[i] = v
        p += 2
    chunks = []
    for _ in range(L):
        _i, n = int(toks[p]), int(toks[p + 1])
        p += 2
        vals = np.array(toks[p:p + 3 * n], dtype=object).reshape(n, 3)[:, 2].astype(np.float64)
        chunks.append(vals)
        p += 3 * n
    return MPS(dims, np.concatenate(chunks), d)


def write_mps(path: str, m: MPS, Dtrunc: int | None = None) -> None:
    L, d = m.L, m.d
    D = int(max(m.dims)) if Dtrunc is None else Dtrunc
    lines = [f"{L}\t{D}\t{d}"]
    lines += [f"{i}\t{int(v)}" for i, v in enumerate(m.dims)]
    off = 0
    for s in range(L):
        n = int(m.dims[s] * m.dims[s + 1] * d)
        lines.append(f"{s}\t{n}")
        lines += [f"{s}\t{j}\t{m.data[off + j]:.17g}" for j in range(n)]
        off += n
    open(path, "w").write("\n".join(lines) + "\n")


def mps_size(dims, d=2) -> int:
    dims = np.asarray(dims)
    return int(np.sum(dims[:-1] * dims[1:]) * d)


# --------------------------------------------------------------------------------------------
# Wrapped oracle calls
# --------------------------------------------------------------------------------------------
def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def inner_product(a: MPS, b: MPS) -> float:
    return lib().orc_inner_product(a.L, a.d, _i32(a.dims), _f64(a.data), _i32(b.dims), _f64(b.data))


def left_normalize(m: MPS) -> tuple[MPS, float]:
    out = m.copy()
    r = lib().orc_left_normalize(out.L, out.d, _i32(out.dims), out.data)
    return out, r


def change_phase(m: MPS) -> MPS:
    out = m.copy()
    lib().orc_change_phase(out.L, out.d, _i32(out.dims), out.data)
    return out


def apply_grid_op(m: MPS, i, j, S, U, VT, x) -> MPS:
    out = m.copy()
    lib().orc_apply_grid_op(out.L, out.d, _i32(out.dims), out.data, i, j, _f64(S), _f64(U), _f64(VT), _f64(x))
    return out


def apply_svd_op(m: MPS, i, j, S, U, VT, k, l, hc=True) -> MPS:
    out = m.copy()
    lib().orc_apply_svd_op(out.L, out.d, _i32(out.dims), out.data, i, j, _f64(S), _f64(U), _f64(VT),
                           k, l, int(hc))
    return out


def grid_marsaglia(ppc: int = 4, dim: int = 4) -> np.ndarray:
    cap = ppc ** dim
    out = np.zeros(cap * dim)
    n = lib().orc_grid_marsaglia(dim, ppc, out, cap)
    return out[: n * dim].reshape(n, dim)


def grid_simple(denom: int = 4, dim: int = 4) -> np.ndarray:
    cap = 4096
    out = np.zeros(cap * dim)
    n = lib().orc_grid_simple(dim, denom, out, cap)
    return out[: n * dim].reshape(n, dim)


def trotter(J: float, dtau: float, d: int = 2):
    n = d * d
    U, S, VT = np.zeros(n * n), np.zeros(n), np.zeros(n * n)
    lib().orc_trotter(d, J, dtau, U, S, VT)
    return U, S, VT


def energy_numerator(trial: MPS, walker: MPS, ci, cj, cJ, h=0.0) -> float:
    return lib().orc_local_energy_numerator(trial.L, trial.d, _i32(trial.dims), _f64(trial.data),
                                            _i32(walker.dims), _f64(walker.data), len(ci), _i32(ci),
                                            _i32(cj), _f64(cJ), float(h))


def compress(m: MPS, D: int) -> MPS:
    dims = _i32(m.dims).copy()
    out = np.zeros_like(m.data)
    lib().orc_compress(m.L, m.d, dims, _f64(m.data), out, D)
    return MPS(dims, out[: mps_size(dims, m.d)].copy(), m.d)


def chain_couplings(L: int, J: float = 1.0):
    ci = np.arange(L - 1, dtype=np.int32)
    return ci, ci + 1, np.full(L - 1, J)


@dataclass
class WalkResult:
    status: int
    E0: float
    sumw: np.ndarray
    EP: np.ndarray
    ET: np.ndarray
    omega: np.ndarray
    n: np.ndarray
    weight: np.ndarray    # [steps, cap] pre-branching
    overlap: np.ndarray
    energy: np.ndarray
    parent: np.ndarray
    trace: np.ndarray | None
    walkers: np.ndarray   # final [N, size]
    weights: np.ndarray
    overlaps: np.ndarray
    ehist: np.ndarray
    draws: int
    wdims: np.ndarray | None = None


def walk(trial: MPS, walkers: np.ndarray, dimsW, weights, overlaps, ehist, *, ci, cj, cJ, Jvals,
         U, S, VT, grid, dtau, nsteps, Ndesired, capacity, seed, skip=0, h=0.0, trace=False,
         nthreads=0, popctl_interval=1, comb=False, wdims=None) -> WalkResult:
    """MPSQMC2::Walk on the CPU (restatement).  walkers: [N, size(dimsW)] float64; with wdims
    ([N, L+1]) walker w has its own bond dims and its tensors at the start of its row."""
    N = walkers.shape[0]
    size = mps_size(dimsW, trial.d)
    buf = np.zeros((capacity, size))
    buf[:N] = walkers
    wd = None
    if wdims is not None:
        wd = np.zeros((capacity, trial.L + 1), dtype=np.int32)
        wd[:N] = wdims
    w = np.zeros(capacity); w[:N] = weights
    o = np.zeros(capacity); o[:N] = overlaps
    eh = np.zeros(capacity); eh[:N] = ehist
    n = C.c_int(N)
    E0 = C.c_double(0)
    st = [np.zeros(nsteps) for _ in range(4)]
    stn = np.zeros(nsteps, dtype=np.int32)
    pw = [np.zeros((nsteps, capacity)) for _ in range(3)]
    par = np.full((nsteps, capacity), -1, dtype=np.int32)
    n2 = trial.d ** 2
    nC = len(ci)
    tr = np.zeros((nsteps, capacity, nC, n2 * n2 + 5)) if trace else None
    draws = C.c_ulonglong(0)
    cfg = WalkConfig(L=trial.L, d=trial.d, nC=nC, nJ=len(Jvals), G=grid.shape[0], Ndesired=Ndesired,
                     capacity=capacity, nsteps=nsteps, nthreads=nthreads, dtau=dtau, h=h, seed=seed,
                     skip=skip, popctl_interval=popctl_interval, comb=int(comb))
    ptr = lambda a: a.ctypes.data_as(C.c_void_p) if a is not None else None
    status = lib().orc_walk_dims(C.byref(cfg), _i32(trial.dims), _f64(trial.data), _i32(ci), _i32(cj),
                                 _f64(cJ), _f64(Jvals), _f64(U), _f64(S), _f64(VT), _f64(grid), _i32(dimsW),
                                 ptr(wd), buf, w, o, eh, C.byref(n), C.byref(E0), st[0], st[1], st[2], st[3], stn,
                                 ptr(pw[0]), ptr(pw[1]), ptr(pw[2]), ptr(par), ptr(tr), C.byref(draws))
    Nf = n.value
    return WalkResult(status, E0.value, st[0], st[1], st[2], st[3], stn, pw[0], pw[1], pw[2], par, tr,
                      buf[:Nf].copy(), w[:Nf].copy(), o[:Nf].copy(), eh[:Nf].copy(), draws.value,
                      None if wd is None else wd[:Nf].copy())


# --------------------------------------------------------------------------------------------
# Reference harness (the reference's own code, built from its sources)
# --------------------------------------------------------------------------------------------
def harness_available() -> bool:
    return os.path.exists(HARNESS_PATH)


def run_harness(*args: str, env_extra: dict | None = None, cwd: str | None = None) -> str:
    env = dict(os.environ)
    env.setdefault("OMP_NUM_THREADS", "1")
    if env_extra:
        env.update(env_extra)
    r = subprocess.run([HARNESS_PATH, *map(str, args)], check=True, capture_output=True, text=True,
                       env=env, cwd=cwd)
    return r.stdout


def load_npy_dir(path: str) -> dict:
    out = {}
    for f in os.listdir(path):
        if f.endswith(".npy"):
            out[f[:-4]] = np.load(os.path.join(path, f))
        elif f.endswith(".json"):
            out[f[:-5]] = json.load(open(os.path.join(path, f)))
    return out


def harness_legacy(L: int, D: int, Nw: int, dtau: float, steps: int, seed: int, field: float = 0.0,
                   lattice: str | None = None) -> dict:
    """The reference's MPO-term projector MPSQMC (oracle/_ref/ref_harness legacy): its own DMRG
    trial, walkers = trial copies, and the per-step quantities of MPSQMC::Walk."""
    with tempfile.TemporaryDirectory() as tmp:
        extra = {"MPSQMC_REF_SEED": str(seed)}
        if field:
            extra["MPSQMC_REF_FIELD"] = repr(float(field))
        if lattice:
            extra["MPSQMC_REF_LATTICE"] = lattice
        run_harness("legacy", L, D, Nw, dtau, steps, tmp, env_extra=extra)
        return load_npy_dir(tmp)


def harness_walk(trial_path: str, DW: int, Nw: int, dtau: float, steps: int, trace=True,
                 tensors=False, seed: int | None = None, field: float = 0.0, lattice: str | None = None) -> dict:
    """The reference's MPSQMC2 walk (oracle/_ref/ref_harness walk); lattice "snake:WxH" selects the
    open square lattice on the snake path instead of the chain."""
    with tempfile.TemporaryDirectory() as tmp:
        extra = {"MPSQMC_REF_SEED": str(seed)} if seed is not None else {}
        if field:
            extra["MPSQMC_REF_FIELD"] = repr(float(field))
        if lattice:
            extra["MPSQMC_REF_LATTICE"] = lattice
        args = ["walk", trial_path, DW, Nw, dtau, steps, tmp] + (["trace"] if trace else []) + \
               (["tensors"] if tensors else [])
        run_harness(*args, env_extra=extra)
        return load_npy_dir(tmp)
