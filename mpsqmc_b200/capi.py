"""ctypes binding of the C ABI in include/mpsqmc_gpu.h (libmpsqmc_b200.so).

There is no CPU fallback: loading fails loudly when the library is missing, and creating an
engine fails with MPSQMC_E_NODEVICE when no CUDA device is visible.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

OK = 0
E_ARG, E_CUDA, E_NODEVICE, E_UNSUPPORTED, E_CAPACITY, E_NUMERIC, E_EXTINCT = -1, -2, -3, -4, -5, -6, -7
TRACE_STRIDE = 21
OPT_SWEEP = 1
SWEEP_AUTO, SWEEP_NEAREST, SWEEP_GENERAL = 0, 1, 2
OPT_WORKSPACE = 2
WORKSPACE_AUTO, WORKSPACE_GLOBAL = 0, 1
OPT_POPCONTROL_INTERVAL = 3
OPT_RESAMPLING = 4
RESAMPLE_THRESHOLD, RESAMPLE_COMB = 0, 1
OPT_PROJECTOR = 5
PROJECTOR_TROTTER, PROJECTOR_MPO_TERMS = 0, 1
OPT_CANONICAL_INTERVAL = 6
OPT_PRECISION = 7
PRECISION_FP64, PRECISION_TF32, PRECISION_TF32X3, PRECISION_TF32X3_TC, PRECISION_TF32_TC = 0, 1, 2, 3, 4
PRECISION_BF16_TC = 5  # the tcgen05 sweep with one bfloat16 pass per product
TC_PASSES_BF16 = 16    # tc_gemm's `passes` for one bfloat16 pass
OPT_PROPOSAL = 8
PROPOSAL_GRID, PROPOSAL_LEARNED = 0, 1
OPT_PROPOSAL_TRAINING = 9
OPT_PROPOSAL_MIX = 10  # thousandths of the exact PDF in the learned proposal's defensive mixture
OPT_TC_STACK_TN, OPT_TC_WIDE_TN, OPT_TC_STAGES, OPT_TC_SPLIT_OUT, OPT_TC_KC = 11, 12, 13, 14, 15  # tcgen05 choices

# Every symbol include/mpsqmc_gpu.h declares.
EXPORTED = [
    "mpsqmc_create", "mpsqmc_destroy", "mpsqmc_last_error", "mpsqmc_version", "mpsqmc_walker_size",
    "mpsqmc_set_walkers", "mpsqmc_get_walkers", "mpsqmc_set_rng", "mpsqmc_get_rng_draws",
    "mpsqmc_energy", "mpsqmc_walk", "mpsqmc_last_step_walkers", "mpsqmc_set_trace",
    "mpsqmc_get_trace", "mpsqmc_last_timing", "mpsqmc_local_energy_noalloc", "mpsqmc_set_step", "mpsqmc_tc_gemm",
    "mpsqmc_set_option", "mpsqmc_get_option", "mpsqmc_set_walkers_dims", "mpsqmc_get_walker_dims",
    "mpsqmc_compress_walkers", "mpsqmc_autotune", "mpsqmc_proposal_params", "mpsqmc_proposal_loss_grad",
    "mpsqmc_proposal_stats", "mpsqmc_step_propagate", "mpsqmc_step_control", "mpsqmc_record_size",
    "mpsqmc_export_walkers", "mpsqmc_import_walkers",
]


class MpsqmcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"mpsqmc error {code}: {msg}")
        self.code = code


class Config(C.Structure):
    _fields_ = [
        ("L", C.c_int), ("d", C.c_int), ("nC", C.c_int),
        ("ci", C.POINTER(C.c_int)), ("cj", C.POINTER(C.c_int)), ("cJ", C.POINTER(C.c_double)),
        ("h", C.c_double), ("dtau", C.c_double),
        ("trial_dims", C.POINTER(C.c_int)), ("trial", C.POINTER(C.c_double)),
        ("nJ", C.c_int), ("Jvals", C.POINTER(C.c_double)), ("U", C.POINTER(C.c_double)),
        ("S", C.POINTER(C.c_double)), ("VT", C.POINTER(C.c_double)),
        ("G", C.c_int), ("grid", C.POINTER(C.c_double)),
        ("Ndesired", C.c_int), ("capacity", C.c_int),
        ("walker_dims", C.POINTER(C.c_int)), ("device", C.c_int),
    ]


class EnergyLayout(C.Structure):
    """mpsqmc_energy_layout: host-side description of the problem for the no-allocation entry point."""
    _fields_ = [
        ("L", C.c_int), ("d", C.c_int), ("trial_dims", C.POINTER(C.c_int)),
        ("walker_dims", C.POINTER(C.c_int)), ("nC", C.c_int), ("ci", C.POINTER(C.c_int)),
        ("cj", C.POINTER(C.c_int)), ("cJ", C.POINTER(C.c_double)), ("h", C.c_double),
    ]


class StepStats(C.Structure):
    _fields_ = [
        ("step", C.c_int), ("n_walkers", C.c_int), ("n_after", C.c_int),
        ("sum_weight", C.c_double), ("avg_weight", C.c_double), ("E_P", C.c_double),
        ("E_T", C.c_double), ("omega", C.c_double), ("scaling", C.c_double),
        ("draws", C.c_uint64),
    ]


_lib = None


def library_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load libmpsqmc_b200.so (building it with nvcc if absent and allowed)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_build.LIB):
        if not build_if_missing:
            raise FileNotFoundError(f"{_build.LIB} is missing; run mpsqmc_b200.build.build()")
        _build.build()
    lib = C.CDLL(_build.LIB)
    P = C.c_void_p
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    fp = C.POINTER(C.c_float)
    sig = {
        "mpsqmc_create": (C.c_int, [C.POINTER(Config), C.POINTER(P)]),
        "mpsqmc_destroy": (C.c_int, [P]),
        "mpsqmc_last_error": (C.c_char_p, []),
        "mpsqmc_version": (C.c_char_p, []),
        "mpsqmc_walker_size": (C.c_long, [P]),
        "mpsqmc_set_walkers": (C.c_int, [P, C.c_int, dp, dp, dp, dp, C.c_int]),
        "mpsqmc_get_walkers": (C.c_int, [P, ip, dp, dp, dp, dp]),
        "mpsqmc_set_rng": (C.c_int, [P, C.c_uint32, C.c_uint64]),
        "mpsqmc_get_rng_draws": (C.c_int, [P, C.POINTER(C.c_uint64)]),
        "mpsqmc_energy": (C.c_int, [P, dp]),
        "mpsqmc_walk": (C.c_int, [P, C.c_int, C.POINTER(StepStats)]),
        "mpsqmc_last_step_walkers": (C.c_int, [P, ip, dp, dp, dp, ip, ip]),
        "mpsqmc_set_trace": (C.c_int, [P, C.c_int]),
        "mpsqmc_get_trace": (C.c_int, [P, dp, ip]),
        "mpsqmc_last_timing": (C.c_int, [P, dp, dp, ip]),
        "mpsqmc_set_step": (C.c_int, [P, C.c_int]),
        "mpsqmc_set_option": (C.c_int, [P, C.c_int, C.c_long]),
        "mpsqmc_set_walkers_dims": (C.c_int, [P, C.c_int, ip, dp, dp, dp, dp, C.c_int]),
        "mpsqmc_get_walker_dims": (C.c_int, [P, ip, ip]),
        "mpsqmc_compress_walkers": (C.c_int, [P, ip, C.c_int]),
        "mpsqmc_autotune": (C.c_int, [P, C.c_int, ip, ip]),
        "mpsqmc_get_option": (C.c_int, [P, C.c_int, C.POINTER(C.c_long)]),
        "mpsqmc_local_energy_noalloc": (C.c_int, [C.POINTER(EnergyLayout), P, P, C.c_long, P, C.c_int, P,
                                                  C.c_int, P]),
        "mpsqmc_tc_gemm": (C.c_int, [P, P, P, C.c_int, C.c_int, C.c_int, C.c_long, C.c_long, C.c_int, C.c_long,
                                     C.c_long, C.c_long, C.c_int, C.c_long, C.c_int, C.c_int, C.c_float, C.c_int,
                                     C.c_int, C.c_long, C.c_long, C.c_long, P, P]),
        "mpsqmc_proposal_params": (C.c_int, [P, fp, fp, C.POINTER(C.c_long)]),
        "mpsqmc_proposal_loss_grad": (C.c_int, [P, C.c_int, fp, fp, dp, fp]),
        "mpsqmc_proposal_stats": (C.c_int, [P, dp, ip]),
        "mpsqmc_step_propagate": (C.c_int, [P, dp]),
        "mpsqmc_step_control": (C.c_int, [P, dp, C.c_long, C.POINTER(StepStats)]),
        "mpsqmc_record_size": (C.c_long, [P]),
        "mpsqmc_export_walkers": (C.c_int, [P, C.c_int, P]),
        "mpsqmc_import_walkers": (C.c_int, [P, C.c_int, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int)) if a is not None else None


def check(rc: int):
    if rc != OK:
        raise MpsqmcError(rc, load().mpsqmc_last_error().decode())
    return rc


class Engine:
    """One device-resident walker population (an mpsqmc_ctx)."""

    def __init__(self, *, L, ci, cj, cJ, h, dtau, trial_dims, trial, Jvals, U, S, VT, grid,
                 Ndesired, capacity, walker_dims, device=0, d=2):
        lib = load()
        self._keep = dict(
            ci=np.ascontiguousarray(ci, dtype=np.int32), cj=np.ascontiguousarray(cj, dtype=np.int32),
            cJ=np.ascontiguousarray(cJ, dtype=np.float64),
            trial_dims=np.ascontiguousarray(trial_dims, dtype=np.int32),
            trial=np.ascontiguousarray(trial, dtype=np.float64),
            Jvals=np.ascontiguousarray(Jvals, dtype=np.float64), U=np.ascontiguousarray(U, dtype=np.float64),
            S=np.ascontiguousarray(S, dtype=np.float64), VT=np.ascontiguousarray(VT, dtype=np.float64),
            grid=np.ascontiguousarray(grid, dtype=np.float64),
            walker_dims=np.ascontiguousarray(walker_dims, dtype=np.int32))
        k = self._keep
        cfg = Config(L=L, d=d, nC=len(k["ci"]), ci=_ip(k["ci"]), cj=_ip(k["cj"]), cJ=_dp(k["cJ"]), h=h,
                     dtau=dtau, trial_dims=_ip(k["trial_dims"]), trial=_dp(k["trial"]), nJ=len(k["Jvals"]),
                     Jvals=_dp(k["Jvals"]), U=_dp(k["U"]), S=_dp(k["S"]), VT=_dp(k["VT"]),
                     G=k["grid"].shape[0], grid=_dp(k["grid"]), Ndesired=Ndesired, capacity=capacity,
                     walker_dims=_ip(k["walker_dims"]), device=device)
        self._ctx = C.c_void_p()
        check(lib.mpsqmc_create(C.byref(cfg), C.byref(self._ctx)))
        self.lib = lib
        self.L, self.nC, self.capacity = L, len(k["ci"]), capacity
        self.walker_size = lib.mpsqmc_walker_size(self._ctx)

    def close(self):
        if self._ctx:
            self.lib.mpsqmc_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_walkers(self, walkers, weights, overlaps=None, ehist=None, normalize=True):
        w = np.ascontiguousarray(walkers, dtype=np.float64)
        N = w.shape[0]
        wt = np.ascontiguousarray(weights, dtype=np.float64)
        ov = None if overlaps is None else np.ascontiguousarray(overlaps, dtype=np.float64)
        eh = None if ehist is None else np.ascontiguousarray(ehist, dtype=np.float64)
        check(self.lib.mpsqmc_set_walkers(self._ctx, N, _dp(w), _dp(wt), _dp(ov), _dp(eh), int(normalize)))

    def set_walkers_dims(self, dims, walkers, weights, overlaps=None, ehist=None, normalize=True):
        """Walkers of individual bond dims: dims [N, L+1]; walkers a list of 1-D tensor arrays (or
        one packed array)."""
        dm = np.ascontiguousarray(dims, dtype=np.int32)
        N = dm.shape[0]
        packed = np.ascontiguousarray(np.concatenate([np.ravel(x) for x in walkers])
                                      if isinstance(walkers, (list, tuple)) else walkers, dtype=np.float64)
        wt = np.ascontiguousarray(weights, dtype=np.float64)
        ov = None if overlaps is None else np.ascontiguousarray(overlaps, dtype=np.float64)
        eh = None if ehist is None else np.ascontiguousarray(ehist, dtype=np.float64)
        check(self.lib.mpsqmc_set_walkers_dims(self._ctx, N, _ip(dm), _dp(packed), _dp(wt), _dp(ov), _dp(eh),
                                               int(normalize)))

    def autotune(self, steps: int = 2):
        """Time the kernel choices on a subset of the population and keep the fastest; returns
        (sweep, workspace)."""
        a, b = C.c_int(0), C.c_int(0)
        check(self.lib.mpsqmc_autotune(self._ctx, steps, C.byref(a), C.byref(b)))
        return a.value, b.value

    def compress_walkers(self, target_D, normalize=True):
        """MPSstate::CompressState on the device: walker w to bond dimension target_D[w] (scalar: all)."""
        n = C.c_int(0)
        check(self.lib.mpsqmc_get_walker_dims(self._ctx, C.byref(n), None))
        t = np.ascontiguousarray(np.broadcast_to(np.asarray(target_D, dtype=np.int32), (n.value,)))
        check(self.lib.mpsqmc_compress_walkers(self._ctx, _ip(t), int(normalize)))

    def get_walker_dims(self):
        n = C.c_int(0)
        check(self.lib.mpsqmc_get_walker_dims(self._ctx, C.byref(n), None))
        dm = np.zeros((n.value, self.L + 1), dtype=np.int32)
        check(self.lib.mpsqmc_get_walker_dims(self._ctx, C.byref(n), _ip(dm)))
        return dm

    def get_walkers(self, out=None):
        """(walkers [N, walker_size], weights, overlaps, energy histories).  out: optional
        float64 C-contiguous array of at least capacity rows (e.g. pinned host memory) that
        receives the walkers; the returned walkers are a view of it."""
        n = C.c_int(0)
        check(self.lib.mpsqmc_get_walkers(self._ctx, C.byref(n), None, None, None, None))
        N = n.value
        if out is not None:
            if out.dtype != np.float64 or not out.flags.c_contiguous or out.shape[0] < N or \
                    out.shape[1] != self.walker_size:
                raise ValueError("out must be C-contiguous float64 [>= N, walker_size]")
            w = out[:N]
        else:
            w = np.zeros((N, self.walker_size))
        wt, ov, eh = np.zeros(N), np.zeros(N), np.zeros(N)
        check(self.lib.mpsqmc_get_walkers(self._ctx, C.byref(n), _dp(w), _dp(wt), _dp(ov), _dp(eh)))
        return w, wt, ov, eh

    def set_rng(self, seed: int, skip: int = 0):
        check(self.lib.mpsqmc_set_rng(self._ctx, seed & 0xFFFFFFFF, skip))

    def rng_draws(self) -> int:
        v = C.c_uint64(0)
        check(self.lib.mpsqmc_get_rng_draws(self._ctx, C.byref(v)))
        return v.value

    def energy(self) -> float:
        e = C.c_double(0)
        check(self.lib.mpsqmc_energy(self._ctx, C.byref(e)))
        return e.value

    @staticmethod
    def _stats(s):
        return dict(step=s.step, n_walkers=s.n_walkers, n_after=s.n_after, sum_weight=s.sum_weight,
                    avg_weight=s.avg_weight, E_P=s.E_P, E_T=s.E_T, omega=s.omega, scaling=s.scaling, draws=s.draws)

    def walk(self, nsteps: int):
        st = (StepStats * max(nsteps, 1))()
        check(self.lib.mpsqmc_walk(self._ctx, nsteps, st))
        return [self._stats(s) for s in st[:nsteps]]

    # walks split over ranks
    def step_propagate(self):
        """One step's propagation; this population's five sums (Sum w, Sum w E, Sum e, Sum e^2, N)."""
        out = np.zeros(5)
        check(self.lib.mpsqmc_step_propagate(self._ctx, _dp(out)))
        return out

    def step_control(self, global_sums, ndesired_total: int):
        g = np.ascontiguousarray(global_sums, dtype=np.float64)
        st = StepStats()
        check(self.lib.mpsqmc_step_control(self._ctx, _dp(g), int(ndesired_total), C.byref(st)))
        return self._stats(st)

    def record_size(self) -> int:
        return int(self.lib.mpsqmc_record_size(self._ctx))

    def export_walkers(self, k: int, records_ptr: int):
        """The last k walkers into k records at a device address (e.g. a torch tensor's data_ptr())."""
        check(self.lib.mpsqmc_export_walkers(self._ctx, int(k), C.c_void_p(records_ptr)))

    def import_walkers(self, k: int, records_ptr: int):
        check(self.lib.mpsqmc_import_walkers(self._ctx, int(k), C.c_void_p(records_ptr)))

    @property
    def n_walkers(self) -> int:
        n = C.c_int(0)
        check(self.lib.mpsqmc_get_walkers(self._ctx, C.byref(n), None, None, None, None))
        return n.value

    def set_step(self, completed_steps: int):
        check(self.lib.mpsqmc_set_step(self._ctx, completed_steps))

    def last_step_walkers(self):
        nb, na = C.c_int(0), C.c_int(0)
        check(self.lib.mpsqmc_last_step_walkers(self._ctx, C.byref(nb), None, None, None, C.byref(na), None))
        w, o, e = np.zeros(nb.value), np.zeros(nb.value), np.zeros(nb.value)
        par = np.zeros(max(na.value, 1), dtype=np.int32)
        check(self.lib.mpsqmc_last_step_walkers(self._ctx, C.byref(nb), _dp(w), _dp(o), _dp(e), C.byref(na),
                                                _ip(par)))
        return dict(weight=w, overlap=o, energy=e, parent=par[:na.value])

    def set_trace(self, on: bool):
        check(self.lib.mpsqmc_set_trace(self._ctx, int(on)))

    def get_trace(self):
        n = C.c_int(0)
        buf = np.zeros((self.capacity, self.nC, TRACE_STRIDE))
        check(self.lib.mpsqmc_get_trace(self._ctx, _dp(buf), C.byref(n)))
        return buf[: n.value]

    def set_option(self, option: int, value: int):
        check(self.lib.mpsqmc_set_option(self._ctx, option, value))

    def get_option(self, option: int) -> int:
        v = C.c_long(0)
        check(self.lib.mpsqmc_get_option(self._ctx, option, C.byref(v)))
        return v.value

    def last_timing(self):
        k, t, n = C.c_double(0), C.c_double(0), C.c_int(0)
        check(self.lib.mpsqmc_last_timing(self._ctx, C.byref(k), C.byref(t), C.byref(n)))
        return dict(step_kernel_ms=k.value, total_ms=t.value, launches=n.value)

    # learned proposal
    def proposal_params(self, new=None):
        """The network's FP32 parameter vector; with `new`, replaces it (and resets Adam)."""
        n = C.c_long(0)
        check(self.lib.mpsqmc_proposal_params(self._ctx, None, None, C.byref(n)))
        out = np.zeros(n.value, dtype=np.float32)
        src = None if new is None else np.ascontiguousarray(new, dtype=np.float32)
        check(self.lib.mpsqmc_proposal_params(self._ctx, _fp(out), _fp(src), None))
        return out

    def proposal_loss_grad(self, features, targets):
        X = np.ascontiguousarray(features, dtype=np.float32)
        Pt = np.ascontiguousarray(targets, dtype=np.float32)
        n = C.c_long(0)
        check(self.lib.mpsqmc_proposal_params(self._ctx, None, None, C.byref(n)))
        grad = np.zeros(n.value, dtype=np.float32)
        loss = C.c_double(0)
        check(self.lib.mpsqmc_proposal_loss_grad(self._ctx, X.shape[0], _fp(X), _fp(Pt), C.byref(loss), _fp(grad)))
        return loss.value, grad

    def proposal_stats(self):
        loss, upd = C.c_double(0), C.c_int(0)
        check(self.lib.mpsqmc_proposal_stats(self._ctx, C.byref(loss), C.byref(upd)))
        return dict(loss=loss.value, updates=upd.value)


def local_energy_noalloc(*, L, trial_dims, walker_dims, ci, cj, cJ, h, trial_ptr, walkers_ptr, walker_stride,
                         overlaps_ptr, n_walkers, energies_ptr, device=0, stream=None):
    """Call mpsqmc_local_energy_noalloc on caller-owned device buffers (raw device addresses).

    The call allocates nothing on the device; results are valid after the stream is synchronised."""
    lib = load()
    keep = [np.ascontiguousarray(a, dtype=t) for a, t in ((trial_dims, np.int32), (walker_dims, np.int32),
                                                           (ci, np.int32), (cj, np.int32), (cJ, np.float64))]
    lay = EnergyLayout(L=L, d=2, trial_dims=_ip(keep[0]), walker_dims=_ip(keep[1]), nC=len(keep[2]),
                       ci=_ip(keep[2]), cj=_ip(keep[3]), cJ=_dp(keep[4]), h=h)
    return lib.mpsqmc_local_energy_noalloc(C.byref(lay), trial_ptr, walkers_ptr, walker_stride, overlaps_ptr,
                                           n_walkers, energies_ptr, device, stream)


def tc_gemm(*, D, A, B, M, N, K, lda, a_zstride, adiv, a_zcount, ldb, b_zstride, bdiv, b_zcount, Z, bstack=1,
            alpha=1.0, beta=0, passes=3, dz, dm, dn, err, stream=None):
    """Call mpsqmc_tc_gemm on device buffers (raw addresses): one batched FP32 product on the
    tcgen05 tensor cores, D_z = alpha A_{z/adiv} B_{z/bdiv}^T (+ D_z).  Returns the status."""
    return load().mpsqmc_tc_gemm(D, A, B, M, N, K, lda, a_zstride, adiv, a_zcount, ldb, b_zstride, bdiv, b_zcount,
                                 Z, bstack, alpha, beta, passes, dz, dm, dn, err, stream)
