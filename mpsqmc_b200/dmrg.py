"""Trial-state generator: two-site DMRG with a compact MPO (bond dimension 5 on a chain,
2 + 3 x (open sites) for couplings of any range, e.g. 2D lattices on a snake path).

The reference's DMRG (DMRG.cpp:13-604) rebuilds the full generic MPO product every step, whose
bond grows to (2 + 3 L/2) * D_T, which is out of reach for L = 64, D_T = 64.  This host-side
solver keeps the same algorithm shape (two-site sweeps, lowest eigenvector of the effective
Hamiltonian, SVD truncation to D; DMRG.cpp:70-100) with environments of the compact
nearest-neighbour Heisenberg MPO
    W = [[I, 0, 0, 0, 0], [J Sx, 0, 0, 0, 0], [-J iSy, 0, 0, 0, 0], [J Sz, 0, 0, 0, 0],
         [-h Sz, Sx, iSy, Sz, I]]
(rows: incoming channel, columns: outgoing; channel 4 = nothing placed, channel 0 = done).
The result is returned in the reference's storage layout and bond profile.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse.linalg as sla

from .problem import MPS, spin_ops, virtual_dims


def chain_mpo(L: int, J: np.ndarray, h: float = 0.0, d: int = 2) -> list[np.ndarray]:
    """W[k] with shape (w_in, w_out, d_out, d_in); J[k] couples sites k and k+1."""
    sz, sx, isy = spin_ops(d)
    eye = np.eye(d)
    Ws = []
    for k in range(L):
        W = np.zeros((5, 5, d, d))
        Jp = J[k - 1] if k > 0 else 0.0
        W[0, 0] = eye
        W[1, 0] = Jp * sx
        W[2, 0] = -Jp * isy
        W[3, 0] = Jp * sz
        W[4, 0] = -h * sz
        W[4, 1] = sx
        W[4, 2] = isy
        W[4, 3] = sz
        W[4, 4] = eye
        if k == 0:
            W = W[4:5]
        if k == L - 1:
            W = W[:, 0:1]
        Ws.append(W)
    return Ws


def coupling_mpo(L: int, ci, cj, cJ, h: float = 0.0, d: int = 2) -> list[np.ndarray]:
    """Compact MPO of H = sum_c J_c S_i.S_j - h sum_k S^z_k for couplings (i < j) of any range.

    Channels on the cut before site k: 0 = done, then (Sx, iSy, Sz) of every site i < k that still
    has a partner j >= k (in order of i), last = nothing placed yet.  Site k closes the channels
    of its partners i (J_ik times Sx, -iSy, Sz on site k), carries on the ones that stay open,
    opens its own when it has a partner beyond k, and places the field.  Same layout as chain_mpo:
    W[k] of shape (w_in, w_out, d_out, d_in)."""
    sz, sx, isy = spin_ops(d)
    ops = (sx, isy, sz)
    eye = np.eye(d)
    last = [-1] * L
    J = {}
    for i, j, c in zip(ci, cj, cJ):
        i, j = int(i), int(j)
        last[i] = max(last[i], j)
        J[(i, j)] = J.get((i, j), 0.0) + float(c)
    opened = [[i for i in range(k) if last[i] >= k] for k in range(L + 1)]  # open sites on cut k
    Ws = []
    for k in range(L):
        inn, out = opened[k], opened[k + 1]
        w_in, w_out = 2 + 3 * len(inn), 2 + 3 * len(out)
        W = np.zeros((w_in, w_out, d, d))
        W[0, 0] = eye
        W[w_in - 1, w_out - 1] = eye
        W[w_in - 1, 0] = -h * sz
        for q, i in enumerate(inn):
            Jik = J.get((i, k), 0.0)
            for a in range(3):
                if Jik != 0.0:
                    W[1 + 3 * q + a, 0] = (-Jik if a == 1 else Jik) * ops[a]
                if i in out:
                    W[1 + 3 * q + a, 1 + 3 * out.index(i) + a] = eye
        if k in out:
            r = out.index(k)
            for a in range(3):
                W[w_in - 1, 1 + 3 * r + a] = ops[a]
        if k == 0:
            W = W[w_in - 1:w_in]
        if k == L - 1:
            W = W[:, 0:1]
        Ws.append(W)
    return Ws


def mpo_energy(m: MPS, Ws) -> float:
    """<m|H|m> / <m|m> of an MPS in the reference layout with the MPO Ws."""
    A = [m.site(k).transpose(1, 0, 2) for k in range(m.L)]  # (Dl, s, Dr)
    E = np.ones((1, 1, 1))
    N = np.ones((1, 1))
    for k in range(m.L):
        E = _left_env(E, A[k], Ws[k])
        N = np.einsum("ab,asc,bsd->cd", N, A[k], A[k])
    return float(E[0, 0, 0] / N[0, 0])


def _left_env(Lprev, A, W):
    # Lprev (a, w, A'), A (A', s, C) ket, bra = A (real)
    t = np.tensordot(Lprev, A, axes=([2], [0]))            # a w s C
    t = np.tensordot(t, W, axes=([1, 2], [0, 3]))           # a C v p
    return np.tensordot(A, t, axes=([0, 1], [0, 3])).transpose(0, 2, 1)  # (bra c, w v, ket C)


def _right_env(Rnext, A, W):
    # Rnext (c, u, C'), A (a, s, C')
    t = np.tensordot(A, Rnext, axes=([2], [2]))             # a s c u
    t = np.tensordot(t, W, axes=([1, 3], [3, 1]))           # a c v p
    return np.tensordot(A, t, axes=([1, 2], [3, 1])).transpose(0, 2, 1)  # a v a'  -> (bra, w, ket)


def _heff(Lenv, W1, W2, Renv, shape):
    def mv(x):
        th = x.reshape(shape)                                      # A s t C
        t = np.tensordot(Lenv, th, axes=([2], [0]))                # a w s t C
        t = np.tensordot(t, W1, axes=([1, 2], [0, 3]))             # a t C v p
        t = np.tensordot(t, W2, axes=([3, 1], [0, 3]))             # a C p u q
        t = np.tensordot(t, Renv, axes=([1, 3], [2, 1]))           # a p q c
        return t.reshape(-1)
    n = int(np.prod(shape))
    return sla.LinearOperator((n, n), matvec=mv, dtype=np.float64)


def dmrg(L: int, D: int, J=1.0, h: float = 0.0, sweeps: int = 8, tol: float = 1e-10, seed: int = 7,
         schedule=None, verbose: bool = False, couplings=None):
    """Ground state of the open Heisenberg chain (or, with couplings = (ci, cj, cJ), of any
    coupling list) as an MPS of bond dimension <= D.

    Returns (MPS in reference layout, left-normalized; energy)."""
    d = 2
    if couplings is not None:
        Ws = coupling_mpo(L, *couplings, h=h, d=d)
    else:
        Jv = np.full(L - 1, float(J)) if np.isscalar(J) else np.asarray(J, dtype=np.float64)
        Ws = chain_mpo(L, Jv, h, d)
    rng = np.random.default_rng(seed)
    dims0 = virtual_dims(L, min(D, 4), d)
    A = [rng.standard_normal((dims0[k], d, dims0[k + 1])) for k in range(L)]
    # right-normalize the start
    for k in range(L - 1, 0, -1):
        m = A[k].reshape(A[k].shape[0], -1)
        q, r = np.linalg.qr(m.T)
        A[k] = q.T.reshape(-1, d, A[k].shape[2])
        A[k - 1] = np.tensordot(A[k - 1], r.T, axes=([2], [0]))
    A[0] /= np.linalg.norm(A[0])
    one = np.ones((1, 1, 1))
    R = [None] * (L + 1)
    R[L] = one
    for k in range(L - 1, 0, -1):
        R[k] = _right_env(R[k + 1], A[k], Ws[k])
    Lenvs = [None] * (L + 1)
    Lenvs[0] = one
    if schedule is None:
        schedule = [min(D, x) for x in (8, 16, 32, 64, 128, 256) if x < D] + [D] * sweeps
    E_prev, E = None, 0.0
    for sweep, Dcur in enumerate(schedule):
        # left-to-right
        for k in range(0, L - 1):
            th = np.tensordot(A[k], A[k + 1], axes=([2], [0]))
            shape = th.shape
            H = _heff(Lenvs[k], Ws[k], Ws[k + 1], R[k + 2], shape)
            w, v = sla.eigsh(H, k=1, which="SA", v0=th.reshape(-1), tol=1e-12, ncv=min(20, H.shape[0] - 1)) \
                if H.shape[0] > 3 else np.linalg.eigh(np.array([H.matvec(e) for e in np.eye(H.shape[0])]).T)
            E = float(w[0])
            m = v[:, 0].reshape(shape[0] * d, d * shape[3])
            u, s, vt = np.linalg.svd(m, full_matrices=False)
            keep = max(1, min(Dcur, int(np.sum(s > 1e-14 * s[0]))))
            A[k] = u[:, :keep].reshape(shape[0], d, keep)
            A[k + 1] = (s[:keep, None] * vt[:keep]).reshape(keep, d, shape[3])
            Lenvs[k + 1] = _left_env(Lenvs[k], A[k], Ws[k])
        # right-to-left
        for k in range(L - 2, -1, -1):
            th = np.tensordot(A[k], A[k + 1], axes=([2], [0]))
            shape = th.shape
            H = _heff(Lenvs[k], Ws[k], Ws[k + 1], R[k + 2], shape)
            w, v = sla.eigsh(H, k=1, which="SA", v0=th.reshape(-1), tol=1e-12, ncv=min(20, H.shape[0] - 1)) \
                if H.shape[0] > 3 else np.linalg.eigh(np.array([H.matvec(e) for e in np.eye(H.shape[0])]).T)
            E = float(w[0])
            m = v[:, 0].reshape(shape[0] * d, d * shape[3])
            u, s, vt = np.linalg.svd(m, full_matrices=False)
            keep = max(1, min(Dcur, int(np.sum(s > 1e-14 * s[0]))))
            A[k] = (u[:, :keep] * s[None, :keep]).reshape(shape[0], d, keep)
            A[k + 1] = vt[:keep].reshape(keep, d, shape[3])
            R[k + 1] = _right_env(R[k + 2], A[k + 1], Ws[k + 1])
        if verbose:
            print(f"sweep {sweep} D={Dcur} E={E:.12f}")
        if E_prev is not None and Dcur == D and abs(E - E_prev) < tol:
            break
        E_prev = E if Dcur == D else None
    # left-normalize (QR sweep) and export in the reference layout
    for k in range(L - 1):
        m = A[k].reshape(-1, A[k].shape[2])
        q, r = np.linalg.qr(m)
        A[k] = q.reshape(A[k].shape[0], d, -1)
        A[k + 1] = np.tensordot(r, A[k + 1], axes=([1], [0]))
    A[L - 1] /= np.linalg.norm(A[L - 1])
    sites = [a.transpose(1, 0, 2) for a in A]  # [sigma, Dl, Dr]
    return MPS.from_sites(sites, d), E


# --------------------------------------------------------------------------------------------
# The same two-site sweeps on the GPU (set-up code: the D_T = 256 trials of the 8x8 lattice)
# --------------------------------------------------------------------------------------------
def _lanczos_lowest(mv, x0, maxit: int = 60, tol: float = 1e-9):
    """Lowest eigenpair of the symmetric operator mv by Lanczos with full reorthogonalisation,
    started from x0 (all vectors on x0's device, FP64).  Stops when the residual estimate
    |beta_m s_m| falls below tol * max(1, |theta|)."""
    import torch
    from scipy.linalg import eigh_tridiagonal

    n = x0.numel()
    m = min(maxit, n)
    V = torch.empty((m, n), dtype=x0.dtype, device=x0.device)
    V[0] = x0 / torch.linalg.vector_norm(x0)
    alphas, betas = [], []
    w = mv(V[0])
    a = float(torch.dot(w, V[0]))
    alphas.append(a)
    w = w - a * V[0]
    theta, s = np.array([a]), np.ones((1, 1))
    k = 1
    for k in range(1, m):
        w = w - V[:k].T @ (V[:k] @ w)
        b = float(torch.linalg.vector_norm(w))
        if b < 1e-14:
            break
        V[k] = w / b
        betas.append(b)
        w = mv(V[k]) - b * V[k - 1]
        a = float(torch.dot(w, V[k]))
        alphas.append(a)
        w = w - a * V[k]
        if k % 3 == 0 or k == m - 1:
            theta, s = eigh_tridiagonal(np.array(alphas), np.array(betas), select="i", select_range=(0, 0))
            res = abs(float(torch.linalg.vector_norm(w - V[:k + 1].T @ (V[:k + 1] @ w)))) * abs(s[-1, 0])
            if res < tol * max(1.0, abs(theta[0])):
                break
    kk = len(alphas)
    theta, s = eigh_tridiagonal(np.array(alphas), np.array(betas[:kk - 1]), select="i", select_range=(0, 0))
    coef = torch.as_tensor(s[:, 0], dtype=x0.dtype, device=x0.device)
    x = V[:kk].T @ coef
    return float(theta[0]), x / torch.linalg.vector_norm(x)


def dmrg_device(L: int, D: int, couplings=None, J=1.0, h: float = 0.0, init: MPS | None = None, schedule=None,
                sweeps: int = 6, tol: float = 1e-8, seed: int = 7, device: str = "cuda", verbose: bool = False):
    """dmrg() with every contraction, eigensolver vector and SVD on a GPU in FP64 (torch).

    The effective-Hamiltonian matvec, environments and truncation are those of dmrg(); the lowest
    eigenvector comes from a Lanczos solver (full reorthogonalisation) on the device.  init: a
    starting MPS (e.g. a stored trial of smaller bond dimension); else a seeded random one.
    Returns (MPS in reference layout, left-normalised; energy of the last two-site solve)."""
    import torch

    dev = torch.device(device)
    f64 = torch.float64
    d = 2
    if couplings is not None:
        Ws = coupling_mpo(L, *couplings, h=h, d=d)
    else:
        Jv = np.full(L - 1, float(J)) if np.isscalar(J) else np.asarray(J, dtype=np.float64)
        Ws = chain_mpo(L, Jv, h, d)
    W = [torch.as_tensor(w, dtype=f64, device=dev) for w in Ws]
    if init is None:
        rng = np.random.default_rng(seed)
        dims0 = virtual_dims(L, min(D, 4), d)
        A = [torch.as_tensor(rng.standard_normal((dims0[k], d, dims0[k + 1])), dtype=f64, device=dev)
             for k in range(L)]
    else:
        A = [torch.as_tensor(init.site(k).transpose(1, 0, 2).copy(), dtype=f64, device=dev) for k in range(L)]
    td = lambda a, b, axes: torch.tensordot(a, b, dims=axes)  # noqa: E731

    def left_env(Lp, a, w):
        t = td(Lp, a, ([2], [0]))
        t = td(t, w, ([1, 2], [0, 3]))
        return td(a, t, ([0, 1], [0, 3])).permute(0, 2, 1).contiguous()

    def right_env(Rn, a, w):
        t = td(a, Rn, ([2], [2]))
        t = td(t, w, ([1, 3], [3, 1]))
        return td(a, t, ([1, 2], [3, 1])).permute(0, 2, 1).contiguous()

    for k in range(L - 1, 0, -1):  # right-normalise the start
        m = A[k].reshape(A[k].shape[0], -1)
        q, r = torch.linalg.qr(m.T)
        A[k] = q.T.reshape(-1, d, A[k].shape[2])
        A[k - 1] = td(A[k - 1], r.T, ([2], [0]))
    A[0] = A[0] / torch.linalg.vector_norm(A[0])
    one = torch.ones((1, 1, 1), dtype=f64, device=dev)
    R = [None] * (L + 1)
    R[L] = one
    for k in range(L - 1, 0, -1):
        R[k] = right_env(R[k + 1], A[k], W[k])
    Lenvs = [None] * (L + 1)
    Lenvs[0] = one
    if schedule is None:
        start = max(a.shape[2] for a in A)
        schedule = [x for x in (8, 16, 32, 64, 128, 256, 512) if start < x < D] + [D] * sweeps

    def solve(k):
        th = td(A[k], A[k + 1], ([2], [0]))
        shape = th.shape
        Le, W1, W2, Re = Lenvs[k], W[k], W[k + 1], R[k + 2]

        def mv(x):
            t = td(Le, x.reshape(shape), ([2], [0]))
            t = td(t, W1, ([1, 2], [0, 3]))
            t = td(t, W2, ([3, 1], [0, 3]))
            return td(t, Re, ([1, 3], [2, 1])).reshape(-1)

        e, v = _lanczos_lowest(mv, th.reshape(-1))
        return e, v.reshape(shape[0] * d, d * shape[3]), shape

    def split(mat, shape, Dcur):
        u, s, vt = torch.linalg.svd(mat, full_matrices=False)
        keep = max(1, min(Dcur, int(torch.count_nonzero(s > 1e-14 * s[0]))))
        return u[:, :keep], s[:keep], vt[:keep], keep

    E_prev, E = None, 0.0
    for sweep, Dcur in enumerate(schedule):
        for k in range(0, L - 1):
            E, mat, shape = solve(k)
            u, s, vt, keep = split(mat, shape, Dcur)
            A[k] = u.reshape(shape[0], d, keep)
            A[k + 1] = (s[:, None] * vt).reshape(keep, d, shape[3])
            Lenvs[k + 1] = left_env(Lenvs[k], A[k], W[k])
        for k in range(L - 2, -1, -1):
            E, mat, shape = solve(k)
            u, s, vt, keep = split(mat, shape, Dcur)
            A[k] = (u * s[None, :]).reshape(shape[0], d, keep)
            A[k + 1] = vt.reshape(keep, d, shape[3])
            R[k + 1] = right_env(R[k + 2], A[k + 1], W[k + 1])
        if verbose:
            print(f"sweep {sweep} D={Dcur} E={E:.12f}", flush=True)
        if E_prev is not None and Dcur == D and abs(E - E_prev) < tol:
            break
        E_prev = E if Dcur == D else None
    for k in range(L - 1):
        m = A[k].reshape(-1, A[k].shape[2])
        q, r = torch.linalg.qr(m)
        A[k] = q.reshape(A[k].shape[0], d, -1)
        A[k + 1] = td(r, A[k + 1], ([1], [0]))
    A[L - 1] = A[L - 1] / torch.linalg.vector_norm(A[L - 1])
    sites = [a.permute(1, 0, 2).cpu().numpy() for a in A]  # [sigma, Dl, Dr]
    return MPS.from_sites(sites, d), E
