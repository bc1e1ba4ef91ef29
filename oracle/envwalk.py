"""Test infrastructure: an FP64 numpy restatement of one MPSQMC2 walker step that gets the
per-coupling overlaps from transfer environments instead of stored trial-term copies, so that
it runs at the bond dimensions the CUDA engine is benchmarked on (L = 64 chains at D_T = 64,
8x8 lattices at D_T = 256), where the literal restatement (liboracle's orc_walk, 16 full-chain
InnerProducts per coupling against nC*16 stored copies of Psi_T) does not fit in memory or time.

Only tests import this module, as the checker; the product never does.

What it restates (file:line in the reference tree):
  - MPSQMC2::PropagateSeparately, MPSQMC2.cpp:518-611: one-site propagator and setOverlap,
    then per coupling the 16 numbers <Psi_T|(sqrt(s_k) U_k)_i (sqrt(s_l) V_l)_j|phi> (540-549),
    the PDF over the grid (551-566), the weight update (568-575), the CDF scan with one uniform
    (577-588), the grid operator on sites i and j (MPSstate.cpp:575-633) and setOverlap
    (Walker.cpp:54-66); the one-site propagator and setOverlap again (603-604);
  - the local energy <H Psi_T|phi> / <Psi_T|phi> of EnergyFunctionAndHistory
    (MPSQMC2.cpp:688-747, Walker.cpp:72-77) for H = sum_c J_c S_i.S_j - h sum_k S^z_k;
  - Random: MT19937 (the standard generator) and the one-draw uniform x / 2^32 (Random.cpp:14-59).

Every quantity the reference takes from the normalised walker is a ratio in which the norm
cancels (PDF = max(0, sum C x x) d^2 / (ov G) with C and ov of the same state), so the walker is
carried unnormalised and normalised once, at the end of the step.  The 16 numbers are formed as
closures of four left branches B_i[s]^T L A_i[t], carried through the sites between i and j, with
four right branches B_j[s'] R A_j[t']^T: M[p + 4q] = <Psi_T|(E_p)_i (E_q)_j|phi> for the
elementary operators E_{s + 2t} = |s><t|, and C_kl = sqrt(s_k s_l) sum U[p + 4k] M[p + 4q] VT[l + 4q].

Pinned: tests/test_envwalk_pin.py checks it against the reference's own first-step values stored
in tests/golden (walk_* fixtures) and against liboracle's literal restatement on random states.
"""
from __future__ import annotations

import numpy as np

SX = np.array([[0.0, 0.5], [0.5, 0.0]])
ISY = np.array([[0.0, -0.5], [0.5, 0.0]])
SZ = np.array([[-0.5, 0.0], [0.0, 0.5]])


def flat(o: np.ndarray) -> np.ndarray:
    """2x2 operator O(s, t) as the vector O[s + 2t]."""
    return np.asarray(o).reshape(-1, order="F")


# --------------------------------------------------------------------------------------------
# Random.cpp: MT19937 and the one-draw uniform
# --------------------------------------------------------------------------------------------
class MT19937:
    """The standard 32-bit Mersenne twister (seeding by init_genrand)."""

    def __init__(self, seed: int):
        mt = [0] * 624
        mt[0] = seed & 0xFFFFFFFF
        for i in range(1, 624):
            mt[i] = (1812433253 * (mt[i - 1] ^ (mt[i - 1] >> 30)) + i) & 0xFFFFFFFF
        self.mt, self.i = mt, 624

    def _twist(self):
        mt = self.mt
        for i in range(624):
            y = (mt[i] & 0x80000000) | (mt[(i + 1) % 624] & 0x7FFFFFFF)
            v = mt[(i + 397) % 624] ^ (y >> 1)
            if y & 1:
                v ^= 0x9908B0DF
            mt[i] = v
        self.i = 0

    def next_u32(self) -> int:
        if self.i >= 624:
            self._twist()
        y = self.mt[self.i]
        self.i += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        return y & 0xFFFFFFFF


def uniforms(seed: int, skip: int, n: int) -> np.ndarray:
    """Draws skip .. skip + n - 1 of RN->rand(): x / 2^32 (one 32-bit output per draw)."""
    g = MT19937(seed)
    for _ in range(skip):
        g.next_u32()
    return np.array([g.next_u32() / 4294967296.0 for _ in range(n)])


# --------------------------------------------------------------------------------------------
# MPS in the reference layout: site k is [r + Dl (c + Dr sigma)] -> array (sigma, Dl, Dr)
# --------------------------------------------------------------------------------------------
def sites_of(dims, data) -> list[np.ndarray]:
    out, off = [], 0
    for k in range(len(dims) - 1):
        dl, dr = int(dims[k]), int(dims[k + 1])
        n = 2 * dl * dr
        out.append(np.asarray(data[off:off + n], dtype=np.float64).reshape(2, dr, dl).transpose(0, 2, 1).copy())
        off += n
    return out


def data_of(sites) -> np.ndarray:
    return np.concatenate([s.transpose(0, 2, 1).reshape(-1) for s in sites])


def left_step(Lk, B, A):
    """L_{k+1} = sum_s B[s]^T L_k A[s]."""
    return B[0].T @ Lk @ A[0] + B[1].T @ Lk @ A[1]


def right_step(Rn, B, A):
    """R_k = sum_s B[s] R_{k+1} A[s]^T."""
    return B[0] @ Rn @ A[0].T + B[1] @ Rn @ A[1].T


def left_branches(Li, B, A):
    """P[s + 2t] = B[s]^T L_i A[t], stacked (4, a, b)."""
    return np.stack([B[s].T @ Li @ A[t] for t in range(2) for s in range(2)])


def carry(P, B, A):
    """Each branch through one site without an operator: P <- sum_s B[s]^T P A[s]."""
    return np.matmul(np.matmul(B[0].T, P), A[0]) + np.matmul(np.matmul(B[1].T, P), A[1])


def right_branches(Rn, B, A):
    """Z[s' + 2t'] = B[s'] R_{j+1} A[t']^T, stacked (4, a, b)."""
    return np.stack([B[s] @ Rn @ A[t].T for t in range(2) for s in range(2)])


class Envs:
    """Trial-walker transfer environments of one walker with lazy right environments."""

    def __init__(self, T, W):
        self.T, self.W = T, W
        L = len(T)
        self.L = L
        self.R = [None] * (L + 1)
        self.R[L] = np.ones((1, 1))
        self.rv = L          # R[k] valid for k >= rv
        for k in range(L - 1, -1, -1):
            self.R[k] = right_step(self.R[k + 1], T[k], W[k])
        self.rv = 0

    def invalidate(self, site: int):
        """Site `site` changed: R[k] with k <= site are stale."""
        self.rv = max(self.rv, site + 1)

    def right(self, k: int):
        while self.rv > k:
            self.rv -= 1
            self.R[self.rv] = right_step(self.R[self.rv + 1], self.T[self.rv], self.W[self.rv])
        return self.R[k]


def closures(T, W, Li, i, j, Rj1) -> np.ndarray:
    """M[p + 4q] = <Psi_T|(E_p)_i (E_q)_j|phi> from the left environment L_i and R_{j+1}."""
    P = left_branches(Li, T[i], W[i])
    for m in range(i + 1, j):
        P = carry(P, T[m], W[m])
    Z = right_branches(Rj1, T[j], W[j])
    M = np.empty(16)
    for q in range(4):
        for p in range(4):
            M[p + 4 * q] = np.sum(P[p] * Z[q])
    return M


def apply_op(A, O):
    """Site operator O (O[s + 2t]) on the sigma index: A'[s] = sum_t O(s, t) A[t]."""
    a0, a1 = A[0].copy(), A[1].copy()
    A[0] = O[0] * a0 + O[2] * a1
    A[1] = O[1] * a0 + O[3] * a1


def overlap(T, W) -> float:
    Lk = np.ones((1, 1))
    for k in range(len(T)):
        Lk = left_step(Lk, T[k], W[k])
    return float(Lk[0, 0])


def norm2(W) -> float:
    Lk = np.ones((1, 1))
    for A in W:
        Lk = A[0].T @ Lk @ A[0] + A[1].T @ Lk @ A[1]
    return float(Lk[0, 0])


def energy_numerator(T, W, ci, cj, cJ, h=0.0) -> float:
    """<Psi_T|H|phi> for H = sum_c J_c S_i.S_j - h sum_k S^z_k (unnormalised phi)."""
    L = len(T)
    Ls = [np.ones((1, 1))]
    for k in range(L):
        Ls.append(left_step(Ls[-1], T[k], W[k]))
    Rs = [None] * (L + 1)
    Rs[L] = np.ones((1, 1))
    for k in range(L - 1, -1, -1):
        Rs[k] = right_step(Rs[k + 1], T[k], W[k])
    sx, isy, sz = flat(SX), flat(ISY), flat(SZ)
    H2 = np.outer(sx, sx) - np.outer(isy, isy) + np.outer(sz, sz)  # H2[p, q]
    e = 0.0
    for i, j, J in zip(ci, cj, cJ):
        M = closures(T, W, Ls[i], int(i), int(j), Rs[int(j) + 1]).reshape(4, 4, order="F")  # M[p, q]
        e += float(J) * float(np.sum(H2 * M))
    if h != 0.0:
        for k in range(L):
            P = left_branches(Ls[k], T[k], W[k])
            e -= h * sum(sz[p] * float(np.sum(P[p] * Rs[k + 1])) for p in range(4))
    return e


def local_energy(trial_dims, trial, walker_dims, walker, ci, cj, cJ, h=0.0) -> float:
    T, W = sites_of(trial_dims, trial), sites_of(walker_dims, walker)
    return energy_numerator(T, W, ci, cj, cJ, h) / overlap(T, W)


def step(trial_dims, trial, walker_dims, walker, weight, *, ci, cj, cJ, Jvals, U, S, VT, grid, dtau, u,
         h=0.0):
    """One PropagateSeparately of one walker followed by its local energy.

    u: the walker's nC uniforms.  U, S, VT: Trotter tables per distinct J ([nJ,16], [nJ,4],
    [nJ,16]).  Returns dict(weight, overlap, energy, index[nC], walker (normalised, reference
    layout, sign as the reference leaves it))."""
    T = sites_of(trial_dims, trial)
    W = sites_of(walker_dims, walker)
    L = len(T)
    G = grid.shape[0]
    U = np.asarray(U).reshape(-1, 16)
    VT = np.asarray(VT).reshape(-1, 16)
    Sq = np.sqrt(np.asarray(S).reshape(-1, 4))
    jidx = [int(np.argmin(np.abs(np.asarray(Jvals) - J))) for J in cJ]
    onesite = np.exp(0.5 * h * dtau * np.array([-0.5, 0.5]))

    def field():
        if h != 0.0:
            for A in W:
                A[0] *= onesite[0]
                A[1] *= onesite[1]

    field()
    env = Envs(T, W)
    ov = float(env.right(0)[0, 0])
    if ov < 0.0:  # ChangePhase (MPSstate.cpp:307-315)
        W[0] *= -1.0
        env = Envs(T, W)
        ov = -ov
    wt = float(weight)
    idx = []
    Li = np.ones((1, 1))
    cur = 0  # Li is the left environment of site cur
    order = np.lexsort((np.asarray(cj), np.asarray(ci)))
    assert np.all(order == np.arange(len(ci))), "couplings must be ordered by (i, j)"
    for c, (i, j) in enumerate(zip(ci, cj)):
        i, j = int(i), int(j)
        while cur < i:
            Li = left_step(Li, T[cur], W[cur])
            cur += 1
        M = closures(T, W, Li, i, j, env.right(j + 1))
        q = jidx[c]
        Uq, VTq, Sqq = U[q], VT[q], Sq[q]
        Cm = np.empty(16)
        for l in range(4):
            for k in range(4):
                acc = 0.0
                for qq in range(4):
                    inner = 0.0
                    for pp in range(4):
                        inner += Uq[pp + 4 * k] * M[pp + 4 * qq]
                    acc += inner * VTq[l + 4 * qq]
                Cm[k + 4 * l] = Sqq[k] * Sqq[l] * acc
        fac = 4.0 / (ov * G)
        Cmat = Cm.reshape(4, 4, order="F")  # Cmat[l, r] = Cm[l + 4 r]
        pdf = np.maximum(0.0, np.einsum("gl,lr,gr->g", grid, Cmat, grid)) * fac
        pnorm = float(np.sum(pdf))
        pdf = pdf * (1.0 / pnorm)
        wt *= pnorm
        uu = float(u[c])
        count = 0
        cum = pdf[0]
        while cum <= uu and count < G - 1:
            count += 1
            cum += pdf[count]
        idx.append(count)
        x = grid[count]
        nm = float(x @ Cmat @ x)
        O1 = np.array([sum(2.0 * Sqq[k] * x[k] * Uq[o + 4 * k] for k in range(4)) for o in range(4)])
        O2 = np.array([sum(2.0 * Sqq[k] * x[k] * VTq[k + 4 * o] for k in range(4)) for o in range(4)])
        apply_op(W[i], O1)
        apply_op(W[j], O2)
        env.invalidate(j)
        ov = 4.0 * nm
    field()
    ovr = overlap(T, W)
    nrm = np.sqrt(norm2(W))
    scale = (-1.0 if ovr < 0.0 else 1.0) / nrm
    en = energy_numerator(T, W, ci, cj, cJ, h) / ovr
    W[-1] = W[-1] * scale
    return dict(weight=wt, overlap=abs(ovr) / nrm, energy=en, index=np.array(idx), walker=data_of(W))
