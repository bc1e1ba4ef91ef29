"""Test infrastructure: exact diagonalisation of the open spin-1/2 Heisenberg chain in the
S^z_tot = 0 sector (sparse Lanczos via scipy's eigsh).  The reference has no ED; its main.cpp:153
quotes E_FCI = -4.25803520728288 for L = 10, which pins this routine.
"""
from __future__ import annotations

from functools import lru_cache
from itertools import combinations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as sla


def chain_hamiltonian(L: int, J: float = 1.0, bonds=None) -> sp.csr_matrix:
    """H = sum_(i,j) J S_i.S_j on the half-filled (S^z = 0) sector; bonds default to the open chain."""
    if bonds is None:
        bonds = [(i, i + 1, J) for i in range(L - 1)]
    states = np.array([sum(1 << i for i in c) for c in combinations(range(L), L // 2)], dtype=np.int64)
    index = {int(s): k for k, s in enumerate(states)}
    rows, cols, vals = [], [], []
    for k, s in enumerate(states):
        s = int(s)
        diag = 0.0
        for i, j, Jb in bonds:
            bi, bj = (s >> i) & 1, (s >> j) & 1
            diag += Jb * (0.25 if bi == bj else -0.25)
            if bi != bj:
                t = s ^ ((1 << i) | (1 << j))
                rows.append(index[t])
                cols.append(k)
                vals.append(0.5 * Jb)
        rows.append(k)
        cols.append(k)
        vals.append(diag)
    n = len(states)
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))


@lru_cache(maxsize=None)
def ground_energy(L: int, J: float = 1.0) -> float:
    H = chain_hamiltonian(L, J)
    if H.shape[0] < 64:
        return float(np.linalg.eigvalsh(H.toarray())[0])
    w = sla.eigsh(H, k=1, which="SA", tol=1e-14, return_eigenvectors=False)
    return float(w[0])


def ground_energy_couplings(L: int, ci, cj, cJ) -> float:
    """Ground energy of H = sum_c J_c S_ci.S_cj (any couplings, e.g. a 2D lattice on a snake path)
    in the sector with L//2 up spins (it holds the ground state: S^z = 0, or -1/2 for odd L)."""
    H = chain_hamiltonian(L, bonds=[(int(i), int(j), float(J)) for i, j, J in zip(ci, cj, cJ)])
    if H.shape[0] < 64:
        return float(np.linalg.eigvalsh(H.toarray())[0])
    w = sla.eigsh(H, k=1, which="SA", tol=1e-14, return_eigenvectors=False)
    return float(w[0])
