"""Host-side set-up of a walk: the inputs the reference's constructors derive, in numpy.

Everything here runs once per run, before the device walk starts:
  - Heisenberg couplings of a chain (main.cpp:36-41),
  - the Marsaglia auxiliary-field grid (GridGenerator.cpp:167-225),
  - the two-site propagator factor tables (TrotterHeisenberg.cpp:102-285),
  - the MPS text format (MPSstate.cpp:92-128 reader, 661-686 writer),
  - walker initialisation: compression to D_W (MPSstate.cpp:379-404) and seeded noise.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class MPS:
    """Bond dims [L+1] and concatenated site storages, element [r + Dl*(c + Dr*sigma)]."""
    dims: np.ndarray
    data: np.ndarray
    d: int = 2

    @property
    def L(self) -> int:
        return len(self.dims) - 1

    def copy(self) -> "MPS":
        return MPS(self.dims.copy(), self.data.copy(), self.d)

    def offsets(self) -> np.ndarray:
        sz = self.dims[:-1] * self.dims[1:] * self.d
        return np.concatenate([[0], np.cumsum(sz)])

    def site(self, s: int) -> np.ndarray:
        """Site s as array [sigma, Dl, Dr] (a copy)."""
        o = self.offsets()
        dl, dr = int(self.dims[s]), int(self.dims[s + 1])
        return self.data[o[s]:o[s + 1]].reshape(self.d, dr, dl).transpose(0, 2, 1).copy()

    @staticmethod
    def from_sites(sites: list[np.ndarray], d: int = 2) -> "MPS":
        dims = [sites[0].shape[1]] + [s.shape[2] for s in sites]
        data = np.concatenate([s.transpose(0, 2, 1).reshape(-1) for s in sites])
        return MPS(np.asarray(dims, dtype=np.int32), data, d)


def virtual_dims(L: int, D: int, d: int = 2) -> np.ndarray:
    """Bond profile min(d^k, d^(L-k), D) of MPSstate.cpp:20-28."""
    v = [1] * (L + 1)
    for c in range(1, L):
        v[c] = min(v[c - 1] * d, D)
    for c in range(L - 1, 0, -1):
        v[c] = min(min(v[c + 1] * d, D), v[c])
    return np.asarray(v, dtype=np.int32)


def chain(L: int, J: float = 1.0):
    """Open nearest-neighbour chain: couplings (i, i+1) in the order MPSQMC2.cpp:286-299 lists them."""
    ci = np.arange(L - 1, dtype=np.int32)
    return ci, ci + 1, np.full(L - 1, float(J))


def snake_site(W: int, r: int, c: int) -> int:
    """MPS position of lattice site (row r, column c) on the snake path: even rows left to
    right, odd rows right to left."""
    return r * W + (c if r % 2 == 0 else W - 1 - c)


def snake(W: int, H: int, J: float = 1.0):
    """Open W x H square lattice, nearest-neighbour couplings J, as MPS couplings (i < j) along
    the snake path, ordered by first site then second site (MPSQMC2.cpp:286-299)."""
    pairs = set()
    for r in range(H):
        for c in range(W):
            s = snake_site(W, r, c)
            if c + 1 < W:
                t = snake_site(W, r, c + 1)
                pairs.add((min(s, t), max(s, t)))
            if r + 1 < H:
                t = snake_site(W, r + 1, c)
                pairs.add((min(s, t), max(s, t)))
    pairs = sorted(pairs)
    ci = np.array([p[0] for p in pairs], dtype=np.int32)
    cj = np.array([p[1] for p in pairs], dtype=np.int32)
    return ci, cj, np.full(len(pairs), float(J))


def lattice(name: str, J: float = 1.0):
    """Couplings by name: "chain:L" or "snake:WxH"."""
    kind, _, shape = name.partition(":")
    if kind == "chain":
        return chain(int(shape), J)
    if kind == "snake":
        W, H = (int(x) for x in shape.split("x"))
        return snake(W, H, J)
    raise ValueError(f"unknown lattice {name!r}")


def _erf_inv(z: float) -> float:
    if z == 0.0:
        return 0.0
    sgn, t = (-1.0 if z < 0 else 1.0), abs(z)
    lo, hi = 0.0, 6.0
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        if math.erf(mid) < t:
            lo = mid
        else:
            hi = mid
    x = 0.5 * (lo + hi)
    for _ in range(4):
        x -= (math.erf(x) - t) / (2.0 / math.sqrt(math.pi) * math.exp(-x * x))
    return sgn * x


def grid_marsaglia(points_per_co: int = 4, dim: int = 4) -> np.ndarray:
    """Unit vectors of R^dim from inverse-normal quantiles, duplicates removed (GridGenerator.cpp:167-225).

    Returns [G, dim]; the default (4, 4) gives the reference's 240-point grid."""
    one = [_erf_inv(2 * (c + 0.5) / points_per_co - 1.0) for c in range(points_per_co)]
    pts: list[np.ndarray] = []
    for cnt in range(points_per_co ** dim):
        cc, att = cnt, np.zeros(dim)
        for k in range(dim):
            rem = cc % points_per_co
            att[k] = one[rem]
            cc = (cc - rem) // points_per_co
        nrm = float(np.sum(att * att))
        if nrm > 1e-16:
            att = att / math.sqrt(nrm)
            if all(float(np.sum((att - p) ** 2)) >= 1e-16 for p in pts):
                pts.append(att)
    return np.asarray(pts)


def spin_ops(d: int = 2):
    """S^z, S^x and i S^y in the basis m = -S..S (OpSz.cpp:9, OpSx.cpp:11, OpISy.cpp:11-21)."""
    sz = np.diag([0.5 * (1 - d) + i for i in range(d)])
    lad = [0.25 * math.sqrt(d * d - 1.0 - (1.0 - d + 2 * k) * (3.0 - d + 2 * k)) for k in range(d - 1)]
    sx, isy = np.zeros((d, d)), np.zeros((d, d))
    for k in range(d - 1):
        sx[k + 1, k] = sx[k, k + 1] = lad[k]
        isy[k + 1, k] = lad[k]
        isy[k, k + 1] = -lad[k]
    return sz, sx, isy


def trotter_tables(J: float, dtau: float, d: int = 2):
    """SVD factors of exp(-dtau J S_1.S_2) reshuffled to (site-1 op) x (site-2 op).

    Returns U [d^4] (U[i + d(j + d k)]), S [d^2], VT [d^4] (VT[k + d^2 (i + d j)]) as in
    TrotterHeisenberg.cpp:102-285.  Singular vectors of the degenerate singular values are
    basis-dependent, so runs that must replay a reference trajectory pass its tables instead."""
    sz, sx, isy = spin_ops(d)
    n = d * d
    H = np.zeros((n, n))
    for r1 in range(d):
        for c1 in range(d):
            for r2 in range(d):
                for c2 in range(d):
                    H[r1 + d * r2, c1 + d * c2] = sx[r1, c1] * sx[r2, c2] - isy[r1, c1] * isy[r2, c2] + \
                        sz[r1, c1] * sz[r2, c2]
    lam, V = np.linalg.eigh(H)
    W = V * np.exp(-0.5 * dtau * J * lam)[None, :]
    P = W @ W.T
    Q = np.zeros((n, n))
    for r1 in range(d):
        for c1 in range(d):
            for r2 in range(d):
                for c2 in range(d):
                    Q[r1 + d * c1, r2 + d * c2] = P[r1 + d * r2, c1 + d * c2]
    u, s, vt = np.linalg.svd(Q)
    return u.reshape(-1, order="F").copy(), s.copy(), vt.reshape(-1, order="F").copy()


def read_mps(path: str, d_default: int = 2) -> MPS:
    """MPS text format of MPSstate.cpp:661-686 (reader: 92-128)."""
    toks = open(path).read().split()
    L, _D, d = int(toks[0]), int(toks[1]), int(toks[2])
    p = 3
    dims = np.zeros(L + 1, dtype=np.int32)
    for _ in range(L + 1):
        dims[int(toks[p])] = int(toks[p + 1])
        p += 2
    chunks = []
    for _ in range(L):
        n = int(toks[p + 1])
        p += 2
        chunks.append(np.array(toks[p:p + 3 * n], dtype=object).reshape(n, 3)[:, 2].astype(np.float64))
        p += 3 * n
    return MPS(dims, np.concatenate(chunks), d)


def write_mps(path: str, m: MPS) -> None:
    L, d = m.L, m.d
    lines = [f"{L}\t{int(max(m.dims))}\t{d}"] + [f"{i}\t{int(v)}" for i, v in enumerate(m.dims)]
    o = m.offsets()
    for s in range(L):
        n = int(o[s + 1] - o[s])
        lines.append(f"{s}\t{n}")
        lines += [f"{s}\t{j}\t{m.data[o[s] + j]:.17g}" for j in range(n)]
    open(path, "w").write("\n".join(lines) + "\n")


def left_normalize(m: MPS) -> MPS:
    """Left-canonical form by QR sweeps (numpy's QR; the last site carries the norm, which is
    divided out).  For synthetic inputs: the reference-exact LeftNormalize is the engine's
    set_overlap and the oracle's."""
    L, d = m.L, 2
    dims = list(m.dims)
    sites = []
    off = 0
    for k in range(L):
        n = dims[k] * dims[k + 1] * d
        sites.append(m.data[off:off + n].reshape((d, dims[k + 1], dims[k])).transpose(2, 0, 1))  # [r, s, c]
        off += n
    out = []
    carry = np.ones((1, 1))
    for k in range(L):
        A = np.einsum("ab,bsc->asc", carry, sites[k])
        a, s_, c = A.shape
        if k < L - 1:
            Q, R = np.linalg.qr(A.reshape(a * s_, c))
            r = Q.shape[1]
            out.append(Q.reshape(a, s_, r))
            carry = R
            dims[k + 1] = r
        else:
            A = A / np.linalg.norm(A)
            out.append(A)
    data = np.concatenate([t.transpose(1, 2, 0).ravel() for t in out])  # [s, c, r] -> r fastest
    return MPS(np.asarray(dims, np.int32), data)


def compress(m: MPS, D: int, cut: float = 1e-13) -> MPS:
    """Two-sweep two-site SVD truncation to bond dimension D (MPSstate.cpp:379-404 with
    TwoSiteObject.cpp:71-184): left-to-right with S pushed right, then right-to-left with S
    pushed left; Schmidt values below `cut` are always dropped."""
    sites = [m.site(s) for s in range(m.L)]
    d = m.d

    def step(s, movingright):
        A, B = sites[s], sites[s + 1]
        DL, DR = A.shape[1], B.shape[2]
        theta = np.einsum("iab,jbc->aicj", A, B).reshape(DL * d, DR * d)
        u, sv, vt = np.linalg.svd(theta, full_matrices=False)
        keep = min(D, int(np.sum(sv >= cut)) if np.any(sv < cut) else len(sv))
        keep = max(keep, 1)
        u, sv, vt = u[:, :keep], sv[:keep], vt[:keep]
        if movingright:
            vt = sv[:, None] * vt
        else:
            u = u * sv[None, :]
        sites[s] = u.reshape(DL, d, keep).transpose(1, 0, 2).copy()
        sites[s + 1] = vt.reshape(keep, DR, d).transpose(2, 0, 1).copy()

    for s in range(m.L - 1):
        step(s, True)
    for s in range(m.L - 2, -1, -1):
        step(s, False)
    return MPS.from_sites(sites, d)


def add_noise(m: MPS, sigma: float, rng: np.random.Generator) -> MPS:
    """Trial-derived walker with i.i.d. N(0, sigma^2) added to every tensor element."""
    out = m.copy()
    out.data = out.data + rng.normal(0.0, sigma, size=out.data.shape)
    return out
