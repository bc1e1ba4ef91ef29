"""Statistics of a walk's energy series: blocking error of the mean and the variance-normalised
throughput used to compare walk variants at equal accuracy.

VN = (walker-steps/s) / sigma2_ws, with sigma2_ws = Var(mean E_P) * N_ws: the variance of the
mean that one walker-step buys.  Two variants reach the same error of the mean in wall-clock
time inversely proportional to their VN.
"""
from __future__ import annotations

import numpy as np


def blocking_levels(x):
    """Flyvbjerg-Petersen blocking: (number of blocks, error of the mean) at every level, halving
    the series by averaging neighbours until fewer than 4 blocks remain."""
    x = np.asarray(x, dtype=np.float64)
    out = []
    while x.size >= 4:
        n = x.size
        out.append((n, float(np.std(x, ddof=1) / np.sqrt(n))))
        m = n // 2
        x = 0.5 * (x[0:2 * m:2] + x[1:2 * m:2])
    return out


def blocking_error(x, min_blocks: int = 16) -> float:
    """Error of the mean of a correlated series: the largest blocking estimate among the levels
    that keep at least min_blocks blocks (the plateau for series much longer than their
    correlation time)."""
    lv = [e for n, e in blocking_levels(x) if n >= min_blocks]
    if not lv:
        lv = [e for _, e in blocking_levels(x)]
    return max(lv) if lv else float("nan")


def variance_normalised(walker_steps_per_s: float, energies, walkers_per_step, equil_frac: float = 0.2):
    """VN and the numbers behind it for the series of per-step mixed energies."""
    e = np.asarray(energies, dtype=np.float64)
    n = np.asarray(walkers_per_step, dtype=np.float64)
    k0 = int(len(e) * equil_frac)
    e, n = e[k0:], n[k0:]
    err = blocking_error(e)
    n_ws = float(n.sum())
    sigma2_ws = err * err * n_ws
    return {"steps_used": int(len(e)), "equil_steps": k0, "E_mean": float(e.mean()), "E_err": err,
            "walker_steps": n_ws, "sigma2_ws": sigma2_ws,
            "vn": walker_steps_per_s / sigma2_ws if sigma2_ws > 0 else float("nan")}


def proposal_gain_bound(weights_per_step):
    """The largest factor by which any auxiliary-field proposal could lower the variance of the
    weighted mean energy, from the walkers' weights after propagation.

    With the grid PDF every coupling multiplies a weight by sum P whatever x is drawn, so the
    weights of a step differ only through the product of those sums along each walker's path.  A
    proposal that made all weights equal (the best case, zero weight variance) would turn the
    weighted mean's variance Var(E) / N_eff into Var(E) / N, N_eff = (sum w)^2 / sum w^2: a gain of
    N / N_eff = N sum w^2 / (sum w)^2 at most.  Returns its mean over the steps."""
    g = []
    for w in weights_per_step:
        w = np.asarray(w, dtype=np.float64)
        if w.size and w.sum() > 0:
            g.append(w.size * float(np.sum(w * w)) / float(w.sum()) ** 2)
    return float(np.mean(g)) if g else float("nan")
