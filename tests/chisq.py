"""Chi-square goodness of fit of drawn outcomes against exact probabilities.

Outcomes are binned so that every bin expects at least `min_expected` draws:
outcomes are taken in decreasing order of probability and a bin is closed once
its expected count reaches the floor (an underfull last bin joins the one
before it). The
statistic sum (observed - expected)^2 / expected has (bins - 1) degrees of
freedom under the null hypothesis that the draws follow the probabilities.
"""
from __future__ import annotations

import numpy as np
from scipy.stats import chi2

P_VALUE_FLOOR = 1e-4  # a draw from the right distribution fails with this probability


def bit_reverse_index(words: np.ndarray, n: int) -> np.ndarray:
    """Result words (bit q = qubit q) -> index into the reference's get_state order
    (qubit 0 is the most significant bit)."""
    w = np.asarray(words, np.uint64)
    out = np.zeros_like(w)
    for q in range(n):
        out |= ((w >> np.uint64(q)) & np.uint64(1)) << np.uint64(n - 1 - q)
    return out


def chi_square(prob: np.ndarray, outcomes: np.ndarray, min_expected: float = 20.0) -> dict:
    """Goodness of fit of `outcomes` (indices into `prob`) against `prob`."""
    prob = np.asarray(prob, np.float64)
    prob = prob / prob.sum()
    shots = len(outcomes)
    counts = np.bincount(np.asarray(outcomes, np.int64), minlength=prob.size).astype(np.float64)
    order = np.argsort(-prob, kind="stable")
    exp_sorted = prob[order] * shots
    obs_sorted = counts[order]
    # greedy bins in that order; an underfull last bin joins the one before it
    bin_of = np.empty(prob.size, np.int64)
    b, acc = 0, 0.0
    for i, x in enumerate(exp_sorted):
        bin_of[i] = b
        acc += x
        if acc >= min_expected:
            b, acc = b + 1, 0.0
    if b > 0 and 0.0 < acc < min_expected:
        bin_of[bin_of == b] = b - 1
    nb = int(bin_of.max()) + 1
    e = np.bincount(bin_of, weights=exp_sorted, minlength=nb)
    o = np.bincount(bin_of, weights=obs_sorted, minlength=nb)
    keep = e > 0
    stat = float(np.sum((o[keep] - e[keep]) ** 2 / e[keep]))
    dof = int(keep.sum()) - 1
    return {"stat": stat, "dof": dof, "p_value": float(chi2.sf(stat, dof)), "bins": int(keep.sum()),
            "min_expected": float(e[keep].min())}
