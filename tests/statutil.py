"""Error bars of Monte Carlo energy series (test infrastructure).

reblock: mean and standard error of a serially correlated series by
Flyvbjerg-Petersen blocking (pairs of neighbours averaged level by level);
the error is the largest standard error over the levels that still hold at
least 32 blocks, which covers a correlation time up to a few blocks.
combine: independent estimates of the same length (one per process) merged
with equal weights (weights from the estimated errors would correlate with
the means).
"""
from __future__ import annotations

import numpy as np


def reblock(x, min_blocks: int = 32):
    x = np.asarray(x, float)
    mean = float(np.mean(x))
    errs = []
    while len(x) >= min_blocks:
        errs.append(float(np.std(x, ddof=1) / np.sqrt(len(x))))
        n = len(x) // 2 * 2
        x = 0.5 * (x[0:n:2] + x[1:n:2])
    if not errs:
        errs.append(float(np.std(x, ddof=1) / np.sqrt(max(len(x), 1))))
    return mean, max(errs)


def combine(estimates):
    m = np.array([e[0] for e in estimates], float)
    s = np.array([e[1] for e in estimates], float)
    return float(np.mean(m)), float(np.sqrt(np.sum(s ** 2)) / len(s))
