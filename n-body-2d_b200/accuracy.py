"""Force-error statistics against the FP64 all-pairs oracle kernel.

Relative error per body: |a - a_exact| / |a_exact|, with a_exact the FP64
all-pairs sum of the reference pair law (BarnesHutCuda.cu:427-431) computed on
the GPU by nb_allpairs_accelerations.  Errors are measured on a seeded random
subsample of target bodies (65,536 by default) against all sources.
"""
from __future__ import annotations

import numpy as np

from .simulation import allpairs_accelerations


def sample_targets(n: int, k: int = 65536, seed: int = 12345) -> np.ndarray:
    if k >= n:
        return np.arange(n, dtype=np.int64)
    return np.sort(np.random.default_rng(seed).choice(n, size=k, replace=False)).astype(np.int64)


def relative_errors(acc: np.ndarray, exact: np.ndarray) -> np.ndarray:
    return np.linalg.norm(acc - exact, axis=1) / np.linalg.norm(exact, axis=1)


def summary(err: np.ndarray) -> dict:
    return {"p50": float(np.percentile(err, 50)), "p99": float(np.percentile(err, 99)),
            "max": float(err.max()), "samples": int(err.shape[0])}


def force_errors(acc_all: np.ndarray, mass: np.ndarray, pos: np.ndarray, epsilon_squared: float,
                 k: int = 65536, device: int = 0, seed: int = 12345) -> dict:
    """acc_all: accelerations of every body (original order) for the state (mass, pos)."""
    tgt = sample_targets(mass.shape[0], k, seed)
    exact = allpairs_accelerations(mass, pos, tgt, epsilon_squared, device)
    return summary(relative_errors(acc_all[tgt], exact))


def ensemble_force_errors(acc_all: np.ndarray, mass: np.ndarray, pos: np.ndarray,
                          counts: np.ndarray, epsilon_squared: float, k: int = 65536,
                          device: int = 0, seed: int = 12345) -> dict:
    """Batched universes: each sampled target against all-pairs over its own
    universe only (universes do not interact)."""
    tgt = sample_targets(mass.shape[0], k, seed)
    off = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
    uni = np.searchsorted(off, tgt, side="right") - 1
    err = np.empty(tgt.shape[0])
    for u in np.unique(uni):
        sel = np.nonzero(uni == u)[0]
        a, b = off[u], off[u + 1]
        exact = allpairs_accelerations(mass[a:b], pos[a:b], tgt[sel] - a, epsilon_squared, device)
        err[sel] = relative_errors(acc_all[tgt[sel]], exact)
    return summary(err)
