"""CPU model of the standardised genotype Gram operator (test helper; uses the oracle)."""

from __future__ import annotations

import numpy as np


def standardized_xtx_reference(oracle, ploidy: int, has_missing: bool, v: np.ndarray) -> np.ndarray:
    """``Zᵀ Z v`` computed on the CPU through the oracle: the same steps as
    ``grg_spmv_b200.xtx.StandardizedXTX.apply`` (reference ``scripts/pca_bench/__main__.py:201-236,
    326-347``), in NumPy FP64."""
    M = oracle.num_mutations
    ones = np.ones((1, oracle.num_individuals))
    miss = np.zeros((1, M))
    counts = oracle.matmul(ones, "up", by_individual=True, miss=miss if has_missing else None)[0]
    miss_counts = miss[0] if has_missing else np.zeros(M)
    denom = float(oracle.num_samples) - miss_counts
    valid = denom != 0.0
    freqs = np.where(valid, counts / np.where(valid, denom, 1.0), 0.0)
    center = ploidy * freqs
    sigma = np.sqrt(ploidy * freqs * (1.0 - freqs))
    sigma = np.where(sigma == 0.0, 1.0, sigma)
    d = (v / sigma[:, None]).T
    c_down = d @ center
    dmiss = d * freqs[None, :] if has_missing else None
    u = oracle.matmul(d, "down", by_individual=True, miss=dmiss) - c_down[:, None]
    c_up = u.sum(axis=1)
    um = np.zeros((u.shape[0], M))
    res = oracle.matmul(u, "up", by_individual=True, miss=um if has_missing else None)
    if has_missing:
        res = res + um * freqs[None, :]
    res = res / sigma[None, :] - c_up[:, None] * (center / sigma)[None, :]
    return res.T
