"""Seeded synthetic sparse tensors for the tests (numpy, small sizes).

Indices per mode are uniform or bounded Zipf(alpha) with P(k) ~ (k+1)^-alpha
(index 0 most frequent), drawn by inverse CDF; values uniform(0,1). The raw
draw keeps duplicates; callers clean it (duplicates summed in input order,
empty slices compacted) with the oracle or the GPU.
"""
import numpy as np


def draw_coo(dims, nnz, seed, alpha=None):
    rng = np.random.default_rng(seed)
    inds = []
    for m, d in enumerate(dims):
        a = alpha[m] if isinstance(alpha, (list, tuple)) else alpha
        if a is None or a <= 0:
            inds.append(rng.integers(0, d, nnz))
        else:
            w = np.arange(1, d + 1, dtype=np.float64) ** (-a)
            cdf = np.cumsum(w) / w.sum()
            cdf[-1] = 1.0
            inds.append(np.searchsorted(cdf, rng.random(nnz), side="right"))
    inds = np.stack(inds).astype(np.uint64)
    vals = rng.random(nnz)
    return inds, vals, [int(d) for d in dims]


def dense_mttkrp(inds, vals, dims, mats, mode):
    """Brute-force MTTKRP: sum over nonzeros of v * Hadamard of the other rows."""
    R = mats[0].shape[1]
    out = np.zeros((dims[mode], R))
    prod = np.ones((inds.shape[1], R))
    for m in range(len(dims)):
        if m != mode:
            prod *= mats[m][inds[m].astype(np.int64)]
    np.add.at(out, inds[mode].astype(np.int64), vals[:, None] * prod)
    return out
