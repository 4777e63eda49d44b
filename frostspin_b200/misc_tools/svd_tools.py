"""Truncation helpers (frostspin/misc_tools/svd_tools.py:7-74).

find_block_cuts runs on the host on the (small) vectors of leading singular
values copied back from the device: its decisions must be bit-identical to the
reference's greedy loop, so it uses the same float64 comparisons in the same
order.
"""

import numpy as np


def find_block_cuts(block_values, cut_target, *, dims=None, atol=0.0, rtol=None,
                    degen_ratio=1.0):
    """Number of values to keep per block.

    Greedy (svd_tools.py:57-74): repeatedly take the block whose next value is
    the largest; take together every value >= degen_ratio * that value
    (multiplets); a value of block i counts dims[i]; stop once cut_target is
    reached or the next value is <= atol + rtol * max(values).  rtol defaults to
    (number of values) * eps.
    """
    vals = [np.asarray(b, dtype=np.float64).ravel() for b in block_values]
    n = len(vals)
    if n == 0:
        return np.zeros(0, dtype=np.int64)
    dims = np.ones(n, dtype=np.int64) if dims is None else np.asarray(dims, dtype=np.int64)
    if dims.shape != (n,):
        raise ValueError("dims does not match the number of blocks")
    if rtol is None:
        rtol = sum(v.size for v in vals) * np.finfo(np.float64).eps
    cutoff = float(atol + rtol * max(float(v[0]) for v in vals))
    degen_ratio = float(degen_ratio)
    if degen_ratio > 1.0:
        raise ValueError("degen_ratio must be <= 1")
    cur = np.array([v[0] for v in vals], dtype=np.float64)
    cuts = np.zeros(n, dtype=np.int64)
    kept = 0
    bi = int(cur.argmax())
    cut_target = int(cut_target)
    while cur[bi] > cutoff and kept < cut_target:
        c = degen_ratio * cur[bi]
        while cur[bi] >= c:
            cuts[bi] += 1
            kept += int(dims[bi])
            cur[bi] = vals[bi][cuts[bi]] if cuts[bi] < vals[bi].size else -1.0
            bi = int(cur.argmax())
    return cuts
