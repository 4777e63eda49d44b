"""Truncation helpers (frostspin/misc_tools/svd_tools.py:7-74).

find_block_cuts runs on the host on the (small) vectors of leading singular
values copied back from the device: its decisions must be bit-identical to the
reference's greedy loop, so it uses the same float64 comparisons in the same
order.
"""

import numpy as np
import torch


def truncated_svd_block(m, k, *, full, n_iter=3, oversampling=None):
    """Leading singular triplets of one device block.

    full=True: dense SVD (cuSOLVER), all values, like the reference's robust_svd
    path (svd_tools.py:116-151).  Otherwise the k leading triplets by subspace
    iteration with re-orthogonalisation (Halko, Martinsson, Tropp 2011,
    Algorithm 4.4) on a basis of k + oversampling vectors -- the role ARPACK on
    X^H X plays in the reference's sparse_svd (svd_tools.py:154-197), with the
    products on the device.  Returns (U, s, Vh) with s decreasing.
    """
    from .. import instrument, linalg

    nr, nc = m.shape
    dmin = min(nr, nc)
    if full or k >= dmin // 2:
        with instrument.region("svd_dense", elems=float(nr * nc)):
            u, s, vh = torch.linalg.svd(m, full_matrices=False)
        return u, s, vh

    p = k + 10 if oversampling is None else oversampling
    kk = min(dmin, k + p)
    g = torch.Generator(device=m.device)
    g.manual_seed(1234 + nr * 7 + nc)
    omega = torch.randn(nc, kk, dtype=m.dtype, device=m.device, generator=g)
    _, _, _, (y,) = linalg.matmul_blocks([m], [omega])
    with instrument.region("svd_qr"):
        q, _ = torch.linalg.qr(y, mode="reduced")
    for _ in range(n_iter):
        _, _, _, (z,) = linalg.matmul_blocks([m.T], [q])
        with instrument.region("svd_qr"):
            z, _ = torch.linalg.qr(z, mode="reduced")
        _, _, _, (y,) = linalg.matmul_blocks([m], [z])
        with instrument.region("svd_qr"):
            q, _ = torch.linalg.qr(y, mode="reduced")
    _, _, _, (b,) = linalg.matmul_blocks([q.T], [m])
    with instrument.region("svd_small"):
        ub, s, vh = torch.linalg.svd(b, full_matrices=False)
    _, _, _, (u,) = linalg.matmul_blocks([q], [ub])
    return u[:, :k], s[:k], vh[:k]


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
