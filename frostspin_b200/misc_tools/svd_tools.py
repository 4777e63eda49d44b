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


_QR_STREAMS = 4
_STREAMS = {}


def _qr_streams():
    dev = torch.cuda.current_device()
    st = _STREAMS.get(dev)
    if st is None:
        st = [torch.cuda.Stream(device=dev) for _ in range(_QR_STREAMS)]
        _STREAMS[dev] = st
    return st


def truncated_svd_blocks(blocks, ks, fulls, *, n_iter=3, oversampling=None):
    """truncated_svd_block for many device blocks at once, with the same
    arithmetic per block (same seeds, same steps): the randomized blocks
    advance in lock step, every product of a step in one grouped GEMM launch
    over all of them, and the SVDs that synchronise with the host (cuSOLVER
    checks its status) come last, so that the device never waits for the host
    to plan the next block.  Returns lists (U, s, Vh)."""
    from .. import instrument, linalg

    n = len(blocks)
    out_u, out_s, out_v = [None] * n, [None] * n, [None] * n
    dense, rand = [], []
    for i, m in enumerate(blocks):
        nr, nc = m.shape
        if fulls[i] or ks[i] >= min(nr, nc) // 2:
            dense.append(i)
        else:
            rand.append(i)
    if rand:
        ms = [blocks[i] for i in rand]
        omegas = []
        for i in rand:
            m = blocks[i]
            nr, nc = m.shape
            k = int(ks[i])
            p = k + 10 if oversampling is None else oversampling
            kk = min(min(nr, nc), k + p)
            g = torch.Generator(device=m.device)
            g.manual_seed(1234 + nr * 7 + nc)
            omegas.append(torch.randn(nc, kk, dtype=m.dtype, device=m.device, generator=g))

        def qr_all(ys):
            # the QRs of the blocks are independent and each is a chain of
            # small panel kernels: spread them over side streams so that they
            # overlap, then join the main stream before the next grouped GEMM
            main = torch.cuda.current_stream()
            ready = torch.cuda.Event()
            ready.record(main)
            out = []
            with instrument.region("svd_qr"):
                for j, y in enumerate(ys):
                    side = _qr_streams()[j % _QR_STREAMS]
                    side.wait_event(ready)
                    y.record_stream(side)
                    with torch.cuda.stream(side):
                        q, _ = torch.linalg.qr(y, mode="reduced")
                    q.record_stream(main)
                    out.append(q)
                for side in _qr_streams()[: min(len(ys), _QR_STREAMS)]:
                    done = torch.cuda.Event()
                    done.record(side)
                    main.wait_event(done)
            return out

        _, _, _, ys = linalg.matmul_blocks(ms, omegas)
        qs = qr_all(ys)
        for _ in range(n_iter):
            _, _, _, zs = linalg.matmul_blocks([m.T for m in ms], qs)
            zs = qr_all(zs)
            _, _, _, ys = linalg.matmul_blocks(ms, zs)
            qs = qr_all(ys)
        _, _, _, bs = linalg.matmul_blocks([q.T for q in qs], ms)
        ubs = []
        for j, i in enumerate(rand):
            with instrument.region("svd_small"):
                ub, sv, vh = torch.linalg.svd(bs[j], full_matrices=False)
            k = int(ks[i])
            ubs.append(ub)
            out_s[i] = sv[:k]
            out_v[i] = vh[:k]
        _, _, _, us = linalg.matmul_blocks(qs, ubs)
        for j, i in enumerate(rand):
            out_u[i] = us[j][:, : int(ks[i])]
    for i in dense:
        m = blocks[i]
        with instrument.region("svd_dense", elems=float(m.shape[0] * m.shape[1])):
            u, sv, vh = torch.linalg.svd(m, full_matrices=False)
        out_u[i], out_s[i], out_v[i] = u, sv, vh
    return out_u, out_s, out_v


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
