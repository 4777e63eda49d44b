"""Device dispatch for block-list linear algebra: grouped GEMM and reductions.

A *block reference* is (buffer, element offset, m, n, trans): the logical m x n
block stored C-order at buffer[offset:] when trans is False, or as its n x m
transpose (F-order view) when trans is True.
"""

import contextlib

import numpy as np
import torch

from . import _native
from . import device as dev

# ----------------------------------------------------------------- precision

_PRECISION = {"gemm": "fp64"}
PRECISIONS = ("fp64",)


def gemm_precision():
    return _PRECISION["gemm"]


def set_gemm_precision(mode):
    """Select the sector-GEMM arithmetic: "fp64" (plain double precision)."""
    if mode not in PRECISIONS:
        msg = f"unknown GEMM precision {mode!r}; choose from {PRECISIONS}"
        raise ValueError(msg)
    _PRECISION["gemm"] = mode


@contextlib.contextmanager
def gemm_precision_mode(mode):
    old = gemm_precision()
    set_gemm_precision(mode)
    try:
        yield
    finally:
        set_gemm_precision(old)


# ------------------------------------------------------------- grouped GEMM

_TILE = None


def _tile_shape():
    global _TILE
    if _TILE is None:
        _TILE = _native.dgemm_tile_shape()
    return _TILE


def grouped_gemm(problems):
    """Run C = alpha op(A) op(B) + beta C for every problem in one launch.

    problems: list of dicts with keys A, B, C (torch buffers), a_off, b_off,
    c_off (element offsets), M, N, K, a_trans, b_trans, alpha, beta.  C blocks
    are C-order (ldc = N).  A with a_trans False is C-order M x K (lda = K);
    with a_trans True it is stored K x M (lda = M).  Likewise for B.
    """
    n = len(problems)
    if n == 0:
        return
    arr = np.zeros(n, dtype=_native.GEMM_PROBLEM_DTYPE)
    tm, tn = _tile_shape()
    ntile = []
    for i, p in enumerate(problems):
        M, N, K = int(p["M"]), int(p["N"]), int(p["K"])
        arr["A"][i] = p["A"].data_ptr() + 8 * int(p["a_off"])
        arr["B"][i] = p["B"].data_ptr() + 8 * int(p["b_off"])
        arr["C"][i] = p["C"].data_ptr() + 8 * int(p["c_off"])
        arr["lda"][i] = M if p["a_trans"] else K
        arr["ldb"][i] = K if p["b_trans"] else N
        arr["ldc"][i] = N
        arr["M"][i], arr["N"][i], arr["K"][i] = M, N, K
        arr["transA"][i] = int(bool(p["a_trans"]))
        arr["transB"][i] = int(bool(p["b_trans"]))
        arr["alpha"][i] = p.get("alpha", 1.0)
        arr["beta"][i] = p.get("beta", 0.0)
        ntile.append(((M + tm - 1) // tm) * ((N + tn - 1) // tn))
    if gemm_precision() == "fp64":
        _dgemm(arr, problems, tm, tn, np.array(ntile, dtype=np.int64))
    else:  # pragma: no cover - guarded by set_gemm_precision
        raise ValueError(gemm_precision())


def _tile_table(arr, tm, tn, ntile):
    total = int(ntile.sum())
    tiles = np.zeros(total, dtype=_native.GEMM_TILE_DTYPE)
    pid = np.repeat(np.arange(arr.size), ntile)
    first = np.repeat(np.cumsum(ntile) - ntile, ntile)
    k = np.arange(total) - first
    ncol = (arr["N"].astype(np.int64) + tn - 1) // tn
    tiles["problem"] = pid
    tiles["tm"] = k // ncol[pid]
    tiles["tn"] = k % ncol[pid]
    # largest problems first: long tiles start early in the static schedule
    order = np.argsort(-arr["K"][pid].astype(np.int64), kind="stable")
    return tiles[order]


def _dgemm(arr, problems, tm, tn, ntile):
    tiles = _tile_table(arr, tm, tn, ntile)
    d_prob = dev.upload(arr)
    d_tiles = dev.upload(tiles)
    _native.call(
        "fs_grouped_dgemm",
        d_prob.data_ptr(),
        arr.size,
        d_tiles.data_ptr(),
        tiles.size,
        dev.stream(),
    )
    return d_prob, d_tiles


# --------------------------------------------------------------- reductions


def weighted_reduce(buf, offsets, lengths, weights, *, squares):
    """sum_s w_s sum_i f(buf[off_s + i]) with f = x^2 or x; returns a 0-d device
    tensor (no host synchronisation)."""
    out = torch.empty(1, dtype=torch.float64, device=buf.device)
    segs = np.zeros(len(offsets), dtype=_native.SEGMENT_DTYPE)
    segs["offset"] = offsets
    segs["length"] = lengths
    segs["weight"] = weights
    part = dev.scratch_partials()
    d_segs = dev.upload(segs)
    name = "fs_weighted_sumsq" if squares else "fs_weighted_sum"
    _native.call(
        name,
        dev.ptr(buf),
        d_segs.data_ptr(),
        segs.size,
        part.data_ptr(),
        part.numel(),
        out.data_ptr(),
        dev.stream(),
    )
    return out[0]


def pair_contract(abuf, bbuf, pairs):
    """pairs: list of (a_off, b_off, m, n, a_trans, b_trans, weight); b_off < 0
    means trace of the A block.  Returns a 0-d device tensor."""
    out = torch.empty(1, dtype=torch.float64, device=abuf.device)
    tab = np.zeros(len(pairs), dtype=_native.PAIR_BLOCK_DTYPE)
    for i, (ao, bo, m, n, at, bt, w) in enumerate(pairs):
        tab[i] = (ao, bo, m, n, int(at), int(bt), w)
    part = dev.scratch_partials()
    d_tab = dev.upload(tab)
    _native.call(
        "fs_pair_contract",
        dev.ptr(abuf),
        dev.ptr(bbuf) if bbuf is not None else None,
        d_tab.data_ptr(),
        tab.size,
        part.data_ptr(),
        part.numel(),
        out.data_ptr(),
        dev.stream(),
    )
    return out[0]


def axpby(x, y, a, b):
    """y = a x + b y over whole buffers (same length)."""
    if x.numel() != y.numel():
        raise ValueError("axpby length mismatch")
    _native.call("fs_axpby", dev.ptr(x), dev.ptr(y), x.numel(), float(a), float(b),
                 dev.stream())


def scale_(x, alpha):
    _native.call("fs_scale", dev.ptr(x), x.numel(), float(alpha), dev.stream())


def power(x, p):
    y = torch.empty_like(x)
    _native.call("fs_pow", dev.ptr(x), dev.ptr(y), x.numel(), float(p), dev.stream())
    return y


def diag_mul(xbuf, dbuf, entries, out_len):
    """entries: list of (x_off, out_off, d_off, m, n, x_trans, left)."""
    out = dev.empty_f64(out_len)
    tab = np.zeros(len(entries), dtype=_native.DIAG_BLOCK_DTYPE)
    for i, e in enumerate(entries):
        tab[i] = (e[0], e[1], e[2], e[3], e[4], int(e[5]), int(e[6]))
    d_tab = dev.upload(tab)
    _native.call(
        "fs_diag_mul",
        dev.ptr(xbuf),
        dev.ptr(dbuf),
        dev.ptr(out),
        d_tab.data_ptr(),
        tab.size,
        dev.stream(),
    )
    return out
