"""Device dispatch for block-list linear algebra: grouped GEMM and reductions.

A *block reference* is (buffer, element offset, m, n, trans): the logical m x n
block stored C-order at buffer[offset:] when trans is False, or as its n x m
transpose (F-order view) when trans is True.
"""

import contextlib

import numpy as np
import torch

from . import _native, autotune, instrument
from . import device as dev

# ----------------------------------------------------------------- precision

_PRECISION = {"gemm": "fp64", "dispatch": "cost", "pair": True}
PRECISIONS = (
    ("fp64",)
    + tuple(f"ozaki{s}" for s in range(3, _native.FS_OZAKI_MAX_SLICES + 1))
    + tuple(f"ozaki2_{n}" for n in range(_native.FS_OZAKI2_MIN_MODULI,
                                         _native.FS_OZAKI2_MAX_MODULI + 1))
)


def gemm_precision():
    return _PRECISION["gemm"]


def set_gemm_precision(mode):
    """Select the sector-GEMM arithmetic: "fp64" (plain double precision on the
    FP64 pipes), "ozakiS" (FP64 operands split into S int8 digit slices, exact
    int32 products on the tcgen05 tensor cores, FP64 recombination; relative
    error ~2^-7S of the row/column maxima, S = 3..8; S(S+1)/2 int8 products) or
    "ozaki2_N" (operands rounded to scaled integers, one int8 product per
    modulus for N = 8..14 coprime moduli, exact CRT reconstruction in FP64;
    relative error ~2^-min(a, b) with a, b from fs_ozaki2_bits, 2^-48 at
    N = 14 and K = 2048)."""
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


@contextlib.contextmanager
def ozaki_dispatch_mode(kind):
    """Which sector GEMMs take the Ozaki path in an ozakiS mode: "cost" (the
    default: those the cost model finds faster than FP64) or "all"."""
    if kind not in ("cost", "all"):
        raise ValueError(kind)
    old = _PRECISION["dispatch"]
    _PRECISION["dispatch"] = kind
    try:
        yield
    finally:
        _PRECISION["dispatch"] = old


def set_ozaki_pair(enabled):
    """Default for ozaki_pair_mode (see there)."""
    _PRECISION["pair"] = bool(enabled)


@contextlib.contextmanager
def ozaki_pair_mode(enabled):
    """Whether Ozaki problems with more than 128 rows run on CTA pairs
    (fs_ozaki_gemm_pair, the default: 15 % faster SU(2) CTMRG iterations at
    chi = 256 than on single CTAs) or on single CTAs (fs_ozaki_gemm); the
    results are bit-identical."""
    old = _PRECISION["pair"]
    _PRECISION["pair"] = bool(enabled)
    try:
        yield
    finally:
        _PRECISION["pair"] = old


# ------------------------------------------------------------- grouped GEMM

# when a list: every grouped_gemm call appends its problem table (the shapes the
# autotuner and the profiling scripts replay)
_RECORDER = None

# when a dict: grouped GEMM problems and abelian permutes are collected and
# launched together when the shared_launches block ends
_SHARED = None


@contextlib.contextmanager
def shared_launches():
    """Collect the sector GEMMs and abelian permutes issued inside the block
    and launch them together on exit: one grouped GEMM launch for all GEMM
    problems and one multi-buffer permute launch for all permutes.  The
    operations inside must be independent of each other (one step of many
    independent runs); their output buffers exist as soon as the call
    returns, their contents once the block has ended."""
    global _SHARED
    old, _SHARED = _SHARED, {"gemm": [], "perm": []}
    try:
        yield
        pend = _SHARED
        _SHARED = old
        if pend["perm"]:
            _flush_permutes(pend["perm"])
        if pend["gemm"]:
            grouped_gemm(pend["gemm"])
    finally:
        _SHARED = old


def defer_permute(ebs, tasks, src, out, nbytes):
    """Queue one abelian permute (its host EB and task tables, source and
    destination buffers) for the enclosing shared_launches block; returns
    False when no block is open."""
    if _SHARED is None:
        return False
    _SHARED["perm"].append((ebs, tasks, src, out, nbytes))
    return True


def _flush_permutes(items):
    bufs = np.zeros(len(items), dtype=_native.PERM_BUFFERS_DTYPE)
    ebs_all, tasks_all = [], []
    n_eb = 0
    nbytes = 0.0
    for i, (ebs, tasks, src, out, nb) in enumerate(items):
        bufs[i] = (dev.ptr(src), int(src.numel()), dev.ptr(out), int(out.numel()))
        e = ebs.copy()
        e["pad"] = i
        t = tasks.copy()
        t["eb"] += n_eb
        n_eb += e.size
        ebs_all.append(e)
        tasks_all.append(t)
        nbytes += nb
    ebs_all = np.concatenate(ebs_all)
    tasks_all = np.concatenate(tasks_all)
    if tasks_all.size == 0:
        return
    d_bufs, d_ebs, d_tasks = dev.upload(bufs), dev.upload(ebs_all), dev.upload(tasks_all)
    with instrument.region("permute", bytes=nbytes):
        _native.call("fs_abelian_permute_multi", d_bufs.data_ptr(), bufs.size,
                     d_ebs.data_ptr(), ebs_all.size, d_tasks.data_ptr(), tasks_all.size,
                     None, dev.stream())


@contextlib.contextmanager
def record_gemm_calls():
    """Collect the FsGemmProblem tables of every grouped_gemm call made inside."""
    global _RECORDER
    old, _RECORDER = _RECORDER, []
    try:
        yield _RECORDER
    finally:
        _RECORDER = old

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
    if _SHARED is not None:
        _SHARED["gemm"].extend(problems)
        return
    arr = np.zeros(n, dtype=_native.GEMM_PROBLEM_DTYPE)
    tm, tn = _tile_shape()
    ntile = []
    for i, p in enumerate(problems):
        M, N, K = int(p["M"]), int(p["N"]), int(p["K"])
        arr["A"][i] = p["A"].data_ptr() + 8 * int(p["a_off"])
        arr["B"][i] = p["B"].data_ptr() + 8 * int(p["b_off"])
        arr["C"][i] = p["C"].data_ptr() + 8 * int(p["c_off"])
        arr["lda"][i] = p.get("lda", M if p["a_trans"] else K)
        arr["ldb"][i] = p.get("ldb", K if p["b_trans"] else N)
        arr["ldc"][i] = N
        arr["M"][i], arr["N"][i], arr["K"][i] = M, N, K
        arr["transA"][i] = int(bool(p["a_trans"]))
        arr["transB"][i] = int(bool(p["b_trans"]))
        arr["alpha"][i] = p.get("alpha", 1.0)
        arr["beta"][i] = p.get("beta", 0.0)
        ntile.append(((M + tm - 1) // tm) * ((N + tn - 1) // tn))
    if _RECORDER is not None:
        _RECORDER.append(arr.copy())
    mode = gemm_precision()
    ntile = np.array(ntile, dtype=np.int64)
    flops = 2.0 * (arr["M"].astype(np.float64) * arr["N"] * arr["K"])
    if mode == "fp64":
        with instrument.region("gemm_fp64", flops=float(flops.sum())):
            _dgemm(arr, problems, tm, tn, ntile)
    elif mode.startswith("ozaki2_"):
        nmod = int(mode[7:])
        fits = arr["K"].astype(np.int64) <= _native.FS_OZAKI2_MAX_K
        if _PRECISION["dispatch"] == "all":
            use = fits
        else:
            use = fits & _tuned(arr, mode, ozaki2_pays(arr, nmod))
        if use.any():
            # regions inside: the split kernels and the tcgen05 GEMM apart
            ozaki2_gemm(arr[use], nmod, flops=float(flops[use].sum()),
                        int8_ops=ozaki2_int8_ops(arr[use], nmod))
        if (~use).any():
            with instrument.region("gemm_fp64", flops=float(flops[~use].sum())):
                _dgemm(arr[~use], None, tm, tn, ntile[~use])
    elif mode.startswith("ozaki"):
        S = int(mode[5:])
        if _PRECISION["dispatch"] == "all":
            use = np.ones(arr.size, dtype=bool)
        else:
            use = _tuned(arr, mode, ozaki_pays(arr, S))
        if use.any():
            with instrument.region("gemm_ozaki", flops=float(flops[use].sum()),
                                   int8_ops=ozaki_int8_ops(arr[use], S)):
                ozaki_gemm(arr[use], S)
        if (~use).any():
            with instrument.region("gemm_fp64", flops=float(flops[~use].sum())):
                _dgemm(arr[~use], None, tm, tn, ntile[~use])
    else:  # pragma: no cover - guarded by set_gemm_precision
        raise ValueError(mode)


_THIN = None


def _thin_shape():
    global _THIN
    if _THIN is None:
        _THIN = _native.thin_dgemm_shape()
    return _THIN


def grouped_dgemm_table(arr, region="gemm_fp64"):
    """FP64 grouped GEMM over a prepared FsGemmProblem table (pointers already
    set); always FP64, whatever the precision mode.  Thin row-major problems
    (M, K <= 32) go to the bandwidth kernel, the rest to the DMMA kernel."""
    if arr.size == 0:
        return
    max_m, max_k, thin_n = _thin_shape()
    M = arr["M"].astype(np.int64)
    N = arr["N"].astype(np.int64)
    K = arr["K"].astype(np.int64)
    thin = (M <= max_m) & (K <= max_k) & (arr["transA"] == 0) & (arr["transB"] == 0)
    if thin.any():
        sub = arr[thin]
        nt = (N[thin] + thin_n - 1) // thin_n
        runs, total = _tile_runs(nt, nt, np.arange(sub.size))
        d_prob = dev.upload(sub)
        d_tiles = _device_tiles(runs, total)
        flops = 2.0 * float((M[thin].astype(np.float64) * N[thin] * K[thin]).sum())
        with instrument.region(region + "_thin", flops=flops,
                               bytes=8.0 * float((N[thin] * (M[thin] + K[thin])).sum())):
            _native.call("fs_grouped_dgemm_thin", d_prob.data_ptr(), sub.size,
                         d_tiles.data_ptr(), total, dev.stream())
    if (~thin).any():
        sub = arr[~thin]
        tm, tn = _tile_shape()
        ntile = ((M[~thin] + tm - 1) // tm) * ((N[~thin] + tn - 1) // tn)
        flops = 2.0 * float((M[~thin].astype(np.float64) * N[~thin] * K[~thin]).sum())
        with instrument.region(region, flops=flops):
            _dgemm(sub, None, tm, tn, ntile)


# rates of the two paths on B200 inside the SU(2) CTMRG workload (int8: the
# CTA-pair k_oz_gemm_pair; FP64: k_grouped_dgemm averaged over the sector
# shapes it receives), used only to decide which path a sector GEMM takes in a
# mixed-precision run
_INT8_OPS = 1.8e15
_FP64_FLOPS = 2.0e13
_EPILOGUE_BPS = 2.0e12
_SPLIT_BPS = 3.0e12


def _pad(x, a):
    return (x + a - 1) // a * a


def ozaki_int8_ops(arr, S):
    M = _pad(arr["M"].astype(np.float64), 128)
    N = _pad(arr["N"].astype(np.float64), 256)
    K = _pad(np.maximum(arr["K"].astype(np.float64), 1), 128)
    return float((2 * M * N * K).sum() * S * (S + 1) / 2)


def ozaki_pays(arr, S):
    """Per problem: True when the tcgen05 path is estimated faster than FP64."""
    M = arr["M"].astype(np.float64)
    N = arr["N"].astype(np.float64)
    K = arr["K"].astype(np.float64)
    t_oz = (S * (S + 1) / 2 * 2 * _pad(M, 128) * _pad(N, 256) * _pad(np.maximum(K, 1), 128)
            / _INT8_OPS + S * M * N * 16 / _EPILOGUE_BPS + (M * K + K * N) * (8 + S) / _SPLIT_BPS)
    t_64 = 2 * _pad(M, 64) * _pad(N, 64) * K / _FP64_FLOPS
    return t_oz < t_64


def _tuned(arr, mode, model):
    """The autotuner's per-problem choice where it measured the shape class,
    the cost model's elsewhere."""
    if not autotune.enabled():
        return model
    dec = autotune.decide(arr, mode)
    return np.array([m if d is None else d for d, m in zip(dec, model, strict=True)],
                    dtype=bool)


_CRT_S_PER_ENTRY = 2.0e-12   # CRT epilogue per output entry (FP64 pipe, not hidden)


def ozaki2_int8_ops(arr, nmod):
    M = _pad(arr["M"].astype(np.float64), 256)
    N = _pad(arr["N"].astype(np.float64), 256)
    K = _pad(np.maximum(arr["K"].astype(np.float64), 1), 128)
    return float((2 * M * N * K).sum() * nmod)


def ozaki2_pays(arr, nmod):
    """Per problem: True when the Ozaki II path is estimated faster than FP64."""
    M = arr["M"].astype(np.float64)
    N = arr["N"].astype(np.float64)
    K = arr["K"].astype(np.float64)
    t_oz = (nmod * 2 * _pad(M, 256) * _pad(N, 256) * _pad(np.maximum(K, 1), 128) / _INT8_OPS
            + M * N * _CRT_S_PER_ENTRY + (M * K + K * N) * (8 + nmod) / _SPLIT_BPS)
    t_64 = 2 * _pad(M, 64) * _pad(N, 64) * K / _FP64_FLOPS
    return t_oz < t_64


def _tile_runs(ntile, ncol, order, nrow=None):
    """FsTileRun table: the problems in `order`, each a run of ntile tiles over
    nrow x ncol tiles; problems with more tile columns than rows run
    column-major (their few row tiles share each B column block in L2)."""
    nt = np.asarray(ntile, dtype=np.int64)[order]
    runs = np.zeros(order.size, dtype=_native.TILE_RUN_DTYPE)
    runs["start"] = np.cumsum(nt) - nt
    runs["problem"] = order
    nc = np.asarray(ncol, dtype=np.int64)[order]
    runs["ncol"] = nc
    if nrow is not None:
        nr = np.asarray(nrow, dtype=np.int64)[order]
        runs["nrow"] = nr
        runs["col_major"] = nc > nr
    else:
        runs["nrow"] = 1
    return runs, int(nt.sum())


def _device_tiles(runs, total):
    """The tile table of a launch, expanded on the device (fs_expand_tiles):
    only the per-problem runs cross PCIe, not one entry per output tile."""
    d_tiles = torch.empty(max(total, 1) * _native.GEMM_TILE_DTYPE.itemsize, dtype=torch.uint8,
                          device=dev.device())
    keep = runs[runs["start"] < total] if total else runs[:0]
    if total:
        d_runs = dev.upload(keep)
        _native.call("fs_expand_tiles", d_runs.data_ptr(), keep.size, total,
                     d_tiles.data_ptr(), dev.stream())
    return d_tiles


def _tile_table(arr, tm, tn, ntile):
    """Device tile table of a DMMA launch: largest K first (long tiles start
    early in the static schedule), each problem's tiles row-major."""
    order = np.argsort(-arr["K"].astype(np.int64), kind="stable")
    ncol = (arr["N"].astype(np.int64) + tn - 1) // tn
    nrow = (arr["M"].astype(np.int64) + tm - 1) // tm
    runs, total = _tile_runs(ntile, ncol, order, nrow)
    return _device_tiles(runs, total), total


_SPLITK_CHUNK = 1024        # smallest K chunk of a split problem
_SPLITK_TARGET_TILES = 3 * 148 * 2   # two waves of 3 CTAs per SM


def _split_k(arr, tm, tn, ntile):
    """Cut long-K problems of a launch that has too few output tiles into K
    chunks writing partial products to a workspace; returns the new problem
    table and tile counts, the reduction items and the workspace (or None
    when the launch already fills the GPU)."""
    total = int(ntile.sum())
    if total == 0 or total >= _SPLITK_TARGET_TILES:
        return None
    factor = min(16, -(-_SPLITK_TARGET_TILES // total))
    K = arr["K"].astype(np.int64)
    ks = np.minimum(factor, K // _SPLITK_CHUNK)
    split = ks >= 2
    if not split.any():
        return None
    M = arr["M"].astype(np.int64)
    N = arr["N"].astype(np.int64)
    w_sizes = np.where(split, ks * M * N, 0)
    w_off = np.concatenate([[0], np.cumsum(w_sizes)[:-1]])
    work = torch.empty(max(int(w_sizes.sum()), 1), dtype=torch.float64, device=dev.device())
    base = work.data_ptr()
    rows, items = [], np.zeros(int(split.sum()), dtype=_native.SPLIT_REDUCE_DTYPE)
    n_items = 0
    for i in range(arr.size):
        if not split[i]:
            rows.append(arr[i : i + 1])
            continue
        k_i, n_chunks = int(K[i]), int(ks[i])
        chunk = -(-k_i // n_chunks)
        chunk = -(-chunk // 16) * 16
        starts = np.arange(0, k_i, chunk)
        sub = np.repeat(arr[i : i + 1], starts.size)
        a_step = int(arr["lda"][i]) if arr["transA"][i] else 1
        b_step = 1 if arr["transB"][i] else int(arr["ldb"][i])
        sub["A"] = arr["A"][i] + (8 * starts * a_step).astype(np.uint64)
        sub["B"] = arr["B"][i] + (8 * starts * b_step).astype(np.uint64)
        sub["K"] = np.minimum(chunk, k_i - starts)
        sub["C"] = np.uint64(base) + (8 * (w_off[i] + np.arange(starts.size) * M[i] * N[i])).astype(np.uint64)
        sub["ldc"] = N[i]
        sub["alpha"] = 1.0
        sub["beta"] = 0.0
        rows.append(sub)
        items[n_items] = (base + 8 * int(w_off[i]), arr["C"][i], arr["ldc"][i], M[i] * N[i],
                          starts.size, M[i], N[i], 0, arr["alpha"][i], arr["beta"][i])
        n_items += 1
    new = np.concatenate(rows)
    nt = ((new["M"].astype(np.int64) + tm - 1) // tm) * ((new["N"].astype(np.int64) + tn - 1) // tn)
    return new, nt, items[:n_items], work


_STREAM_MAX_K = 256   # longest K of a launch that goes to the streaming kernel


def _launch_dgemm(arr, d_prob, d_tiles, n_tiles):
    """One DMMA launch over a problem table: the streaming kernel when every
    problem has the same transpose flags and a short K (pipeline fill and
    padded fragments dominate there), else the per-tile kernel (faster on long
    K, where it keeps a few registers more for the DMMA loop)."""
    ta, tb = arr["transA"], arr["transB"]
    if (arr.size and (ta == ta[0]).all() and (tb == tb[0]).all()
            and int(arr["K"].max()) <= _STREAM_MAX_K):
        _native.call("fs_grouped_dgemm_uniform", d_prob.data_ptr(), arr.size,
                     d_tiles.data_ptr(), n_tiles, int(ta[0]), int(tb[0]), dev.stream())
    else:
        _native.call("fs_grouped_dgemm", d_prob.data_ptr(), arr.size, d_tiles.data_ptr(),
                     n_tiles, dev.stream())


def _dgemm(arr, problems, tm, tn, ntile):
    sk = _split_k(arr, tm, tn, ntile)
    if sk is not None:
        arr, ntile, items, work = sk
        d_tiles, n_tiles = _tile_table(arr, tm, tn, ntile)
        d_prob = dev.upload(arr)
        _launch_dgemm(arr, d_prob, d_tiles, n_tiles)
        d_items = dev.upload(items)
        max_elems = int((items["M"].astype(np.int64) * items["N"]).max())
        for start in range(0, items.size, 65535):
            cnt = min(65535, items.size - start)
            _native.call("fs_splitk_reduce", d_items.data_ptr() + start * items.itemsize, cnt,
                         max_elems, dev.stream())
        return d_prob, d_tiles, work
    d_tiles, n_tiles = _tile_table(arr, tm, tn, ntile)
    d_prob = dev.upload(arr)
    _launch_dgemm(arr, d_prob, d_tiles, n_tiles)
    return d_prob, d_tiles


def _operand(t):
    """(buffer, element offset, trans, leading dim) of a 2-D torch view whose
    rows or columns are unit-stride; other views are made contiguous."""
    if t.dim() != 2:
        raise ValueError("block operands must be 2-D")
    m, n = t.shape
    s0, s1 = t.stride()
    if s1 == 1 and (s0 >= n or m <= 1):
        return t, max(s0, n), False
    if s0 == 1 and (s1 >= m or n <= 1):
        return t, max(s1, m), True
    t = t.contiguous()
    return t, n, False


def matmul_blocks(lefts, rights, *, alpha=1.0):
    """C_i = alpha * lefts[i] @ rights[i] for lists of 2-D device views, all in
    one grouped GEMM launch; returns (buffer, offsets, shapes, views)."""
    n = len(lefts)
    shapes = np.array([(a.shape[0], b.shape[1]) for a, b in zip(lefts, rights, strict=True)],
                      dtype=np.int64).reshape(-1, 2)
    sizes = shapes[:, 0] * shapes[:, 1]
    offsets = np.zeros(n, dtype=np.int64)
    if n > 1:
        offsets[1:] = np.cumsum(sizes[:-1])
    out = dev.empty_f64(int(sizes.sum()))
    problems = []
    keep = []
    for i, (a, b) in enumerate(zip(lefts, rights, strict=True)):
        if a.shape[1] != b.shape[0]:
            raise ValueError("inner dimensions do not match")
        ta, lda, a_t = _operand(a)
        tb, ldb, b_t = _operand(b)
        keep += [ta, tb]
        problems.append({
            "A": ta, "a_off": 0, "a_trans": a_t, "lda": lda,
            "B": tb, "b_off": 0, "b_trans": b_t, "ldb": ldb,
            "C": out, "c_off": offsets[i], "M": a.shape[0], "N": b.shape[1],
            "K": a.shape[1], "alpha": alpha,
        })
    for p in problems:
        # data_ptr() of a view already includes its storage offset
        p["a_off"] = 0
        p["b_off"] = 0
    if problems:
        grouped_gemm(problems)
    views = [out[o : o + m * k].view(m, k) for o, (m, k) in zip(offsets, shapes, strict=True)]
    return out, offsets, shapes, views


# ------------------------------------------------- tcgen05 (Ozaki int8) GEMM

OZ_TILE_M = 128
OZ_TILE_N = 256
OZ_TILE_K = 128
OZ_SPLIT_ROWS = 128
OZ_TILE_BYTES = OZ_SPLIT_ROWS * OZ_TILE_K


def ozaki_chunk_ktiles(nslices):
    """Largest number of k-tiles whose int32 diagonal sums cannot overflow."""
    return max(1, (2**31 - 1) // (nslices * OZ_TILE_K * 127 * 127))


def _round_up(x, a):
    return (x + a - 1) // a * a


def ozaki_plan(arr, nslices, pair=False):
    """Operand/problem/tile tables and workspace layout for a problem array
    (GEMM_PROBLEM_DTYPE).  Returns (ops, probs, tiles, pair_tiles,
    workspace_bytes) with pointer fields relative to the workspace base
    (patched on launch).  With `pair`, problems of more than 128 rows get an
    even number of A row tiles and 256-row tiles in `pair_tiles` (CTA-pair
    kernel); the others stay in `tiles`."""
    n = arr.size
    ops = np.zeros(2 * n, dtype=_native.OZ_OPERAND_DTYPE)
    probs = np.zeros(n, dtype=_native.OZ_PROBLEM_DTYPE)
    off = 0
    rel = {"a_slices": [], "b_slices": [], "a_exps": [], "b_exps": []}
    tiles = []
    pair_tiles = []
    for i in range(n):
        M, N, K = int(arr["M"][i]), int(arr["N"][i]), int(arr["K"][i])
        kt = max(1, (K + OZ_TILE_K - 1) // OZ_TILE_K)
        art = (M + OZ_SPLIT_ROWS - 1) // OZ_SPLIT_ROWS
        is_pair = pair and M > OZ_TILE_M
        if is_pair:
            art += art % 2
        brt = 2 * ((N + OZ_TILE_N - 1) // OZ_TILE_N)
        a_bytes = nslices * kt * art * OZ_TILE_BYTES
        b_bytes = nslices * kt * brt * OZ_TILE_BYTES
        a_sl, off = off, off + a_bytes
        b_sl, off = off, off + b_bytes
        a_ex, off = off, off + _round_up(4 * max(M, 1), 256)
        b_ex, off = off, off + _round_up(4 * max(N, 1), 256)
        off = _round_up(off, 1024)
        lda, ldb = int(arr["lda"][i]), int(arr["ldb"][i])
        ta, tb = int(arr["transA"][i]), int(arr["transB"][i])
        # operand A: element (i, k) of op(A)
        ops[2 * i] = (arr["A"][i], 1 if ta else lda, lda if ta else 1, a_sl, a_ex, M, K, art, kt)
        # operand B^T: element (j, k) = op(B)[k, j]
        ops[2 * i + 1] = (arr["B"][i], ldb if tb else 1, 1 if tb else ldb, b_sl, b_ex, N, K, brt, kt)
        probs[i] = (a_sl, b_sl, a_ex, b_ex, arr["C"][i], arr["ldc"][i], M, N, K, art, brt, kt,
                    arr["alpha"][i], arr["beta"][i])
        for tm_ in range(art // 2 if is_pair else art):
            for tn_ in range((N + OZ_TILE_N - 1) // OZ_TILE_N):
                (pair_tiles if is_pair else tiles).append((i, tm_, tn_, 0, K))
        rel["a_slices"].append(a_sl)

    def table(lst):
        out = np.zeros(len(lst), dtype=_native.OZ_TILE_DTYPE)
        if lst:
            t = np.array(lst, dtype=np.int64)
            t = t[np.argsort(-t[:, 4], kind="stable")]
            out["problem"] = t[:, 0]
            out["tm"] = t[:, 1]
            out["tn"] = t[:, 2]
        return out

    return ops, probs, table(tiles), table(pair_tiles), off


def ozaki_gemm(arr, nslices, workspace=None):
    """Run the problems of `arr` (GEMM_PROBLEM_DTYPE) on the tcgen05 Ozaki path.
    The workspace is a caller-owned uint8 device buffer (allocated here from
    torch's caching allocator when not given)."""
    ops, probs, tiles, pair_tiles, nbytes = ozaki_plan(arr, nslices, _PRECISION["pair"])
    if tiles.size == 0 and pair_tiles.size == 0:
        return
    if workspace is None or workspace.numel() < nbytes:
        # at least one 128 x 128-byte tile: the CTA-pair kernel's tensor map
        # needs whole 128-row boxes
        workspace = torch.empty(max(nbytes, 128 * 128), dtype=torch.uint8, device=dev.device())
    base = workspace.data_ptr()
    for f in ("slices", "exps"):
        ops[f] += np.uint64(base)
    for f in ("a_slices", "b_slices", "a_exps", "b_exps"):
        probs[f] += np.uint64(base)
    d_ops = dev.upload(ops)
    d_probs = dev.upload(probs)
    max_rows = int(ops["rows"].max())
    max_tiles = int((ops["rowtiles"].astype(np.int64) * ops["ktiles"]).max())
    for start in range(0, ops.size, 65534):
        sub = slice(start, min(ops.size, start + 65534))
        _native.call(
            "fs_ozaki_split",
            d_ops.data_ptr() + start * ops.itemsize,
            ops[sub].size,
            max_rows,
            max_tiles,
            nslices,
            dev.stream(),
        )
    flag = torch.zeros(1, dtype=torch.int32, device=dev.device())
    if pair_tiles.size:
        d_tiles = dev.upload(pair_tiles)
        _native.call(
            "fs_ozaki_gemm_pair", d_probs.data_ptr(), probs.size, d_tiles.data_ptr(),
            pair_tiles.size, nslices, ozaki_chunk_ktiles(nslices), base,
            (workspace.numel() // 128) * 128, flag.data_ptr(), dev.stream(),
        )
    if tiles.size:
        d_tiles = dev.upload(tiles)
        _native.call(
            "fs_ozaki_gemm", d_probs.data_ptr(), probs.size, d_tiles.data_ptr(), tiles.size,
            nslices, ozaki_chunk_ktiles(nslices), flag.data_ptr(), dev.stream(),
        )
    _OZ_FLAGS.append(flag)
    if len(_OZ_FLAGS) > 64:
        check_ozaki_flags()
    return workspace


_OZ_FLAGS = []

OZ2_MODULI = (256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199)
_OZ2_PRODUCT_BITS = {}


def ozaki2_bits(nmod, K):
    """(a, b) operand bits for nmod moduli and inner size K: the largest
    (at most 50 each) with K 2^(a+b) <= P / 4, P the product of the moduli
    (the same rule as fs_ozaki2_bits)."""
    if nmod not in _OZ2_PRODUCT_BITS:
        P = 1
        for p in OZ2_MODULI[:nmod]:
            P *= p
        _OZ2_PRODUCT_BITS[nmod] = P.bit_length() - 1
    K = max(int(K), 1)
    L = _OZ2_PRODUCT_BITS[nmod] - 2 - (int(K - 1).bit_length() if K > 1 else 0)
    return min(50, L // 2), min(50, L - L // 2)


def ozaki2_plan(arr, nmod):
    """Operand/problem/tile tables and the slice workspace size of the Ozaki II
    path for a problem array (GEMM_PROBLEM_DTYPE); pointer fields are relative
    to the workspace base.  Every problem runs on 256 x 256 CTA-pair tiles."""
    n = arr.size
    ops = np.zeros(2 * n, dtype=_native.OZ2_OPERAND_DTYPE)
    probs = np.zeros(n, dtype=_native.OZ2_PROBLEM_DTYPE)
    off = 0
    tiles = []
    for i in range(n):
        M, N, K = int(arr["M"][i]), int(arr["N"][i]), int(arr["K"][i])
        kt = max(1, (K + OZ_TILE_K - 1) // OZ_TILE_K)
        art = 2 * ((M + 255) // 256)
        ntn = (N + OZ_TILE_N - 1) // OZ_TILE_N
        brt = 2 * ntn
        a_bits, b_bits = ozaki2_bits(nmod, K)
        a_sl, off = off, off + nmod * kt * art * OZ_TILE_BYTES
        b_sl, off = off, off + nmod * kt * brt * OZ_TILE_BYTES
        a_ex, off = off, off + _round_up(4 * max(M, 1), 256)
        b_ex, off = off, off + _round_up(4 * max(N, 1), 256)
        off = _round_up(off, 1024)
        lda, ldb = int(arr["lda"][i]), int(arr["ldb"][i])
        ta, tb = int(arr["transA"][i]), int(arr["transB"][i])
        ops[2 * i] = (arr["A"][i], 1 if ta else lda, lda if ta else 1, a_sl, a_ex, M, K, art, kt,
                      a_bits, 0)
        ops[2 * i + 1] = (arr["B"][i], ldb if tb else 1, 1 if tb else ldb, b_sl, b_ex, N, K, brt,
                          kt, b_bits, 0)
        probs[i] = (a_sl, b_sl, a_ex, b_ex, arr["C"][i], arr["ldc"][i], M, N, K, art, brt, kt,
                    arr["alpha"][i], arr["beta"][i], a_bits, b_bits)
        for tm_ in range(art // 2):
            for tn_ in range(ntn):
                tiles.append((i, tm_, tn_, K))
    table = np.zeros(len(tiles), dtype=_native.OZ_TILE_DTYPE)
    if tiles:
        t = np.array(tiles, dtype=np.int64)
        t = t[np.argsort(-t[:, 3], kind="stable")]
        table["problem"] = t[:, 0]
        table["tm"] = t[:, 1]
        table["tn"] = t[:, 2]
    return ops, probs, table, off


_OZ2_SCRATCH = {}


def ozaki2_gemm(arr, nmod, *, flops=0.0, int8_ops=0.0):
    """Run the problems of `arr` (GEMM_PROBLEM_DTYPE) on the Ozaki II path
    (fs_ozaki2_split + fs_ozaki2_gemm_pair); the slice workspace and the CRT
    scratch come from torch's caching allocator.  Instrumented as two
    regions: "ozaki_split" (exponent and residue-slice kernels, 8 + 8 bytes
    read and nmod written per operand entry) and "gemm_ozaki" (the GEMM)."""
    ops, probs, tiles, nbytes = ozaki2_plan(arr, nmod)
    if tiles.size == 0:
        return None
    if nmod not in _OZ2_SCRATCH:
        _OZ2_SCRATCH[nmod] = _native.ozaki2_scratch_bytes(nmod)
    ws_bytes = _round_up(max(nbytes, 128 * 128), 1024)
    scratch_bytes = _OZ2_SCRATCH[nmod]
    buf = torch.empty(ws_bytes + scratch_bytes, dtype=torch.uint8, device=dev.device())
    base = buf.data_ptr()
    for f in ("slices", "exps"):
        ops[f] += np.uint64(base)
    for f in ("a_slices", "b_slices", "a_exps", "b_exps"):
        probs[f] += np.uint64(base)
    d_ops = dev.upload(ops)
    d_probs = dev.upload(probs)
    d_tiles = dev.upload(tiles)
    max_rows = int(ops["rows"].max())
    max_units = int((ops["rowtiles"].astype(np.int64) * 4 * ops["ktiles"]).max())
    entries = float((ops["rows"].astype(np.float64) * ops["K"]).sum())
    with instrument.region("ozaki_split", bytes=entries * (16 + nmod)):
        for start in range(0, ops.size, 65534):
            cnt = min(65534, ops.size - start)
            _native.call("fs_ozaki2_split", d_ops.data_ptr() + start * ops.itemsize, cnt,
                         max_rows, max_units, nmod, dev.stream())
    flag = torch.zeros(1, dtype=torch.int32, device=dev.device())
    with instrument.region("gemm_ozaki", flops=flops, int8_ops=int8_ops):
        _native.call("fs_ozaki2_gemm_pair", d_probs.data_ptr(), probs.size, d_tiles.data_ptr(),
                     tiles.size, nmod, base, ws_bytes, base + ws_bytes, scratch_bytes,
                     flag.data_ptr(), dev.stream())
    _OZ_FLAGS.append(flag)
    if len(_OZ_FLAGS) > 64:
        check_ozaki_flags()
    return buf


def check_ozaki_flags():
    """Synchronise on the error flags of past tcgen05 launches; raise if a bounded
    device wait ran out."""
    flags = list(_OZ_FLAGS)
    _OZ_FLAGS.clear()
    for f in flags:
        v = int(f.item())
        if v != 0:
            _native.check(v, "fs_ozaki_gemm (device flag)")


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
    """x *= alpha; alpha a number, or a 1-element device tensor (no host sync)."""
    if isinstance(alpha, torch.Tensor):
        s = alpha.reshape(1).to(torch.float64)
        _native.call("fs_scale_by", dev.ptr(x), x.numel(), s.data_ptr(), 0, dev.stream())
    else:
        _native.call("fs_scale", dev.ptr(x), x.numel(), float(alpha), dev.stream())


def divide_(x, s):
    """x /= s for a 1-element device tensor s (no host sync)."""
    s = s.reshape(1).to(torch.float64)
    _native.call("fs_scale_by", dev.ptr(x), x.numel(), s.data_ptr(), 1, dev.stream())


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
