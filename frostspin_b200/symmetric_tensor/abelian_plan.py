"""Host plan builder for the abelian (U(1) / Z2) permute kernel.

Reference behaviour (frostspin/symmetric_tensor/abelian_symmetric_tensor.py
:103-250, ``_numba_abelian_transpose``, and :78-100 ``_numpy_get_indices``):
the rows of an irrep block are the fused row indices carrying that irrep, in
ascending C-order flat index; columns likewise with the column legs' signature
flipped.  A permute moves every entry to the block, row and column it occupies
under the new leg order.  New blocks are all allowed irreps (present in both the
new row and the new column representation), sorted; entries with no source
block are zero.

Design: instead of per-entry index arithmetic, each leg representation is cut
into segments (maximal runs of one irrep).  A tuple of one segment per leg is
an *elementary block* (EB).  Within a group of legs fused into rows (or
columns), the rank of a row among the rows of its irrep is affine in the local
indices of the legs inside their segments, with strides given by suffix charge
counts:

    stride_m = #{combinations of legs m+1.. with charge Q - prefix_m - c_m}
    base     = sum_m sum_{segments t of leg m before s_m} len(t) * #{... Q - prefix_m - c(t)}

So every EB is a strided copy between the old and new block buffers.  Charges
are handled modulo 256, which is exactly the int8 wraparound the reference
relies on for Z2 = {-128, 0} (examples/ising_classical_ctmrg.py:369-378).
"""

import numpy as np

from .._native import FS_PERM_MAXR, PERM_EB_DTYPE, PERM_TASK_DTYPE

TASK_CHUNK = 8192


def to_int8(c):
    """Map charges modulo 256 to their int8 label."""
    return ((np.asarray(c, dtype=np.int64) + 128) % 256 - 128).astype(np.int8)


def segments(rep):
    """Maximal runs of equal irrep in a 1-D int8 representation."""
    rep = np.asarray(rep)
    n = rep.size
    if n == 0:
        z = np.zeros(0, dtype=np.int64)
        return z, z, z
    change = np.flatnonzero(rep[1:] != rep[:-1]) + 1
    starts = np.concatenate(([0], change)).astype(np.int64)
    lens = np.diff(np.concatenate((starts, [n]))).astype(np.int64)
    q = rep[starts].astype(np.int64)
    return starts, lens, q


def _cyclic_conv(h, s):
    c = np.arange(256)
    idx = (c[:, None] - c[None, :]) % 256
    return (h[None, :] * s[idx]).sum(axis=1)


class GroupInfo:
    """Rank structure of a group of legs fused into rows (or columns).

    Attributes per tuple of segments (C-order over the legs of the group):
    ``irrep`` (mod 256), ``base`` (rank of the tuple's first entry inside its
    block) and ``strides`` (rank step per leg).  ``counts[c]`` is the block size
    (number of fused indices) of irrep c.
    """

    def __init__(self, segs, coefs):
        p = len(segs)
        self.nseg = np.array([len(s[0]) for s in segs], dtype=np.int64)
        charges = [(cf * s[2]) % 256 for s, cf in zip(segs, coefs, strict=True)]
        hists = []
        for s, ch in zip(segs, charges, strict=True):
            h = np.zeros(256, dtype=np.int64)
            np.add.at(h, ch, s[1])
            hists.append(h)
        suf = [None] * (p + 1)
        suf[p] = np.zeros(256, dtype=np.int64)
        suf[p][0] = 1
        for m in range(p - 1, -1, -1):
            suf[m] = _cyclic_conv(hists[m], suf[m + 1])
        self.counts = suf[0]

        # before[m][sigma, x]: entries of leg m ahead of segment sigma, weighted by
        # the number of completions of legs m+1.. reaching total x.
        before = []
        xs = np.arange(256)
        for m in range(p):
            lens = segs[m][1]
            ch = charges[m]
            contrib = lens[:, None] * suf[m + 1][(xs[None, :] - ch[:, None]) % 256]
            b = np.zeros((lens.size, 256), dtype=np.int64)
            if lens.size > 1:
                b[1:] = np.cumsum(contrib[:-1], axis=0)
            before.append(b)

        grids = np.indices(tuple(self.nseg), dtype=np.int64).reshape(p, -1).T
        nt = grids.shape[0]
        c = np.empty((nt, p), dtype=np.int64)
        for m in range(p):
            c[:, m] = charges[m][grids[:, m]]
        prefix = np.zeros((nt, p), dtype=np.int64)
        if p > 1:
            prefix[:, 1:] = np.cumsum(c[:, :-1], axis=1)
        irrep = c.sum(axis=1) % 256
        base = np.zeros(nt, dtype=np.int64)
        strides = np.empty((nt, p), dtype=np.int64)
        for m in range(p):
            x = (irrep - prefix[:, m]) % 256
            base += before[m][grids[:, m], x]
            strides[:, m] = suf[m + 1][(x - c[:, m]) % 256]
        self.seg_index = grids
        self.irrep = irrep
        self.base = base
        self.strides = strides

    def tuple_id(self, seg_idx):
        """Mixed-radix id of segment-index rows (n, p), C order."""
        tid = np.zeros(seg_idx.shape[0], dtype=np.int64)
        for m in range(seg_idx.shape[1]):
            tid = tid * self.nseg[m] + seg_idx[:, m]
        return tid


def leg_coefficients(signature, nrr):
    """Signed charge coefficient of each leg: rows (1-2s), columns -(1-2s)."""
    sig = np.asarray(signature, dtype=bool)
    cf = 1 - 2 * sig.astype(np.int64)
    cf[nrr:] *= -1
    return cf


def magic_divisor(d):
    """Granlund-Montgomery constants (m, s) for 32-bit division by d >= 1."""
    d = np.asarray(d, dtype=np.uint64)
    # s = ceil(log2 d) = bit length of d - 1 (frexp is exact below 2^53)
    s = np.frexp((d - np.uint64(1)).astype(np.float64))[1].astype(np.uint64)
    m = ((np.uint64(1) << np.uint64(32)) * ((np.uint64(1) << s) - d)) // d + np.uint64(1)
    return m.astype(np.uint32), s.astype(np.uint32)


class AbelianPermutePlan:
    """Everything needed to run one abelian permute: output block structure plus
    the EB and task tables (numpy; uploaded lazily by the tensor class)."""

    __slots__ = (
        "block_irreps",
        "block_shapes",
        "offsets",
        "size",
        "ebs",
        "tasks",
        "in_len",
        "device_tables",
    )


def build_abelian_permute_plan(
    reps,
    signature,
    nrr,
    old_block_irreps,
    old_offsets,
    old_shapes,
    old_trans,
    in_len,
    axes,
    new_nrr,
):
    """Plan a permute of an abelian tensor.

    Parameters
    ----------
    reps : list of int8 arrays, old leg order (row legs then column legs)
    signature : bool array, old leg order
    nrr : number of old row legs
    old_block_irreps, old_offsets, old_shapes : present old blocks (sorted irreps),
        element offsets into the input buffer and logical (m, n) shapes
    old_trans : True if every old block is stored transposed (F-order)
    in_len : input buffer length in elements
    axes : new leg order (tuple of old leg indices)
    new_nrr : number of new row legs
    """
    ndim = len(reps)
    axes = tuple(int(a) for a in axes)
    segs = [segments(r) for r in reps]
    coef = leg_coefficients(signature, nrr)

    old_rows = GroupInfo([segs[k] for k in range(nrr)], coef[:nrr])
    old_cols = GroupInfo([segs[k] for k in range(nrr, ndim)], coef[nrr:])
    new_sig = np.asarray(signature, dtype=bool)[list(axes)]
    new_coef = leg_coefficients(new_sig, new_nrr)
    # the leg coefficient travels with the leg: same signature, but the column
    # sign flips when a leg moves between rows and columns, which only changes
    # the irrep label, not the conservation law
    new_rows = GroupInfo([segs[a] for a in axes[:new_nrr]], new_coef[:new_nrr])
    new_cols = GroupInfo([segs[a] for a in axes[new_nrr:]], new_coef[new_nrr:])

    # new blocks: irreps allowed in both new rows and new columns
    allowed = np.flatnonzero((new_rows.counts > 0) & (new_cols.counts > 0))
    irr8 = to_int8(allowed)
    order = np.argsort(irr8, kind="stable")
    allowed = allowed[order]
    new_block_irreps = irr8[order]
    new_m = new_rows.counts[allowed]
    new_n = new_cols.counts[allowed]
    sizes = new_m * new_n
    new_offsets = np.zeros(allowed.size, dtype=np.int64)
    if allowed.size > 1:
        new_offsets[1:] = np.cumsum(sizes[:-1])
    total = int(sizes.sum())
    nb_index = np.full(256, -1, dtype=np.int64)
    nb_index[allowed] = np.arange(allowed.size)

    # old blocks present
    ob_index = np.full(256, -1, dtype=np.int64)
    old_irr_mod = np.asarray(old_block_irreps, dtype=np.int64) % 256
    ob_index[old_irr_mod] = np.arange(old_irr_mod.size)
    old_offsets = np.asarray(old_offsets, dtype=np.int64)
    old_shapes = np.asarray(old_shapes, dtype=np.int64).reshape(-1, 2)
    for i, q in enumerate(old_irr_mod):
        exp = (old_rows.counts[q], old_cols.counts[q])
        if tuple(old_shapes[i]) != exp:
            msg = f"old block {i} has shape {tuple(old_shapes[i])}, expected {exp}"
            raise ValueError(msg)

    # join old row tuples with old column tuples of equal irrep
    rq = old_rows.irrep
    cq = old_cols.irrep
    corder = np.argsort(cq, kind="stable")
    cq_sorted = cq[corder]
    lo = np.searchsorted(cq_sorted, rq, side="left")
    hi = np.searchsorted(cq_sorted, rq, side="right")
    cnt = hi - lo
    keep_r = np.flatnonzero(cnt > 0)
    cnt_k = cnt[keep_r]
    n_eb = int(cnt_k.sum())
    eb_r = np.repeat(keep_r, cnt_k)
    starts = np.repeat(lo[keep_r], cnt_k)
    within = np.arange(n_eb) - np.repeat(np.cumsum(cnt_k) - cnt_k, cnt_k)
    eb_c = corder[starts + within]

    q = rq[eb_r]
    # per-leg segment index in old leg order
    seg_idx = np.empty((n_eb, ndim), dtype=np.int64)
    seg_idx[:, :nrr] = old_rows.seg_index[eb_r]
    seg_idx[:, nrr:] = old_cols.seg_index[eb_c]
    # old per-leg strides (rank units) in old leg order
    ostr_rank = np.empty((n_eb, ndim), dtype=np.int64)
    ostr_rank[:, :nrr] = old_rows.strides[eb_r]
    ostr_rank[:, nrr:] = old_cols.strides[eb_c]
    obase_r = old_rows.base[eb_r]
    obase_c = old_cols.base[eb_c]

    ob = ob_index[q]
    present = ob >= 0
    om = np.where(present, old_shapes[np.maximum(ob, 0), 0], 0)
    on = np.where(present, old_shapes[np.maximum(ob, 0), 1], 0)
    ooff = np.where(present, old_offsets[np.maximum(ob, 0)], -1)
    if old_trans:
        row_mul, col_mul = np.ones_like(om), om
    else:
        row_mul, col_mul = on, np.ones_like(on)
    obase = np.where(present, ooff + obase_r * row_mul + obase_c * col_mul, -1)

    # new side
    nr_t = new_rows.tuple_id(seg_idx[:, list(axes[:new_nrr])])
    nc_t = new_cols.tuple_id(seg_idx[:, list(axes[new_nrr:])])
    nq = new_rows.irrep[nr_t]
    if not (nq == new_cols.irrep[nc_t]).all():
        raise AssertionError("charge conservation broken in permute plan")
    nb = nb_index[nq]
    if (nb < 0).any():
        raise AssertionError("elementary block maps to a forbidden new block")
    nn = new_n[nb]
    nbase = new_offsets[nb] + new_rows.base[nr_t] * nn + new_cols.base[nc_t]

    # per leg in new order: dims, old stride, new stride (elements)
    dims = np.empty((n_eb, ndim), dtype=np.int64)
    ostride = np.empty((n_eb, ndim), dtype=np.int64)
    nstride = np.empty((n_eb, ndim), dtype=np.int64)
    for i, a in enumerate(axes):
        dims[:, i] = segs[a][1][seg_idx[:, a]]
        mul = row_mul if a < nrr else col_mul
        ostride[:, i] = np.where(present, ostr_rank[:, a] * mul, 0)
        if i < new_nrr:
            nstride[:, i] = new_rows.strides[nr_t, i] * nn
        else:
            nstride[:, i] = new_cols.strides[nc_t, i - new_nrr]

    ebs, vol = _pack_ebs(dims, ostride, nstride, obase, nbase, present)

    # host-side bounds validation of every EB against both buffers
    span_o = ((np.maximum(dims - 1, 0)) * ostride).sum(axis=1)
    span_n = ((np.maximum(dims - 1, 0)) * nstride).sum(axis=1)
    if present.any() and (
        (obase[present] < 0).any() or (obase + span_o)[present].max() >= in_len
    ):
        raise AssertionError("permute plan reads outside the input buffer")
    if n_eb and ((nbase < 0).any() or (nbase + span_n).max() >= max(total, 1)):
        raise AssertionError("permute plan writes outside the output buffer")
    if int(vol.sum()) != total:
        raise AssertionError(f"plan covers {int(vol.sum())} entries, expected {total}")

    plan = AbelianPermutePlan()
    plan.block_irreps = new_block_irreps
    plan.block_shapes = np.stack([new_m, new_n], axis=1).astype(np.int64)
    plan.offsets = new_offsets
    plan.size = total
    plan.ebs = ebs
    plan.tasks = _make_tasks(ebs)
    plan.in_len = int(in_len)
    plan.device_tables = None
    return plan


def _pack_ebs(dims, ostride, nstride, obase, nbase, present):
    """Canonicalise (drop unit legs, sort by output stride, merge legs contiguous
    in both layouts) and pack into the FsPermEB table."""
    n_eb, ndim = dims.shape
    out = np.zeros(n_eb, dtype=PERM_EB_DTYPE)
    vol = np.prod(dims, axis=1)
    if (vol >= 2**31).any():
        raise ValueError("elementary block too large for 32-bit positions")
    out["obase"] = obase
    out["nbase"] = nbase
    out["volume"] = vol
    out["tile_leg"] = -1
    out["dims"] = 1
    if n_eb == 0:
        return out, vol
    # unit legs sort last, the rest by decreasing output stride (stable)
    big = np.iinfo(np.int64).max
    key = np.where(dims > 1, -nstride, big)
    order = np.argsort(key, axis=1, kind="stable")
    d = np.take_along_axis(dims, order, axis=1)
    o = np.take_along_axis(ostride, order, axis=1)
    s = np.take_along_axis(nstride, order, axis=1)
    md = np.ones((n_eb, ndim), dtype=np.int64)
    mo = np.zeros((n_eb, ndim), dtype=np.int64)
    mn = np.zeros((n_eb, ndim), dtype=np.int64)
    r = np.zeros(n_eb, dtype=np.int64)
    rows = np.arange(n_eb)
    for k in range(ndim):
        valid = d[:, k] > 1
        prev = np.maximum(r - 1, 0)
        merge = (
            valid
            & (r > 0)
            & (mo[rows, prev] == o[:, k] * d[:, k])
            & (mn[rows, prev] == s[:, k] * d[:, k])
        )
        mi = rows[merge]
        md[mi, prev[merge]] *= d[merge, k]
        mo[mi, prev[merge]] = o[merge, k]
        mn[mi, prev[merge]] = s[merge, k]
        new = valid & ~merge
        ni = rows[new]
        md[ni, r[new]] = d[new, k]
        mo[ni, r[new]] = o[new, k]
        mn[ni, r[new]] = s[new, k]
        r[new] += 1
    r = np.maximum(r, 1)
    if r.max() > FS_PERM_MAXR:
        msg = f"elementary block needs {r.max()} legs after merging (max {FS_PERM_MAXR})"
        raise ValueError(msg)
    w = min(ndim, FS_PERM_MAXR)
    out["ndim"] = r
    out["dims"][:, :w] = md[:, :w]
    out["ostride"][:, :w] = np.where(present[:, None], mo[:, :w], 0)
    out["nstride"][:, :w] = mn[:, :w]
    m, s = magic_divisor(out["dims"])
    out["divm"] = m
    out["divs"] = s
    return out, vol


MAX_TASK_ROWS = 1024


def _make_tasks(ebs, chunk=TASK_CHUNK):
    """Split every EB into tasks of whole rows (runs along the last leg): about
    `chunk` entries and at most MAX_TASK_ROWS rows per task."""
    n_eb = ebs.size
    if n_eb == 0:
        return np.zeros(0, dtype=PERM_TASK_DTYPE)
    r = ebs["ndim"].astype(np.int64)
    inner = ebs["dims"][np.arange(n_eb), r - 1].astype(np.int64)
    rows = ebs["volume"].astype(np.int64) // inner
    per = np.clip(chunk // inner, 1, MAX_TASK_ROWS)
    nchunk = (rows + per - 1) // per
    n = int(nchunk.sum())
    tasks = np.zeros(n, dtype=PERM_TASK_DTYPE)
    eb = np.repeat(np.arange(n_eb), nchunk)
    first = np.repeat(np.cumsum(nchunk) - nchunk, nchunk)
    start = (np.arange(n) - first) * per[eb]
    tasks["eb"] = eb
    tasks["start"] = start
    tasks["count"] = np.minimum(per[eb], rows[eb] - start)
    return tasks


def emulate_permute(plan, data_in):
    """Apply a plan with numpy, mirroring the kernel's index arithmetic (test aid;
    never used by the device path)."""
    out = np.full(plan.size, np.nan)
    for e in plan.ebs:
        r = int(e["ndim"])
        dims = e["dims"][:r].astype(np.int64)
        idx = np.indices(tuple(dims)).reshape(r, -1)
        dst = e["nbase"] + (idx * e["nstride"][:r, None]).sum(axis=0)
        if e["obase"] < 0:
            out[dst] = 0.0
        else:
            src = e["obase"] + (idx * e["ostride"][:r, None]).sum(axis=0)
            out[dst] = data_in[src]
    return out
