"""Tables of the fused SU(2) permute (fs_su2_permute_fused).

The SU(2) permute of frostspin (lie_group_symmetric_tensor.py:96-265,
:735-835) is, per simple block, gather -> recoupling product -> scatter.  The
structure code of lie_group_symmetric_tensor.py describes every (simple
block, sector) piece as a strided copy: dims (s_r, s_c, external legs...),
source and destination strides and bases (_block_gather / _block_scatter).
This module turns the pieces of the simple blocks with small recoupling
matrices (M = K <= the kernel's row limit) into the fused kernel's group,
piece and task tables: the external legs of a group in output order (unit
legs dropped), per piece the structural strides and the stride of every
external leg.  `emulate` applies the tables with numpy exactly as the kernel
indexes them (a test aid; the device path never calls it).
"""

import numpy as np

from .._native import FS_PERM_MAXR, PERM_TASK_DTYPE, SU2_GROUP_DTYPE, SU2_PIECE_DTYPE
from .abelian_plan import magic_divisor

MAXD = 8
TASK_COLUMNS = 4096
TASK_ROWS = 48      # FS_SU2_TASK_ROWS: outer-leg values one task may span


def fusable(M, K, E, e_out, n_in, n_out, max_rows, max_pieces):
    """Per simple block: True when the fused kernel can take it."""
    nonunit = (e_out > 1).sum(axis=1)
    return ((M <= max_rows) & (K <= max_rows) & (M == K) & (n_in <= max_pieces)
            & (n_out <= max_pieces) & (nonunit <= MAXD) & (E < 2**31) & (E > 0))


def build(groups_sel, e_out, E, M, K, u_off, gather, gin_group, gin_row, scatter,
          sout_group, sout_row, axes):
    """Fused tables for the simple blocks `groups_sel` (indices).

    gather / scatter: the raw piece arrays (dims, ostride, nstride, obase, nbase,
    present) of _block_gather / _block_scatter; gin_group / sout_group: the
    simple block of every piece, gin_row / sout_row its first row in the
    group (structural offset koff / moff).  Input pieces take their strides
    from the source side (ostride, obase; absent sources get base -1), output
    pieces from the destination side (nstride, nbase).  Vectorised over the
    groups: the legs of a group in output order with unit legs dropped, every
    piece's leg strides reordered the same way."""
    axes = np.asarray(axes, dtype=np.int64)
    sel = np.asarray(groups_sel, dtype=np.int64)
    ng = sel.size
    gtab = np.zeros(ng, dtype=SU2_GROUP_DTYPE)
    gd, go, _, gob, _, gpres = gather
    sd, _, sn, _, snb, _ = scatter
    n_sb = e_out.shape[0]
    nleg = e_out.shape[1]
    pos = np.full(n_sb, -1, dtype=np.int64)
    pos[sel] = np.arange(ng)
    eo = e_out[sel]
    keep = eo > 1
    nkeep = keep.sum(axis=1)
    order = np.argsort(~keep, axis=1, kind="stable")    # kept legs first, in order
    live = np.arange(nleg)[None, :] < nkeep[:, None]
    dims = np.where(live, np.take_along_axis(eo, order, axis=1), 1)

    def pieces_of(groups):
        # the pieces of the selected groups, grouped, in their original order
        idx = np.flatnonzero(pos[groups] >= 0)
        return idx[np.argsort(pos[groups[idx]], kind="stable")]

    pi = pieces_of(gin_group)
    po = pieces_of(sout_group)
    gi_in = pos[gin_group[pi]]
    gi_out = pos[sout_group[po]]
    tin = np.zeros(pi.size, dtype=SU2_PIECE_DTYPE)
    tin["base"] = np.where(gpres[pi], gob[pi], -1)
    tin["sr_stride"] = go[pi, 0]
    tin["sc_stride"] = go[pi, 1]
    ext_in = np.take_along_axis(go[pi][:, 2:][:, axes], order[gi_in], axis=1)
    tin["ext"][:, :nleg] = np.where(live[gi_in], ext_in, 0)[:, :MAXD]
    tin["sr"] = gd[pi, 0]
    tin["sc"] = gd[pi, 1]
    tin["row0"] = gin_row[pi]
    tout = np.zeros(po.size, dtype=SU2_PIECE_DTYPE)
    tout["base"] = snb[po]
    tout["sr_stride"] = sn[po, 0]
    tout["sc_stride"] = sn[po, 1]
    ext_out = np.take_along_axis(sn[po][:, 2:], order[gi_out], axis=1)
    tout["ext"][:, :nleg] = np.where(live[gi_out], ext_out, 0)[:, :MAXD]
    tout["sr"] = sd[po, 0]
    tout["sc"] = sd[po, 1]
    tout["row0"] = sout_row[po]
    gtab["u_off"] = u_off[sel]
    gtab["ncols"] = E[sel]
    gtab["dims"] = 1
    gtab["dims"][:, :nleg] = dims[:, :MAXD]
    m, sh = magic_divisor(np.maximum(gtab["dims"].astype(np.int64), 1))
    gtab["divm"] = m
    gtab["divs"] = sh
    gtab["ndim"] = nkeep
    gtab["M"] = M[sel]
    gtab["K"] = K[sel]
    counts_in = np.bincount(gi_in, minlength=ng)
    counts_out = np.bincount(gi_out, minlength=ng)
    gtab["in_count"] = counts_in
    gtab["out_count"] = counts_out
    gtab["in_first"] = np.cumsum(counts_in) - counts_in
    gtab["out_first"] = pi.size + np.cumsum(counts_out) - counts_out
    pieces = np.concatenate([tin, tout])
    return gtab, pieces, make_tasks(gtab)


def check(gtab, pieces, src_len, out_len, u_len):
    """Every address the kernel forms lies inside its buffer (host side check
    before the call; the kernel checks again and flags)."""
    if gtab.size == 0:
        return
    if ((gtab["u_off"] < 0) | (gtab["u_off"] + gtab["M"].astype(np.int64) * gtab["K"] > u_len)).any():
        raise AssertionError("recoupling matrix outside the U buffer")
    d = gtab["dims"].astype(np.int64) - 1
    for first, count, length, is_in, rows_key in (
            ("in_first", "in_count", src_len, True, "K"), ("out_first", "out_count", out_len, False, "M")):
        cnt = gtab[count].astype(np.int64)
        idx = np.repeat(gtab[first].astype(np.int64), cnt) + (
            np.arange(int(cnt.sum())) - np.repeat(np.cumsum(cnt) - cnt, cnt))
        gidx = np.repeat(np.arange(gtab.size), cnt)
        pc = pieces[idx]
        ext = pc["ext"].astype(np.int64)
        sr = pc["sr"].astype(np.int64)
        sc = pc["sc"].astype(np.int64)
        lo = pc["base"] + (np.minimum(ext, 0) * d[gidx]).sum(axis=1)
        hi = (pc["base"] + (np.maximum(ext, 0) * d[gidx]).sum(axis=1)
              + (sr - 1) * pc["sr_stride"] + (sc - 1) * pc["sc_stride"])
        live = pc["base"] >= 0 if is_in else np.ones(idx.size, dtype=bool)
        if ((lo < 0) | (hi >= length))[live].any():
            raise AssertionError("fused permute piece outside its buffer")
        lim = gtab[rows_key].astype(np.int64)
        if (pc["row0"] + sr * sc > lim[gidx]).any():
            raise AssertionError("fused permute piece rows outside the group")
        if not np.array_equal(np.bincount(gidx, weights=sr * sc, minlength=gtab.size), lim):
            raise AssertionError("fused permute pieces do not cover the group")


def make_tasks(gtab):
    """Tasks of the fused kernel: whole rows of the innermost output leg (L
    columns each), at most TASK_ROWS rows and about TASK_COLUMNS columns per
    task; a row longer than TASK_COLUMNS is cut into pieces of one row."""
    ng = gtab.size
    ncols = gtab["ncols"].astype(np.int64)
    nd = gtab["ndim"].astype(np.int64)
    L = np.where(nd > 0, gtab["dims"][np.arange(ng), np.maximum(nd - 1, 0)], 1).astype(np.int64)
    per = np.where(L >= TASK_COLUMNS, TASK_COLUMNS,
                   L * np.clip(TASK_COLUMNS // np.maximum(L, 1), 1, TASK_ROWS))
    starts, groups_of = [], []
    for g in range(ng):
        if L[g] >= TASK_COLUMNS:
            rows = np.arange(0, ncols[g], L[g])
            inner = np.arange(0, L[g], TASK_COLUMNS)
            st = (rows[:, None] + inner[None, :]).ravel()
        else:
            st = np.arange(0, ncols[g], per[g])
        starts.append(st)
        groups_of.append(np.full(st.size, g))
    tasks = np.zeros(int(sum(x.size for x in starts)), dtype=PERM_TASK_DTYPE)
    if tasks.size == 0:
        return tasks
    st = np.concatenate(starts)
    gi = np.concatenate(groups_of)
    tasks["eb"] = gi
    tasks["start"] = st
    row_end = np.where(L[gi] >= TASK_COLUMNS, (st // L[gi] + 1) * L[gi], ncols[gi])
    tasks["count"] = np.minimum(np.minimum(per[gi], row_end - st), ncols[gi] - st)
    return tasks


def emulate(gtab, pieces, tasks, U, src, out):
    """numpy application of the fused tables, indexing as the kernel does."""
    for t in tasks:
        g = gtab[int(t["eb"])]
        nd = int(g["ndim"])
        dims = g["dims"][:nd].astype(np.int64)
        cols = np.arange(int(t["start"]), int(t["start"]) + int(t["count"]))
        e = np.array(np.unravel_index(cols, dims)) if nd else np.zeros((0, cols.size), int)
        Kg, Mg = int(g["K"]), int(g["M"])
        x = np.zeros((Kg, cols.size))
        for p in pieces[int(g["in_first"]): int(g["in_first"]) + int(g["in_count"])]:
            ext = (p["ext"][:nd].astype(np.int64)[:, None] * e).sum(axis=0)
            for sr in range(int(p["sr"])):
                for sc in range(int(p["sc"])):
                    k = int(p["row0"]) + sr * int(p["sc"]) + sc
                    if p["base"] >= 0:
                        x[k] = src[p["base"] + ext + sr * p["sr_stride"] + sc * p["sc_stride"]]
        u = U[int(g["u_off"]): int(g["u_off"]) + Mg * Kg].reshape(Mg, Kg)
        y = u @ x
        for p in pieces[int(g["out_first"]): int(g["out_first"]) + int(g["out_count"])]:
            ext = (p["ext"][:nd].astype(np.int64)[:, None] * e).sum(axis=0)
            for sr in range(int(p["sr"])):
                for sc in range(int(p["sc"])):
                    i = int(p["row0"]) + sr * int(p["sc"]) + sc
                    out[p["base"] + ext + sr * p["sr_stride"] + sc * p["sc_stride"]] = y[i]
    return out


assert FS_PERM_MAXR == MAXD
