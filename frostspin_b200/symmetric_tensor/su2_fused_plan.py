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
TASK_COLUMNS = 1024


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
    pieces from the destination side (nstride, nbase)."""
    axes = np.asarray(axes, dtype=np.int64)
    ng = len(groups_sel)
    gtab = np.zeros(ng, dtype=SU2_GROUP_DTYPE)
    gd, go, _, gob, _, gpres = gather
    sd, _, sn, _, snb, _ = scatter
    pieces_in, pieces_out = [], []
    for j, g in enumerate(groups_sel):
        keep = np.flatnonzero(e_out[g] > 1)
        dims = e_out[g][keep]
        pi = np.flatnonzero(gin_group == g)
        po = np.flatnonzero(sout_group == g)
        row_in = gin_row[pi]
        row_out = sout_row[po]
        tin = np.zeros(pi.size, dtype=SU2_PIECE_DTYPE)
        tin["base"] = np.where(gpres[pi], gob[pi], -1)
        tin["sr_stride"] = go[pi, 0]
        tin["sc_stride"] = go[pi, 1]
        ext_in = go[pi][:, 2:][:, axes][:, keep]
        tin["ext"][:, : keep.size] = ext_in
        tin["sr"] = gd[pi, 0]
        tin["sc"] = gd[pi, 1]
        tin["row0"] = row_in
        tout = np.zeros(po.size, dtype=SU2_PIECE_DTYPE)
        tout["base"] = snb[po]
        tout["sr_stride"] = sn[po, 0]
        tout["sc_stride"] = sn[po, 1]
        tout["ext"][:, : keep.size] = sn[po][:, 2:][:, keep]
        tout["sr"] = sd[po, 0]
        tout["sc"] = sd[po, 1]
        tout["row0"] = row_out
        pieces_in.append(tin)
        pieces_out.append(tout)
        gtab["u_off"][j] = u_off[g]
        gtab["ncols"][j] = E[g]
        gtab["dims"][j] = 1
        gtab["dims"][j, : keep.size] = dims
        m, s = magic_divisor(np.maximum(gtab["dims"][j].astype(np.int64), 1))
        gtab["divm"][j] = m
        gtab["divs"][j] = s
        gtab["ndim"][j] = keep.size
        gtab["M"][j] = M[g]
        gtab["K"][j] = K[g]
        gtab["in_count"][j] = pi.size
        gtab["out_count"][j] = po.size
    pin = np.concatenate(pieces_in) if pieces_in else np.zeros(0, dtype=SU2_PIECE_DTYPE)
    pout = np.concatenate(pieces_out) if pieces_out else np.zeros(0, dtype=SU2_PIECE_DTYPE)
    counts_in = gtab["in_count"].astype(np.int64)
    counts_out = gtab["out_count"].astype(np.int64)
    gtab["in_first"] = np.concatenate([[0], np.cumsum(counts_in)[:-1]]) if ng else []
    gtab["out_first"] = (pin.size + np.concatenate([[0], np.cumsum(counts_out)[:-1]])
                         if ng else [])
    pieces = np.concatenate([pin, pout])
    # tasks: runs of TASK_COLUMNS columns of one group
    ncols = gtab["ncols"].astype(np.int64)
    nt = (ncols + TASK_COLUMNS - 1) // TASK_COLUMNS
    tasks = np.zeros(int(nt.sum()), dtype=PERM_TASK_DTYPE)
    gi = np.repeat(np.arange(ng), nt)
    first = np.repeat(np.cumsum(nt) - nt, nt)
    start = (np.arange(tasks.size) - first) * TASK_COLUMNS
    tasks["eb"] = gi
    tasks["start"] = start
    tasks["count"] = np.minimum(TASK_COLUMNS, ncols[gi] - start)
    return gtab, pieces, tasks


def check(gtab, pieces, src_len, out_len, u_len):
    """Every address the kernel forms lies inside its buffer (host side check
    before the call; the kernel checks again and flags)."""
    if gtab.size == 0:
        return
    for j in range(gtab.size):
        g = gtab[j]
        nd = int(g["ndim"])
        if g["u_off"] < 0 or g["u_off"] + int(g["M"]) * int(g["K"]) > u_len:
            raise AssertionError("recoupling matrix outside the U buffer")
        for first, count, length, is_in in ((g["in_first"], g["in_count"], src_len, True),
                                            (g["out_first"], g["out_count"], out_len, False)):
            rows = 0
            for p in pieces[int(first): int(first) + int(count)]:
                rows += int(p["sr"]) * int(p["sc"])
                if is_in and p["base"] < 0:
                    continue
                ext = p["ext"][:nd].astype(np.int64)
                d = g["dims"][:nd].astype(np.int64) - 1
                lo = p["base"] + (np.minimum(ext, 0) * d).sum()
                hi = (p["base"] + (np.maximum(ext, 0) * d).sum()
                      + (int(p["sr"]) - 1) * int(p["sr_stride"])
                      + (int(p["sc"]) - 1) * int(p["sc_stride"]))
                if lo < 0 or hi >= length:
                    raise AssertionError("fused permute piece outside its buffer")
                if int(p["row0"]) + int(p["sr"]) * int(p["sc"]) > (g["K"] if is_in else g["M"]):
                    raise AssertionError("fused permute piece rows outside the group")
            if rows != (g["K"] if is_in else g["M"]):
                raise AssertionError("fused permute pieces do not cover the group")


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
