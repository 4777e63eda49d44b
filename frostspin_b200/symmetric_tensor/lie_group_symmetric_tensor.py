"""Non-abelian (Lie group) SymmetricTensor: permute through fusion trees.

Mirrors frostspin/symmetric_tensor/non_abelian_symmetric_tensor.py and
lie_group_symmetric_tensor.py.  A representation is a 2 x n int array (row 0:
degeneracies, row 1: irreps).  An elementary block fixes one irrep per leg; its
row legs fuse (Clebsch-Gordan tree with depth on the first leg only) into
irreps with structural multiplicities, and a matrix block of irrep b stacks, for
every row elementary block, (structural multiplicity x external degeneracy)
rows, structural index outer.  Columns likewise.

A permute, a dense -> blocks and a blocks -> dense conversion are all one
linear map of the same shape, executed on the device in three launches:

  gather   fs_abelian_permute with strided tables: every (group, sector) piece
           of the input becomes rows of a matrix X_g (structural x external),
           the external axes already in output order;
  GEMM     fs_grouped_dgemm: Y_g = U_g X_g for all groups in one launch, U_g
           the recoupling matrix of the group (host computed, device cached);
  scatter  fs_abelian_permute: the rows of Y_g go to the output sectors.

For a permute a group is a simple block (one elementary block seen from the
input and the output bipartition) and U_g stacks the reference's isometries
(lie_group_symmetric_tensor.py:657-733); for the dense conversions a group is
one (row, column) elementary block and U_g the CG projector of
lie_group_symmetric_tensor.py:856-1109.  Only the structural part is keyed on
irreps; external degeneracies enter the gather/scatter tables, rebuilt (and
cached) per concrete tensor layout.
"""

import itertools
from collections import OrderedDict

import numpy as np

from .. import _native, instrument, linalg
from .. import device as dev
from .._native import FS_PERM_MAXR
from . import su2_fused_plan
from .abelian_plan import _make_tasks, _pack_ebs
from .symmetric_tensor import SymmetricTensor

_MAP_CACHE = OrderedDict()
_MAP_CACHE_SIZE = 256
_FUSED = {"on": True, "limits": None}


def set_fused_permute(enabled):
    """Whether permutes run the simple blocks with small recoupling matrices
    through the one-pass fused kernel (the default: one pass over the data
    instead of three) or through gather -> grouped GEMM -> scatter like the
    others; the results agree to rounding."""
    _FUSED["on"] = bool(enabled)


def fused_permute_enabled():
    return _FUSED["on"]


def _fused_limits():
    if _FUSED["limits"] is None:
        _FUSED["limits"] = _native.su2_fused_limits()
    return _FUSED["limits"]


# ------------------------------------------------------------------ helpers
def _kron_all(arrays):
    """C-order products over legs: out[ravel(j0, j1, ...)] = a0[j0] * a1[j1] ..."""
    out = np.ones(1, dtype=np.int64)
    for a in arrays:
        out = np.multiply.outer(out, np.asarray(a, dtype=np.int64)).ravel()
    return out


def _suffix_prod(e):
    """s[:, k] = prod_{k' > k} e[:, k'] (C-order strides of the legs of e)."""
    s = np.ones_like(e)
    for k in range(e.shape[1] - 2, -1, -1):
        s[:, k] = s[:, k + 1] * e[:, k + 1]
    return s


def _exclusive_cumsum(x):
    out = np.zeros(len(x), dtype=np.int64)
    if len(x) > 1:
        out[1:] = np.cumsum(x[:-1])
    return out


def _segment_offsets(group, sizes):
    """Offset of every entry inside its group (entries sorted by group)."""
    start = _exclusive_cumsum(sizes)
    first = np.zeros(len(group), dtype=np.int64)
    if len(group):
        new = np.ones(len(group), dtype=bool)
        new[1:] = group[1:] != group[:-1]
        idx = np.flatnonzero(new)
        first = np.repeat(start[idx], np.diff(np.append(idx, len(group))))
    return start - first


def _split_wide(dims, ostride, nstride, obase, nbase, present):
    """Enumerate the outermost legs of entries with more than FS_PERM_MAXR
    non-unit legs into separate entries, so that every entry fits the kernel's
    descriptor even when no legs merge."""
    while True:
        wide = (dims > 1).sum(axis=1) > FS_PERM_MAXR
        if not wide.any():
            return dims, ostride, nstride, obase, nbase, present
        w = np.flatnonzero(wide)
        key = np.where(dims[w] > 1, nstride[w], -1)
        k = np.argmax(key, axis=1)
        ext = dims[w, k]
        rep = np.repeat(np.arange(w.size), ext)
        idx = np.arange(int(ext.sum())) - np.repeat(_exclusive_cumsum(ext), ext)
        src = w[rep]
        kk = k[rep]
        nd = dims[src].copy()
        nd[np.arange(src.size), kk] = 1
        no = obase[src] + np.where(present[src], idx * ostride[src, kk], 0)
        nn = nbase[src] + idx * nstride[src, kk]
        keep = ~wide
        dims = np.concatenate([dims[keep], nd])
        ostride = np.concatenate([ostride[keep], ostride[src]])
        nstride = np.concatenate([nstride[keep], nstride[src]])
        obase = np.concatenate([obase[keep], no])
        nbase = np.concatenate([nbase[keep], nn])
        present = np.concatenate([present[keep], present[src]])


def _copy_tables(dims, ostride, nstride, obase, nbase, present, src_len, dst_len):
    """Pack strided copies into the fs_abelian_permute tables, after checking
    every entry against both buffers."""
    dims = np.asarray(dims, dtype=np.int64)
    ostride = np.asarray(ostride, dtype=np.int64)
    nstride = np.asarray(nstride, dtype=np.int64)
    obase = np.asarray(obase, dtype=np.int64)
    nbase = np.asarray(nbase, dtype=np.int64)
    present = np.asarray(present, dtype=bool)
    if dims.shape[0]:
        span_o = ((dims - 1) * ostride).sum(axis=1)
        span_n = ((dims - 1) * nstride).sum(axis=1)
        if present.any() and (
            (obase[present] < 0).any() or (obase + span_o)[present].max() >= src_len
        ):
            raise AssertionError("copy table reads outside its source buffer")
        if (nbase < 0).any() or (nbase + span_n).max() >= dst_len:
            raise AssertionError("copy table writes outside its destination buffer")
    dims, ostride, nstride, obase, nbase, present = _split_wide(
        dims, ostride, nstride, np.where(present, obase, -1), nbase, present
    )
    ebs, _ = _pack_ebs(dims, ostride, nstride, np.where(present, obase, -1), nbase, present)
    return ebs, _make_tasks(ebs)


class LieMap:
    """One gather -> grouped GEMM -> scatter on the device (numpy tables; device
    copies made on first use)."""

    __slots__ = (
        "gather", "scatter", "x_size", "out_size", "zero_out", "M", "N", "K",
        "u_off", "x_off", "u_host", "device", "out_offsets", "out_shapes",
        "out_irreps", "in_len", "fused", "fused_coeffs",
    )

    def run(self, src, out=None):
        if self.device is None:
            fz = self.fused
            self.device = (
                dev.upload(self.gather[0]), dev.upload(self.gather[1]),
                dev.upload(self.scatter[0]), dev.upload(self.scatter[1]),
                dev.upload_f64(self.u_host),
                None if fz is None else tuple(dev.upload(a) for a in fz),
            )
        g_ebs, g_tasks, s_ebs, s_tasks, d_u, d_fz = self.device
        if out is None:
            out = dev.zeros_f64(self.out_size) if self.zero_out else dev.empty_f64(self.out_size)
        if src.numel() < self.in_len:
            raise ValueError("source buffer is smaller than the plan expects")
        if d_fz is not None:
            d_groups, d_pieces, d_tasks = d_fz
            with instrument.region("permute_fused", bytes=16.0 * self.fused_coeffs):
                _native.call(
                    "fs_su2_permute_fused", dev.ptr(src), int(src.numel()), dev.ptr(out),
                    int(out.numel()), d_groups.data_ptr(), int(self.fused[0].size),
                    d_pieces.data_ptr(), int(self.fused[1].size), d_u.data_ptr(),
                    int(self.u_host.size), d_tasks.data_ptr(), int(self.fused[2].size), None,
                    dev.stream(),
                )
        if self.x_size == 0:
            return out
        x = dev.empty_f64(self.x_size)
        y = dev.empty_f64(int((self.M * self.N).sum()))
        with instrument.region("permute", bytes=16.0 * self.x_size):
            _native.call(
                "fs_abelian_permute", dev.ptr(src), int(src.numel()), dev.ptr(x),
                int(x.numel()), g_ebs.data_ptr(), int(self.gather[0].size),
                g_tasks.data_ptr(), int(self.gather[1].size), None, dev.stream(),
            )
        arr = np.zeros(self.M.size, dtype=_native.GEMM_PROBLEM_DTYPE)
        y_off = _exclusive_cumsum(self.M * self.N)
        arr["A"] = d_u.data_ptr() + 8 * self.u_off
        arr["B"] = x.data_ptr() + 8 * self.x_off
        arr["C"] = y.data_ptr() + 8 * y_off
        arr["lda"] = self.K
        arr["ldb"] = self.N
        arr["ldc"] = self.N
        arr["M"], arr["N"], arr["K"] = self.M, self.N, self.K
        arr["alpha"] = 1.0
        linalg.grouped_dgemm_table(arr, region="gemm_recoupling")
        with instrument.region("permute", bytes=16.0 * int(y.numel())):
            _native.call(
                "fs_abelian_permute", dev.ptr(y), int(y.numel()), dev.ptr(out),
                int(out.numel()), s_ebs.data_ptr(), int(self.scatter[0].size),
                s_tasks.data_ptr(), int(self.scatter[1].size), None, dev.stream(),
            )
        return out


def _block_gather(e, nrr, axes, sr, sc, row0, col0, src_off, rs, cs, present, dst, koff, E):
    """Strided copy of block sectors (s_r, e_rows..., s_c, e_cols...) into rows
    s_r * s_c + s_c of X, columns the external legs in the order ``axes``
    (lie_group_symmetric_tensor.py:130-164: numba_transpose_reshape with
    data_perm = (0, nrr + 1, *(axes + 1 + (axes >= nrr))))."""
    ndim = e.shape[1]
    edir = e[:, :nrr].prod(axis=1)
    edic = e[:, nrr:].prod(axis=1)
    rpre = _suffix_prod(e[:, :nrr])
    cpre = _suffix_prod(e[:, nrr:])
    npre = _suffix_prod(e[:, axes])
    inv = np.argsort(axes)
    dims = np.concatenate([sr[:, None], sc[:, None], e], axis=1)
    ostride = np.concatenate(
        [(edir * rs)[:, None], (edic * cs)[:, None], rpre * rs[:, None], cpre * cs[:, None]],
        axis=1,
    )
    nstride = np.concatenate([(sc * E)[:, None], E[:, None], npre[:, inv]], axis=1)
    obase = src_off + row0 * rs + col0 * cs
    nbase = dst + koff * E
    assert dims.shape[1] == ndim + 2
    return dims, ostride, nstride, obase, nbase, present


def _block_scatter(e_new, new_nrr, sr, sc, row0, col0, dst_off, ncols, src, moff, E):
    """Rows s_r * s_c + s_c of Y (columns: external legs in output order) into
    output block sectors (s_r, e_rows..., s_c, e_cols...)
    (lie_group_symmetric_tensor.py:184-212)."""
    edor = e_new[:, :new_nrr].prod(axis=1)
    edoc = e_new[:, new_nrr:].prod(axis=1)
    npre = _suffix_prod(e_new)
    nrpre = _suffix_prod(e_new[:, :new_nrr])
    ncpre = _suffix_prod(e_new[:, new_nrr:])
    dims = np.concatenate([sr[:, None], sc[:, None], e_new], axis=1)
    ostride = np.concatenate([(sc * E)[:, None], E[:, None], npre], axis=1)
    nstride = np.concatenate(
        [(edor * ncols)[:, None], edoc[:, None], nrpre * ncols[:, None], ncpre], axis=1
    )
    obase = src + moff * E
    nbase = dst_off + row0 * ncols + col0
    return dims, ostride, nstride, obase, nbase, np.ones(len(sr), dtype=bool)


def _dense_copy(irr, e, shifts_base, dstride, xy_off, E, to_dense):
    """Between a dense tensor (leg index shift + e * irr + m) and X/Y matrices
    (rows: m of all legs, columns: e of all legs), lie_group_symmetric_tensor.py
    :920-925 and :1104-1107."""
    mpre = _suffix_prod(irr)
    epre = _suffix_prod(e)
    n = irr.shape[0]
    dims = np.concatenate([irr, e], axis=1)
    dense_s = np.concatenate([np.broadcast_to(dstride, irr.shape), irr * dstride], axis=1)
    mat_s = np.concatenate([mpre * E[:, None], epre], axis=1)
    dense_base = (shifts_base * dstride).sum(axis=1)
    present = np.ones(n, dtype=bool)
    if to_dense:
        return dims, mat_s, dense_s, xy_off, dense_base, present
    return dims, dense_s, mat_s, dense_base, xy_off, present


# ------------------------------------------------------------------ classes
class NonAbelianSymmetricTensor(SymmetricTensor):
    """non_abelian_symmetric_tensor.py:7-90."""

    @staticmethod
    def init_representation(degen, irreps):
        rep = np.empty((2, len(degen)), dtype=np.int64)
        rep[0] = degen
        rep[1] = irreps
        return rep

    @classmethod
    def get_block_sizes(cls, row_reps, col_reps, signature):
        """non_abelian_symmetric_tensor.py:36-67."""
        signature = np.asarray(signature, dtype=bool)
        nrr = len(row_reps)
        row_tot = cls.combine_representations(row_reps, signature[:nrr])
        col_tot = cls.combine_representations(col_reps, ~signature[nrr:])
        rinds, cinds = (row_tot[1, :, None] == col_tot[1]).nonzero()
        block_irreps = np.asarray(row_tot[1, rinds], dtype=np.int64)
        block_shapes = np.empty((rinds.size, 2), dtype=np.int64)
        block_shapes[:, 0] = row_tot[0, rinds]
        block_shapes[:, 1] = col_tot[0, cinds]
        return block_irreps, block_shapes

    def check_blocks_fit_representations(self):
        """non_abelian_symmetric_tensor.py:69-84."""
        assert self._block_irreps.size == self._nblocks
        row_rep = self.get_row_representation()
        col_rep = self.get_column_representation()
        r_indices = row_rep[1].searchsorted(self._block_irreps)
        c_indices = col_rep[1].searchsorted(self._block_irreps)
        assert (r_indices < row_rep.shape[1]).all() and (c_indices < col_rep.shape[1]).all()
        assert (row_rep[1, r_indices] == self._block_irreps).all()
        assert (col_rep[1, c_indices] == self._block_irreps).all()
        for bi in range(self._nblocks):
            assert tuple(self._bshapes[bi]) == (row_rep[0, r_indices[bi]], col_rep[0, c_indices[bi]])
        return True

    def update_signature(self, sign_update):
        # the reference leaves this unimplemented for non-abelian groups
        # (lie_group_symmetric_tensor.py:1136-1147)
        raise NotImplementedError("To do!")


class LieGroupSymmetricTensor(NonAbelianSymmetricTensor):
    """lie_group_symmetric_tensor.py:298-1176: permute, transpose and the dense
    conversions of a tensor whose symmetry is a Lie group, through CG trees."""

    _tree_cache = {}
    _fuse_cache = {}
    _iso_cache = {}
    _proj_cache = {}
    _struct_cache = {}

    @classmethod
    def compute_clebsch_gordan_tree(cls, rep_in, signature, *, target_irreps=None):
        raise NotImplementedError("Must be defined in derived class")

    @classmethod
    def clear_structure_caches(cls):
        for c in (cls._tree_cache, cls._fuse_cache, cls._iso_cache, cls._proj_cache,
                  cls._struct_cache):
            c.clear()
        _MAP_CACHE.clear()

    # ------------------------------------------------- elementary structure
    @classmethod
    def _fuse_elementary(cls, irreps):
        """Fused (multiplicities, irreps) of one irrep per leg."""
        key = (cls._symmetry, irreps)
        r = cls._fuse_cache.get(key)
        if r is None:
            reps = [np.array([[1], [irr]], dtype=np.int64) for irr in irreps]
            r = cls.combine_representations(reps, None)
            r = (np.asarray(r[0], dtype=np.int64), np.asarray(r[1], dtype=np.int64))
            cls._fuse_cache[key] = r
        return r

    @classmethod
    def elementary_trees(cls, irreps, signature, target):
        """CG trees of one elementary block sliced by target irrep
        (sliced_elementary_trees, lie_group_symmetric_tensor.py:365-430, for a
        single elementary block): dict irrep -> array (*irrep dims, multiplicity,
        irrep dim)."""
        key = (cls._symmetry, irreps, signature, target)
        trees = cls._tree_cache.get(key)
        if trees is not None:
            return trees
        reps = [np.array([[1], [irr]], dtype=np.int64) for irr in irreps]
        rep, tree = cls.compute_clebsch_gordan_tree(
            reps, np.array(signature, dtype=bool), target_irreps=np.array(target)
        )
        trees = {}
        dims = [cls.irrep_dimension(irr) for irr in irreps]
        k = 0
        tset = set(target)
        for i in range(rep.shape[1]):
            deg, irr = int(rep[0, i]), int(rep[1, i])
            d = cls.irrep_dimension(irr)
            if irr in tset:
                sub = np.ascontiguousarray(tree[:, k : k + deg * d].reshape(*dims, deg, d))
                sub.setflags(write=False)
                trees[irr] = sub
            k += deg * d
        assert k == tree.shape[1]
        cls._tree_cache[key] = trees
        return trees

    @classmethod
    def _multiplicities(cls, irreps_per_leg, legs, targets):
        """(n elementary blocks over ``legs`` in C order, len(targets))
        structural multiplicity of every target irrep."""
        lists = [irreps_per_leg[k] for k in legs]
        n = int(np.prod([len(x) for x in lists]))
        out = np.zeros((n, len(targets)), dtype=np.int64)
        for i, combo in enumerate(itertools.product(*lists)):
            deg, irr = cls._fuse_elementary(tuple(int(c) for c in combo))
            pos = np.searchsorted(targets, irr)
            ok = pos < len(targets)
            ok[ok] = targets[pos[ok]] == irr[ok]
            out[i, pos[ok]] = deg[ok]
        return out

    @classmethod
    def _pair_projector(cls, rtree, ctree):
        """Projector of one sector of a (row, column) elementary block:
        (prod row dims * prod col dims, s_r * s_c)
        (lie_group_symmetric_tensor.py:949-955, :1086-1094)."""
        d = rtree.shape[-1]
        sr, sc = rtree.shape[-2], ctree.shape[-2]
        rt = rtree.reshape(-1, d)
        ct = ctree.reshape(-1, d)
        p = rt @ ct.T
        rdim = rt.shape[0] // sr
        cdim = ct.shape[0] // sc
        return p.reshape(rdim, sr, cdim, sc).swapaxes(1, 2).reshape(rdim * cdim, sr * sc)

    @classmethod
    def _recoupling(cls, irr, nrr, axes, new_nrr, signature):
        """Isometry of one simple block, all input sectors side by side
        (overlap_cg_trees, lie_group_symmetric_tensor.py:657-733): rows = output
        sectors (increasing irrep) x (s_or, s_oc); columns = input sectors x
        (s_ir, s_ic).  Entries below 1e-14 are set to zero before the division
        by the output irrep dimension, as in the reference."""
        key = (cls._symmetry, irr, nrr, axes, new_nrr, signature)
        u = cls._iso_cache.get(key)
        if u is not None:
            return u
        ndim = len(irr)
        sig = np.array(signature, dtype=bool)
        irr_out = tuple(irr[a] for a in axes)
        sig_out = sig[list(axes)]
        _, ri = cls._fuse_elementary(irr[:nrr])
        _, ci = cls._fuse_elementary(irr[nrr:])
        _, ro = cls._fuse_elementary(irr_out[:new_nrr])
        _, co = cls._fuse_elementary(irr_out[new_nrr:])
        shared_in = tuple(sorted(set(ri.tolist()) & set(ci.tolist())))
        shared_out = tuple(sorted(set(ro.tolist()) & set(co.tolist())))
        tri = cls.elementary_trees(irr[:nrr], tuple(bool(s) for s in sig[:nrr]), shared_in)
        tci = cls.elementary_trees(irr[nrr:], tuple(bool(s) for s in ~sig[nrr:]), shared_in)
        tro = cls.elementary_trees(
            irr_out[:new_nrr], tuple(bool(s) for s in sig_out[:new_nrr]), shared_out
        )
        tco = cls.elementary_trees(
            irr_out[new_nrr:], tuple(bool(s) for s in ~sig_out[new_nrr:]), shared_out
        )
        out_proj = [cls._pair_projector(tro[b], tco[b]).T for b in shared_out]
        dims_out = [cls.irrep_dimension(b) for b in shared_out]
        ax = np.array(axes)
        perm = np.empty(ndim + 2, dtype=np.int64)
        perm[:ndim] = (ax >= nrr) + ax
        perm[ndim] = nrr
        perm[ndim + 1] = ndim + 1
        n_rows = sum(op.shape[0] for op in out_proj)
        n_cols = sum(tri[b].shape[-2] * tci[b].shape[-2] for b in shared_in)
        u = np.empty((n_rows, n_cols))
        c0 = 0
        for b in shared_in:
            rtree, ctree = tri[b], tci[b]
            d = rtree.shape[-1]
            p = rtree.reshape(-1, d) @ ctree.reshape(-1, d).T
            p = p.reshape(rtree.shape[:-1] + ctree.shape[:-1]).transpose(perm)
            w = rtree.shape[-2] * ctree.shape[-2]
            p = p.reshape(-1, w)
            r0 = 0
            for op, dim in zip(out_proj, dims_out, strict=True):
                iso = op @ p
                iso[np.abs(iso) < 1e-14] = 0
                u[r0 : r0 + iso.shape[0], c0 : c0 + w] = iso / dim
                r0 += iso.shape[0]
            c0 += w
        u.setflags(write=False)
        cls._iso_cache[key] = u
        return u

    # ------------------------------------------------------ permute structure
    @classmethod
    def _permute_structure(cls, irreps_per_leg, nrr, axes, new_nrr, signature):
        """Degeneracy-independent part of a permute
        (_compute_structural_data, lie_group_symmetric_tensor.py:432-655),
        cached on (irreps per leg, nrr, axes, new nrr, signature) like the
        reference's _structural_data_dic."""
        key = (cls._symmetry, irreps_per_leg, nrr, axes, new_nrr, signature)
        st = cls._struct_cache.get(key)
        if st is not None:
            return st
        ndim = len(irreps_per_leg)
        ax = np.array(axes, dtype=np.int64)
        sig = np.array(signature, dtype=bool)
        sig_out = sig[ax]
        ones = [np.array([np.ones(len(x), dtype=np.int64), x]) for x in irreps_per_leg]
        bi_in, _ = cls.get_block_sizes(ones[:nrr], ones[nrr:], sig)
        if bi_in.size == 0:
            raise ValueError("Representations do not allow any block")
        out_ones = [ones[a] for a in axes]
        bi_out, _ = cls.get_block_sizes(out_ones[:new_nrr], out_ones[new_nrr:], sig_out)
        idirb = cls._multiplicities(irreps_per_leg, range(nrr), bi_in)
        idicb = cls._multiplicities(irreps_per_leg, range(nrr, ndim), bi_in)
        idorb = cls._multiplicities(irreps_per_leg, axes[:new_nrr], bi_out)
        idocb = cls._multiplicities(irreps_per_leg, axes[new_nrr:], bi_out)
        nseg = np.array([len(x) for x in irreps_per_leg], dtype=np.int64)
        shared = (idirb > 0).astype(np.int64) @ (idicb > 0).T.astype(np.int64)
        ir, ic = np.nonzero(shared)
        mul = np.concatenate(
            [np.array(np.unravel_index(ir, nseg[:nrr])).T.reshape(-1, nrr),
             np.array(np.unravel_index(ic, nseg[nrr:])).T.reshape(-1, ndim - nrr)],
            axis=1,
        ).astype(np.int64)
        ir_out = np.ravel_multi_index(mul[:, ax[:new_nrr]].T, nseg[ax[:new_nrr]])
        ic_out = np.ravel_multi_index(mul[:, ax[new_nrr:]].T, nseg[ax[new_nrr:]])
        in_sb, in_b = np.nonzero((idirb[ir] > 0) & (idicb[ic] > 0))
        out_sb, out_b = np.nonzero((idorb[ir_out] > 0) & (idocb[ic_out] > 0))
        in_sr, in_sc = idirb[ir[in_sb], in_b], idicb[ic[in_sb], in_b]
        out_sr, out_sc = idorb[ir_out[out_sb], out_b], idocb[ic_out[out_sb], out_b]
        n_sb = ir.size
        K = np.bincount(in_sb, in_sr * in_sc, minlength=n_sb).astype(np.int64)
        M = np.bincount(out_sb, out_sr * out_sc, minlength=n_sb).astype(np.int64)
        if not np.array_equal(K, M):
            raise AssertionError("number of coefficients not conserved")
        us = []
        sigt = tuple(bool(s) for s in sig)
        for s in range(n_sb):
            irr = tuple(int(irreps_per_leg[k][mul[s, k]]) for k in range(ndim))
            u = cls._recoupling(irr, nrr, axes, new_nrr, sigt)
            if u.shape != (M[s], K[s]):
                raise AssertionError("recoupling matrix does not match the sectors")
            us.append(u.ravel())
        st = {
            "bi_in": bi_in, "bi_out": bi_out, "idirb": idirb, "idicb": idicb,
            "idorb": idorb, "idocb": idocb, "ir": ir, "ic": ic, "ir_out": ir_out,
            "ic_out": ic_out, "mul": mul, "in_sb": in_sb, "in_b": in_b, "in_sr": in_sr,
            "in_sc": in_sc, "in_koff": _segment_offsets(in_sb, in_sr * in_sc),
            "out_sb": out_sb, "out_b": out_b, "out_sr": out_sr, "out_sc": out_sc,
            "out_moff": _segment_offsets(out_sb, out_sr * out_sc), "M": M, "K": K,
            "u_host": np.concatenate(us) if us else np.zeros(0),
            "u_off": _exclusive_cumsum(M * K),
        }
        cls._struct_cache[key] = st
        return st

    def _irreps_key(self):
        return tuple(
            tuple(int(x) for x in r[1]) for r in self._row_reps + self._col_reps
        )

    def _layout_key(self):
        return (
            tuple(tuple(int(x) for x in r[0]) for r in self._row_reps + self._col_reps),
            self._block_irreps.tobytes(), self._offsets.tobytes(), self._bshapes.tobytes(),
            self._trans, int(self._data.numel()),
        )

    def _source_blocks(self, all_irreps):
        """For every allowed block irrep: index of the stored block or -1."""
        pos = np.searchsorted(self._block_irreps, all_irreps)
        pos = np.minimum(pos, max(self._nblocks - 1, 0))
        ok = (self._nblocks > 0) & (self._block_irreps[pos] == all_irreps)
        return np.where(ok, pos, -1)

    def _block_source_arrays(self, bidx):
        """Offsets and (row, column) strides of stored blocks (index -1: absent)."""
        p = np.maximum(bidx, 0)
        present = bidx >= 0
        R = self._bshapes[p, 0]
        C = self._bshapes[p, 1]
        if self._trans:
            rs, cs = np.ones_like(R), R
        else:
            rs, cs = C, np.ones_like(C)
        return self._offsets[p], rs, cs, present

    def _permute_map(self, axes, new_nrr):
        key = ("permute", type(self).__name__, self._irreps_key(), self._layout_key(),
               self._signature.tobytes(), self._nrr, axes, new_nrr, _FUSED["on"])
        m = _MAP_CACHE.get(key)
        if m is not None:
            _MAP_CACHE.move_to_end(key)
            return m
        nrr = self._nrr
        st = self._permute_structure(
            self._irreps_key(), nrr, axes, new_nrr, tuple(bool(s) for s in self._signature)
        )
        reps = self._row_reps + self._col_reps
        degs = [np.asarray(r[0], dtype=np.int64) for r in reps]
        ax = np.array(axes, dtype=np.int64)
        mul = st["mul"]
        e = np.stack([degs[k][mul[:, k]] for k in range(self._ndim)], axis=1).reshape(
            -1, self._ndim
        )
        E = e.prod(axis=1)
        edir = _kron_all(degs[:nrr])
        edic = _kron_all(degs[nrr:])
        edor = _kron_all([degs[a] for a in axes[:new_nrr]])
        edoc = _kron_all([degs[a] for a in axes[new_nrr:]])
        cum_ir = np.cumsum(edir[:, None] * st["idirb"], axis=0)
        cum_ic = np.cumsum(edic[:, None] * st["idicb"], axis=0)
        cum_or = np.cumsum(edor[:, None] * st["idorb"], axis=0)
        cum_oc = np.cumsum(edoc[:, None] * st["idocb"], axis=0)
        row_start = cum_ir - edir[:, None] * st["idirb"]
        col_start = cum_ic - edic[:, None] * st["idicb"]
        orow_start = cum_or - edor[:, None] * st["idorb"]
        ocol_start = cum_oc - edoc[:, None] * st["idocb"]
        src_block = self._source_blocks(st["bi_in"])
        have = src_block >= 0
        if not np.array_equal(
            self._bshapes[src_block[have]],
            np.stack([cum_ir[-1], cum_ic[-1]], axis=1)[have],
        ):
            raise ValueError("block shapes do not match the representations")
        out_shapes = np.stack([cum_or[-1], cum_oc[-1]], axis=1).astype(np.int64)
        out_sizes = out_shapes[:, 0] * out_shapes[:, 1]
        out_offsets = _exclusive_cumsum(out_sizes)
        out_size = int(out_sizes.sum())
        n_sb = E.size
        e_out = e[:, ax]
        if _FUSED["on"] and n_sb:
            max_rows, max_pieces, _ = _fused_limits()
            fz = su2_fused_plan.fusable(
                st["M"], st["K"], E, e_out, np.bincount(st["in_sb"], minlength=n_sb),
                np.bincount(st["out_sb"], minlength=n_sb), max_rows, max_pieces)
        else:
            fz = np.zeros(n_sb, dtype=bool)
        rest = ~fz
        # X and Y hold the simple blocks that go through the grouped GEMM only
        x_off = _exclusive_cumsum(st["K"] * E * rest)
        x_size = int((st["K"] * E * rest).sum())

        sb = st["in_sb"]
        b = st["in_b"]
        src_off, rs, cs, present = self._block_source_arrays(src_block[b])
        raw_g = _block_gather(
            e[sb], nrr, ax, st["in_sr"], st["in_sc"], row_start[st["ir"][sb], b],
            col_start[st["ic"][sb], b], src_off, rs, cs, present, x_off[sb],
            st["in_koff"], E[sb],
        )
        sel = rest[sb]
        gather = _copy_tables(*(a[sel] for a in raw_g), int(self._data.numel()), x_size)
        sb = st["out_sb"]
        b = st["out_b"]
        raw_s = _block_scatter(
            e_out[sb], new_nrr, st["out_sr"], st["out_sc"],
            orow_start[st["ir_out"][sb], b], ocol_start[st["ic_out"][sb], b],
            out_offsets[b], out_shapes[b, 1], x_off[sb], st["out_moff"], E[sb],
        )
        sel = rest[sb]
        # M == K: Y has the layout of X
        scatter = _copy_tables(*(a[sel] for a in raw_s), x_size, out_size)
        fused, fused_coeffs = None, 0
        if fz.any():
            fused = su2_fused_plan.build(
                np.flatnonzero(fz), e_out, E, st["M"], st["K"], st["u_off"], raw_g,
                st["in_sb"], st["in_koff"], raw_s, st["out_sb"], st["out_moff"], ax)
            su2_fused_plan.check(fused[0], fused[1], int(self._data.numel()), out_size,
                                 int(st["u_host"].size))
            fused_coeffs = int((st["M"] * E)[fz].sum())
        if int(gather[0]["volume"].astype(np.int64).sum()) != x_size or int(
            scatter[0]["volume"].astype(np.int64).sum()
        ) + fused_coeffs != out_size:
            raise AssertionError("permute tables do not cover their buffers")
        m = LieMap()
        m.gather, m.scatter = gather, scatter
        m.x_size, m.out_size, m.zero_out = x_size, out_size, False
        m.M, m.N, m.K = st["M"][rest], E[rest], st["K"][rest]
        m.u_off, m.x_off, m.u_host = st["u_off"][rest], x_off[rest], st["u_host"]
        m.fused, m.fused_coeffs = fused, fused_coeffs
        m.device = None
        m.out_offsets, m.out_shapes, m.out_irreps = out_offsets, out_shapes, st["bi_out"]
        m.in_len = int(self._data.numel())
        _MAP_CACHE[key] = m
        if len(_MAP_CACHE) > _MAP_CACHE_SIZE:
            _MAP_CACHE.popitem(last=False)
        return m

    def _permute_data(self, axes, nrr):
        """lie_group_symmetric_tensor.py:1116-1134 -> _lie_permute_data
        (:735-835) on the device.  Every allowed output block is produced."""
        if self._nblocks == 0:  # symmetric_tensor.py:200-201
            return (dev.empty_f64(0), np.zeros(0, dtype=np.int64),
                    np.zeros((0, 2), dtype=np.int64), self._block_irreps)
        m = self._permute_map(tuple(int(a) for a in axes), int(nrr))
        out = m.run(self._data)
        return out, m.out_offsets, m.out_shapes, m.out_irreps

    def _transpose_data(self):
        """lie_group_symmetric_tensor.py:1111-1114: a full permute."""
        axes = tuple(range(self._nrr, self._ndim)) + tuple(range(self._nrr))
        data, offsets, shapes, irreps = self._permute_data(axes, self._ndim - self._nrr)
        return data, offsets, shapes, irreps, False

    # ----------------------------------------------------- dense conversions
    @classmethod
    def _dense_structure(cls, irreps_per_leg, nrr, signature, targets, to_dense):
        """Groups (row, column elementary blocks sharing an irrep of
        ``targets``) and their CG projectors for the dense conversions."""
        key = (cls._symmetry, irreps_per_leg, nrr, signature, targets, to_dense)
        st = cls._struct_cache.get(key)
        if st is not None:
            return st
        ndim = len(irreps_per_leg)
        tg = np.array(targets, dtype=np.int64)
        sig = np.array(signature, dtype=bool)
        idrb = cls._multiplicities(irreps_per_leg, range(nrr), tg)
        idcb = cls._multiplicities(irreps_per_leg, range(nrr, ndim), tg)
        nseg = np.array([len(x) for x in irreps_per_leg], dtype=np.int64)
        shared = (idrb > 0).astype(np.int64) @ (idcb > 0).T.astype(np.int64)
        ir, ic = np.nonzero(shared)
        mul = np.concatenate(
            [np.array(np.unravel_index(ir, nseg[:nrr])).T.reshape(-1, nrr),
             np.array(np.unravel_index(ic, nseg[nrr:])).T.reshape(-1, ndim - nrr)],
            axis=1,
        ).astype(np.int64)
        sec_g, sec_b = np.nonzero((idrb[ir] > 0) & (idcb[ic] > 0))
        sr, sc = idrb[ir[sec_g], sec_b], idcb[ic[sec_g], sec_b]
        irr = np.stack(
            [np.asarray(irreps_per_leg[k], dtype=np.int64)[mul[:, k]] for k in range(ndim)],
            axis=1,
        ).reshape(-1, ndim)
        dims = np.vectorize(cls.irrep_dimension, otypes=[np.int64])(irr) if irr.size else irr
        rc = dims.prod(axis=1)
        us = []
        sig_r = tuple(bool(s) for s in sig[:nrr])
        sig_c = tuple(bool(s) for s in ~sig[nrr:])
        tset = tuple(int(t) for t in tg)
        for g in range(ir.size):
            row_irr = tuple(int(x) for x in irr[g, :nrr])
            col_irr = tuple(int(x) for x in irr[g, nrr:])
            tri = cls.elementary_trees(row_irr, sig_r, tset)
            tci = cls.elementary_trees(col_irr, sig_c, tset)
            parts = []
            for b in sec_b[sec_g == g]:
                q = int(tg[b])
                p = cls._pair_projector(tri[q], tci[q])
                parts.append(p if to_dense else p.T / cls.irrep_dimension(q))
            u = np.hstack(parts) if to_dense else np.vstack(parts)
            us.append(np.ascontiguousarray(u).ravel())
        KS = np.bincount(sec_g, sr * sc, minlength=ir.size).astype(np.int64)
        M = rc if to_dense else KS
        K = KS if to_dense else rc
        st = {
            "idrb": idrb, "idcb": idcb, "ir": ir, "ic": ic, "mul": mul, "irr": irr,
            "dims": dims, "sec_g": sec_g, "sec_b": sec_b, "sr": sr, "sc": sc,
            "soff": _segment_offsets(sec_g, sr * sc), "M": M, "K": K,
            "u_host": np.concatenate(us) if us else np.zeros(0),
            "u_off": _exclusive_cumsum(M * K),
        }
        cls._struct_cache[key] = st
        return st

    @classmethod
    def _dense_geometry(cls, reps, st):
        ndim = len(reps)
        degs = [np.asarray(r[0], dtype=np.int64) for r in reps]
        mul = st["mul"]
        e = np.stack([degs[k][mul[:, k]] for k in range(ndim)], axis=1).reshape(-1, ndim)
        shape = np.array([cls.representation_dimension(r) for r in reps], dtype=np.int64)
        dstride = _suffix_prod(shape[None, :])[0]
        seg_start = []
        for r in reps:
            d = np.array([cls.irrep_dimension(x) for x in r[1]], dtype=np.int64)
            seg_start.append(_exclusive_cumsum(np.asarray(r[0], dtype=np.int64) * d))
        base = np.stack([seg_start[k][mul[:, k]] for k in range(ndim)], axis=1).reshape(-1, ndim)
        return degs, e, e.prod(axis=1), dstride, base, int(shape.prod())

    @classmethod
    def _from_dense_map(cls, row_reps, col_reps, signature):
        """The dense -> blocks map of a structure, with the allowed block irreps."""
        reps = tuple(row_reps) + tuple(col_reps)
        nrr = len(row_reps)
        signature = np.asarray(signature, dtype=bool)
        irreps_key = tuple(tuple(int(x) for x in r[1]) for r in reps)
        degs_key = tuple(tuple(int(x) for x in r[0]) for r in reps)
        key = ("from_dense", cls.__name__, irreps_key, degs_key, nrr, signature.tobytes())
        m = _MAP_CACHE.get(key)
        if m is not None:
            _MAP_CACHE.move_to_end(key)
            return m
        block_irreps, block_shapes = cls.get_block_sizes(row_reps, col_reps, signature)
        st = cls._dense_structure(
            irreps_key, nrr, tuple(bool(s) for s in signature),
            tuple(int(b) for b in block_irreps), False,
        )
        degs, e, E, dstride, base, dense_size = cls._dense_geometry(reps, st)
        m = cls._dense_map(st, degs, e, E, dstride, base, dense_size, nrr, block_shapes,
                           to_dense=False)
        m.out_irreps = block_irreps
        _MAP_CACHE[key] = m
        if len(_MAP_CACHE) > _MAP_CACHE_SIZE:
            _MAP_CACHE.popitem(last=False)
        return m

    @classmethod
    def _blocks_from_dense(cls, arr, row_reps, col_reps, signature):
        """lie_group_symmetric_tensor.py:856-967 on the device: every elementary
        block of the dense tensor is projected onto the block irreps by one
        group of the gather -> GEMM -> scatter map."""
        import torch

        m = cls._from_dense_map(row_reps, col_reps, signature)
        if isinstance(arr, torch.Tensor):
            src = arr.to(device=dev.device(), dtype=torch.float64).reshape(-1).contiguous()
        else:
            src = dev.upload_f64(np.asarray(arr).reshape(-1))
        out = m.run(src)
        return cls._from_storage(row_reps, col_reps, out, m.out_offsets, m.out_shapes,
                                 m.out_irreps, np.asarray(signature, dtype=bool))

    @classmethod
    def _dense_map(cls, st, degs, e, E, dstride, base, dense_size, nrr, block_shapes,
                   *, to_dense, tensor=None):
        ndim = e.shape[1]
        edr = _kron_all(degs[:nrr])
        edc = _kron_all(degs[nrr:])
        cum_r = np.cumsum(edr[:, None] * st["idrb"], axis=0)
        cum_c = np.cumsum(edc[:, None] * st["idcb"], axis=0)
        row_start = cum_r - edr[:, None] * st["idrb"]
        col_start = cum_c - edc[:, None] * st["idcb"]
        x_off = _exclusive_cumsum(st["K"] * E)
        x_size = int((st["K"] * E).sum())
        y_off = _exclusive_cumsum(st["M"] * E)
        y_size = int((st["M"] * E).sum())
        g = st["sec_g"]
        b = st["sec_b"]
        ident = np.arange(ndim, dtype=np.int64)
        irr_dims = st["dims"]
        m = LieMap()
        m.fused, m.fused_coeffs = None, 0
        if to_dense:
            # the targets are the stored blocks: sector b reads stored block b
            src_off, rs, cs, present = tensor._block_source_arrays(b)
            gather = _copy_tables(
                *_block_gather(e[g], nrr, ident, st["sr"], st["sc"], row_start[st["ir"][g], b],
                               col_start[st["ic"][g], b], src_off, rs, cs, present, x_off[g],
                               st["soff"], E[g]),
                int(tensor._data.numel()), x_size,
            )
            scatter = _copy_tables(
                *_dense_copy(irr_dims, e, base, dstride[None, :], y_off, E, True),
                y_size, dense_size,
            )
            out_size = dense_size
            m.zero_out = True
            m.in_len = int(tensor._data.numel())
            m.out_offsets = m.out_shapes = None
        else:
            gather = _copy_tables(
                *_dense_copy(irr_dims, e, base, dstride[None, :], x_off, E, False),
                dense_size, x_size,
            )
            out_shapes = np.asarray(block_shapes, dtype=np.int64).reshape(-1, 2)
            if not np.array_equal(out_shapes, np.stack([cum_r[-1], cum_c[-1]], axis=1)):
                raise AssertionError("block shapes do not match the representations")
            out_sizes = out_shapes[:, 0] * out_shapes[:, 1]
            out_offsets = _exclusive_cumsum(out_sizes)
            out_size = int(out_sizes.sum())
            scatter = _copy_tables(
                *_block_scatter(e[g], nrr, st["sr"], st["sc"], row_start[st["ir"][g], b],
                                col_start[st["ic"][g], b], out_offsets[b], out_shapes[b, 1],
                                y_off[g], st["soff"], E[g]),
                y_size, out_size,
            )
            if int(scatter[0]["volume"].astype(np.int64).sum()) != out_size:
                raise AssertionError("dense -> blocks tables do not cover the blocks")
            m.zero_out = False
            m.in_len = dense_size
            m.out_offsets, m.out_shapes = out_offsets, out_shapes
        m.gather, m.scatter = gather, scatter
        m.x_size, m.out_size = x_size, out_size
        m.M, m.N, m.K = st["M"], E, st["K"]
        m.u_off, m.x_off, m.u_host = st["u_off"], x_off, st["u_host"]
        m.device = None
        return m

    def _to_dense_map(self):
        """The blocks -> dense map of this tensor's layout."""
        reps = self._row_reps + self._col_reps
        nrr = self._nrr
        key = ("to_dense", type(self).__name__, self._irreps_key(), self._layout_key(),
               self._signature.tobytes(), nrr)
        m = _MAP_CACHE.get(key)
        if m is not None:
            _MAP_CACHE.move_to_end(key)
            return m
        st = self._dense_structure(
            self._irreps_key(), nrr, tuple(bool(s) for s in self._signature),
            tuple(int(b) for b in self._block_irreps), True,
        )
        degs, e, E, dstride, base, dense_size = self._dense_geometry(reps, st)
        m = self._dense_map(st, degs, e, E, dstride, base, dense_size, nrr, None,
                            to_dense=True, tensor=self)
        _MAP_CACHE[key] = m
        if len(_MAP_CACHE) > _MAP_CACHE_SIZE:
            _MAP_CACHE.popitem(last=False)
        return m

    def _tomatrix(self):
        """lie_group_symmetric_tensor.py:969-1109 on the device (dense result
        copied to the host)."""
        if self._nblocks == 0:
            return np.zeros(self.matrix_shape)
        out = self._to_dense_map().run(self._data)
        return out.cpu().numpy().reshape(self.matrix_shape)
