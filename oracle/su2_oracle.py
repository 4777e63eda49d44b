"""CPU oracle for SU(2) symmetric tensors -- TEST INFRASTRUCTURE ONLY.

A plain numpy restatement of the reference's SU(2) tensor (ogauthe/frostspin
1.0.0: symmetric_tensor/su2_symmetric_tensor.py, lie_group_symmetric_tensor.py,
non_abelian_symmetric_tensor.py, groups/su2_clebsch_gordan.py), following the
reference's own loop structure: Clebsch-Gordan coefficients from sympy,
fusion trees with depth on the first leg, per-simple-block isometries, and a
permute that loops over simple blocks, gathering each old sector through a
reshape/transpose view, multiplying by the isometry and scattering into the
new blocks.  Function names and signatures match frostspin_oracle (the abelian
oracle), so the CTMRG oracle runs on either.

Only tests/ and bench.py's CPU-baseline leg may import this module, as the
checker and the timed CPU baseline; the device package never imports it.
Parity pin: tests/test_oracle_su2.py checks it against fixtures written by the
reference itself (tests/golden/su2.npz, tests/golden/simple_update_su2.npz).
"""

import functools

import numpy as np

from .frostspin_oracle import find_block_cuts, validated_signature  # noqa: F401

SYMMETRY = "SU2"


# ------------------------------------------------------------- group data


@functools.lru_cache(maxsize=None)
def cg_tensor(d1, d2, d3):
    """<s1 m1; s2 m2 | s3 m3> as p[i1, i2, i3], irreps labelled by dimension,
    basis by decreasing S_z, evaluated exactly by sympy and cast to float64
    (groups/su2_clebsch_gordan.py:8-32)."""
    import sympy as sp
    from sympy.physics.quantum.cg import CG

    p = np.zeros((d1, d2, d3))
    s1, s2, s3 = (sp.Rational(d - 1, 2) for d in (d1, d2, d3))
    for i1 in range(d1):
        for i2 in range(d2):
            i3 = i1 + i2 - (d1 + d2 - d3 - 1) // 2
            if 0 <= i3 < d3:
                p[i1, i2, i3] = float(CG(s1, s1 - i1, s2, s2 - i2, s3, s3 - i3).doit())
    p.setflags(write=False)
    return p


def singlet():
    return np.ones((2, 1), dtype=np.int64)


def irrep_dims(irreps):
    return np.asarray(irreps, dtype=np.int64)


def elementary_combine(deg1, irr1, deg2, irr2):
    """su2_symmetric_tensor.py:109-119."""
    degen = np.zeros(int(irr1[-1]) + int(irr2[-1]) - 1, dtype=np.int64)
    for d1, i1 in zip(deg1, irr1, strict=True):
        for d2, i2 in zip(deg2, irr2, strict=True):
            for irr in range(abs(int(i1) - int(i2)), int(i1) + int(i2) - 1, 2):
                degen[irr] += int(d1) * int(d2)
    nz = degen.nonzero()[0]
    return degen[nz], nz + 1


def combine(reps):
    """su2_symmetric_tensor.py:122-127."""
    degen, irreps = reps[0][0], reps[0][1]
    for r in reps[1:]:
        degen, irreps = elementary_combine(degen, irreps, r[0], r[1])
    return np.array([degen, irreps], dtype=np.int64)


def init_representation(degen, irreps):
    """non_abelian_symmetric_tensor.py:16-26."""
    return np.array([np.asarray(degen, dtype=np.int64), np.asarray(irreps, dtype=np.int64)])


def fusion_tensor(rep1, rep2, s1, s2, max_irrep=2**30):
    """compute_fusion_tensor, su2_symmetric_tensor.py:12-106."""
    degen, irreps = elementary_combine(rep1[0], rep1[1], rep2[0], rep2[1])
    keep = irreps <= max_irrep
    degen, irreps = degen[keep], irreps[keep]
    proj = np.zeros((int(rep1[0] @ rep1[1]), int(rep2[0] @ rep2[1]), int(degen @ irreps)))
    if irreps.size == 0:
        return np.zeros((2, 0), dtype=np.int64), proj
    start = {}
    n = 0
    for d, irr in zip(degen, irreps, strict=True):
        start[int(irr)] = n
        n += int(d * irr)
    sh1 = 0
    for d1, irr1 in rep1.T:
        sh2 = 0
        for d2, irr2 in rep2.T:
            for irr3 in range(abs(irr1 - irr2) + 1, min(irr1 + irr2, max_irrep + 1), 2):
                p = cg_tensor(int(irr1), int(irr2), int(irr3))
                if s1:  # spin reversal on the first input
                    p = p[::-1] * (np.arange(irr1 % 2, irr1 + irr1 % 2) % 2 * 2 - 1)[:, None, None]
                if s2:
                    p = p[:, ::-1] * (np.arange(irr2 % 2, irr2 + irr2 % 2) % 2 * 2 - 1)[None, :, None]
                for i3 in range(d1 * d2):
                    i1, i2 = divmod(i3, d2)
                    c = start[irr3] + i3 * irr3
                    proj[sh1 + i1 * irr1 : sh1 + (i1 + 1) * irr1,
                         sh2 + i2 * irr2 : sh2 + (i2 + 1) * irr2, c : c + irr3] = p
                start[irr3] += d1 * d2 * irr3
            sh2 += d2 * irr2
        sh1 += d1 * irr1
    return np.array([degen, irreps], dtype=np.int64), proj


def cg_tree(reps, signature, target_max=None):
    """compute_clebsch_gordan_tree, su2_symmetric_tensor.py:178-218."""
    reps = list(reps)
    signature = list(signature)
    if len(reps) == 1:
        reps.append(singlet())
        signature.append(False)
    n = len(reps)
    max_irrep = 2**30 if target_max is None else target_max + sum(int(r[1, -1]) for r in reps[2:]) - n + 2
    nr, p = fusion_tensor(reps[0], reps[1], signature[0], signature[1], max_irrep)
    if nr.size == 0:
        return nr, np.zeros((p.shape[0] * p.shape[1], 0))
    proj = p
    for i in range(2, n):
        max_irrep -= int(reps[i][1, -1]) - 1
        nr, p = fusion_tensor(nr, reps[i], False, signature[i], max_irrep)
        if nr.size == 0:
            return nr, np.zeros((p.shape[0] * p.shape[1], 0))
        proj = proj.reshape(-1, p.shape[0]) @ p.reshape(p.shape[0], -1)
    return nr, proj.reshape(-1, p.shape[2])


@functools.lru_cache(maxsize=None)
def elementary_trees(irreps, signature, target):
    """sliced_elementary_trees for one elementary block
    (lie_group_symmetric_tensor.py:365-430): irrep -> (*dims, mult, dim)."""
    reps = [np.array([[1], [i]], dtype=np.int64) for i in irreps]
    rep, tree = cg_tree(reps, signature, max(target) if target else None)
    out = {}
    k = 0
    for deg, irr in rep.T:
        w = int(deg * irr)
        if int(irr) in target:
            out[int(irr)] = tree[:, k : k + w].reshape(*irreps, int(deg), int(irr))
        k += w
    return out


# ------------------------------------------------------------------ tensors


class OTensor:
    """SU(2) tensor: 2 x n int reps, sorted int block irreps, numpy blocks."""

    def __init__(self, row_reps, col_reps, blocks, block_irreps, signature):
        self.row_reps = tuple(np.asarray(r, dtype=np.int64) for r in row_reps)
        self.col_reps = tuple(np.asarray(c, dtype=np.int64) for c in col_reps)
        self.blocks = [np.ascontiguousarray(b, dtype=np.float64) for b in blocks]
        self.block_irreps = np.asarray(block_irreps, dtype=np.int64)
        self.signature = np.asarray(signature, dtype=bool)
        self.nrr = len(self.row_reps)
        self.ndim = self.nrr + len(self.col_reps)
        self.shape = tuple(int(r[0] @ r[1]) for r in self.row_reps + self.col_reps)


def get_block_sizes(row_reps, col_reps, signature):
    """non_abelian_symmetric_tensor.py:36-67."""
    r = combine(row_reps) if len(row_reps) > 1 else np.asarray(row_reps[0])
    c = combine(col_reps) if len(col_reps) > 1 else np.asarray(col_reps[0])
    ri, ci = (r[1, :, None] == c[1]).nonzero()
    return r[1, ri].astype(np.int64), np.stack([r[0, ri], c[0, ci]], axis=1).reshape(-1, 2)


def random(row_reps, col_reps, signature=None, *, rng):
    signature = validated_signature(signature, len(row_reps), len(col_reps))
    irr, shapes = get_block_sizes(row_reps, col_reps, signature)
    return OTensor(row_reps, col_reps, [rng.random(tuple(s)) - 0.5 for s in shapes], irr,
                   signature)


def _ele_multiplicities(reps, target):
    """Per elementary block (C order over legs): multiplicity of each target."""
    lists = [r[1] for r in reps]
    grids = np.indices([len(x) for x in lists]).reshape(len(lists), -1).T
    out = np.zeros((grids.shape[0], len(target)), dtype=np.int64)
    for i, g in enumerate(grids):
        ele = [np.array([[1], [lists[k][g[k]]]]) for k in range(len(lists))]
        deg, irr = combine(ele) if len(ele) > 1 else ele[0]
        for dd, q in zip(deg, irr, strict=True):
            j = np.searchsorted(target, q)
            if j < len(target) and target[j] == q:
                out[i, j] = dd
    return grids, out


def _ext(reps, grid):
    return np.array([reps[k][0, grid[k]] for k in range(len(reps))], dtype=np.int64)


def _pair_projector(rt, ct):
    d = rt.shape[-1]
    sr, sc = rt.shape[-2], ct.shape[-2]
    p = rt.reshape(-1, d) @ ct.reshape(-1, d).T
    rd = p.shape[0] // sr
    cd = p.shape[1] // sc
    return p.reshape(rd, sr, cd, sc).swapaxes(1, 2).reshape(rd * cd, sr * sc)


def _sector_starts(edeg, mult):
    """Row (or column) offset of every (elementary block, irrep) inside its
    matrix block: cumulative ext * multiplicity (lie_group_symmetric_tensor.py
    :802-805)."""
    cum = np.cumsum(edeg[:, None] * mult, axis=0)
    return cum - edeg[:, None] * mult, cum[-1] if cum.size else np.zeros(mult.shape[1], int)


def from_array(arr, row_reps, col_reps, signature=None):
    """_blocks_from_dense, lie_group_symmetric_tensor.py:856-967."""
    signature = validated_signature(signature, len(row_reps), len(col_reps))
    reps = tuple(row_reps) + tuple(col_reps)
    nrr = len(row_reps)
    irr, shapes = get_block_sizes(row_reps, col_reps, signature)
    blocks = [np.zeros(tuple(s)) for s in shapes]
    rg, rm = _ele_multiplicities(row_reps, irr)
    cg, cm = _ele_multiplicities(col_reps, irr)
    re_ = np.array([_ext(row_reps, g).prod() for g in rg])
    ce_ = np.array([_ext(col_reps, g).prod() for g in cg])
    rs, _ = _sector_starts(re_, rm)
    cs, _ = _sector_starts(ce_, cm)
    shifts = [np.concatenate([[0], np.cumsum(r[0] * r[1])]) for r in reps]
    for i, g in enumerate(rg):
        for j, h in enumerate(cg):
            shared = (rm[i] > 0) & (cm[j] > 0)
            if not shared.any():
                continue
            gg = np.concatenate([g, h])
            e = _ext(reps, gg)
            dims = np.array([reps[k][1, gg[k]] for k in range(len(reps))])
            sl = tuple(slice(shifts[k][gg[k]], shifts[k][gg[k] + 1]) for k in range(len(reps)))
            n = len(reps)
            data = np.asarray(arr)[sl].reshape(np.stack([e, dims], axis=1).ravel())
            data = data.transpose(tuple(range(1, 2 * n, 2)) + tuple(range(0, 2 * n, 2)))
            data = data.reshape(dims.prod(), e.prod())
            rt = elementary_trees(tuple(int(x) for x in dims[:nrr]),
                                  tuple(bool(s) for s in signature[:nrr]), tuple(int(q) for q in irr))
            ct = elementary_trees(tuple(int(x) for x in dims[nrr:]),
                                  tuple(bool(s) for s in ~signature[nrr:]), tuple(int(q) for q in irr))
            for b in np.flatnonzero(shared):
                q = int(irr[b])
                sr, sc = rm[i, b], cm[j, b]
                blk = _pair_projector(rt[q], ct[q]).T @ data / q
                blk = blk.reshape(sr, sc, re_[i], ce_[j]).swapaxes(1, 2).reshape(sr * re_[i], sc * ce_[j])
                blocks[b][rs[i, b] : rs[i, b] + sr * re_[i], cs[j, b] : cs[j, b] + sc * ce_[j]] = blk
    return OTensor(row_reps, col_reps, blocks, irr, signature)


def toarray(t, *, as_matrix=False):
    """_tomatrix, lie_group_symmetric_tensor.py:969-1109."""
    reps = t.row_reps + t.col_reps
    nrr = t.nrr
    out = np.zeros(t.shape)
    rg, rm = _ele_multiplicities(t.row_reps, t.block_irreps)
    cg, cm = _ele_multiplicities(t.col_reps, t.block_irreps)
    re_ = np.array([_ext(t.row_reps, g).prod() for g in rg])
    ce_ = np.array([_ext(t.col_reps, g).prod() for g in cg])
    rs, _ = _sector_starts(re_, rm)
    cs, _ = _sector_starts(ce_, cm)
    shifts = [np.concatenate([[0], np.cumsum(r[0] * r[1])]) for r in reps]
    n = len(reps)
    for i, g in enumerate(rg):
        for j, h in enumerate(cg):
            shared = (rm[i] > 0) & (cm[j] > 0)
            if not shared.any():
                continue
            gg = np.concatenate([g, h])
            e = _ext(reps, gg)
            dims = np.array([reps[k][1, gg[k]] for k in range(n)])
            rt = elementary_trees(tuple(int(x) for x in dims[:nrr]),
                                  tuple(bool(s) for s in t.signature[:nrr]),
                                  tuple(int(q) for q in t.block_irreps))
            ct = elementary_trees(tuple(int(x) for x in dims[nrr:]),
                                  tuple(bool(s) for s in ~t.signature[nrr:]),
                                  tuple(int(q) for q in t.block_irreps))
            dense = np.zeros((dims.prod(), e.prod()))
            for b in np.flatnonzero(shared):
                q = int(t.block_irreps[b])
                sr, sc = rm[i, b], cm[j, b]
                blk = t.blocks[b][rs[i, b] : rs[i, b] + sr * re_[i], cs[j, b] : cs[j, b] + sc * ce_[j]]
                blk = blk.reshape(sr, re_[i], sc, ce_[j]).swapaxes(1, 2).reshape(sr * sc, -1)
                dense += _pair_projector(rt[q], ct[q]) @ blk
            dense = dense.reshape(np.concatenate([dims, e]))
            inv = np.argsort(tuple(range(1, 2 * n, 2)) + tuple(range(0, 2 * n, 2)))
            dense = dense.transpose(inv).reshape(tuple(dims * e))
            sl = tuple(slice(shifts[k][gg[k]], shifts[k][gg[k] + 1]) for k in range(n))
            out[sl] = dense.reshape(np.stack([e, dims], axis=1).ravel()).reshape(
                tuple(e * dims))
    if as_matrix:
        return out.reshape(int(np.prod(t.shape[:nrr])), -1)
    return out


@functools.lru_cache(maxsize=None)
def _isometry(irreps, nrr, axes, new_nrr, signature):
    """overlap_cg_trees, lie_group_symmetric_tensor.py:657-733, for one simple
    block; rows: output sectors (increasing irrep), columns: input sectors."""
    n = len(irreps)
    sig = np.array(signature)
    out_irr = tuple(irreps[a] for a in axes)
    out_sig = sig[list(axes)]
    ri = combine([np.array([[1], [i]]) for i in irreps[:nrr]])[1]
    ci = combine([np.array([[1], [i]]) for i in irreps[nrr:]])[1]
    ro = combine([np.array([[1], [i]]) for i in out_irr[:new_nrr]])[1]
    co = combine([np.array([[1], [i]]) for i in out_irr[new_nrr:]])[1]
    sin = tuple(int(q) for q in np.intersect1d(ri, ci))
    sout = tuple(int(q) for q in np.intersect1d(ro, co))
    tri = elementary_trees(irreps[:nrr], tuple(bool(s) for s in sig[:nrr]), sin)
    tci = elementary_trees(irreps[nrr:], tuple(bool(s) for s in ~sig[nrr:]), sin)
    tro = elementary_trees(out_irr[:new_nrr], tuple(bool(s) for s in out_sig[:new_nrr]), sout)
    tco = elementary_trees(out_irr[new_nrr:], tuple(bool(s) for s in ~out_sig[new_nrr:]), sout)
    ax = np.array(axes)
    perm = list((ax >= nrr) + ax) + [nrr, n + 1]
    cols = []
    for q in sin:
        rt, ct = tri[q], tci[q]
        p = rt.reshape(-1, q) @ ct.reshape(-1, q).T
        p = p.reshape(rt.shape[:-1] + ct.shape[:-1]).transpose(perm)
        p = p.reshape(-1, rt.shape[-2] * ct.shape[-2])
        rows = []
        for qo in sout:
            iso = _pair_projector(tro[qo], tco[qo]).T @ p
            iso[np.abs(iso) < 1e-14] = 0
            rows.append(iso / qo)
        cols.append(np.vstack(rows))
    return sin, sout, np.hstack(cols)


def permute(t, row_axes, col_axes):
    """symmetric_tensor.py:166-212 -> _lie_permute_data,
    lie_group_symmetric_tensor.py:735-835 and permute_simple_block :96-212."""
    axes = tuple(row_axes) + tuple(col_axes)
    new_nrr = len(row_axes)
    nrr = t.nrr
    n = t.ndim
    if axes == tuple(range(n)) and new_nrr == nrr:
        return t
    reps = t.row_reps + t.col_reps
    sig = t.signature
    new_reps = [reps[a] for a in axes]
    new_sig = sig[list(axes)]
    irr_out, shapes_out = get_block_sizes(new_reps[:new_nrr], new_reps[new_nrr:], new_sig)
    irr_in, _ = get_block_sizes(reps[:nrr], reps[nrr:], sig)
    out = [np.zeros(tuple(s)) for s in shapes_out]
    rg, rm = _ele_multiplicities(reps[:nrr], irr_in)
    cg, cm = _ele_multiplicities(reps[nrr:], irr_in)
    org, orm = _ele_multiplicities(new_reps[:new_nrr], irr_out)
    ocg, ocm = _ele_multiplicities(new_reps[new_nrr:], irr_out)
    re_ = np.array([_ext(reps[:nrr], g).prod() for g in rg])
    ce_ = np.array([_ext(reps[nrr:], g).prod() for g in cg])
    ore = np.array([_ext(new_reps[:new_nrr], g).prod() for g in org])
    oce = np.array([_ext(new_reps[new_nrr:], g).prod() for g in ocg])
    rs, _ = _sector_starts(re_, rm)
    cs, _ = _sector_starts(ce_, cm)
    ors, _ = _sector_starts(ore, orm)
    ocs, _ = _sector_starts(oce, ocm)
    nseg = [r.shape[1] for r in reps]
    present = {int(q): b for q, b in zip(t.block_irreps, t.blocks, strict=True)}
    data_perm = [0, nrr + 1] + [a + 1 + (a >= nrr) for a in axes]
    sigt = tuple(bool(s) for s in sig)
    for i, g in enumerate(rg):
        for j, h in enumerate(cg):
            if not ((rm[i] > 0) & (cm[j] > 0)).any():
                continue
            gg = np.concatenate([g, h])
            e = _ext(reps, gg)
            irreps = tuple(int(reps[k][1, gg[k]]) for k in range(n))
            sin, sout, U = _isometry(irreps, nrr, axes, new_nrr, sigt)
            E = int(e.prod())
            parts = []
            for q in sin:
                b = int(np.searchsorted(irr_in, q))
                sr, sc = rm[i, b], cm[j, b]
                if q not in present:
                    parts.append(np.zeros((sr * sc, E)))
                    continue
                blk = present[q][rs[i, b] : rs[i, b] + sr * re_[i], cs[j, b] : cs[j, b] + sc * ce_[j]]
                blk = blk.reshape((sr, *e[:nrr], sc, *e[nrr:])).transpose(data_perm)
                parts.append(blk.reshape(sr * sc, E))
            Y = U @ np.vstack(parts)
            go = np.array([gg[a] for a in axes])
            io = np.ravel_multi_index(go[:new_nrr], [nseg[a] for a in axes[:new_nrr]])
            jo = np.ravel_multi_index(go[new_nrr:], [nseg[a] for a in axes[new_nrr:]])
            k = 0
            for q in sout:
                b = int(np.searchsorted(irr_out, q))
                sr, sc = orm[io, b], ocm[jo, b]
                blk = Y[k : k + sr * sc].reshape(sr, sc, ore[io], oce[jo]).swapaxes(1, 2)
                out[b][ors[io, b] : ors[io, b] + sr * ore[io],
                       ocs[jo, b] : ocs[jo, b] + sc * oce[jo]] = blk.reshape(sr * ore[io], -1)
                k += sr * sc
    return OTensor(new_reps[:new_nrr], new_reps[new_nrr:], out, irr_out, new_sig)


def transpose(t):
    """symmetric_tensor.py:569-576 with _transpose_data = a permute
    (lie_group_symmetric_tensor.py:1111-1114)."""
    n, nrr = t.ndim, t.nrr
    return permute(t, tuple(range(nrr, n)), tuple(range(nrr)))


def dagger(t):
    """symmetric_tensor.py:596-609."""
    s = np.concatenate([~t.signature[t.nrr :], ~t.signature[: t.nrr]])
    return OTensor(t.col_reps, t.row_reps, [b.T for b in t.blocks], t.block_irreps, s)


def matmul(a, b):
    """symmetric_tensor.py:453-489."""
    common, i1, i2 = np.intersect1d(a.block_irreps, b.block_irreps, return_indices=True)
    sig = np.concatenate([a.signature[: a.nrr], b.signature[b.nrr :]])
    return OTensor(a.row_reps, b.col_reps, [a.blocks[x] @ b.blocks[y] for x, y in zip(i1, i2)],
                   common, sig)


def norm(t):
    """symmetric_tensor.py:624-631."""
    return float(np.sqrt(sum(q * np.vdot(b, b) for q, b in zip(t.block_irreps, t.blocks))))


def trace(t):
    return float(sum(q * np.trace(b) for q, b in zip(t.block_irreps, t.blocks)))


def full_contract(a, b):
    common, i1, i2 = np.intersect1d(a.block_irreps, b.block_irreps, return_indices=True)
    return float(sum(q * np.vdot(a.blocks[x].T, b.blocks[y])
                     for q, x, y in zip(common, i1, i2)))


def scale(t, x):
    return OTensor(t.row_reps, t.col_reps, [x * b for b in t.blocks], t.block_irreps,
                   t.signature)
