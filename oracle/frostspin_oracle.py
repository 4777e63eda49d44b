"""CPU oracle for the frostspin_b200 hot path -- TEST INFRASTRUCTURE ONLY.

A plain numpy restatement of the reference algorithms (ogauthe/frostspin 1.0.0)
for the block-sparse abelian (U(1) / Z2) symmetric tensor: representation
fusion, block extraction, permute, matmul, diagonal products, reductions,
the greedy multiplet-aware truncation and truncated SVD / eigh, plus the C4v
classical CTMRG iteration used by the Ising workload.  Each function cites the
reference file:line it follows.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import
this module, and only as the checker.  The device package never imports it.

Parity pin: the functions here are checked against golden fixtures written by
the reference itself (tests/golden/make_golden.py imports frostspin from the
read-only reference tree and stores its outputs) in tests/test_oracle.py.
"""

import numpy as np

# ------------------------------------------------------------------ data model


class OTensor:
    """Minimal abelian symmetric tensor: reps, signature, sorted block irreps and
    C-order numpy blocks (symmetric_tensor.py:245-261)."""

    def __init__(self, row_reps, col_reps, blocks, block_irreps, signature):
        self.row_reps = tuple(np.asarray(r, dtype=np.int8) for r in row_reps)
        self.col_reps = tuple(np.asarray(c, dtype=np.int8) for c in col_reps)
        self.blocks = [np.ascontiguousarray(b, dtype=np.float64) for b in blocks]
        self.block_irreps = np.asarray(block_irreps, dtype=np.int8)
        self.signature = np.asarray(signature, dtype=bool)
        self.nrr = len(self.row_reps)
        self.ndim = self.nrr + len(self.col_reps)
        self.shape = tuple(r.size for r in self.row_reps + self.col_reps)

    def row_irreps(self):
        return combine_u1(self.row_reps, self.signature[: self.nrr])

    def col_irreps(self):
        return combine_u1(self.col_reps, ~self.signature[self.nrr :])


def combine_u1(reps, signature):
    """Fused irreps of a leg group, int8 arithmetic with wraparound
    (u1_symmetric_tensor.py:8-19, :36-40): Kronecker sum of (1-2s)*rep."""
    signature = np.asarray(signature, dtype=bool)
    out = (np.int8(1) - np.int8(2) * signature[0].astype(np.int8)) * np.asarray(
        reps[0], dtype=np.int8
    )
    for r, s in zip(reps[1:], signature[1:], strict=True):
        rs = (np.int8(1) - np.int8(2) * np.int8(s)) * np.asarray(r, dtype=np.int8)
        out = (out[:, None] + rs[None, :]).ravel()
    return out.astype(np.int8)


def validated_signature(signature, nrr, ncr):
    """symmetric_tensor.py:24-32."""
    if signature is None:
        s = np.zeros(nrr + ncr, dtype=bool)
        s[nrr:] = True
        return s
    s = np.ascontiguousarray(signature, dtype=bool)
    if s.shape != (nrr + ncr,):
        raise ValueError("Invalid signature shape")
    return s


def get_block_sizes(row_reps, col_reps, signature):
    """abelian_symmetric_tensor.py:287-318."""
    nrr = len(row_reps)
    rt = combine_u1(row_reps, signature[:nrr])
    ct = combine_u1(col_reps, ~np.asarray(signature[nrr:], dtype=bool))
    ri, rs = np.unique(rt, return_counts=True)
    ci, cs = np.unique(ct, return_counts=True)
    a, b = (ri[:, None] == ci).nonzero()
    return ri[a], np.array([rs[a], cs[b]]).T.copy()


def from_array(arr, row_reps, col_reps, signature=None):
    """symmetric_tensor.py:118-146 with abelian _blocks_from_dense
    (abelian_symmetric_tensor.py:19-40, :361-371)."""
    sig = validated_signature(signature, len(row_reps), len(col_reps))
    t = OTensor(row_reps, col_reps, [], [], sig)
    ri = t.row_irreps()
    ci = t.col_irreps()
    m = np.asarray(arr, dtype=np.float64).reshape(ri.size, ci.size)
    blocks, irreps = [], []
    for q in np.unique(ri):
        cols = np.flatnonzero(ci == q)
        if cols.size:
            rows = np.flatnonzero(ri == q)
            blocks.append(m[np.ix_(rows, cols)])
            irreps.append(q)
    t.blocks = blocks
    t.block_irreps = np.array(irreps, dtype=np.int8)
    return t


def toarray(t, *, as_matrix=False):
    """abelian_symmetric_tensor.py:63-75, :373-383 (blocks -> dense)."""
    ri = t.row_irreps()
    ci = t.col_irreps()
    m = np.zeros((ri.size, ci.size))
    for q, b in zip(t.block_irreps, t.blocks, strict=True):
        m[np.ix_(np.flatnonzero(ri == q), np.flatnonzero(ci == q))] = b
    return m if as_matrix else m.reshape(t.shape)


def random(row_reps, col_reps, signature=None, *, rng):
    """symmetric_tensor.py:514-546: uniform [-0.5, 0.5) blocks in block order."""
    sig = validated_signature(signature, len(row_reps), len(col_reps))
    irreps, shapes = get_block_sizes(row_reps, col_reps, sig)
    blocks = [rng.random(tuple(sh)) - 0.5 for sh in shapes]
    return OTensor(row_reps, col_reps, blocks, irreps, sig)


# --------------------------------------------------------------------- permute


def _block_positions(irreps):
    """For each fused index: rank among indices with the same irrep (C order),
    abelian_symmetric_tensor.py:78-100 (_numpy_get_indices)."""
    order = np.argsort(irreps, kind="mergesort")
    s = irreps[order]
    start = np.r_[0, np.flatnonzero(s[1:] != s[:-1]) + 1]
    grp_start = np.repeat(start, np.diff(np.r_[start, s.size]))
    pos = np.empty(irreps.size, dtype=np.int64)
    pos[order] = np.arange(s.size) - grp_start
    return pos


def permute(t, row_axes, col_axes):
    """symmetric_tensor.py:166-212 + abelian_symmetric_tensor.py:395-430, with
    the scatter of _numba_abelian_transpose (:103-250) written with numpy:
    old flat row/col -> per-leg index (// strides % dims) -> new flat index
    (* new strides) -> divmod by new column count -> new block/row/col."""
    row_axes, col_axes = tuple(row_axes), tuple(col_axes)
    axes = row_axes + col_axes
    if sorted(axes) != list(range(t.ndim)):
        raise ValueError("Axes do not match tensor")
    if row_axes == tuple(range(t.nrr)) and col_axes == tuple(range(t.nrr, t.ndim)):
        return t
    if row_axes == tuple(range(t.nrr, t.ndim)) and col_axes == tuple(range(t.nrr)):
        return transpose(t)
    reps = list(t.row_reps + t.col_reps)
    sig = t.signature[list(axes)]
    nrr = len(row_axes)
    new_reps = [reps[a] for a in axes]
    nri = combine_u1(new_reps[:nrr], sig[:nrr])
    nci = combine_u1(new_reps[nrr:], ~sig[nrr:])
    shape = np.array(t.shape, dtype=np.int64)
    ndim = t.ndim
    new_strides = np.ones(ndim, dtype=np.int64)
    for i in range(ndim - 1, 0, -1):
        new_strides[axes[i - 1]] = new_strides[axes[i]] * shape[axes[i]]
    row_shape = shape[: t.nrr]
    col_shape = shape[t.nrr :]
    rstr = np.r_[np.cumprod(row_shape[::-1])[::-1][1:], 1]
    cstr = np.r_[np.cumprod(col_shape[::-1])[::-1][1:], 1]

    uq = np.unique(nri)
    rpos = _block_positions(nri)
    cpos = _block_positions(nci)
    rblk = np.searchsorted(uq, nri)
    ncols_per = np.array([(nci == q).sum() for q in uq], dtype=np.int64)
    nrows_per = np.array([(nri == q).sum() for q in uq], dtype=np.int64)
    new_blocks = [np.zeros((nrows_per[i], ncols_per[i])) for i in range(uq.size)]
    ncs = nci.size
    ori_all = t.row_irreps()
    oci_all = t.col_irreps()
    for q, b in zip(t.block_irreps, t.blocks, strict=True):
        rows = np.flatnonzero(ori_all == q)
        cols = np.flatnonzero(oci_all == q)
        ori = ((rows[:, None] // rstr) % row_shape * new_strides[: t.nrr]).sum(axis=1)
        oci = ((cols[:, None] // cstr) % col_shape * new_strides[t.nrr :]).sum(axis=1)
        flat = ori[:, None] + oci[None, :]
        nr, nc = np.divmod(flat, ncs)
        bi = rblk[nr]
        for i in np.unique(bi):
            sel = bi == i
            new_blocks[i][rpos[nr[sel]], cpos[nc[sel]]] = b[sel]
    blocks, irreps = [], []
    for i, q in enumerate(uq):
        if new_blocks[i].size:
            blocks.append(new_blocks[i])
            irreps.append(q)
    return OTensor(new_reps[:nrr], new_reps[nrr:], blocks, irreps, sig)


def transpose(t):
    """symmetric_tensor.py:569-576 + abelian_symmetric_tensor.py:385-393."""
    conj = (-t.block_irreps.astype(np.int8)).astype(np.int8)
    so = np.argsort(conj, kind="stable")
    blocks = [t.blocks[i].T.copy() for i in so]
    s = t.signature[np.arange(-t.ndim + t.nrr, t.nrr) % t.ndim]
    return OTensor(t.col_reps, t.row_reps, blocks, conj[so], s)


def dagger(t):
    """symmetric_tensor.py:596-609."""
    s = np.empty(t.ndim, dtype=bool)
    s[: t.ndim - t.nrr] = ~t.signature[t.nrr :]
    s[t.ndim - t.nrr :] = ~t.signature[: t.nrr]
    return OTensor(
        t.col_reps, t.row_reps, [b.T.copy() for b in t.blocks], t.block_irreps, s
    )


# ---------------------------------------------------------------- linear algebra


def matmul(a, b):
    """symmetric_tensor.py:453-489: merge-join over sorted block irreps."""
    i1 = i2 = 0
    blocks, irreps = [], []
    while i1 < len(a.blocks) and i2 < len(b.blocks):
        if a.block_irreps[i1] == b.block_irreps[i2]:
            blocks.append(a.blocks[i1] @ b.blocks[i2])
            irreps.append(a.block_irreps[i1])
            i1 += 1
            i2 += 1
        elif a.block_irreps[i1] < b.block_irreps[i2]:
            i1 += 1
        else:
            i2 += 1
    sig = np.r_[a.signature[: a.nrr], b.signature[b.nrr :]]
    return OTensor(a.row_reps, b.col_reps, blocks, irreps, sig)


def norm(t):
    """symmetric_tensor.py:624-631 (abelian irrep dimension 1)."""
    return float(np.sqrt(sum(float((b * b).sum()) for b in t.blocks)))


def trace(t):
    """symmetric_tensor.py:633-637."""
    return float(sum(np.trace(b) for b in t.blocks))


def full_contract(a, b):
    """symmetric_tensor.py:639-653."""
    x = 0.0
    for i1, q in enumerate(a.block_irreps):
        j = np.flatnonzero(b.block_irreps == q)
        if j.size:
            x += float(np.einsum("ij,ji->", a.blocks[i1], b.blocks[j[0]]))
    return x


def diagonal_mul(t, diag_blocks, diag_irreps, *, left=False):
    """symmetric_tensor.py:1189-1248."""
    diag_irreps = np.asarray(diag_irreps, dtype=np.int8)
    if (left and t.signature[0]) or (not left and not t.signature[-1]):
        conj = (-diag_irreps).astype(np.int8)
        so = conj.argsort(kind="stable")
        diag_irreps = conj[so]
        diag_blocks = [diag_blocks[i] for i in so]
    blocks, irreps = [], []
    i1 = i2 = 0
    while i1 < len(t.blocks) and i2 < len(diag_blocks):
        if t.block_irreps[i1] == diag_irreps[i2]:
            d = np.asarray(diag_blocks[i2])
            blocks.append(t.blocks[i1] * (d[:, None] if left else d))
            irreps.append(t.block_irreps[i1])
            i1 += 1
            i2 += 1
        elif t.block_irreps[i1] < diag_irreps[i2]:
            i1 += 1
        else:
            i2 += 1
    return OTensor(t.row_reps, t.col_reps, blocks, irreps, t.signature)


def find_block_cuts(block_values, cut_target, *, dims=None, atol=0.0, rtol=None,
                    degen_ratio=1.0):
    """svd_tools.py:7-74: greedy selection of the largest values across blocks,
    keeping values >= degen_ratio * current together (multiplets); each value of
    block i counts dims[i]; stop at cut_target or below atol + rtol * max."""
    vals = [np.asarray(v, dtype=np.float64) for v in block_values]
    n = len(vals)
    dims = np.ones(n, dtype=np.int64) if dims is None else np.asarray(dims, dtype=np.int64)
    if rtol is None:
        rtol = sum(len(v) for v in vals) * np.finfo(np.float64).eps
    cutoff = float(atol + rtol * max(v[0] for v in vals))
    degen_ratio = float(degen_ratio)
    cur = np.array([v[0] for v in vals], dtype=np.float64)
    cuts = np.zeros(n, dtype=np.int64)
    kept = 0
    bi = int(cur.argmax())
    while cur[bi] > cutoff and kept < cut_target:
        c = degen_ratio * cur[bi]
        while cur[bi] >= c:
            cuts[bi] += 1
            kept += dims[bi]
            cur[bi] = vals[bi][cuts[bi]] if cuts[bi] < vals[bi].size else -1.0
            bi = int(cur.argmax())
    return cuts


def singlet():
    """abelian_symmetric_tensor.py:48-50."""
    return np.zeros(1, dtype=np.int8)


def irrep_dims(irreps):
    """Abelian irreps are one-dimensional."""
    return np.ones(len(irreps), dtype=np.int64)


def init_representation(degen, irreps):
    """abelian_symmetric_tensor.py:254-261."""
    return np.repeat(np.asarray(irreps, dtype=np.int8), np.asarray(degen, dtype=np.int64))


def truncated_eigh(t, nvals, *, atol=0.0, rtol=None, degen_ratio=1.0):
    """symmetric_tensor.py:1087-1132 -> _sparse_eig (:1250-1434) on the dense
    path (every block small): per block eigh, sort by |value| descending, keep
    nvals//dim+1 per block, find_block_cuts, truncate.  Missing allowed blocks
    contribute a zero value that find_block_cuts then drops."""
    irreps, shapes = get_block_sizes(t.row_reps, t.col_reps, t.signature)
    vals, vecs, absv = [], [], []
    for q, sh in zip(irreps, shapes, strict=True):
        k = nvals + 1
        j = np.flatnonzero(t.block_irreps == q)
        if j.size:
            w, v = np.linalg.eigh(t.blocks[j[0]])
            a = np.abs(w)
            so = a.argsort()[: -k - 1 : -1]
            vals.append(w[so])
            vecs.append(v[:, so])
            absv.append(a[so])
        else:
            vals.append(np.zeros(0))
            vecs.append(np.zeros((sh[0], 0)))
            absv.append(np.zeros(1))
    cuts = find_block_cuts(absv, nvals, atol=atol, rtol=rtol, degen_ratio=degen_ratio)
    keep = np.flatnonzero(cuts)
    s_blocks = [vals[i][: cuts[i]] for i in keep]
    s_irreps = irreps[keep]
    mid = init_representation(cuts[keep], s_irreps)
    usign = np.r_[t.signature[: t.nrr], True]
    u = OTensor(t.row_reps, (mid,), [vecs[i][:, : cuts[i]] for i in keep], s_irreps, usign)
    return s_blocks, s_irreps, u


def truncated_svd(t, cut, *, atol=0.0, rtol=None, degen_ratio=1.0):
    """symmetric_tensor.py:835-877 on the dense path (robust_svd per block,
    svd_tools.py:116-151), then find_block_cuts and truncate_values_vectors
    (:1436-1477)."""
    us, ss, vs = [], [], []
    for b in t.blocks:
        u, s, v = np.linalg.svd(b, full_matrices=False)
        us.append(u)
        ss.append(s)
        vs.append(v)
    cuts = find_block_cuts(ss, cut, atol=atol, rtol=rtol, degen_ratio=degen_ratio)
    keep = np.flatnonzero(cuts)
    irr = t.block_irreps[keep]
    mid = init_representation(cuts[keep], irr)
    U = OTensor(
        t.row_reps, (mid,), [us[i][:, : cuts[i]] for i in keep], irr,
        np.r_[t.signature[: t.nrr], True],
    )
    V = OTensor(
        (mid,), t.col_reps, [vs[i][: cuts[i]] for i in keep], irr,
        np.r_[False, t.signature[t.nrr :]],
    )
    return U, [ss[i][: cuts[i]] for i in keep], irr, V


def add(a, b):
    """symmetric_tensor.py:326-352 (merge of possibly missing blocks)."""
    blocks, irreps = [], []
    i1 = i2 = 0
    while i1 < len(a.blocks) and i2 < len(b.blocks):
        if a.block_irreps[i1] == b.block_irreps[i2]:
            blocks.append(a.blocks[i1] + b.blocks[i2])
            irreps.append(a.block_irreps[i1])
            i1 += 1
            i2 += 1
        elif a.block_irreps[i1] < b.block_irreps[i2]:
            blocks.append(a.blocks[i1].copy())
            irreps.append(a.block_irreps[i1])
            i1 += 1
        else:
            blocks.append(b.blocks[i2].copy())
            irreps.append(b.block_irreps[i2])
            i2 += 1
    blocks += [x.copy() for x in a.blocks[i1:]] + [x.copy() for x in b.blocks[i2:]]
    irreps += list(a.block_irreps[i1:]) + list(b.block_irreps[i2:])
    return OTensor(a.row_reps, a.col_reps, blocks, irreps, a.signature)


def scale(t, x):
    return OTensor(t.row_reps, t.col_reps, [x * b for b in t.blocks], t.block_irreps,
                   t.signature)


# --------------------------------------------------- C4v classical CTMRG (Ising)


def ising_c4v_iteration(s_blocks, s_irreps, T, a, a2, chi):
    """One iteration of examples/ising_classical_ctmrg.py:115-204 (iterate_ctm)
    on oracle tensors; s is the corner spectrum as (blocks, irreps)."""
    Tp = permute(T, (0, 1), (2,))
    matC = diagonal_mul(Tp, s_blocks, s_irreps)
    matC = matmul(matC, T)
    matC = permute(matC, (1, 2), (0, 3))
    matC = matmul(a2, matC)
    matC = permute(matC, (0, 2), (1, 3))
    ns_blocks, ns_irreps, U = truncated_eigh(matC, chi)
    nrm = np.sqrt(sum(float((b * b).sum()) for b in ns_blocks))
    ns_blocks = [b / nrm for b in ns_blocks]
    newT = permute(U, (1,), (0, 2))
    newT = matmul(Tp, newT)
    newT = permute(newT, (1, 2), (0, 3))
    newT = matmul(a, newT)
    newT = permute(newT, (0, 2), (1, 3))
    newT = matmul(dagger(U), newT)
    newT = scale(newT, 1.0 / norm(newT))
    return ns_blocks, ns_irreps, newT


def ising_tensors(beta):
    """Site tensors of examples/ising_classical_ctmrg.py:44-64 and :362-384 in the
    Z2 basis (irreps {-128, 0}); returns (a, a2, a0_diag, magn_op_diag)."""
    import scipy.linalg as lg

    d = 2
    h = -2 * np.eye(2) + 1
    sq_bw = lg.sqrtm(np.exp(-beta * h)).real
    delta = np.zeros((d,) * 4)
    delta[0, 0, 0, 0] = delta[1, 1, 1, 1] = 1
    a0 = np.einsum("abcd,ai,bj,ck,dl->ijkl", delta, sq_bw, sq_bw, sq_bw, sq_bw)
    mop = delta.copy()
    mop[1, 1, 1, 1] = -1
    mop = np.einsum("abcd,ai,bj,ck,dl->ijkl", mop, sq_bw, sq_bw, sq_bw, sq_bw)
    K = np.array([[-1.0, 1.0], [1.0, 1.0]]) / np.sqrt(2)
    a0d = np.einsum("abcd,ai,bj,ck,dl->ijkl", a0, K, K, K, K)
    mopd = np.einsum("abcd,ai,bj,ck,dl->ijkl", mop, K, K, K, K)
    rep = np.array([-128, 0], dtype=np.int8)
    siga = np.array([False, False, True, True])
    a = from_array(a0d, (rep, rep), (rep, rep), siga)
    siga2 = np.array([False, True, True, True])
    a2 = OTensor(a.row_reps, a.col_reps, a.blocks, a.block_irreps, siga2)
    return a, a2, a0d, mopd


def ising_initial_env(chi, rng):
    """Seeded initial Z2 corner spectrum and symmetric edge tensor,
    examples/ising_classical_ctmrg.py:386-412."""
    d0o = chi // 2
    d0e = chi // 2
    s_odd = rng.normal(size=(d0o,))
    s_odd = s_odd[np.abs(s_odd).argsort()[::-1]] / np.linalg.norm(s_odd)
    s_even = rng.normal(size=(d0e,))
    s_even = s_even[np.abs(s_even).argsort()[::-1]] / np.linalg.norm(s_even)
    corner = np.array([-128] * d0o + [0] * d0e, dtype=np.int8)
    bond = np.array([-128, 0], dtype=np.int8)
    sigT = np.array([False, False, True])
    T0 = random((corner,), (bond, corner), sigT, rng=rng)
    temp = OTensor(T0.row_reps, T0.col_reps, T0.blocks, T0.block_irreps, [1, 0, 0])
    temp = permute(temp, (2,), (1, 0))
    T0 = add(T0, temp)
    T0 = scale(T0, 1.0 / norm(T0))
    return [s_odd, s_even], np.array([-128, 0], dtype=np.int8), T0


def ising_energy_per_bond(s_blocks, s_irreps, T, a0d, mopd):
    """Energy per bond -<s s> from the two-site environment
    (examples/ising_classical_ctmrg.py:254-304, :344-350; the example's energy is
    per site = 2 bonds)."""
    Tp = permute(T, (0, 1), (2,))
    env = diagonal_mul(Tp, s_blocks, s_irreps)
    env = matmul(env, permute(env, (0,), (1, 2)))
    env = matmul(Tp, permute(env, (0,), (1, 2, 3)))
    left = permute(env, (1, 2, 3), (0, 4))
    right = permute(env, (4, 0), (1, 2, 3))
    env2 = toarray(matmul(left, right))
    nr = np.einsum("abcdef,bgdc,afeg->", env2, a0d, a0d)
    sdsr = np.einsum("abcdef,bgdc,afeg->", env2, mopd, mopd)
    return -sdsr / nr


def ising_correlation_length(T):
    """xi = -1/ln|lambda_2/lambda_1| of the C4v edge transfer operator
    M[(l1, l2), (r1, r2)] = sum_p T[l1, p, r1] T[l2, p, r2] (dense, FP64).
    The reference example (examples/ising_classical_ctmrg.py) computes no
    correlation length; this restates the definition used for the Z2 Ising
    benchmark, applied to the reference's own edge tensors."""
    Td = toarray(T)
    chi = Td.shape[0]
    M = np.einsum("apc,bpd->abcd", Td, Td).reshape(chi * chi, -1)
    lam = np.linalg.eigvals(M)
    lam = lam[np.argsort(-np.abs(lam), kind="stable")]
    return -1.0 / np.log(abs(lam[1]) / abs(lam[0])), lam[:4]
