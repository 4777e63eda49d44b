"""CPU oracle for O(2) symmetric tensors -- TEST INFRASTRUCTURE ONLY.

A plain numpy restatement of the reference's O(2) tensor (ogauthe/frostspin
1.0.0, symmetric_tensor/o2_symmetric_tensor.py).  O(2) = U(1) x| Z2.  Irrep -1
is the odd and irrep 0 the even one-dimensional irrep; irrep n > 0 is the
two-dimensional irrep pairing U(1) charges +n and -n.  A tensor stores its 0odd
and 0even blocks and the U(1) blocks of charge n > 0.  The charge -n blocks
follow from the Sz reflection; the U(1) charge-0 block is an orthogonal mix of
the 0odd and 0even blocks.  The permute here goes through U(1): cast, abelian
permute (frostspin_oracle), cast back.  The reference's own tests pin that
equivalence at 1e-15 (tests/test_o2_tensor.py:20-33).

Only tests/ may import this module, as the checker; the device package never
imports it.  Parity pin: tests/test_oracle_o2.py checks it against fixtures
written by the reference itself (tests/golden/o2.npz).
"""

import numpy as np

from . import frostspin_oracle as u1
from .frostspin_oracle import validated_signature

SYMMETRY = "O2"


# ------------------------------------------------------------- group data
def singlet():
    """o2_symmetric_tensor.py:620-622."""
    return np.array([[1], [0]])


def irrep_dims(irreps):
    """o2_symmetric_tensor.py:628-630: 1 for 0odd / 0even, 2 for n > 0."""
    return 1 + (np.asarray(irreps) > 0).astype(np.int64)


def representation_dimension(rep):
    """o2_symmetric_tensor.py:56-58."""
    rep = np.asarray(rep)
    return int((rep[0] * irrep_dims(rep[1])).sum())


def elementary_combine(deg1, irr1, deg2, irr2):
    """o2_symmetric_tensor.py:20-53: 0o x 0o = 0e x 0e = 0e, 0e x 0o = 0o,
    0 x n = n, n x n = 0o + 0e + 2n, n x m = |n - m| + (n + m)."""
    nmax = max(int(irr1[-1]), 0) + max(int(irr2[-1]), 0)
    degen = np.zeros(nmax + 2, dtype=np.int64)
    for d1, a in zip(deg1, irr1, strict=True):
        for d2, b in zip(deg2, irr2, strict=True):
            d = int(d1) * int(d2)
            if a < 1 and b < 1:
                degen[(a + b + 1) % 2] += d
            elif a < 1:
                degen[b + 1] += d
            elif b < 1:
                degen[a + 1] += d
            elif a == b:
                degen[0] += d
                degen[1] += d
                degen[2 * a + 1] += d
            else:
                degen[a + b + 1] += d
                degen[abs(a - b) + 1] += d
    irreps = np.arange(-1, nmax + 1)
    nz = degen.nonzero()[0]
    return degen[nz], irreps[nz]


def combine(reps):
    """o2_symmetric_tensor.py:12-17 (signature plays no role: every O(2)
    representation is self-conjugate)."""
    deg, irr = np.asarray(reps[0][0]), np.asarray(reps[0][1])
    for r in reps[1:]:
        deg, irr = elementary_combine(deg, irr, r[0], r[1])
    return np.array([deg, irr])


def rep_to_u1(rep):
    """o2_symmetric_tensor.py:61-89: 0odd states, 0even states, then for each
    n > 0 its degeneracy at charge +n followed by the same at -n."""
    out = []
    for d, irr in zip(rep[0], rep[1], strict=True):
        if irr < 1:
            out += [0] * int(d)
        else:
            out += [int(irr)] * int(d) + [-int(irr)] * int(d)
    return np.array(out, dtype=np.int8)


def reflection_perm_sign(rep):
    """o2_symmetric_tensor.py:92-115: the Sz reflection on one leg maps the +n
    copy of a state to its -n copy and back; 0odd states get sign -1, and for
    odd n the -n -> +n direction gets sign -1."""
    dim = representation_dimension(rep)
    perm = np.arange(dim)
    sign = np.ones(dim, dtype=np.int64)
    k = 0
    for d, irr in zip(rep[0], rep[1], strict=True):
        d = int(d)
        if irr < 1:
            if irr == -1:
                sign[k : k + d] = -1
            k += d
            continue
        perm[k : k + d] = np.arange(k + d, k + 2 * d)
        perm[k + d : k + 2 * d] = np.arange(k, k + d)
        if irr % 2:
            sign[k + d : k + 2 * d] = -1
        k += 2 * d
    return perm, sign


def _reflect_states(o2_reps, states):
    """Reflected fused index and sign of each fused index in ``states``."""
    dims = [representation_dimension(r) for r in o2_reps]
    digits = np.unravel_index(np.asarray(states, dtype=np.int64), dims)
    refl = np.zeros(len(states), dtype=np.int64)
    sign = np.ones(len(states), dtype=np.int64)
    stride = 1
    for leg in range(len(o2_reps) - 1, -1, -1):
        p, s = reflection_perm_sign(o2_reps[leg])
        refl += p[digits[leg]] * stride
        sign *= s[digits[leg]]
        stride *= dims[leg]
    return refl, sign


def b0_arrays(o2_reps, sz_values):
    """o2_symmetric_tensor.py:118-266: projectors of the U(1) charge-0 states
    onto 0odd and 0even.  Fixed points of the reflection come first (sign -1:
    odd, +1: even), in state order; then one odd and one even combination per
    doublet (a, b = reflected a, a < b): (a - sign_b b) / sqrt 2 and
    (a + sign_b b) / sqrt 2.  Returns (ocoeff, ocols, ecoeff, ecols), each
    (rows, 2), columns being positions among the charge-0 states."""
    sz0 = np.flatnonzero(np.asarray(sz_values) == 0)
    refl, sign = _reflect_states(o2_reps, sz0)
    pos = {int(s): i for i, s in enumerate(sz0)}
    ofix, efix, doublets = [], [], []
    for i, (s, r) in enumerate(zip(sz0, refl, strict=True)):
        if s == r:
            (ofix if sign[i] < 0 else efix).append(i)
        elif s < r:
            doublets.append(i)
    c = 1.0 / np.sqrt(2)
    ocols = [[i, i] for i in ofix]
    ocoeff = [[1.0, 0.0] for _ in ofix]
    ecols = [[i, i] for i in efix]
    ecoeff = [[1.0, 0.0] for _ in efix]
    for i in doublets:
        j = pos[int(refl[i])]
        ocols.append([i, j])
        ocoeff.append([c, -sign[j] / np.sqrt(2)])
        ecols.append([i, j])
        ecoeff.append([c, sign[j] / np.sqrt(2)])

    def arr(x, dt):
        return np.array(x, dtype=dt).reshape(-1, 2)

    return arr(ocoeff, float), arr(ocols, np.int64), arr(ecoeff, float), arr(ecols, np.int64)


# ------------------------------------------------------------- tensors
class OTensor:
    def __init__(self, row_reps, col_reps, blocks, block_irreps, signature):
        self.row_reps = tuple(np.asarray(r, dtype=np.int64) for r in row_reps)
        self.col_reps = tuple(np.asarray(c, dtype=np.int64) for c in col_reps)
        self.blocks = [np.ascontiguousarray(b, dtype=np.float64) for b in blocks]
        self.block_irreps = np.asarray(block_irreps, dtype=np.int64)
        self.signature = np.asarray(signature, dtype=bool)
        self.nrr = len(self.row_reps)
        self.ndim = self.nrr + len(self.col_reps)
        self.shape = tuple(representation_dimension(r) for r in self.row_reps + self.col_reps)


def get_block_sizes(row_reps, col_reps, signature):
    """non_abelian_symmetric_tensor.py:36-67."""
    rt = combine(row_reps)
    ct = combine(col_reps)
    ri, ci = (rt[1][:, None] == ct[1]).nonzero()
    return rt[1][ri], np.array([rt[0][ri], ct[0][ci]]).T.reshape(-1, 2)


def random(row_reps, col_reps, signature=None, *, rng):
    sig = validated_signature(signature, len(row_reps), len(col_reps))
    irreps, shapes = get_block_sizes(row_reps, col_reps, sig)
    return OTensor(row_reps, col_reps, [rng.random(tuple(s)) - 0.5 for s in shapes], irreps, sig)


def _u1_sz(t):
    rows = u1.combine_u1([rep_to_u1(r) for r in t.row_reps], t.signature[: t.nrr])
    cols = u1.combine_u1([rep_to_u1(r) for r in t.col_reps], ~t.signature[t.nrr :])
    return rows, cols


def _neg_blocks(t):
    """o2_symmetric_tensor.py:798-851 and :327-354: the charge -n U(1) block of
    each stored n > 0 block, refl[rank(r'), rank(c')] = sign_r sign_c b[r, c],
    r' (c') the reflected row (column) state.  Returned for increasing n."""
    rows, cols = _u1_sz(t)
    out = {}
    for n, b in zip(t.block_irreps, t.blocks, strict=True):
        if n < 1:
            continue
        rs = np.flatnonzero(rows == n)
        cs = np.flatnonzero(cols == n)
        rr, rsg = _reflect_states(t.row_reps, rs)
        cr, csg = _reflect_states(t.col_reps, cs)
        rso = rr.argsort().argsort()
        cso = cr.argsort().argsort()
        nb = np.empty_like(b)
        for i in range(rs.size):
            for j in range(cs.size):
                nb[rso[i], cso[j]] = rsg[i] * csg[j] * b[i, j]
        out[int(n)] = nb
    return out


def to_u1(t):
    """o2_symmetric_tensor.py:682-733: charge -n blocks from the reflection,
    charge-0 block merged from 0odd and 0even (:269-288), charge n > 0 blocks
    as stored."""
    rows, cols = _u1_sz(t)
    neg = _neg_blocks(t)
    blocks, irreps = [], []
    for n in sorted(neg, reverse=True):
        blocks.append(neg[n])
        irreps.append(-n)
    irr = list(t.block_irreps)
    if -1 in irr or 0 in irr:
        ro, rocol, re_, recol = b0_arrays(t.row_reps, rows)
        co, cocol, ce, cecol = b0_arrays(t.col_reps, cols)
        b0 = np.zeros((ro.shape[0] + re_.shape[0], co.shape[0] + ce.shape[0]))
        for q, (rc, rcol, cc, ccol) in ((-1, (ro, rocol, co, cocol)), (0, (re_, recol, ce, cecol))):
            if q not in irr:
                continue
            bq = t.blocks[irr.index(q)]
            for i in range(bq.shape[0]):
                for j in range(bq.shape[1]):
                    for k1 in range(2):
                        for k2 in range(2):
                            b0[rcol[i, k1], ccol[j, k2]] += rc[i, k1] * bq[i, j] * cc[j, k2]
        blocks.append(b0)
        irreps.append(0)
    for n, b in zip(t.block_irreps, t.blocks, strict=True):
        if n > 0:
            blocks.append(b)
            irreps.append(n)
    return u1.OTensor([rep_to_u1(r) for r in t.row_reps], [rep_to_u1(r) for r in t.col_reps],
                      blocks, irreps, t.signature)


def from_u1(tu1, row_reps, col_reps):
    """o2_symmetric_tensor.py:650-675, :778-793 and split_b0 (:291-325): keep
    charges n >= 0; the charge-0 block is split into 0odd and 0even.  An empty
    half is dropped."""
    rows, cols = tu1.row_irreps(), tu1.col_irreps()
    blocks, irreps = [], []
    q = list(tu1.block_irreps)
    if 0 in q:
        b0 = tu1.blocks[q.index(0)]
        ro, rocol, re_, recol = b0_arrays(row_reps, rows)
        co, cocol, ce, cecol = b0_arrays(col_reps, cols)
        halves = []
        for rc, rcol, cc, ccol in ((ro, rocol, co, cocol), (re_, recol, ce, cecol)):
            h = np.empty((rc.shape[0], cc.shape[0]))
            for i in range(h.shape[0]):
                for j in range(h.shape[1]):
                    v = rc[i, 0] * b0[rcol[i, 0], ccol[j, 0]] * cc[j, 0]
                    v += rc[i, 0] * b0[rcol[i, 0], ccol[j, 1]] * cc[j, 1]
                    v += rc[i, 1] * b0[rcol[i, 1], ccol[j, 0]] * cc[j, 0]
                    v += rc[i, 1] * b0[rcol[i, 1], ccol[j, 1]] * cc[j, 1]
                    h[i, j] = v
            halves.append(h)
        for irr, h in zip((-1, 0), halves, strict=True):
            if h.size:
                blocks.append(h)
                irreps.append(irr)
    for n, b in zip(tu1.block_irreps, tu1.blocks, strict=True):
        if n > 0:
            blocks.append(b)
            irreps.append(int(n))
    return OTensor(row_reps, col_reps, blocks, irreps, tu1.signature)


def from_array(arr, row_reps, col_reps, signature=None):
    """o2_symmetric_tensor.py:766-776: through the U(1) blocks."""
    sig = validated_signature(signature, len(row_reps), len(col_reps))
    tu1 = u1.from_array(arr, [rep_to_u1(r) for r in row_reps],
                        [rep_to_u1(r) for r in col_reps], sig)
    return from_u1(tu1, row_reps, col_reps)


def toarray(t, *, as_matrix=False):
    """o2_symmetric_tensor.py:795-796."""
    return u1.toarray(to_u1(t), as_matrix=as_matrix)


def permute(t, row_axes, col_axes):
    """The O(2) permute as cast -> abelian permute -> cast back (equal to
    _numba_O2_transpose, o2_symmetric_tensor.py:357-580, :853-936, to
    rounding)."""
    p = u1.permute(to_u1(t), row_axes, col_axes)
    reps = t.row_reps + t.col_reps
    axes = tuple(row_axes) + tuple(col_axes)
    nrr = len(row_axes)
    return from_u1(p, [reps[a] for a in axes[:nrr]], [reps[a] for a in axes[nrr:]])


def transpose(t):
    """o2_symmetric_tensor.py:938-942 with symmetric_tensor.py:569-576: 0odd and
    0even blocks transposed, block n > 0 becomes the transposed charge -n
    block."""
    neg = _neg_blocks(t)
    blocks = []
    for n, b in zip(t.block_irreps, t.blocks, strict=True):
        blocks.append(b.T if n < 1 else neg[int(n)].T)
    s = t.signature[np.arange(-t.ndim + t.nrr, t.nrr) % t.ndim]
    return OTensor(t.col_reps, t.row_reps, blocks, t.block_irreps, s)


def norm(t):
    return float(np.sqrt(sum(d * (b**2).sum() for d, b in
                             zip(irrep_dims(t.block_irreps), t.blocks, strict=True))))


def dagger(t):
    """symmetric_tensor.py:596-609 (blocks transposed, signature flipped)."""
    s = np.empty(t.ndim, dtype=bool)
    s[: t.ndim - t.nrr] = ~t.signature[t.nrr :]
    s[t.ndim - t.nrr :] = ~t.signature[: t.nrr]
    return OTensor(t.col_reps, t.row_reps, [b.T for b in t.blocks], t.block_irreps, s)


def matmul(a, b):
    """symmetric_tensor.py:453-489: products of the blocks with equal irreps."""
    common, i1, i2 = np.intersect1d(a.block_irreps, b.block_irreps, return_indices=True)
    sig = np.r_[a.signature[: a.nrr], b.signature[b.nrr :]]
    return OTensor(a.row_reps, b.col_reps, [a.blocks[i] @ b.blocks[j] for i, j in
                                            zip(i1, i2, strict=True)], common, sig)


def su2_leg_to_o2(rep):
    """su2_symmetric_tensor.py:272-304 for one leg: O(2) representation, the
    state order taking the leg to O(2) order and the sign of every state."""
    sz, lab, sign = [], [], []
    for d, irr in zip(rep[0], rep[1], strict=True):
        irr = int(irr)
        for _ in range(int(d)):
            for s in range(irr - 1, -irr, -2):
                lb = abs(s)
                if s == 0 and irr % 4 == 3:
                    lb = -1
                flip = s < 0 and s % 4 == ((irr + 1) % 4 if irr % 2 else (irr - 1) % 4)
                sz.append(s)
                lab.append(lb)
                sign.append(-1.0 if flip else 1.0)
    order = sorted(range(len(sz)), key=lambda i: (lab[i], -sz[i], i))
    irreps = sorted(set(lab))
    degen = [lab.count(q) // (2 if q > 0 else 1) for q in irreps]
    return np.array([degen, irreps]), np.array(order), np.array(sign)


def from_su2_dense(arr, su2_row_reps, su2_col_reps, signature):
    """SU2SymmetricTensor.toO2 (su2_symmetric_tensor.py:249-318) from the dense
    SU(2) tensor: legs reordered and signed, then from_array."""
    reps = []
    for ax, r in enumerate(list(su2_row_reps) + list(su2_col_reps)):
        rep, order, sign = su2_leg_to_o2(r)
        reps.append(rep)
        arr = np.moveaxis(np.moveaxis(arr, ax, 0)[order] * sign[order].reshape(
            (-1,) + (1,) * (arr.ndim - 1)), 0, ax)
    nrr = len(su2_row_reps)
    return from_array(arr, reps[:nrr], reps[nrr:], signature)
