"""O(2) symmetric device tensor.

Mirrors frostspin/symmetric_tensor/o2_symmetric_tensor.py (O2SymmetricTensor,
:584-945).  O(2) = U(1) x| Z2: irrep -1 is the odd and irrep 0 the even
one-dimensional irrep, irrep n > 0 the two-dimensional irrep pairing U(1)
charges +n and -n.  Representations are 2 x n int arrays [degen; irrep] with
irreps sorted; a tensor stores its 0odd and 0even blocks and the U(1) blocks of
charge n > 0 (rows and columns in U(1) fused order).

The data plane is the U(1) one.  The cast to U(1) (charge -n blocks from the
Sz reflection, the charge-0 block merged from 0odd and 0even) and the cast
back (charges n >= 0 kept, charge 0 split) are each one launch of
fs_o2_recombine over host-built row / column tables; the permute is cast ->
abelian permute (fs_abelian_permute) -> cast back.  The reference's own tests
pin that equivalence at 1e-15 (tests/test_o2_tensor.py:20-33).
"""

from collections import OrderedDict

import numpy as np

from .. import _native
from .. import device as dev
from .. import instrument
from .lie_group_symmetric_tensor import NonAbelianSymmetricTensor
from .tools import symmetric_tensor_types
from .u1_symmetric_tensor import U1SymmetricTensor, combine_u1

_PLAN_CACHE = OrderedDict()
_PLAN_CACHE_SIZE = 256
_MAX_BLOCKS_PER_CALL = 65535


def plan_cache_clear():
    _PLAN_CACHE.clear()


# ------------------------------------------------------------ group data
def elementary_combine(degen1, irreps1, degen2, irreps2):
    """o2_symmetric_tensor.py:20-53: 0o x 0o = 0e x 0e = 0e, 0e x 0o = 0o,
    0 x n = n, n x n = 0o + 0e + 2n, n x m = |n - m| + (n + m)."""
    degen1 = np.asarray(degen1, dtype=np.int64)
    degen2 = np.asarray(degen2, dtype=np.int64)
    irreps1 = np.asarray(irreps1, dtype=np.int64)
    irreps2 = np.asarray(irreps2, dtype=np.int64)
    nmax = max(int(irreps1[-1]), 0) + max(int(irreps2[-1]), 0)
    degen = np.zeros(nmax + 2, dtype=np.int64)
    a, b = np.meshgrid(irreps1, irreps2, indexing="ij")
    d = np.outer(degen1, degen2)
    zz = (a < 1) & (b < 1)       # 0 x 0: parity product
    np.add.at(degen, ((a + b + 1) % 2)[zz], d[zz])
    zn = (a < 1) & (b >= 1)      # 0 x n = n
    np.add.at(degen, (b + 1)[zn], d[zn])
    nz = (a >= 1) & (b < 1)      # n x 0 = n
    np.add.at(degen, (a + 1)[nz], d[nz])
    same = (a >= 1) & (a == b)   # n x n = 0o + 0e + 2n
    degen[0] += d[same].sum()
    degen[1] += d[same].sum()
    np.add.at(degen, (2 * a + 1)[same], d[same])
    diff = (a >= 1) & (b >= 1) & (a != b)   # n x m = |n - m| + (n + m)
    np.add.at(degen, (a + b + 1)[diff], d[diff])
    np.add.at(degen, (np.abs(a - b) + 1)[diff], d[diff])
    irreps = np.arange(-1, nmax + 1)
    keep = degen.nonzero()[0]
    return degen[keep], irreps[keep]


def combine_o2(reps):
    """o2_symmetric_tensor.py:12-17."""
    degen = np.asarray(reps[0][0], dtype=np.int64)
    irreps = np.asarray(reps[0][1], dtype=np.int64)
    for r in reps[1:]:
        degen, irreps = elementary_combine(degen, irreps, r[0], r[1])
    return np.array([degen, irreps], dtype=np.int64)


def rep_to_u1(rep):
    """o2_symmetric_tensor.py:61-89: the 0odd states, the 0even states, then for
    every n > 0 its degeneracy at charge +n followed by the same at -n."""
    rep = np.asarray(rep, dtype=np.int64)
    parts = []
    for d, irr in zip(rep[0], rep[1], strict=True):
        if irr < 1:
            parts.append(np.zeros(d, dtype=np.int8))
        else:
            parts.append(np.full(d, irr, dtype=np.int8))
            parts.append(np.full(d, -irr, dtype=np.int8))
    return np.concatenate(parts) if parts else np.zeros(0, dtype=np.int8)


def reflection_perm_sign(rep):
    """o2_symmetric_tensor.py:92-115: the Sz reflection of one leg swaps the +n
    and -n copies of every n > 0 state; 0odd states and, for odd n, the -n -> +n
    direction carry a sign -1."""
    rep = np.asarray(rep, dtype=np.int64)
    dim = int((rep[0] * (1 + (rep[1] > 0))).sum())
    perm = np.arange(dim, dtype=np.int64)
    sign = np.ones(dim, dtype=np.int64)
    k = 0
    for d, irr in zip(rep[0], rep[1], strict=True):
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


def reflect_states(o2_reps, states):
    """Sz-reflected fused index and sign of each fused (C-order) index."""
    dims = [int((np.asarray(r)[0] * (1 + (np.asarray(r)[1] > 0))).sum()) for r in o2_reps]
    states = np.asarray(states, dtype=np.int64)
    refl = np.zeros(states.size, dtype=np.int64)
    sign = np.ones(states.size, dtype=np.int64)
    if states.size == 0:
        return refl, sign
    digits = np.unravel_index(states, dims)
    stride = 1
    for leg in range(len(o2_reps) - 1, -1, -1):
        p, s = reflection_perm_sign(o2_reps[leg])
        refl += p[digits[leg]] * stride
        sign *= s[digits[leg]]
        stride *= dims[leg]
    return refl, sign


def b0_arrays(o2_reps, sz_values):
    """o2_symmetric_tensor.py:118-266: projectors of the U(1) charge-0 states on
    0odd and 0even.  Fixed points of the reflection first, in state order (sign
    -1: odd, +1: even, coefficient 1); then, for every doublet (a, b = reflected
    a, a < b) in order of a, the odd row (a - sign_b b) / sqrt 2 and the even row
    (a + sign_b b) / sqrt 2.  Returns (ocoeff, ocols, ecoeff, ecols), each
    (rows, 2); columns are positions among the charge-0 states."""
    sz0 = np.flatnonzero(np.asarray(sz_values) == 0)
    refl, sign = reflect_states(o2_reps, sz0)
    fixed = sz0 == refl
    ofix = np.flatnonzero(fixed & (sign < 0))
    efix = np.flatnonzero(fixed & (sign > 0))
    dbl = np.flatnonzero(sz0 < refl)
    j = np.searchsorted(sz0, refl[dbl])
    c = 1.0 / np.sqrt(2)
    ocols = np.concatenate([np.stack([ofix, ofix], 1), np.stack([dbl, j], 1)]).reshape(-1, 2)
    ecols = np.concatenate([np.stack([efix, efix], 1), np.stack([dbl, j], 1)]).reshape(-1, 2)
    fo = np.zeros((ofix.size, 2))
    fo[:, 0] = 1.0
    fe = np.zeros((efix.size, 2))
    fe[:, 0] = 1.0
    do = np.stack([np.full(dbl.size, c), -sign[j] / np.sqrt(2)], 1)
    de = np.stack([np.full(dbl.size, c), sign[j] / np.sqrt(2)], 1)
    ocoeff = np.concatenate([fo, do]).reshape(-1, 2)
    ecoeff = np.concatenate([fe, de]).reshape(-1, 2)
    return ocoeff, ocols.astype(np.int64), ecoeff, ecols.astype(np.int64)


def _merge_rows(coeff, cols, n0):
    """Transpose of a charge-0 projector as per-state tables: the one O(2) row
    every charge-0 state belongs to and its coefficient (0 for states the
    projector does not reach)."""
    idx = np.zeros(n0, dtype=np.int64)
    cf = np.zeros(n0)
    rows = np.arange(coeff.shape[0], dtype=np.int64)
    for k in range(2):
        idx[cols[:, k]] = rows
        np.add.at(cf, cols[:, k], coeff[:, k])
    return idx, cf


# --------------------------------------------------------------- tables
class _Recombine:
    """Host tables of one fs_o2_recombine map, their device copies and the
    structure of the output storage."""

    def __init__(self):
        self._blocks = []
        self._index = []
        self._coef = []
        self._n_index = 0
        self._n_coef = 0
        self._pushed = {}
        self.out_len = 0
        self.max_rows = 0
        self.offsets = []
        self.shapes = []
        self.irreps = []
        self.device_tables = None
        self._all_terms = []

    def _push(self, arr, kind):
        key = (kind, id(arr))
        if key in self._pushed:
            return self._pushed[key][0]
        if kind == "i":
            off = self._n_index
            self._index.append(np.asarray(arr, dtype=np.int64))
            self._n_index += arr.size
        else:
            off = self._n_coef
            self._coef.append(np.asarray(arr, dtype=np.float64))
            self._n_coef += arr.size
        self._pushed[key] = (off, arr)
        return off

    @staticmethod
    def strides(shape, trans):
        m, n = int(shape[0]), int(shape[1])
        return (1, m) if trans else (n, 1)

    def term(self, src_off, shape, trans, ridx, cidx, rcoef, ccoef):
        """One source term; ridx / cidx index rows / columns of the logical
        source block of the given shape (validated here)."""
        m, n = int(shape[0]), int(shape[1])
        if ridx.size and (ridx.min() < 0 or ridx.max() >= m):
            raise ValueError("O(2) table row index outside its source block")
        if cidx.size and (cidx.min() < 0 or cidx.max() >= n):
            raise ValueError("O(2) table column index outside its source block")
        if ridx.shape != rcoef.shape or cidx.shape != ccoef.shape:
            raise ValueError("O(2) table index and coefficient lengths differ")
        rs, cs = self.strides(shape, trans)
        return (int(src_off), rs, cs, self._push(ridx, "i"), self._push(cidx, "i"),
                self._push(rcoef, "c"), self._push(ccoef, "c"), m * n, ridx.size, cidx.size)

    def identity(self, src_off, shape, trans):
        m, n = int(shape[0]), int(shape[1])
        return self.term(src_off, shape, trans, np.arange(m), np.arange(n), np.ones(m),
                         np.ones(n))

    def block(self, nrows, ncols, terms, irrep):
        nrows, ncols = int(nrows), int(ncols)
        if len(terms) > _native.FS_O2_MAXTERMS:
            raise ValueError("too many terms for one O(2) block")
        rec = np.zeros((), dtype=_native.O2_BLOCK_DTYPE)
        rec["out_off"] = self.out_len
        rec["nrows"] = nrows
        rec["ncols"] = ncols
        rec["nterms"] = len(terms)
        for t, (src_off, rs, cs, ri, ci, rc, cc, _, nr, nc) in enumerate(terms):
            # the kernel reads nrows row entries and ncols column entries
            if (nr, nc) != (nrows, ncols):
                raise ValueError("O(2) table lengths do not match the output block")
            rec["terms"][t] = (src_off, rs, cs, ri, ci, rc, cc)
        self._blocks.append(rec)
        self._all_terms.append(terms)
        self.offsets.append(self.out_len)
        self.shapes.append((nrows, ncols))
        self.irreps.append(int(irrep))
        self.out_len += nrows * ncols
        self.max_rows = max(self.max_rows, nrows)

    def finish(self, src_len):
        """Freeze the tables; every source term must lie inside the source
        buffer of length src_len."""
        for terms in self._all_terms:
            for src_off, _, _, _, _, _, _, size, _, _ in terms:
                if src_off < 0 or src_off + size > src_len:
                    raise ValueError("O(2) table source block outside the source buffer")
        self.blocks = (np.array(self._blocks, dtype=_native.O2_BLOCK_DTYPE)
                       if self._blocks else np.zeros(0, dtype=_native.O2_BLOCK_DTYPE))
        self.index = np.concatenate(self._index) if self._index else np.zeros(1, np.int64)
        self.coef = np.concatenate(self._coef) if self._coef else np.zeros(1)
        self.offsets = np.asarray(self.offsets, dtype=np.int64)
        self.shapes = np.asarray(self.shapes, dtype=np.int64).reshape(-1, 2)
        del self._pushed, self._index, self._coef, self._blocks, self._all_terms
        return self

    def run(self, src):
        """Apply the map to the device buffer ``src``; returns the output."""
        out = dev.empty_f64(self.out_len)
        if self.blocks.size == 0 or self.out_len == 0:
            return out
        if self.device_tables is None:
            self.device_tables = (dev.upload(self.blocks), dev.upload(self.index),
                                  dev.upload(self.coef))
        d_blocks, d_index, d_coef = self.device_tables
        with instrument.region("o2_recombine", bytes=16.0 * self.out_len):
            for start in range(0, self.blocks.size, _MAX_BLOCKS_PER_CALL):
                cnt = min(_MAX_BLOCKS_PER_CALL, self.blocks.size - start)
                _native.call(
                    "fs_o2_recombine", dev.ptr(src), int(src.numel()), dev.ptr(out),
                    self.out_len, d_blocks.data_ptr() + start * self.blocks.itemsize, cnt,
                    d_index.data_ptr(), d_coef.data_ptr(), self.max_rows, None, dev.stream(),
                )
        return out


def _cached(key, build):
    plan = _PLAN_CACHE.get(key)
    if plan is not None:
        _PLAN_CACHE.move_to_end(key)
        return plan
    plan = build()
    _PLAN_CACHE[key] = plan
    if len(_PLAN_CACHE) > _PLAN_CACHE_SIZE:
        _PLAN_CACHE.popitem(last=False)
    return plan


def _reps_key(reps):
    return tuple(np.asarray(r, dtype=np.int64).tobytes() for r in reps)


def _reflection_tables(row_reps, col_reps, row_sz, col_sz, n, shape):
    """Gather form of _numba_generate_refl_block (o2_symmetric_tensor.py:327-354):
    the charge -n block at (i', j') is sign_r sign_c b[r, c] with r (c) the row
    (column) of the charge n block whose reflection has rank i' (j')."""
    rows = np.flatnonzero(row_sz == n)
    cols = np.flatnonzero(col_sz == n)
    if (rows.size, cols.size) != (int(shape[0]), int(shape[1])):
        raise ValueError("O(2) block shape does not match its representations")
    rr, rsg = reflect_states(row_reps, rows)
    cr, csg = reflect_states(col_reps, cols)
    ir = np.argsort(rr, kind="stable")
    ic = np.argsort(cr, kind="stable")
    return ir, ic, rsg[ir].astype(np.float64), csg[ic].astype(np.float64)


def _to_u1_plan(t):
    """o2_symmetric_tensor.py:682-733: charge -n blocks (increasing charge),
    the charge-0 block when a 0odd or 0even block exists, charge n > 0 blocks."""
    key = ("to_u1", _reps_key(t._row_reps + t._col_reps), t._signature.tobytes(), t._nrr,
           t._block_irreps.tobytes(), t._offsets.tobytes(), t._bshapes.tobytes(), t._trans,
           int(t._data.numel()))

    def build():
        nrr = t._nrr
        row_sz = combine_u1([rep_to_u1(r) for r in t._row_reps], t._signature[:nrr])
        col_sz = combine_u1([rep_to_u1(r) for r in t._col_reps], ~t._signature[nrr:])
        irr = np.asarray(t._block_irreps, dtype=np.int64)
        rc = _Recombine()
        pos = np.flatnonzero(irr > 0)
        for b in pos[::-1]:
            ir, ic, rs, cs = _reflection_tables(t._row_reps, t._col_reps, row_sz, col_sz,
                                                irr[b], t._bshapes[b])
            term = rc.term(t._offsets[b], t._bshapes[b], t._trans, ir, ic, rs, cs)
            rc.block(t._bshapes[b][0], t._bshapes[b][1], [term], -irr[b])
        zero = [b for b in range(irr.size) if irr[b] < 1]
        if zero:
            ro, rocol, re_, recol = b0_arrays(t._row_reps, row_sz)
            co, cocol, ce, cecol = b0_arrays(t._col_reps, col_sz)
            n0r = int((row_sz == 0).sum())
            n0c = int((col_sz == 0).sum())
            terms = []
            for q, (rcf, rcol, ccf, ccol) in ((-1, (ro, rocol, co, cocol)),
                                             (0, (re_, recol, ce, cecol))):
                hit = np.flatnonzero(irr == q)
                if hit.size == 0:
                    continue
                b = int(hit[0])
                if tuple(t._bshapes[b]) != (rcf.shape[0], ccf.shape[0]):
                    raise ValueError("O(2) zero block shape does not match its representations")
                ridx, rcoef = _merge_rows(rcf, rcol, n0r)
                cidx, ccoef = _merge_rows(ccf, ccol, n0c)
                terms.append(rc.term(t._offsets[b], t._bshapes[b], t._trans, ridx, cidx,
                                     rcoef, ccoef))
            rc.block(n0r, n0c, terms, 0)
        for b in pos:
            rc.block(t._bshapes[b][0], t._bshapes[b][1],
                     [rc.identity(t._offsets[b], t._bshapes[b], t._trans)], irr[b])
        return rc.finish(int(t._data.numel()))

    return _cached(key, build)


def _from_u1_plan(tu1, row_reps, col_reps):
    """o2_symmetric_tensor.py:778-793 with split_b0 (:291-325): the charge-0
    block split into 0odd and 0even (each as the four products of the
    projectors, in the reference's order; an empty half is dropped), then the
    charge n > 0 blocks."""
    key = ("from_u1", _reps_key(list(row_reps) + list(col_reps)),
           tuple(np.asarray(r, dtype=np.int8).tobytes() for r in tu1._row_reps + tu1._col_reps),
           tu1._signature.tobytes(), tu1._nrr, tu1._block_irreps.tobytes(),
           tu1._offsets.tobytes(), tu1._bshapes.tobytes(), tu1._trans, int(tu1._data.numel()))

    def build():
        irr = np.asarray(tu1._block_irreps, dtype=np.int64)
        rc = _Recombine()
        hit = np.flatnonzero(irr == 0)
        if hit.size:
            b = int(hit[0])
            row_sz = tu1.get_row_representation()
            col_sz = tu1.get_column_representation()
            ro, rocol, re_, recol = b0_arrays(row_reps, row_sz)
            co, cocol, ce, cecol = b0_arrays(col_reps, col_sz)
            if tuple(tu1._bshapes[b]) != (ro.shape[0] + re_.shape[0], co.shape[0] + ce.shape[0]):
                raise ValueError("U(1) charge-0 block does not match the O(2) representations")
            for q, (rcf, rcol, ccf, ccol) in ((-1, (ro, rocol, co, cocol)),
                                             (0, (re_, recol, ce, cecol))):
                if rcf.shape[0] == 0 or ccf.shape[0] == 0:
                    continue
                rows = [np.ascontiguousarray(rcol[:, k]) for k in range(2)]
                cols = [np.ascontiguousarray(ccol[:, k]) for k in range(2)]
                rcs = [np.ascontiguousarray(rcf[:, k]) for k in range(2)]
                ccs = [np.ascontiguousarray(ccf[:, k]) for k in range(2)]
                terms = [rc.term(tu1._offsets[b], tu1._bshapes[b], tu1._trans, rows[k1],
                                 cols[k2], rcs[k1], ccs[k2])
                         for k1 in range(2) for k2 in range(2)]
                rc.block(rcf.shape[0], ccf.shape[0], terms, q)
        for b in np.flatnonzero(irr > 0):
            rc.block(tu1._bshapes[b][0], tu1._bshapes[b][1],
                     [rc.identity(tu1._offsets[b], tu1._bshapes[b], tu1._trans)], irr[b])
        return rc.finish(int(tu1._data.numel()))

    return _cached(key, build)


def _transpose_plan(t):
    """o2_symmetric_tensor.py:938-942: 0odd / 0even blocks as they are, block
    n > 0 replaced by the charge -n block; all written in C order of the
    current logical shape, read back transposed (storage flag)."""
    key = ("transpose", _reps_key(t._row_reps + t._col_reps), t._signature.tobytes(), t._nrr,
           t._block_irreps.tobytes(), t._offsets.tobytes(), t._bshapes.tobytes(), t._trans,
           int(t._data.numel()))

    def build():
        nrr = t._nrr
        row_sz = combine_u1([rep_to_u1(r) for r in t._row_reps], t._signature[:nrr])
        col_sz = combine_u1([rep_to_u1(r) for r in t._col_reps], ~t._signature[nrr:])
        rc = _Recombine()
        for b, q in enumerate(np.asarray(t._block_irreps, dtype=np.int64)):
            sh = t._bshapes[b]
            if q < 1:
                term = rc.identity(t._offsets[b], sh, t._trans)
            else:
                ir, ic, rs, cs = _reflection_tables(t._row_reps, t._col_reps, row_sz, col_sz,
                                                    q, sh)
                term = rc.term(t._offsets[b], sh, t._trans, ir, ic, rs, cs)
            rc.block(sh[0], sh[1], [term], q)
        return rc.finish(int(t._data.numel()))

    return _cached(key, build)


# ---------------------------------------------------------------- class
class O2SymmetricTensor(NonAbelianSymmetricTensor):
    """o2_symmetric_tensor.py:584-945."""

    _symmetry = "O2"

    @staticmethod
    def singlet():
        return np.array([[1], [0]])

    @staticmethod
    def representation_dimension(rep):
        rep = np.asarray(rep)
        return int((rep[0] * (1 + (rep[1] > 0))).sum())

    @staticmethod
    def irrep_dimension(irrep):
        return 1 + int(irrep > 0)

    @staticmethod
    def combine_representations(reps, _signature):
        if len(reps) > 1:
            return combine_o2(reps)
        return np.asarray(reps[0], dtype=np.int64)

    @staticmethod
    def conjugate_irrep(irr):
        return irr

    @staticmethod
    def conjugate_representation(rep):
        return rep

    # ------------------------------------------------------------- casts
    @classmethod
    def from_U1(cls, tu1, row_reps, col_reps):
        """o2_symmetric_tensor.py:649-675: the U(1) tensor must carry the O(2)
        representations cast to U(1); charge -n blocks are not read."""
        row_reps = tuple(np.asarray(r, dtype=np.int64) for r in row_reps)
        col_reps = tuple(np.asarray(r, dtype=np.int64) for r in col_reps)
        if tu1.n_row_reps != len(row_reps) or len(tu1.col_reps) != len(col_reps):
            raise ValueError("U(1) tensor does not match the O(2) representations")
        for r, ru1 in zip(row_reps + col_reps, tu1.row_reps + tu1.col_reps, strict=True):
            if not np.array_equal(rep_to_u1(r), ru1):
                raise ValueError("U(1) tensor does not match the O(2) representations")
        plan = _from_u1_plan(tu1, row_reps, col_reps)
        data = plan.run(tu1.data)
        return cls._from_storage(row_reps, col_reps, data, plan.offsets, plan.shapes,
                                 np.asarray(plan.irreps, dtype=np.int64), tu1.signature)

    def toabelian(self):
        return self.toU1()

    def toO2(self):
        return self

    def toU1(self):
        """o2_symmetric_tensor.py:682-733, on the device."""
        plan = _to_u1_plan(self)
        data = plan.run(self._data)
        return U1SymmetricTensor._from_storage(
            [rep_to_u1(r) for r in self._row_reps], [rep_to_u1(r) for r in self._col_reps],
            data, plan.offsets, plan.shapes, np.asarray(plan.irreps, dtype=np.int8),
            self._signature,
        )

    def update_signature(self, sign_update):
        """o2_symmetric_tensor.py:735-744: every O(2) representation is
        self-conjugate and the coefficients follow the U(1) convention, so only
        the signature changes."""
        up = np.asarray(sign_update, dtype=bool)
        if up.shape != (self._ndim,):
            raise ValueError("sign_update shape does not match the tensor")
        self._signature = self._signature ^ up

    # -------------------------------------------------------- data hooks
    @classmethod
    def _blocks_from_dense(cls, arr, row_reps, col_reps, signature):
        """o2_symmetric_tensor.py:766-776: U(1) blocks first, then the split of
        the charge-0 block."""
        row_reps = tuple(np.asarray(r, dtype=np.int64) for r in row_reps)
        col_reps = tuple(np.asarray(r, dtype=np.int64) for r in col_reps)
        tu1 = U1SymmetricTensor.from_array(arr, [rep_to_u1(r) for r in row_reps],
                                           [rep_to_u1(r) for r in col_reps], signature)
        return cls.from_U1(tu1, row_reps, col_reps)

    def _tomatrix(self):
        """o2_symmetric_tensor.py:795-796."""
        return self.toU1()._tomatrix()

    def _permute_data(self, axes, nrr):
        """o2_symmetric_tensor.py:853-936 as cast -> abelian permute -> cast back."""
        tu1 = self.toU1()
        p = tu1.permute(axes[:nrr], axes[nrr:])
        reps = self._row_reps + self._col_reps
        plan = _from_u1_plan(p, [reps[a] for a in axes[:nrr]], [reps[a] for a in axes[nrr:]])
        return (plan.run(p.data), plan.offsets, plan.shapes,
                np.asarray(plan.irreps, dtype=np.int64))

    def _transpose_data(self):
        """o2_symmetric_tensor.py:938-942."""
        plan = _transpose_plan(self)
        data = plan.run(self._data)
        return (data, plan.offsets, plan.shapes[:, ::-1].copy(),
                np.asarray(plan.irreps, dtype=np.int64), True)


symmetric_tensor_types["O2"] = O2SymmetricTensor
