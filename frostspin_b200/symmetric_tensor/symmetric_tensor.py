"""Device SymmetricTensor: the reference's group-agnostic block-matrix API with
block data resident in B200 HBM.

Mirrors frostspin/symmetric_tensor/symmetric_tensor.py:35-1477.  A tensor is a
matrix (legs split into row and column legs) stored as one dense block per
allowed irrep, blocks sorted by irrep.  Storage here is one contiguous float64
device buffer per tensor with per-block element offsets; ``blocks`` returns
torch views into it.  A tensor may hold all of its blocks transposed (F-order,
flag ``_trans``): transpose()/dagger() are then free, as in the reference where
they return numpy views, and the kernels read through the flag.

Representations, signatures and block irreps stay on the host in the
reference's exact formats, so block structure is bit-identical.
"""

import numpy as np
import torch

from .. import device as dev
from .. import instrument
from .. import linalg
from ..misc_tools.svd_tools import find_block_cuts
from .diagonal_tensor import DiagonalTensor


def validated_signature(signature0, n_row_reps, n_col_reps):
    """symmetric_tensor.py:24-32."""
    if signature0 is None:
        signature = np.zeros((n_row_reps + n_col_reps,), dtype=bool)
        signature[n_row_reps:] = True
    else:
        signature = np.ascontiguousarray(signature0, dtype=bool)
        if signature.shape != (n_row_reps + n_col_reps,):
            raise ValueError("Invalid signature shape")
    return signature


def _is_number(x):
    return isinstance(x, (int, float, np.number)) and not isinstance(x, bool)


def _pack_blocks(blocks):
    """Concatenate 2-D blocks (numpy or torch) into one C-order device buffer."""
    shapes = np.array([tuple(b.shape) for b in blocks], dtype=np.int64).reshape(-1, 2)
    sizes = shapes[:, 0] * shapes[:, 1]
    offsets = np.zeros(len(blocks), dtype=np.int64)
    if len(blocks) > 1:
        offsets[1:] = np.cumsum(sizes[:-1])
    if not blocks:
        return dev.empty_f64(0), offsets, shapes
    if all(isinstance(b, torch.Tensor) for b in blocks):
        data = torch.cat(
            [b.to(device=dev.device(), dtype=torch.float64).reshape(-1) for b in blocks]
        )
    else:
        host = np.concatenate(
            [
                (b.detach().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b))
                .astype(np.float64, copy=False)
                .ravel(order="C")
                for b in blocks
            ]
        )
        data = dev.upload_f64(host)
    return data, offsets, shapes


class SymmetricTensor:
    """Generic base class; symmetry-specific statics and data hooks live in the
    subclasses, exactly as in the reference's plugin design."""

    _symmetry = NotImplemented

    # ------------------------------------------------------ symmetry interface
    @classmethod
    def symmetry(cls):
        return cls._symmetry

    @staticmethod
    def singlet():
        raise NotImplementedError("Must be defined in derived class")

    @staticmethod
    def combine_representations(reps, signature):
        raise NotImplementedError("Must be defined in derived class")

    @staticmethod
    def conjugate_irrep(irr):
        raise NotImplementedError("Must be defined in derived class")

    @staticmethod
    def conjugate_representation(rep):
        raise NotImplementedError("Must be defined in derived class")

    @staticmethod
    def init_representation(degen, irreps):
        raise NotImplementedError("Must be defined in derived class")

    @staticmethod
    def representation_dimension(rep):
        raise NotImplementedError("Must be defined in derived class")

    @staticmethod
    def irrep_dimension(rep):
        raise NotImplementedError("Must be defined in derived class")

    @classmethod
    def get_block_sizes(cls, row_reps, col_reps, signature):
        raise NotImplementedError("Must be defined in derived class")

    # ------------------------------------------------------------ construction
    def __init__(self, row_reps, col_reps, blocks, block_irreps, signature):
        data, offsets, shapes = _pack_blocks(list(blocks))
        self._init_storage(
            row_reps, col_reps, data, offsets, shapes, block_irreps, signature, False
        )
        if __debug__:
            assert self.check_blocks_fit_representations()

    @classmethod
    def _from_storage(cls, row_reps, col_reps, data, offsets, shapes, block_irreps,
                      signature, trans=False):
        t = cls.__new__(cls)
        t._init_storage(row_reps, col_reps, data, offsets, shapes, block_irreps,
                        signature, trans)
        return t

    def _init_storage(self, row_reps, col_reps, data, offsets, shapes, block_irreps,
                      signature, trans):
        self._row_reps = tuple(row_reps)
        self._col_reps = tuple(col_reps)
        self._shape = tuple(
            self.representation_dimension(r) for r in self._row_reps + self._col_reps
        )
        self._ndim = len(self._shape)
        self._nrr = len(self._row_reps)
        self._signature = np.ascontiguousarray(signature, dtype=bool)
        self._data = data
        self._offsets = np.asarray(offsets, dtype=np.int64)
        self._bshapes = np.asarray(shapes, dtype=np.int64).reshape(-1, 2)
        self._block_irreps = np.asarray(block_irreps)
        self._nblocks = int(self._offsets.size)
        self._trans = bool(trans)
        self._views = None
        if not (0 < self._nrr < self._ndim):
            raise ValueError("a SymmetricTensor needs at least one row and one column leg")
        if self._signature.shape != (self._ndim,):
            raise ValueError("signature does not match the number of legs")
        if self._block_irreps.shape[0] != self._nblocks:
            raise ValueError("block_irreps does not match the number of blocks")

    @classmethod
    def from_array(cls, arr, row_reps, col_reps, signature=None):
        """symmetric_tensor.py:118-146 (dense -> blocks, on the device)."""
        row_reps = tuple(row_reps)
        col_reps = tuple(col_reps)
        shape = tuple(cls.representation_dimension(rep) for rep in row_reps + col_reps)
        if tuple(arr.shape) != shape:
            raise ValueError("Representations do not match array shape")
        signature = validated_signature(signature, len(row_reps), len(col_reps))
        return cls._blocks_from_dense(arr, row_reps, col_reps, signature)

    @classmethod
    def from_flat(cls, row_reps, col_reps, flat, block_irreps, signature):
        """Build a tensor from one flat buffer holding its blocks back to back in
        block order, each C-order (the concatenation of the reference's
        ``blocks``).  ``flat`` may be a numpy array, a (pinned) host torch tensor
        or a device tensor; host data is copied to the device in one transfer."""
        signature = validated_signature(signature, len(row_reps), len(col_reps))
        block_irreps = np.asarray(block_irreps)
        irreps, shapes = cls.get_block_sizes(row_reps, col_reps, signature)
        keep = np.isin(irreps, block_irreps) if irreps.ndim == 1 else None
        if keep is None:
            raise NotImplementedError("from_flat needs 1-D irreps")
        shapes = shapes[keep]
        sizes = shapes[:, 0] * shapes[:, 1]
        offsets = np.zeros(sizes.size, dtype=np.int64)
        if sizes.size > 1:
            offsets[1:] = np.cumsum(sizes[:-1])
        if not isinstance(flat, torch.Tensor):
            flat = torch.from_numpy(np.ascontiguousarray(flat, dtype=np.float64))
        if flat.numel() != int(sizes.sum()):
            raise ValueError("flat buffer size does not match the block structure")
        data = flat.to(device=dev.device(), dtype=torch.float64, non_blocking=True)
        if data.data_ptr() == flat.data_ptr():
            data = data.clone()
        return cls._from_storage(row_reps, col_reps, data.reshape(-1), offsets, shapes,
                                 irreps[keep], signature)

    @classmethod
    def from_diagonal_tensor(cls, dt):
        """symmetric_tensor.py:264-275."""
        if type(dt) is not DiagonalTensor:
            raise ValueError(f"Invalid input type: {type(dt)}")
        if cls.symmetry() != dt.symmetry():
            raise ValueError("Symmetries do not match")
        blocks = tuple(torch.diag(db) for db in dt.diagonal_blocks)
        return cls(
            (dt.representation,), (dt.representation,), blocks, dt.block_irreps,
            np.array([False, True]),
        )

    @classmethod
    def random(cls, row_reps, col_reps, signature=None, *, rng=None):
        """symmetric_tensor.py:514-546; same numbers as the reference for the same
        numpy Generator (blocks drawn in block order on the host)."""
        signature = validated_signature(signature, len(row_reps), len(col_reps))
        if rng is None:
            rng = np.random.default_rng()
        block_irreps, block_shapes = cls.get_block_sizes(row_reps, col_reps, signature)
        blocks = [rng.random(tuple(sh)) - 0.5 for sh in block_shapes]
        return cls(row_reps, col_reps, blocks, block_irreps, signature)

    @classmethod
    def init_square_matrix(cls, reps, signature):
        s = np.asarray(signature, dtype=bool)
        return cls(reps, reps, [], [], np.hstack((s, ~s)))

    def cast(self, symmetry):
        return getattr(self, f"to{symmetry}")()

    # ----------------------------------------------------------------- getters
    @property
    def nblocks(self):
        return self._nblocks

    @property
    def ndim(self):
        return self._ndim

    @property
    def n_row_reps(self):
        return self._nrr

    @property
    def shape(self):
        return self._shape

    @property
    def matrix_shape(self):
        return (int(np.prod(self._shape[: self._nrr])), int(np.prod(self._shape[self._nrr :])))

    @property
    def dtype(self):
        return np.dtype(np.float64)

    @property
    def ncoeff(self):
        return int((self._bshapes[:, 0] * self._bshapes[:, 1]).sum())

    @property
    def blocks(self):
        """Tuple of torch views (device) into the tensor buffer."""
        if self._views is None:
            vs = []
            for o, (m, n) in zip(self._offsets, self._bshapes, strict=True):
                flat = self._data[o : o + m * n]
                vs.append(flat.view(n, m).t() if self._trans else flat.view(m, n))
            self._views = tuple(vs)
        return self._views

    @property
    def block_irreps(self):
        return self._block_irreps

    @property
    def block_shapes(self):
        return self._bshapes

    @property
    def row_reps(self):
        return self._row_reps

    @property
    def col_reps(self):
        return self._col_reps

    @property
    def signature(self):
        return self._signature

    @property
    def data(self):
        return self._data

    def host_blocks(self):
        """Blocks copied to the host as C-contiguous numpy arrays."""
        host = self._data.detach().cpu().numpy()
        out = []
        for o, (m, n) in zip(self._offsets, self._bshapes, strict=True):
            b = host[o : o + m * n]
            out.append(np.ascontiguousarray(b.reshape(n, m).T if self._trans else b.reshape(m, n)))
        return out

    def get_row_representation(self):
        return self.combine_representations(self._row_reps, self._signature[: self._nrr])

    def get_column_representation(self):
        return self.combine_representations(self._col_reps, ~self._signature[self._nrr :])

    # ------------------------------------------------------------------ magic
    def __repr__(self):
        bipartition = (self._nrr, self._ndim - self._nrr)
        return (
            f"{self.symmetry()} SymmetricTensor with bipartition {bipartition}"
            f" and shape {self._shape}"
        )

    def _same_structure(self, data, trans=None):
        return type(self)._from_storage(
            self._row_reps, self._col_reps, data, self._offsets, self._bshapes,
            self._block_irreps, self._signature, self._trans if trans is None else trans,
        )

    def _contiguous(self):
        """Same tensor with blocks packed C-order, back to back, in block order."""
        sizes = self._bshapes[:, 0] * self._bshapes[:, 1]
        canon = np.zeros(self._nblocks, dtype=np.int64)
        if self._nblocks > 1:
            canon[1:] = np.cumsum(sizes[:-1])
        if not self._trans and np.array_equal(canon, self._offsets) and (
            self._data.numel() == int(sizes.sum())
        ):
            return self
        data = self._relayout(canon, int(sizes.sum()))
        return type(self)._from_storage(
            self._row_reps, self._col_reps, data, canon, self._bshapes,
            self._block_irreps, self._signature, False,
        )

    def _relayout(self, new_offsets, total):
        from .layout import relayout_blocks

        return relayout_blocks(
            self._data, self._offsets, self._bshapes, self._trans, new_offsets, total
        )

    def __add__(self, other):
        """symmetric_tensor.py:326-352."""
        if not self.match_representations(other):
            raise ValueError("representations do not match")
        a = self._contiguous()
        b = other._contiguous()
        if np.array_equal(a._block_irreps, b._block_irreps):
            out = b._data.clone()
            if out.numel():
                linalg.axpby(a._data, out, 1.0, 1.0)
            return a._same_structure(out)
        irreps = np.union1d(a._block_irreps, b._block_irreps)
        ia = {int(q): i for i, q in enumerate(a._block_irreps)}
        ib = {int(q): i for i, q in enumerate(b._block_irreps)}
        blocks = []
        for q in irreps:
            q = int(q)
            if q in ia and q in ib:
                blocks.append(a.blocks[ia[q]] + b.blocks[ib[q]])
            elif q in ia:
                blocks.append(a.blocks[ia[q]].clone())
            else:
                blocks.append(b.blocks[ib[q]].clone())
        return type(self)(self._row_reps, self._col_reps, blocks,
                          irreps.astype(self._block_irreps.dtype), self._signature)

    def __sub__(self, other):
        return self + (-other)

    def _scaled(self, x):
        out = torch.empty_like(self._data)
        if out.numel():
            linalg.axpby(self._data, out, float(x), 0.0)
        return self._same_structure(out)

    def __mul__(self, other):
        """symmetric_tensor.py:377-403: scalar, or DiagonalTensor on the last leg."""
        if _is_number(other):
            return self._scaled(other)
        if isinstance(other, DiagonalTensor):
            if self._symmetry != other.symmetry():
                raise ValueError("Symmetries do not match")
            return self._diagonal_mul(other)
        raise TypeError("unsupported operation")

    def __rmul__(self, other):
        """symmetric_tensor.py:405-424: scalar, or DiagonalTensor on the 1st leg."""
        if _is_number(other):
            return self._scaled(other)
        if isinstance(other, DiagonalTensor):
            if self._symmetry != other.symmetry():
                raise ValueError("Symmetries do not match")
            return self._diagonal_mul(other, left=True)
        raise TypeError("unsupported operation")

    def __truediv__(self, x):
        return self * (1.0 / x)

    def __rtruediv__(self, x):
        return self * (1.0 / x)

    def __pos__(self):
        return self

    def __neg__(self):
        return self._scaled(-1.0)

    def __imul__(self, x):
        if self._data.numel():
            linalg.scale_(self._data, float(x))
        return self

    def __itruediv__(self, x):
        """In place division; x may be a number or a 1-element device tensor
        (for example norm_device()), which avoids a host synchronisation."""
        if self._data.numel():
            if isinstance(x, torch.Tensor):
                linalg.divide_(self._data, x)
            else:
                linalg.scale_(self._data, 1.0 / float(x))
        return self

    def __matmul__(self, other):
        """symmetric_tensor.py:453-489: every shared irrep block in one grouped
        GEMM launch.  Irreps missing on either side are dropped."""
        if type(self) is not type(other):
            raise TypeError("matmul needs tensors of the same type")
        if self._shape[self._nrr :] != other._shape[: other._nrr]:
            raise ValueError("contracted legs do not match")
        if __debug__:
            assert (self._signature[self._nrr :] ^ other._signature[: other._nrr]).all()
        common, i1, i2 = np.intersect1d(
            self._block_irreps, other._block_irreps, assume_unique=True,
            return_indices=True,
        )
        order = np.argsort(i1)
        i1, i2, common = i1[order], i2[order], common[order]
        M = self._bshapes[i1, 0]
        K = self._bshapes[i1, 1]
        N = other._bshapes[i2, 1]
        if (other._bshapes[i2, 0] != K).any():
            raise ValueError("inner block dimensions do not match")
        sizes = M * N
        offsets = np.zeros(common.size, dtype=np.int64)
        if common.size > 1:
            offsets[1:] = np.cumsum(sizes[:-1])
        out = dev.empty_f64(int(sizes.sum()))
        problems = [
            {
                "A": self._data, "a_off": self._offsets[a], "a_trans": self._trans,
                "B": other._data, "b_off": other._offsets[b], "b_trans": other._trans,
                "C": out, "c_off": offsets[i], "M": M[i], "N": N[i], "K": K[i],
            }
            for i, (a, b) in enumerate(zip(i1, i2, strict=True))
        ]
        linalg.grouped_gemm(problems)
        signature = np.empty((self._nrr + other._ndim - other._nrr,), dtype=bool)
        signature[: self._nrr] = self._signature[: self._nrr]
        signature[self._nrr :] = other._signature[other._nrr :]
        return type(self)._from_storage(
            self._row_reps, other._col_reps, out, offsets, np.stack([M, N], axis=1),
            common, signature,
        )

    # ------------------------------------------------------------------- misc
    def match_representations(self, other):
        """symmetric_tensor.py:494-512."""
        if (
            type(self) is not type(other)
            or self._shape != other.shape
            or (self._signature != other.signature).any()
        ):
            return False
        for r, r2 in zip(self._row_reps, other.row_reps, strict=True):
            if r.shape != r2.shape or (r != r2).any():
                return False
        for r, r2 in zip(self._col_reps, other.col_reps, strict=True):
            if r.shape != r2.shape or (r != r2).any():
                return False
        return True

    def copy(self):
        """Copies blocks only; reps, irreps and signature are shared."""
        return self._same_structure(self._data.clone())

    # ---------------------------------------------------- transpose & permute
    def permute(self, row_axes, col_axes):
        """symmetric_tensor.py:166-212."""
        row_axes = tuple(int(a) for a in row_axes)
        col_axes = tuple(int(a) for a in col_axes)
        axes = row_axes + col_axes
        if sorted(axes) != list(range(self._ndim)):
            raise ValueError("Axes do not match tensor")
        if row_axes == tuple(range(self._nrr)) and col_axes == tuple(
            range(self._nrr, self._ndim)
        ):
            return self
        if row_axes == tuple(range(self._nrr, self._ndim)) and col_axes == tuple(
            range(self._nrr)
        ):
            return self.transpose()
        signature = np.empty((self._ndim,), dtype=bool)
        reps = [None] * self._ndim
        for i, ax in enumerate(axes):
            signature[i] = self._signature[ax]
            reps[i] = self._row_reps[ax] if ax < self._nrr else self._col_reps[ax - self._nrr]
        nrr = len(row_axes)
        data, offsets, shapes, block_irreps = self._permute_data(axes, nrr)
        return type(self)._from_storage(
            reps[:nrr], reps[nrr:], data, offsets, shapes, block_irreps, signature
        )

    def transpose(self):
        """symmetric_tensor.py:569-576."""
        data, offsets, shapes, block_irreps, trans = self._transpose_data()
        s = self._signature[np.arange(-self._ndim + self._nrr, self._nrr) % self._ndim]
        return type(self)._from_storage(
            self._col_reps, self._row_reps, data, offsets, shapes, block_irreps, s, trans
        )

    def dual(self):
        return self.dagger().conjugate().transpose()

    def conjugate(self):
        """Real float64 data: conjugation is the identity on coefficients."""
        return self._same_structure(self._data)

    def dagger(self):
        """symmetric_tensor.py:596-609: free (flips the storage flag)."""
        s = np.empty((self._ndim,), dtype=bool)
        s[: self._ndim - self._nrr] = ~self._signature[self._nrr :]
        s[self._ndim - self._nrr :] = ~self._signature[: self._nrr]
        return type(self)._from_storage(
            self._col_reps, self._row_reps, self._data, self._offsets,
            self._bshapes[:, ::-1].copy(), self._block_irreps, s, not self._trans,
        )

    # --------------------------------------------------------- linear algebra
    def is_square_matrix(self):
        if self._nrr != self._ndim // 2:
            return False
        if (self._signature[: self._nrr] == self._signature[self._nrr :]).any():
            return False
        for r1, r2 in zip(self._row_reps, self._col_reps, strict=True):
            if r1.shape != r2.shape or (r1 != r2).any():
                return False
        return True

    def _irrep_weights(self, irreps):
        return np.array([self.irrep_dimension(r) for r in irreps], dtype=np.float64)

    def norm_device(self):
        """Frobenius norm as a 0-d device tensor (no host sync)."""
        sizes = self._bshapes[:, 0] * self._bshapes[:, 1]
        return torch.sqrt(
            linalg.weighted_reduce(
                self._data, self._offsets, sizes, self._irrep_weights(self._block_irreps),
                squares=True,
            )
        )

    def norm(self):
        """symmetric_tensor.py:624-631: sqrt(sum dim(irr) ||b||^2)."""
        if self._nblocks == 0:
            return 0.0
        return float(self.norm_device())

    def trace(self):
        """symmetric_tensor.py:633-637."""
        if self._nblocks == 0:
            return 0.0
        w = self._irrep_weights(self._block_irreps)
        pairs = [
            (o, -1, m, n, self._trans, False, w[i])
            for i, (o, (m, n)) in enumerate(zip(self._offsets, self._bshapes, strict=True))
        ]
        return float(linalg.pair_contract(self._data, None, pairs))

    def full_contract(self, other):
        """symmetric_tensor.py:639-653: sum dim(irr) tr(A_irr B_irr)."""
        if __debug__:
            assert self.match_representations(other.dagger())
        common, i1, i2 = np.intersect1d(
            self._block_irreps, other.block_irreps, assume_unique=True,
            return_indices=True,
        )
        if common.size == 0:
            return 0.0
        w = self._irrep_weights(common)
        pairs = [
            (self._offsets[a], other._offsets[b], self._bshapes[a, 0],
             self._bshapes[a, 1], self._trans, other._trans, w[i])
            for i, (a, b) in enumerate(zip(i1, i2, strict=True))
        ]
        return float(linalg.pair_contract(self._data, other._data, pairs))

    def _diagonal_mul(self, dt, *, left=False):
        """symmetric_tensor.py:1189-1248: scale the last column leg (right) or the
        first row leg (left) by diagonal blocks; conjugate and re-sort the
        diagonal irreps when the signature does not match."""
        d_irreps = np.asarray(dt.block_irreps)
        d_index = np.arange(dt.nblocks)
        if (left and self._signature[0]) or (not left and not self._signature[-1]):
            conj = np.array([self.conjugate_irrep(r) for r in d_irreps])
            so = conj.argsort(kind="stable") if conj.ndim == 1 else np.lexsort(conj.T[::-1])
            d_irreps = conj[so]
            d_index = d_index[so]
        if left:
            if self._nrr != 1:
                raise ValueError("left diagonal product needs exactly one row leg")
        elif self._ndim - self._nrr != 1:
            raise ValueError("right diagonal product needs exactly one column leg")
        common, i1, i2 = np.intersect1d(
            self._block_irreps, d_irreps, assume_unique=True, return_indices=True
        )
        order = np.argsort(i1)
        i1, i2, common = i1[order], i2[order], common[order]
        shapes = self._bshapes[i1]
        sizes = shapes[:, 0] * shapes[:, 1]
        offsets = np.zeros(common.size, dtype=np.int64)
        if common.size > 1:
            offsets[1:] = np.cumsum(sizes[:-1])
        entries = []
        for i, (a, b) in enumerate(zip(i1, i2, strict=True)):
            m, n = shapes[i]
            db = d_index[b]
            if dt.block_sizes[db] != (m if left else n):
                raise ValueError("diagonal block size does not match")
            entries.append(
                (self._offsets[a], offsets[i], dt.block_offsets[db], m, n, self._trans, left)
            )
        out = linalg.diag_mul(self._data, dt.data, entries, int(sizes.sum()))
        return type(self)._from_storage(
            self._row_reps, self._col_reps, out, offsets, shapes, common, self._signature
        )

    # ------------------------------------------------------- factorisations
    def _per_block(self, fn):
        return [fn(b) for b in self.blocks]

    def qr(self):
        """symmetric_tensor.py:655-671 (economic QR per block, cuSOLVER)."""
        qs, rs = [], []
        for b in self.blocks:
            q, r = torch.linalg.qr(b, mode="reduced")
            qs.append(q)
            rs.append(r)
        degen = np.array([r.shape[0] for r in rs], dtype=np.int64)
        mid_rep = self.init_representation(degen, self._block_irreps)
        qsign = np.ones((self._nrr + 1,), dtype=bool)
        qsign[: self._nrr] = self._signature[: self._nrr]
        Q = type(self)(self._row_reps, (mid_rep,), qs, self._block_irreps, qsign)
        rsign = np.zeros((self._ndim - self._nrr + 1,), dtype=bool)
        rsign[1:] = self._signature[self._nrr :]
        R = type(self)((mid_rep,), self._col_reps, rs, self._block_irreps, rsign)
        return Q, R

    def rq(self):
        """symmetric_tensor.py:673-689 (economic RQ per block).  RQ of B is taken
        from the QR of the row/column-reversed transpose."""
        rs, qs = [], []
        for b in self.blocks:
            q1, r1 = torch.linalg.qr(torch.flip(b, dims=(0, 1)).T, mode="reduced")
            rs.append(torch.flip(r1.T, dims=(0, 1)))
            qs.append(torch.flip(q1.T, dims=(0, 1)))
        degen = np.array([r.shape[1] for r in rs], dtype=np.int64)
        mid_rep = self.init_representation(degen, self._block_irreps)
        rsign = np.ones((self._nrr + 1,), dtype=bool)
        rsign[: self._nrr] = self._signature[: self._nrr]
        R = type(self)(self._row_reps, (mid_rep,), rs, self._block_irreps, rsign)
        qsign = np.zeros((self._ndim - self._nrr + 1,), dtype=bool)
        qsign[1:] = self._signature[self._nrr :]
        Q = type(self)((mid_rep,), self._col_reps, qs, self._block_irreps, qsign)
        return R, Q

    def svd(self):
        """symmetric_tensor.py:691-710 (dense SVD per block, cuSOLVER)."""
        us, ss, vs = [], [], []
        for b in self.blocks:
            u, s, v = torch.linalg.svd(b, full_matrices=False)
            us.append(u)
            ss.append(s)
            vs.append(v)
        degen = np.array([s.shape[0] for s in ss], dtype=np.int64)
        mid_rep = self.init_representation(degen, self._block_irreps)
        usign = np.ones((self._nrr + 1,), dtype=bool)
        usign[: self._nrr] = self._signature[: self._nrr]
        U = type(self)(self._row_reps, (mid_rep,), us, self._block_irreps, usign)
        degens = [self.irrep_dimension(irr) for irr in self._block_irreps]
        s = DiagonalTensor(ss, mid_rep, self._block_irreps, degens, self._symmetry)
        vsign = np.zeros((self._ndim - self._nrr + 1,), dtype=bool)
        vsign[1:] = self._signature[self._nrr :]
        V = type(self)((mid_rep,), self._col_reps, vs, self._block_irreps, vsign)
        return U, s, V

    def truncated_svd(self, cut, *, dmax_full=100, oversampling=0, atol=0.0, rtol=None,
                      degen_ratio=1.0):
        """symmetric_tensor.py:835-877.  Every block takes the dense path here (a
        superset of the values the reference's ARPACK path computes); the kept
        set is decided by the same greedy find_block_cuts."""
        del dmax_full, oversampling
        raw_u, raw_s, raw_v = [], [], []
        for b in self.blocks:
            u, s, v = torch.linalg.svd(b, full_matrices=False)
            raw_u.append(u)
            raw_s.append(s)
            raw_v.append(v)
        if not raw_s:
            raise ValueError("truncated_svd of a tensor without blocks")
        host_s = [s.detach().cpu().numpy() for s in raw_s]
        dims = np.array([self.irrep_dimension(r) for r in self._block_irreps])
        cuts = find_block_cuts(host_s, cut, dims=dims, atol=atol, rtol=rtol,
                               degen_ratio=degen_ratio)
        return self._truncate(raw_s, self._block_irreps, cuts, raw_u, raw_v)

    def _truncate(self, val_blocks, block_irreps, cuts, left=None, right=None):
        """truncate_values_vectors, symmetric_tensor.py:1436-1477."""
        non_empty = np.flatnonzero(cuts)
        nkept = np.asarray(cuts)[non_empty]
        kept_irreps = np.asarray(block_irreps)[non_empty]
        s_blocks = [val_blocks[bi][: cuts[bi]] for bi in non_empty]
        s_rep = self.init_representation(nkept, kept_irreps)
        degens = [self.irrep_dimension(irr) for irr in kept_irreps]
        s = DiagonalTensor(s_blocks, s_rep, kept_irreps, degens, self._symmetry)
        u = v = None
        if left is not None:
            ub = [left[bi][:, : cuts[bi]] for bi in non_empty]
            usign = np.hstack((self._signature[: self._nrr], [True]))
            u = type(self)(self._row_reps, (s.representation,), ub, kept_irreps, usign)
        if right is not None:
            vb = [right[bi][: cuts[bi], :] for bi in non_empty]
            vsign = np.hstack(([False], self._signature[self._nrr :]))
            v = type(self)((s.representation,), self._col_reps, vb, kept_irreps, vsign)
        return u, s, v

    def pinv(self, *, atol=0.0, rtol=None):
        u, s, v = self.truncated_svd(2**31, atol=atol, rtol=rtol)
        return v.dagger() * (1 / s) @ u.dagger()

    def eigh(self, *, compute_vectors=True):
        """symmetric_tensor.py:738-777."""
        if not self.is_square_matrix():
            raise ValueError("Tensor legs do not define a square matrix")
        return self.truncated_eigh(2**31, compute_vectors=compute_vectors)

    def truncated_eigh(self, nvals, *, atol=0.0, rtol=None, degen_ratio=1.0,
                       dmax_full=100, compute_vectors=True, rng=None, maxiter=4000,
                       arpack_tol=0, matmat=None):
        """symmetric_tensor.py:1087-1132 -> _sparse_eig (:1250-1434) with every
        block on the dense path (cuSOLVER syevd): per allowed block keep the
        nvals // dim + 1 largest |eigenvalues|, then find_block_cuts."""
        del dmax_full, rng, maxiter, arpack_tol
        if matmat is not None:
            raise NotImplementedError("matrix-free truncated_eigh is not supported")
        if not self.is_square_matrix():
            raise ValueError("Tensor legs do not define a square matrix")
        irreps, shapes = self.get_block_sizes(self._row_reps, self._col_reps, self._signature)
        nb = len(shapes)
        vals = [None] * nb
        vecs = [None] * nb
        absv = [np.zeros((1,))] * nb
        lookup = {self._irrep_key(q): i for i, q in enumerate(self._block_irreps)}
        dims = np.empty(nb, dtype=np.int64)
        pending = []
        for bi in range(nb):
            dims[bi] = self.irrep_dimension(irreps[bi])
            k = nvals // dims[bi] + 1
            j = lookup.get(self._irrep_key(irreps[bi]))
            if j is None:
                continue
            with instrument.region("eigh"):
                w, v = torch.linalg.eigh(self.blocks[j])
            a = torch.abs(w)
            so = torch.argsort(a, descending=True, stable=True)[: min(k, a.numel())]
            vals[bi] = w[so]
            vecs[bi] = v[:, so] if compute_vectors else None
            pending.append((bi, a[so]))
        for bi, a in pending:
            absv[bi] = a.detach().cpu().numpy()
        cuts = find_block_cuts(absv, nvals, dims=dims, atol=atol, rtol=rtol,
                               degen_ratio=degen_ratio)
        u, s, _ = self._truncate(vals, irreps, cuts, vecs if compute_vectors else None)
        if compute_vectors:
            return s, u
        return s

    @staticmethod
    def truncated_eigh_many(tensors, nvals, *, atol=0.0, rtol=None, degen_ratio=1.0):
        """truncated_eigh of many independent tensors (the corners of many
        CTMRG runs advanced in lock step): every block of every tensor is
        diagonalised with the other blocks of the same size in one batched
        cuSOLVER call, the kept eigenvalues of all tensors come to the host in
        one copy, then each tensor is truncated as truncated_eigh does.
        Returns [(s, u)] in the order of `tensors`."""
        jobs = []
        per = []
        for ti, (t, nv) in enumerate(zip(tensors, nvals, strict=True)):
            if not t.is_square_matrix():
                raise ValueError("Tensor legs do not define a square matrix")
            irreps, shapes = t.get_block_sizes(t._row_reps, t._col_reps, t._signature)
            nb = len(shapes)
            lookup = {t._irrep_key(q): i for i, q in enumerate(t._block_irreps)}
            dims = np.array([t.irrep_dimension(irreps[bi]) for bi in range(nb)], dtype=np.int64)
            per.append((irreps, dims, [None] * nb, [None] * nb, [np.zeros((1,))] * nb))
            for bi in range(nb):
                j = lookup.get(t._irrep_key(irreps[bi]))
                if j is not None:
                    jobs.append((ti, bi, t.blocks[j], int(nv // dims[bi] + 1)))
        by_shape = {}
        for job in jobs:
            by_shape.setdefault(tuple(job[2].shape), []).append(job)
        pending = []
        for group in by_shape.values():
            w, v = torch.linalg.eigh(torch.stack([job[2] for job in group]))
            for gi, (ti, bi, _, k) in enumerate(group):
                a = torch.abs(w[gi])
                so = torch.argsort(a, descending=True, stable=True)[: min(k, a.numel())]
                per[ti][2][bi] = w[gi][so]
                per[ti][3][bi] = v[gi][:, so]
                pending.append((ti, bi, a[so]))
        host = torch.cat([a for _, _, a in pending]).cpu().numpy() if pending else None
        pos = 0
        for ti, bi, a in pending:
            per[ti][4][bi] = host[pos: pos + a.numel()]
            pos += a.numel()
        out = []
        for t, nv, (irreps, dims, vals, vecs, absv) in zip(tensors, nvals, per, strict=True):
            cuts = find_block_cuts(absv, nv, dims=dims, atol=atol, rtol=rtol,
                                   degen_ratio=degen_ratio)
            u, sv, _ = t._truncate(vals, irreps, cuts, vecs)
            out.append((sv, u))
        return out

    @classmethod
    def eigs(cls, matmat, nvals, reps, signature, *, atol=0.0, rtol=None, degen_ratio=1.0,
             dmax_full=100, compute_vectors=False, rng=None, maxiter=4000, arpack_tol=0):
        """symmetric_tensor.py:880-955 -> _sparse_eig (:1250-1434) for a real
        square matrix known only through ``matmat`` (applied to device tensors).

        Blocks smaller than max(dmax_full, 3k) are built by one ``matmat`` on
        identity blocks and diagonalised on the device (torch.linalg.eigvals);
        larger ones go to ARPACK (scipy.sparse.linalg.eigs), whose matvec copies
        the Krylov vector to the device, applies ``matmat`` there and copies the
        block back.  Returns the kept eigenvalues as the reference's
        ``DiagonalTensor.toarray()`` lays them out (per kept block, each value
        repeated irrep-dimension times), a host numpy array."""
        if compute_vectors:
            raise NotImplementedError("eigenvectors of a matrix-free operator are not returned")
        import scipy.sparse.linalg as slg

        if rng is None:
            rng = np.random.default_rng()
        m = cls.init_square_matrix(reps, signature)
        block_irreps, block_shapes = cls.get_block_sizes(m._row_reps, m._col_reps,
                                                         m._signature)
        nb = len(block_shapes)
        sigv = np.hstack((m._signature[: m._nrr], [True]))
        dims = np.array([cls.irrep_dimension(q) for q in block_irreps], dtype=np.int64)
        val_blocks = [None] * nb
        abs_blocks = [np.zeros((1,))] * nb
        full, sparse = [], []
        for bi in range(nb):
            k = nvals // dims[bi] + 1
            (full if block_shapes[bi, 0] < max(dmax_full, 3 * k) else sparse).append(bi)

        def keep(bi, vals, k):
            a = np.abs(vals)
            so = a.argsort()[: -k - 1 : -1]
            val_blocks[bi] = vals[so]
            abs_blocks[bi] = a[so]

        if full:
            irr_full = np.ascontiguousarray(block_irreps[full])
            rfull = cls.init_representation(block_shapes[full, 0], irr_full)
            eye = [torch.eye(int(block_shapes[bi, 0]), dtype=torch.float64,
                             device=dev.device()) for bi in full]
            st = matmat(cls(m._row_reps, (rfull,), eye, irr_full, sigv))
            for bi in full:
                q = block_irreps[bi]
                bj = int(np.searchsorted(st.block_irreps, q))
                if bj < st.nblocks and st.block_irreps[bj] == q:
                    vals = torch.linalg.eigvals(st.blocks[bj]).cpu().numpy()
                    keep(bi, vals, nvals // dims[bi] + 1)
        for bi in sparse:
            q = block_irreps[bi : bi + 1]
            d = int(block_shapes[bi, 0])
            k = nvals // dims[bi] + 1
            v0 = rng.standard_normal(size=(d,))
            brep = cls.init_representation(np.ones((1,), dtype=np.int64), q)
            st0 = cls(m._row_reps, (brep,), (v0[:, None],), q, sigv)
            st1 = matmat(st0)
            bj = int(np.searchsorted(st1.block_irreps, q[0]))
            if not (bj < st1.nblocks and st1.block_irreps[bj] == q[0]):
                continue

            def matvec(x, st0=st0, bj=bj):
                st0.blocks[0][:, 0].copy_(torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)))
                return matmat(st0).blocks[bj].reshape(-1).cpu().numpy()

            op = slg.LinearOperator((d, d), matvec=matvec, dtype=np.float64)
            try:
                vals = slg.eigs(op, k=k, v0=v0, maxiter=maxiter, tol=arpack_tol,
                                return_eigenvectors=False)
            except slg.ArpackNoConvergence as err:
                vals = err.eigenvalues
            keep(bi, vals, k)
        cuts = find_block_cuts(abs_blocks, nvals, dims=dims, atol=atol, rtol=rtol,
                               degen_ratio=degen_ratio)
        kept = [bi for bi in range(nb) if cuts[bi]]
        dtype = np.result_type(*[val_blocks[bi].dtype for bi in kept]) if kept else np.float64
        out = [np.repeat(val_blocks[bi][: cuts[bi]].astype(dtype), dims[bi]) for bi in kept]
        return np.concatenate(out) if out else np.zeros(0, dtype=dtype)

    @staticmethod
    def _irrep_key(q):
        return int(q) if np.ndim(q) == 0 else tuple(np.ravel(q))

    def expm(self):
        """symmetric_tensor.py:818-824."""
        if not self.is_square_matrix():
            raise ValueError("Tensor legs do not define a square matrix")
        blocks = [torch.linalg.matrix_exp(b) for b in self.blocks]
        return type(self)(self._row_reps, self._col_reps, blocks, self._block_irreps,
                          self._signature)

    def solve(self, b):
        """symmetric_tensor.py:712-732."""
        if not self.is_square_matrix():
            raise ValueError("Tensor legs do not define a square matrix")
        common, i1, i2 = np.intersect1d(self._block_irreps, b.block_irreps,
                                        assume_unique=True, return_indices=True)
        if common.size < b.nblocks:
            raise ValueError("No solution: missing block in A appears in b")
        xb = [torch.linalg.solve(self.blocks[i], b.blocks[j]) for i, j in zip(i1, i2, strict=True)]
        s = np.hstack((~self._signature[self._nrr :], b.signature[b.n_row_reps :]))
        return type(self)(self._col_reps, b.col_reps, xb, common, s)

    # --------------------------------------------------------------------- I/O
    def toarray(self, *, as_matrix=False):
        """symmetric_tensor.py:148-164 (host numpy array)."""
        mat = self._tomatrix()
        return mat if as_matrix else mat.reshape(self._shape)

    def save_to_file(self, savefile):
        np.savez_compressed(savefile, **self.get_data_dic())

    def get_data_dic(self, *, prefix=""):
        """Same keys and formats as symmetric_tensor.py:1145-1167."""
        data = {
            prefix + "_symmetry": self._symmetry,
            prefix + "_n_row_reps": self._nrr,
            prefix + "_n_col_reps": self._ndim - self._nrr,
            prefix + "_block_irreps": self._block_irreps,
            prefix + "_signature": self._signature,
        }
        for ri, r in enumerate(self._row_reps):
            data[f"{prefix}_row_rep_{ri}"] = r
        for ci, c in enumerate(self._col_reps):
            data[f"{prefix}_col_rep_{ci}"] = c
        for bi, b in enumerate(self.host_blocks()):
            data[f"{prefix}_block_{bi}"] = b
        return data

    @classmethod
    def load_from_dic(cls, data, *, prefix=""):
        """symmetric_tensor.py:1169-1180."""
        if cls._symmetry != data[prefix + "_symmetry"][()]:
            raise ValueError(f"Saved SymmetricTensor does not match type {cls}")
        nrr = int(data[prefix + "_n_row_reps"])
        row_reps = [data[f"{prefix}_row_rep_{ri}"] for ri in range(nrr)]
        nrc = int(data[prefix + "_n_col_reps"])
        col_reps = [data[f"{prefix}_col_rep_{ri}"] for ri in range(nrc)]
        block_irreps = data[prefix + "_block_irreps"]
        signature = data[prefix + "_signature"]
        blocks = [np.asarray(data[f"{prefix}_block_{bi}"]) for bi in range(block_irreps.shape[0])]
        return cls(row_reps, col_reps, blocks, block_irreps, signature)

    @classmethod
    def load_from_file(cls, savefile, *, prefix=""):
        with np.load(savefile) as fin:
            return cls.load_from_dic(fin, prefix=prefix)
