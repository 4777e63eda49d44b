"""Device DiagonalTensor: singular values, eigenvalues and bond weights.

Mirrors frostspin/symmetric_tensor/diagonal_tensor.py:5-276.  The 1-D diagonal
blocks live back to back in one float64 device buffer; ``diagonal_blocks``
returns torch views into it.  Metadata (representation, irreps, degeneracies,
symmetry name) stays on the host in the reference's formats.
"""

import numpy as np
import torch

from .. import device as dev
from .. import linalg


def _is_number(x):
    return isinstance(x, (int, float, np.number)) and not isinstance(x, bool)


class DiagonalTensor:
    def __init__(self, diag_blocks, representation, block_irreps, block_degen, symmetry):
        blocks = [
            b if isinstance(b, torch.Tensor) else np.asarray(b, dtype=np.float64)
            for b in diag_blocks
        ]
        sizes = np.array([int(b.shape[0]) for b in blocks], dtype=np.int64)
        if any(b.ndim != 1 for b in blocks):
            raise ValueError("diagonal blocks must be 1-D")
        if blocks and all(isinstance(b, torch.Tensor) for b in blocks):
            data = torch.cat([b.reshape(-1).to(torch.float64) for b in blocks]).to(
                dev.device()
            )
        elif blocks:
            host = np.concatenate(
                [
                    b.detach().cpu().numpy().ravel() if isinstance(b, torch.Tensor) else b
                    for b in blocks
                ]
            )
            data = dev.upload_f64(host)
        else:
            data = dev.empty_f64(0)
        self._set(data, sizes, representation, block_irreps, block_degen, symmetry)

    @classmethod
    def _from_storage(cls, data, sizes, representation, block_irreps, block_degen,
                      symmetry):
        t = cls.__new__(cls)
        t._set(data, np.asarray(sizes, dtype=np.int64), representation, block_irreps,
               block_degen, symmetry)
        return t

    def _set(self, data, sizes, representation, block_irreps, block_degen, symmetry):
        self._data = data
        self._sizes = sizes
        self._offsets = np.zeros(sizes.size, dtype=np.int64)
        if sizes.size > 1:
            self._offsets[1:] = np.cumsum(sizes[:-1])
        self._representation = representation
        self._block_irreps = np.asarray(block_irreps)
        self._block_degen = np.asarray(block_degen)
        self._symmetry = symmetry
        self._nblocks = int(sizes.size)
        self._views = None
        if self._block_degen.shape != (self._nblocks,):
            raise ValueError("block_degen does not match the number of blocks")
        if self._block_irreps.shape[0] != self._nblocks:
            raise ValueError("block_irreps does not match the number of blocks")

    # ------------------------------------------------------------------ getters
    @property
    def diagonal_blocks(self):
        if self._views is None:
            self._views = tuple(
                self._data[o : o + s] for o, s in zip(self._offsets, self._sizes, strict=True)
            )
        return self._views

    @property
    def data(self):
        return self._data

    @property
    def block_sizes(self):
        return self._sizes

    @property
    def block_offsets(self):
        return self._offsets

    @property
    def block_degen(self):
        return self._block_degen

    @property
    def block_irreps(self):
        return self._block_irreps

    @property
    def nblocks(self):
        return self._nblocks

    @property
    def ndim(self):
        return 1

    @property
    def representation(self):
        return self._representation

    @property
    def signature(self):
        return np.array([False, True])

    @property
    def shape(self):
        return (len(self),)

    @property
    def dtype(self):
        return np.dtype(np.float64)

    def symmetry(self):
        return self._symmetry

    # ------------------------------------------------------------------ magic
    def __repr__(self):
        return f"DiagonalTensor with {self.nblocks} blocks and {self.symmetry()} symmetry"

    def __len__(self):
        return int((self._sizes * self._block_degen).sum())

    def _like(self, data):
        return type(self)._from_storage(
            data, self._sizes, self._representation, self._block_irreps,
            self._block_degen, self._symmetry,
        )

    def __mul__(self, x):
        if isinstance(x, DiagonalTensor):
            if not np.array_equal(np.asarray(self._representation),
                                  np.asarray(x.representation)):
                raise ValueError("Representations do not match")
            return self._like(self._data * x.data)
        if _is_number(x):
            out = torch.empty_like(self._data)
            if out.numel():
                linalg.axpby(self._data, out, float(x), 0.0)
            return self._like(out)
        return NotImplemented

    def __rmul__(self, x):
        if _is_number(x):
            return self * x
        msg = f"Unsupported operation for type: {type(x)}"
        raise TypeError(msg)

    def __imul__(self, x):
        if not _is_number(x):
            raise NotImplementedError("Invalid type for *=")
        if self._data.numel():
            linalg.scale_(self._data, float(x))
        return self

    def __truediv__(self, x):
        return self * (1.0 / x)

    def __rtruediv__(self, x):
        if _is_number(x):
            inv = linalg.power(self._data, -1.0)
            if float(x) != 1.0:
                linalg.scale_(inv, float(x))
            return self._like(inv)
        raise NotImplementedError("Invalid type for /")

    def __itruediv__(self, x):
        if isinstance(x, torch.Tensor):
            if self._data.numel():
                linalg.divide_(self._data, x)
            return self
        self *= 1.0 / x
        return self

    def __pow__(self, x):
        if not _is_number(x):
            raise NotImplementedError("Invalid type for **")
        return self._like(linalg.power(self._data, float(x)))

    def __neg__(self):
        return self * -1.0

    def __add__(self, other):
        if not isinstance(other, DiagonalTensor):
            raise NotImplementedError("Invalid type for +")
        if not np.array_equal(np.asarray(self._representation),
                              np.asarray(other.representation)):
            raise ValueError("Representations do not match")
        out = other.data.clone()
        linalg.axpby(self._data, out, 1.0, 1.0)
        return self._like(out)

    def __sub__(self, other):
        return self + (-other)

    def __pos__(self):
        return self

    # ------------------------------------------------------------------ misc
    def copy(self):
        return self._like(self._data.clone())

    def _weights(self):
        return self._block_degen.astype(np.float64)

    def sum_device(self):
        return linalg.weighted_reduce(
            self._data, self._offsets, self._sizes, self._weights(), squares=False
        )

    def sum(self):
        """sum_i degen_i * sum(block_i), diagonal_tensor.py:195-199."""
        if self._nblocks == 0:
            return 0.0
        return float(self.sum_device())

    def norm_device(self):
        return torch.sqrt(
            linalg.weighted_reduce(
                self._data, self._offsets, self._sizes, self._weights(), squares=True
            )
        )

    def norm(self):
        """diagonal_tensor.py:201-205."""
        if self._nblocks == 0:
            return 0.0
        return float(self.norm_device())

    def toarray(self, *, sort=False):
        """diagonal_tensor.py:207-233: host array, blocks repeated by degeneracy,
        optionally sorted by decreasing magnitude."""
        host = self._data.detach().cpu().numpy()
        parts = []
        for o, s, d in zip(self._offsets, self._sizes, self._block_degen, strict=True):
            parts.append(np.repeat(host[o : o + s], int(d)))
        arr = np.concatenate(parts) if parts else np.zeros(0)
        if sort:
            arr = arr[np.abs(arr).argsort()[::-1]]
        return arr

    def host_blocks(self):
        host = self._data.detach().cpu().numpy()
        return [host[o : o + s].copy() for o, s in zip(self._offsets, self._sizes, strict=True)]

    # ------------------------------------------------------------------ I/O
    def save_to_file(self, savefile):
        np.savez_compressed(savefile, **self.get_data_dic())

    def get_data_dic(self, *, prefix=""):
        """Same keys as the reference (diagonal_tensor.py:245-262)."""
        data = {
            prefix + "_block_irreps": self._block_irreps,
            prefix + "_block_degen": self._block_degen,
            prefix + "_representation": self._representation,
            prefix + "_symmetry": self._symmetry,
        }
        for bi, db in enumerate(self.host_blocks()):
            data[f"{prefix}_diagonal_block_{bi}"] = db
        return data

    @classmethod
    def load_from_dic(cls, data, *, prefix=""):
        symmetry = str(data[prefix + "_symmetry"])
        block_irreps = data[prefix + "_block_irreps"]
        block_degen = data[prefix + "_block_degen"]
        representation = data[prefix + "_representation"]
        diag_blocks = tuple(
            np.asarray(data[f"{prefix}_diagonal_block_{bi}"])
            for bi in range(block_irreps.shape[0])
        )
        return cls(diag_blocks, representation, block_irreps, block_degen, symmetry)

    @classmethod
    def load_from_file(cls, savefile, *, prefix=""):
        with np.load(savefile) as fin:
            return cls.load_from_dic(fin, prefix=prefix)
