"""Abelian (U(1) and Z2-as-U(1)) device tensors.

Mirrors frostspin/symmetric_tensor/abelian_symmetric_tensor.py:253-430:
int8 irreps, 1-D int8 representations, irrep dimension 1.  The permute data
plane is the C ABI's fs_abelian_permute driven by a cached elementary-block
plan (abelian_plan.py); transpose is a zero-copy flag flip plus block re-sort.
"""

from collections import OrderedDict

import numpy as np
import torch

from .. import _native, instrument, linalg
from .. import device as dev
from .abelian_plan import (
    GroupInfo,
    build_abelian_permute_plan,
    leg_coefficients,
    segments,
    to_int8,
)
from .symmetric_tensor import SymmetricTensor

_PLAN_CACHE = OrderedDict()
_PLAN_CACHE_SIZE = 512


def plan_cache_clear():
    _PLAN_CACHE.clear()


def _rep_key(reps):
    return tuple(np.asarray(r, dtype=np.int8).tobytes() for r in reps)


class AbelianSymmetricTensor(SymmetricTensor):
    # ----------------------------------------------------------- symmetry
    @staticmethod
    def singlet():
        return np.zeros((1,), dtype=np.int8)

    @staticmethod
    def init_representation(degen, irreps):
        """abelian_symmetric_tensor.py:254-261."""
        return np.repeat(np.asarray(irreps, dtype=np.int8), np.asarray(degen, dtype=np.int64))

    @staticmethod
    def representation_dimension(rep):
        return int(np.asarray(rep).size)

    @staticmethod
    def irrep_dimension(_rep):
        return 1

    @classmethod
    def get_block_sizes(cls, row_reps, col_reps, signature):
        """abelian_symmetric_tensor.py:287-318, from per-irrep index counts (no
        Kronecker expansion of the fused representations)."""
        signature = np.asarray(signature, dtype=bool)
        nrr = len(row_reps)
        coef = leg_coefficients(signature, nrr)
        reps = list(row_reps) + list(col_reps)
        rows = GroupInfo([segments(r) for r in reps[:nrr]], coef[:nrr])
        cols = GroupInfo([segments(r) for r in reps[nrr:]], coef[nrr:])
        allowed = np.flatnonzero((rows.counts > 0) & (cols.counts > 0))
        irr = to_int8(allowed)
        order = np.argsort(irr, kind="stable")
        allowed = allowed[order]
        shapes = np.stack([rows.counts[allowed], cols.counts[allowed]], axis=1)
        return irr[order], shapes.astype(np.int64)

    def toabelian(self):
        return self

    def check_blocks_fit_representations(self):
        """abelian_symmetric_tensor.py:338-349."""
        irreps, shapes = self.get_block_sizes(self._row_reps, self._col_reps, self._signature)
        lookup = {int(q): tuple(s) for q, s in zip(irreps, shapes, strict=True)}
        for q, sh in zip(self._block_irreps, self._bshapes, strict=True):
            if lookup.get(int(q)) != tuple(sh):
                return False
        return sorted(set(self._block_irreps.tolist())) == list(self._block_irreps)

    def update_signature(self, sign_update):
        """abelian_symmetric_tensor.py:320-336 (in place; coefficients unchanged)."""
        up = np.asarray(sign_update, dtype=bool)
        if up.shape != (self._ndim,):
            raise ValueError("sign_update shape does not match the tensor")
        row_reps = list(self._row_reps)
        col_reps = list(self._col_reps)
        for i in up.nonzero()[0]:
            if i < self._nrr:
                row_reps[i] = self.conjugate_representation(row_reps[i])
            else:
                j = i - self._nrr
                col_reps[j] = self.conjugate_representation(col_reps[j])
        self._row_reps = tuple(row_reps)
        self._col_reps = tuple(col_reps)
        self._signature = self._signature ^ up

    # --------------------------------------------------------- data hooks
    @classmethod
    def _blocks_from_dense(cls, arr, row_reps, col_reps, signature):
        """Dense -> blocks (abelian_symmetric_tensor.py:361-371), gathered on the
        device."""
        nrr = len(row_reps)
        ri = cls.combine_representations(row_reps, signature[:nrr])
        ci = cls.combine_representations(col_reps, ~signature[nrr:])
        if isinstance(arr, torch.Tensor):
            m = arr.to(device=dev.device(), dtype=torch.float64).reshape(ri.size, ci.size)
        else:
            m = dev.upload_f64(np.asarray(arr).reshape(ri.size, ci.size))
        blocks, irreps = [], []
        for q in np.unique(ri):
            cols = np.flatnonzero(ci == q)
            if cols.size:
                rows = np.flatnonzero(ri == q)
                r_t = torch.from_numpy(rows).to(m.device)
                c_t = torch.from_numpy(cols).to(m.device)
                blocks.append(m.index_select(0, r_t).index_select(1, c_t))
                irreps.append(q)
        return cls(row_reps, col_reps, blocks, np.array(irreps, dtype=np.int8), signature)

    def _tomatrix(self):
        """Blocks -> dense host matrix (abelian_symmetric_tensor.py:373-383)."""
        ri = self.get_row_representation()
        ci = self.get_column_representation()
        mat = np.zeros((ri.size, ci.size))
        for q, b in zip(self._block_irreps, self.host_blocks(), strict=True):
            mat[np.ix_(np.flatnonzero(ri == q), np.flatnonzero(ci == q))] = b
        return mat

    def _transpose_data(self):
        """abelian_symmetric_tensor.py:385-393: conjugate irreps, re-sort, and
        transpose every block -- here by flipping the storage flag."""
        conj = self.conjugate_representation(self._block_irreps)
        so = np.argsort(conj, kind="stable")
        return (
            self._data,
            self._offsets[so],
            self._bshapes[so][:, ::-1].copy(),
            conj[so],
            not self._trans,
        )

    def _permute_plan(self, axes, nrr):
        key = (
            type(self).__name__,
            _rep_key(self._row_reps + self._col_reps),
            self._signature.tobytes(),
            self._nrr,
            self._block_irreps.tobytes(),
            self._offsets.tobytes(),
            self._bshapes.tobytes(),
            self._trans,
            int(self._data.numel()),
            tuple(axes),
            nrr,
        )
        plan = _PLAN_CACHE.get(key)
        if plan is not None:
            _PLAN_CACHE.move_to_end(key)
            return plan
        plan = build_abelian_permute_plan(
            list(self._row_reps + self._col_reps),
            self._signature,
            self._nrr,
            self._block_irreps,
            self._offsets,
            self._bshapes,
            self._trans,
            int(self._data.numel()),
            axes,
            nrr,
        )
        _PLAN_CACHE[key] = plan
        if len(_PLAN_CACHE) > _PLAN_CACHE_SIZE:
            _PLAN_CACHE.popitem(last=False)
        return plan

    def _permute_data(self, axes, nrr):
        """abelian_symmetric_tensor.py:395-430 on the device."""
        plan = self._permute_plan(axes, nrr)
        out = dev.empty_f64(plan.size)
        if plan.size and linalg.defer_permute(plan.ebs, plan.tasks, self._data, out,
                                              16.0 * plan.size):
            return out, plan.offsets, plan.block_shapes, plan.block_irreps
        if plan.size:
            if plan.device_tables is None:
                plan.device_tables = (dev.upload(plan.ebs), dev.upload(plan.tasks))
            d_ebs, d_tasks = plan.device_tables
            with instrument.region("permute", bytes=16.0 * plan.size):
                _native.call(
                    "fs_abelian_permute",
                    dev.ptr(self._data),
                    int(self._data.numel()),
                    dev.ptr(out),
                    int(out.numel()),
                    d_ebs.data_ptr(),
                    int(plan.ebs.size),
                    d_tasks.data_ptr(),
                    int(plan.tasks.size),
                    None,
                    dev.stream(),
                )
        return out, plan.offsets, plan.block_shapes, plan.block_irreps
