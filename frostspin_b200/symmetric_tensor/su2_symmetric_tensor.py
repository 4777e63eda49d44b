"""SU(2)-symmetric tensor on the device.

Mirrors frostspin/symmetric_tensor/su2_symmetric_tensor.py.  A representation is
a 2 x n int array: first row the degeneracy (external multiplicity) of each
irrep, second row the irrep, labelled by its dimension 2 s + 1, sorted
increasingly.  The basis of an irrep is ordered by decreasing S_z.

Everything structural (fusion of representations, Clebsch-Gordan fusion tensors
and trees, the recoupling isometries of a permute) is host work on small
arrays, cached per structure; block data only ever lives on the device and is
moved by the kernels behind LieGroupSymmetricTensor.
"""

import json
from functools import lru_cache

import numpy as np

from . import su2_cg
from .lie_group_symmetric_tensor import LieGroupSymmetricTensor
from .tools import symmetric_tensor_types


def elementary_combine(degen1, irreps1, degen2, irreps2):
    """Fusion of two SU(2) representations (su2_symmetric_tensor.py:109-119):
    d1 x d2 = |d1 - d2| + 1, |d1 - d2| + 3, ..., d1 + d2 - 1."""
    degen = np.zeros(int(irreps1[-1]) + int(irreps2[-1]) - 1, dtype=np.int64)
    for d1, i1 in zip(degen1, irreps1, strict=True):
        for d2, i2 in zip(degen2, irreps2, strict=True):
            degen[abs(int(i1) - int(i2)) : int(i1) + int(i2) - 1 : 2] += int(d1) * int(d2)
    nz = degen.nonzero()[0]
    return degen[nz], nz + 1


def combine_reps(reps):
    """su2_symmetric_tensor.py:122-127."""
    degen, irreps = np.asarray(reps[0][0]), np.asarray(reps[0][1])
    for r in reps[1:]:
        degen, irreps = elementary_combine(degen, irreps, r[0], r[1])
    return np.array([degen, irreps], dtype=np.int64)


@lru_cache(maxsize=None)
def _reversal_signs(irr):
    """Signs of the S_z-reversal map on irrep irr, applied after reversing the
    basis (su2_symmetric_tensor.py:66, :71)."""
    return np.arange(irr % 2, irr + irr % 2) % 2 * 2 - 1


@lru_cache(maxsize=None)
def _signed_cg(irr1, irr2, irr3, s1, s2):
    p = su2_cg.cg_tensor(irr1, irr2, irr3)
    if s1:
        p = p[::-1] * _reversal_signs(irr1)[:, None, None]
    if s2:
        p = p[:, ::-1] * _reversal_signs(irr2)[None, :, None]
    p = np.ascontiguousarray(p)
    p.setflags(write=False)
    return p


def compute_fusion_tensor(rep1, rep2, s1, s2, *, max_irrep=2**30):
    """Clebsch-Gordan fusion tensor of rep1 x rep2 with signatures s1, s2,
    truncated above max_irrep (su2_symmetric_tensor.py:12-106).

    Returns (new_rep, projector) with projector of shape (dim1, dim2, dim3): the
    output axis holds, irrep by irrep, d1 * d2 copies (i3 = i1 * d2 + i2) of the
    irrep for every pair of input irreps, in input order.  A signature True
    applies the spin-reversal map to that input.
    """
    rep1 = np.asarray(rep1)
    rep2 = np.asarray(rep2)
    degen, irreps = elementary_combine(rep1[0], rep1[1], rep2[0], rep2[1])
    trunc = int(np.searchsorted(irreps, max_irrep + 1))
    degen = degen[:trunc]
    irreps = irreps[:trunc]
    projector = np.zeros(
        (int(rep1[0] @ rep1[1]), int(rep2[0] @ rep2[1]), int(degen @ irreps))
    )
    if trunc == 0:
        return np.zeros((2, 0), dtype=np.int64), projector
    start3 = {}
    n = 0
    for d3, irr3 in zip(degen, irreps, strict=True):
        start3[int(irr3)] = n
        n += int(d3 * irr3)
    shift1 = 0
    for d1, irr1 in zip(rep1[0], rep1[1], strict=True):
        d1, irr1 = int(d1), int(irr1)
        shift2 = 0
        for d2, irr2 in zip(rep2[0], rep2[1], strict=True):
            d2, irr2 = int(d2), int(irr2)
            for irr3 in range(abs(irr1 - irr2) + 1, min(irr1 + irr2, max_irrep + 1), 2):
                p = _signed_cg(irr1, irr2, irr3, bool(s1), bool(s2))
                s3 = start3[irr3]
                for i1 in range(d1):
                    a = shift1 + i1 * irr1
                    for i2 in range(d2):
                        b = shift2 + i2 * irr2
                        c = s3 + (i1 * d2 + i2) * irr3
                        projector[a : a + irr1, b : b + irr2, c : c + irr3] = p
                start3[irr3] = s3 + d1 * d2 * irr3
            shift2 += d2 * irr2
        shift1 += d1 * irr1
    return np.array([degen, irreps], dtype=np.int64), projector


def _o2_leg(rep):
    """O(2) representation of one SU(2) leg, the state order that takes the
    leg to O(2) order and the sign of every state (su2_symmetric_tensor.py:
    272-304).  States of a multiplet of dimension irr have 2 S_z = irr - 1,
    irr - 3, ..., 1 - irr.  O(2) label: |2 S_z|, or -1 (0odd) for S_z = 0 when
    irr = 3 mod 4.  Sign -1 for S_z < 0 with 2 S_z = irr + 1 (mod 4) for integer
    spin, 2 S_z = irr - 1 (mod 4) for half-integer spin.  Order: label
    ascending, then S_z descending, then multiplet order."""
    sz, lab, neg = [], [], []
    for d, irr in zip(np.asarray(rep[0]), np.asarray(rep[1]), strict=True):
        irr = int(irr)
        s = np.arange(irr - 1, -irr, -2, dtype=np.int64)
        lb = np.abs(s)
        if irr % 4 == 3:
            lb[irr // 2] = -1
        target = (irr + 1) % 4 if irr % 2 else (irr - 1) % 4
        flip = (s < 0) & (s % 4 == target)
        sz.append(np.tile(s, int(d)))
        lab.append(np.tile(lb, int(d)))
        neg.append(np.tile(flip, int(d)))
    sz = np.concatenate(sz)
    lab = np.concatenate(lab)
    sign = 1.0 - 2.0 * np.concatenate(neg)
    order = np.lexsort((-sz, lab))
    irreps, degen = np.unique(lab, return_counts=True)
    degen[irreps > 0] //= 2
    return np.array([degen, irreps], dtype=np.int64), order, sign


class SU2SymmetricTensor(LieGroupSymmetricTensor):
    """SU(2) SymmetricTensor (su2_symmetric_tensor.py:130-338)."""

    _symmetry = "SU2"

    @staticmethod
    def singlet():
        return np.ones((2, 1), dtype=int)

    @staticmethod
    def combine_representations(reps, _signature):
        if len(reps) > 1:
            return combine_reps(reps)
        return reps[0]

    @staticmethod
    def conjugate_irrep(irr):
        return irr

    @staticmethod
    def conjugate_representation(rep):
        return rep

    @staticmethod
    def representation_dimension(rep):
        return int(rep[0] @ rep[1])

    @staticmethod
    def irrep_dimension(irr):
        return int(irr)

    @classmethod
    def compute_clebsch_gordan_tree(cls, rep_in, signature, *, target_irreps=None):
        """Chained fusion tensor of rep_in, only the first leg with depth
        (su2_symmetric_tensor.py:178-218).  Intermediate irreps that cannot fuse
        down to the largest target irrep are dropped, which removes only columns
        of irreps above that target.  Returns (rep, matrix (dim_in, dim_out))."""
        n = len(rep_in)
        if n == 1:
            rep_in = [rep_in[0], np.ones((2, 1), dtype=np.int64)]
            signature = [signature[0], False]
            n = 2
        if target_irreps is None:
            max_irrep = 2**30
        else:
            max_irrep = int(target_irreps[-1]) + sum(int(r[1, -1]) for r in rep_in[2:]) - n + 2
        nr, p = compute_fusion_tensor(
            rep_in[0], rep_in[1], signature[0], signature[1], max_irrep=max_irrep
        )
        if nr.size == 0:
            return nr, np.zeros((p.shape[0] * p.shape[1], 0))
        proj = p
        for i in range(2, n):
            max_irrep -= int(rep_in[i][1, -1]) - 1
            nr, p = compute_fusion_tensor(nr, rep_in[i], False, signature[i], max_irrep=max_irrep)
            if nr.size == 0:
                return nr, np.zeros((p.shape[0] * p.shape[1], 0))
            proj = proj.reshape(-1, p.shape[0]) @ p.reshape(p.shape[0], -1)
        return nr, proj.reshape(-1, p.shape[2])

    # ------------------------------------------------------------- casts
    def toSU2(self):
        return self

    def toabelian(self):
        return self.toU1()

    def toU1(self):
        """su2_symmetric_tensor.py:229-247: every multiplet is expanded into its
        S_z states (2 S_z as int8, decreasing), through the dense tensor."""
        from .u1_symmetric_tensor import U1SymmetricTensor

        reps = []
        for r in self._row_reps + self._col_reps:
            sz = [
                np.tile(np.arange(irr - 1, -irr - 1, -2, dtype=np.int8), int(d))
                for d, irr in zip(r[0], r[1], strict=True)
            ]
            reps.append(np.concatenate(sz))
        out = U1SymmetricTensor.from_array(
            self.toarray(), reps[: self._nrr], reps[self._nrr :], self._signature
        )
        if __debug__:
            n1, n2 = self.norm(), out.norm()
            assert abs(n1 - n2) <= 1e-13 * max(n1, 1.0)
        return out

    def toO2(self):
        """su2_symmetric_tensor.py:249-318, through the dense tensor as in the
        reference.  Every leg is reordered into O(2) order (label |2 S_z|,
        except S_z = 0 of an odd integer spin, which is 0odd; +n states before
        -n states) and some S_z < 0 basis vectors change sign to follow the
        O(2) reflection convention; the result is a gauge transform of the
        tensor, invisible once legs are contracted."""
        from .o2_symmetric_tensor import O2SymmetricTensor

        arr = self.toarray()
        o2_reps = []
        for ax, r in enumerate(self._row_reps + self._col_reps):
            rep, order, sign = _o2_leg(r)
            o2_reps.append(rep)
            shape = [1] * arr.ndim
            shape[ax] = sign.size
            arr = np.take(arr * sign.reshape(shape), order, axis=ax)
        out = O2SymmetricTensor.from_array(arr, o2_reps[: self._nrr], o2_reps[self._nrr :],
                                           self._signature)
        if __debug__:
            n1, n2 = self.norm(), out.norm()
            assert abs(n1 - n2) <= 1e-13 * max(n1, 1.0)
        return out

    # --------------------------------------------------- Clebsch-Gordan data
    @classmethod
    def reload_clebsch_gordan(cls, savefile, *, verbosity=0):
        """Replace the on-demand coefficients by a table in the reference's file
        formats (frostspin/groups/su2_clebsch_gordan.py:38-108): json with keys
        "d1,d2,d3" -> [flat indices, values], or npz with i_d1_d2_d3 / c_d1_d2_d3."""
        table = {}
        if str(savefile).endswith(".json"):
            with open(savefile, encoding="utf8") as fin:
                data = json.load(fin)
            for key, val in data.items():
                if key.startswith("!"):
                    continue
                sh = tuple(int(x) for x in key.split(","))
                table[sh] = (np.asarray(val[0], dtype=np.int64), np.asarray(val[1]))
        elif str(savefile).endswith(".npz"):
            with np.load(savefile) as data:
                for key in data.files:
                    if key[0] == "i":
                        sh = tuple(int(x) for x in key[2:].split("_"))
                        table[sh] = (data[key], data["c" + key[1:]])
        else:
            raise RuntimeError("Invalid file extension: must be json or npz")
        su2_cg.set_table(table)
        _signed_cg.cache_clear()
        cls.clear_structure_caches()
        if verbosity > 0:
            print("Clebsch-Gordan maximal spin dimension =", max(k[0] for k in table))


symmetric_tensor_types["SU2"] = SU2SymmetricTensor
