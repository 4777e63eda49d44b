"""U(1) symmetric device tensor (Z2 is U(1) with irreps {-128, 0}).

Mirrors frostspin/symmetric_tensor/u1_symmetric_tensor.py:8-57.
"""

import numpy as np

from .abelian_plan import to_int8
from .abelian_symmetric_tensor import AbelianSymmetricTensor
from .tools import symmetric_tensor_types


def combine_u1(reps, signature):
    """Fused irreps of a leg group: Kronecker sum of (1 - 2 s) * rep in int8 with
    wraparound (u1_symmetric_tensor.py:8-19, :36-40)."""
    signature = np.asarray(signature, dtype=bool)
    c0 = (1 - 2 * signature[0].astype(np.int64)) * np.asarray(reps[0], dtype=np.int64)
    for r, s in zip(reps[1:], signature[1:], strict=True):
        rs = (1 - 2 * int(s)) * np.asarray(r, dtype=np.int64)
        c0 = (c0[:, None] + rs[None, :]).ravel()
    return ((c0 + 128) % 256 - 128).astype(np.int8)


class U1SymmetricTensor(AbelianSymmetricTensor):
    _symmetry = "U1"

    @staticmethod
    def combine_representations(reps, signature):
        signature = np.asarray(signature, dtype=bool)
        if signature.shape != (len(reps),):
            raise ValueError("signature does not match representations")
        return combine_u1(reps, signature)

    @staticmethod
    def conjugate_irrep(irr):
        return to_int8(-np.asarray(irr, dtype=np.int64))

    @staticmethod
    def conjugate_representation(rep):
        return to_int8(-np.asarray(rep, dtype=np.int64))

    def toU1(self):
        return self


symmetric_tensor_types["U1"] = U1SymmetricTensor
