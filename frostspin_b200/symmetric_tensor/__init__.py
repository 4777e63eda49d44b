from .diagonal_tensor import DiagonalTensor
from .o2_symmetric_tensor import O2SymmetricTensor
from .su2_symmetric_tensor import SU2SymmetricTensor
from .tools import get_symmetric_tensor_type, symmetric_tensor_types
from .u1_symmetric_tensor import U1SymmetricTensor

__all__ = [
    "DiagonalTensor",
    "O2SymmetricTensor",
    "SU2SymmetricTensor",
    "U1SymmetricTensor",
    "get_symmetric_tensor_type",
    "symmetric_tensor_types",
]
