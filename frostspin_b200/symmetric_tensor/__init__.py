from .diagonal_tensor import DiagonalTensor
from .tools import get_symmetric_tensor_type, symmetric_tensor_types
from .u1_symmetric_tensor import U1SymmetricTensor

__all__ = [
    "DiagonalTensor",
    "U1SymmetricTensor",
    "get_symmetric_tensor_type",
    "symmetric_tensor_types",
]
