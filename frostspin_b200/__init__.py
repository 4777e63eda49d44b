"""frostspin_b200: block-sparse symmetric tensors for CTMRG and simple update on
NVIDIA B200 (sm_100a).

Device-resident SymmetricTensor types mirror the interface of frostspin 1.0.0
(ogauthe/frostspin); their data plane is a C-ABI CUDA library
(include/frostspin_b200.h) built in-tree by ``frostspin_b200.build``.
"""

from .linalg import gemm_precision, gemm_precision_mode, set_gemm_precision
from .symmetric_tensor import (
    DiagonalTensor,
    O2SymmetricTensor,
    SU2SymmetricTensor,
    U1SymmetricTensor,
    get_symmetric_tensor_type,
)

__version__ = "0.1.0"

__all__ = [
    "DiagonalTensor",
    "O2SymmetricTensor",
    "SU2SymmetricTensor",
    "U1SymmetricTensor",
    "gemm_precision",
    "gemm_precision_mode",
    "get_symmetric_tensor_type",
    "set_gemm_precision",
]
