"""Plugin registry for SymmetricTensor types (frostspin/symmetric_tensor/tools.py:5-23)."""

symmetric_tensor_types = {}


def get_symmetric_tensor_type(symmetry):
    """SymmetricTensor subclass implementing ``symmetry`` ("U1", ...)."""
    try:
        return symmetric_tensor_types[symmetry]
    except KeyError:
        msg = f"Unknown symmetry '{symmetry}'"
        raise RuntimeError(msg) from None


def check_norm(t1, t2, *, tol=4e-13):
    """Relative norm agreement check used as a debug invariant (tools.py:26-39)."""
    n1 = t1.norm() if hasattr(t1, "norm") else float((t1**2).sum() ** 0.5)
    n2 = t2.norm() if hasattr(t2, "norm") else float((t2**2).sum() ** 0.5)
    return abs(n1 - n2) <= tol * max(n1, n2)
