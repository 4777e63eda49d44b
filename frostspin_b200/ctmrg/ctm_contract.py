"""Enlarged corners and norm contractions of the double-layer CTMRG network.

Same tensor conventions as frostspin/ctmrg/ctm_contract.py:7-162 (leg order
(physical, ancilla, *virtual) for site tensors, clockwise virtual legs starting
from up, environment tensors C1..C4 / T1..T4 clockwise from the upper left):
the leg permutations are part of the algorithm and are kept, as data, so that
the device tensors are the reference's tensors.  Every step is a device
permute or grouped GEMM.
"""

# input permutations that bring (C, Tx, Ty, A) of each corner to the upper-left
# template (frostspin/ctmrg/ctm_contract.py:64-100)
_CORNER_LEGS = {
    "ul": (((1, 2, 0), (3,)), ((0,), (1, 2, 3)), ((0, 1, 3, 4), (2, 5))),
    "ur": (((2, 3, 1), (0,)), ((0,), (1, 2, 3)), ((0, 1, 4, 5), (3, 2))),
    "dr": (((0, 1, 3), (2,)), ((1,), (2, 3, 0)), ((0, 1, 5, 2), (4, 3))),
    "dl": (((1, 2, 0), (3,)), ((3,), (0, 1, 2)), ((0, 1, 2, 3), (5, 4))),
}


def contract_enlarged_corner(C, Tx, Ty, A):
    """C-T//T-A with A and its dagger (ctm_contract.py:7-61); the rank-8
    intermediate is the memory peak 2 a d chi^2 D^4."""
    ul = Tx @ C
    ul = ul @ Ty
    ul = ul.permute((0, 3), (1, 4, 2, 5))
    ul = A @ ul
    ul = ul.permute((0, 1, 4, 5), (2, 3, 6, 7))
    ul = A.permute((0, 1, 4, 5), (2, 3)).dagger() @ ul
    return ul.permute((2, 0, 4), (3, 1, 5))


def _corner(kind, C, Tx, Ty, A):
    tx, ty, a = _CORNER_LEGS[kind]
    return contract_enlarged_corner(C, Tx.permute(*tx), Ty.permute(*ty), A.permute(*a))


def contract_ul(C1, T1, T4, A):
    return _corner("ul", C1, T1, T4, A)


def contract_ur(T1, C2, A, T2):
    return _corner("ur", C2, T2, T1, A)


def contract_dr(A, T2, T3, C3):
    """Transposed with respect to clockwise order, as in the reference."""
    return _corner("dr", C3.transpose(), T3, T2, A)


def contract_dl(T4, A, C4, T3):
    return _corner("dl", C4, T4, T3, A)


def contract_C1234(C1, C2, C4, C3):
    """ctm_contract.py:103-106."""
    up = C2 @ C1
    down = C4 @ C3.transpose()
    return up.full_contract(down)


def contract_T1T3(C1, T1, C2, C4, T3, C3):
    """ctm_contract.py:109-127."""
    left = T1.permute((0, 1, 2), (3,)) @ (C1 @ C4)
    right = T3.permute((3, 0, 1), (2,)) @ (C3.transpose() @ C2)
    right = right.permute((0,), (3, 1, 2))
    return left.full_contract(right)


def contract_T2T4(C1, C2, T4, T2, C4, C3):
    """ctm_contract.py:130-138."""
    left = (C2 @ C1) @ T4.permute((0,), (1, 2, 3))
    down = C4 @ C3.transpose()
    left = left.permute((0, 1, 2), (3,)) @ down
    return left.full_contract(T2.permute((1,), (0, 2, 3)))


def contract_norm(C1, T1, C2, T4, A, T2, C4, T3, C3):
    """ctm_contract.py:141-162."""
    ul = contract_ul(C1, T1, T4, A)
    right = C2.transpose() @ T2.permute((0,), (2, 3, 1))
    up = right.permute((3,), (1, 2, 0)) @ ul
    down = C3 @ T3.permute((2,), (0, 1, 3))
    down = C4 @ down.permute((3,), (1, 2, 0))
    down = down.permute((1, 2, 0), (3,))
    return up.full_contract(down)
