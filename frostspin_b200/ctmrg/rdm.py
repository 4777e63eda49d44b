"""Reduced density matrices from a converged CTMRG environment (device tensors).

Same contraction sequences as frostspin/ctmrg/rdm.py:1-189 (the leg orders are
the algorithm's); the result is normalised by its trace.
"""


def rdm_1x1(C1, T1, C2, T4, A, T2, C4, T3, C3):
    """rdm.py:1-27."""
    right = C3.transpose() @ T2.permute((1,), (0, 2, 3))
    right = right.permute((0, 2, 3), (1,)) @ C2
    down = C4 @ T3.permute((3,), (0, 1, 2))
    r = T1.permute((0, 1, 2), (3,)) @ C1
    r = r @ T4.permute((0,), (1, 2, 3))
    r = r.permute((0, 2, 4, 5), (1, 3)) @ A.permute((2, 5), (0, 1, 3, 4))
    down = down.permute((0, 1, 2), (3,)) @ right.permute((0,), (1, 2, 3))
    down = down.permute((2, 4), (5, 3, 0, 1))
    r = r.permute((0, 6, 3, 7), (1, 2, 4, 5))
    down = down @ r
    down = down.permute((4,), (2, 3, 1, 0, 5))
    r = down @ A.permute((0,), (2, 5, 3, 4, 1)).dagger()
    r /= r.trace()
    return r


def contract_open_corner(C1, T1, T4, A):
    """rdm.py:30-66."""
    ul = T1.permute((1, 2, 0), (3,)) @ C1
    ul = ul @ T4.permute((0,), (1, 2, 3))
    ul = ul.permute((0, 3), (1, 4, 2, 5))
    ul = A.permute((1, 0, 3, 4), (2, 5)) @ ul
    ul = ul.permute((0, 4, 5), (1, 2, 3, 6, 7))
    ul = A.permute((1, 2, 5), (0, 3, 4)).dagger() @ ul
    return ul.permute((3, 0, 4, 1, 6), (5, 2, 7))


def contract_open_corner_mirror(T1, C2, A, T2):
    """rdm.py:69-87."""
    ur = C2 @ T1.permute((0,), (1, 2, 3))
    ur = ur.transpose() @ T2.permute((0,), (2, 3, 1))
    ur = ur.permute((0, 3), (1, 4, 2, 5))
    ur = A.permute((1, 0, 4, 5), (2, 3)) @ ur
    ur = ur.permute((0, 4, 5), (1, 2, 3, 6, 7))
    return A.permute((1, 2, 3), (0, 4, 5)).dagger() @ ur


def rdm_1x2(C1, T1l, T1r, C2, T4, Al, Ar, T2, C4, T3l, T3r, C3):
    """Two sites in a row (rdm.py:90-137)."""
    left = T4.permute((0, 1, 2), (3,)) @ C4
    left = contract_open_corner(C1, T1l, left, Al)
    left = left @ T3l.permute((0, 1, 3), (2,))
    left = left.permute((0, 1), (2, 3, 4, 5))
    right = T2.permute((0, 2, 3), (1,)) @ C3
    right = right.permute((0, 3), (1, 2))
    right = contract_open_corner_mirror(T1r, C2, Ar, right)
    right = right.permute((3, 0, 5, 2, 6), (4, 1, 7))
    right = right @ T3r.permute((0, 1, 2), (3,))
    right = right.permute((2, 3, 4, 5), (0, 1))
    r = (left @ right).permute((1, 3), (0, 2))
    r /= r.trace()
    return r


def rdm_2x1(C1, T1, C2, T4u, Au, T2u, T4d, Ad, T2d, C4, T3, C3):
    """Two sites in a column, through rdm_1x2 on rotated tensors (rdm.py:171-189)."""
    return rdm_1x2(
        C2,
        T2u.permute((1, 2, 3), (0,)),
        T2d.permute((1,), (2, 3, 0)),
        C3.transpose(),
        T1,
        Au.permute((0, 1), (3, 4, 5, 2)),
        Ad.permute((0, 1), (3, 4, 5, 2)),
        T3.permute((2, 3, 0), (1,)),
        C1,
        T4u.permute((1, 2, 3), (0,)),
        T4d.permute((1, 2, 3), (0,)),
        C4.transpose(),
    )


def rdm_symmetrized_1x2(C1, T1l, T4, Al, C4, T3l):
    """Two sites in a row when the right half is the mirror image of the left
    one (environment of SymmetrizedCTMRG, B = rotated dagger of A;
    rdm.py:139-153): the left half is contracted once and reused, permuted."""
    left = T4.permute((0, 1, 2), (3,)) @ C4
    left = contract_open_corner(C1, T1l, left, Al)
    left = left @ T3l.permute((0, 1, 3), (2,))
    left = left.permute((0, 1), (2, 3, 4, 5))
    right = left.permute((3, 2, 5, 4), (1, 0))
    r = (left @ right).permute((1, 3), (0, 2))
    r /= r.trace()
    return r


def rdm_symmetrized_2x1(C1, T1, C2, T4u, Au, T2u):
    """Two sites in a column, symmetrized environment (rdm.py:156-168)."""
    return rdm_symmetrized_1x2(
        C2,
        T2u.permute((1, 2, 3), (0,)),
        T1,
        Au.permute((0, 1), (3, 4, 5, 2)),
        C1,
        T4u.permute((1, 2, 3), (0,)),
    )


def rdm_diag_dr(C1, T1l, ur, T4u, Aul, dl, Adr, T2d, T3r, C3):
    """Second neighbours on the down-right diagonal of a 2x2 plaquette
    (rdm.py:190-238): the open upper-left corner, closed with the enlarged
    down-left and upper-right corners, then the open down-right corner."""
    r = contract_open_corner(C1, T1l, T4u, Aul)
    r = r @ dl
    r = r.permute((2, 3, 4), (0, 1, 5, 6, 7))
    r = ur @ r
    r = r.permute((3, 4), (0, 1, 2, 5, 6, 7))
    dr = contract_open_corner_mirror(
        T2d.permute((1, 2, 3), (0,)),
        C3.transpose(),
        Adr.permute((0, 1, 3, 4), (5, 2)),
        T3r.permute((2, 3), (0, 1)),
    )
    dr = dr.permute((5, 2, 6, 4, 1, 7), (3, 0))
    r = (r @ dr).permute((1, 3), (0, 2))
    r /= r.trace()
    return r


def rdm_diag_ur(ul, T1r, C2, Aur, T2u, T4d, Adl, dr_T, C4, T3l):
    """Second neighbours on the up-right diagonal (rdm.py:241-269), through
    rdm_diag_dr on the plaquette rotated by a quarter turn; dr_T is the
    enlarged down-right corner in transposed leg order."""
    r = rdm_diag_dr(
        C4,
        T4d,
        ul,
        T3l.permute((3,), (0, 1, 2)),
        Adl.permute((0, 1), (5, 2, 3, 4)),
        dr_T,
        Aur.permute((0, 1), (5, 2, 3, 4)),
        T1r.permute((3,), (0, 1, 2)),
        T2u.permute((2, 3, 0), (1,)),
        C2.transpose(),
    )
    return r.permute((1, 0), (3, 2))
