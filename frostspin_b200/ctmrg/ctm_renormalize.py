"""Projectors and renormalisation of the double-layer CTMRG, on the device.

Follows frostspin/ctmrg/ctm_renormalize.py:6-341.  construct_projectors works
sector by sector on the irreps shared by the four corners: R = c1 c2,
Rt = c3 c4 and M = R Rt are grouped GEMMs over all sectors (one launch each),
M is decomposed per sector on the device, the kept multiplets are chosen by the
same greedy find_block_cuts, and P = s^-1/2 U^T R, Pt = Rt V^T s^-1/2 are again
grouped GEMMs.
"""

import numpy as np
import torch

from .. import linalg
from ..misc_tools.svd_tools import find_block_cuts, truncated_svd_blocks


def _block_index(tensor, irreps):
    idx = np.searchsorted(tensor.block_irreps, irreps)
    return idx


def construct_projectors(
    corner1,
    corner2,
    corner3,
    corner4,
    chi_target,
    last_renormalized,
    *,
    block_chi_ratio=1.1,
    ncv_ratio=2.0,
    atol=0.0,
    rtol=None,
    degen_ratio=1.0,
):
    """ctm_renormalize.py:6-136.  Returns (P, Pt)."""
    shared = np.intersect1d(
        np.intersect1d(corner1.block_irreps, corner2.block_irreps),
        np.intersect1d(corner3.block_irreps, corner4.block_irreps),
    )
    i1 = _block_index(corner1, shared)
    i2 = _block_index(corner2, shared)
    i3 = _block_index(corner3, shared)
    i4 = _block_index(corner4, shared)
    b1, b2, b3, b4 = corner1.blocks, corner2.blocks, corner3.blocks, corner4.blocks

    # number of values to compute per sector: the last kept count + margin
    # (ctm_renormalize.py:79-88)
    block_chi = np.zeros(shared.shape, dtype=int)
    last = last_renormalized.block_irreps
    pos = np.searchsorted(last, shared)
    for bi, ind in enumerate(pos):
        if ind < last.size and shared[bi] == last[ind]:
            block_chi[bi] = last_renormalized.block_shapes[ind][1]
    block_chi = np.maximum(block_chi + 10, (block_chi_ratio * block_chi).astype(int))
    block_chi = np.minimum(chi_target + 10, block_chi)

    _, _, _, r_blocks = linalg.matmul_blocks([b1[i] for i in i1], [b2[i] for i in i2])
    _, _, _, rt_blocks = linalg.matmul_blocks([b3[i] for i in i3], [b4[i] for i in i4])
    _, _, _, m_blocks = linalg.matmul_blocks(r_blocks, rt_blocks)

    dims = np.array([corner2.irrep_dimension(corner2.block_irreps[i]) for i in i2], dtype=int)
    fulls = []
    for bi, m in enumerate(m_blocks):
        ncv = int(ncv_ratio * block_chi[bi]) + 10
        fulls.append(min(m.shape) < max(100, 4 * ncv))
    u_blocks, s_blocks, v_blocks = truncated_svd_blocks(m_blocks, block_chi, fulls)

    host_s = [s.detach().cpu().numpy() for s in s_blocks]
    cuts = find_block_cuts(host_s, chi_target, dims=dims, atol=atol, rtol=rtol,
                           degen_ratio=degen_ratio)
    non_empty = np.flatnonzero(cuts)

    lefts_p, rights_p, lefts_pt, rights_pt, scales = [], [], [], [], []
    for bi in non_empty:
        cut = int(cuts[bi])
        s12 = torch.rsqrt(s_blocks[bi][:cut])
        scales.append(s12)
        # P^T block = s^-1/2 U^H R : scale the rows of U^H through its columns
        lefts_p.append((u_blocks[bi][:, :cut] * s12).T)
        rights_p.append(r_blocks[bi])
        lefts_pt.append(rt_blocks[bi])
        rights_pt.append(v_blocks[bi][:cut].T * s12)
    _, _, _, p_blocks = linalg.matmul_blocks(lefts_p, rights_p)
    _, _, _, pt_blocks = linalg.matmul_blocks(lefts_pt, rights_pt)

    block_irreps = corner2.block_irreps[i2[non_empty]]
    mid_rep = corner2.init_representation(cuts[non_empty], block_irreps)
    nrr2 = corner2.n_row_reps
    sp = np.zeros(nrr2 + 1, dtype=bool)
    sp[1:] = corner2.signature[nrr2:]
    spt = np.ones(nrr2 + 1, dtype=bool)
    spt[:-1] = ~corner2.signature[nrr2:]
    ST = type(corner2)
    P = ST((mid_rep,), corner2.col_reps, p_blocks, block_irreps, sp).transpose()
    Pt = ST(corner2.col_reps, (mid_rep,), pt_blocks, block_irreps, spt)
    return P, Pt


# ------------------------------------------------------------------ renormalise


def renormalize_T(Pt, T, A, P):
    """ctm_renormalize.py:145-166."""
    nT = T @ P.permute((2,), (0, 1, 3))
    nT = nT.permute((0, 3), (1, 4, 2, 5))
    nT = A @ nT
    nT = nT.permute((0, 1, 4, 5), (2, 3, 6, 7))
    nT = A.permute((0, 1, 4, 5), (2, 3)).dagger() @ nT
    nT = nT.permute((3, 1, 4), (2, 0, 5))
    nT = Pt.transpose() @ nT
    nT /= nT.norm_device()
    return nT


def renormalize_corner_P(C, T, P):
    """ctm_renormalize.py:169-193."""
    nC = (T @ C).permute((0,), (1, 2, 3)) @ P
    nC /= nC.norm_device()
    return nC


def renormalize_corner_Pt(C, T, Pt):
    """ctm_renormalize.py:196-216."""
    nC = (T @ C).permute((0,), (1, 2, 3)) @ Pt
    nC /= nC.norm_device()
    return nC


def renormalize_quadrant(P, quadrant, Pt):
    """ctm_renormalize.py:219-225."""
    nc = P.transpose() @ quadrant @ Pt
    nc /= nc.norm_device()
    return nc


# per direction: leg permutations of the edge and site tensors around the
# generic routines (ctm_renormalize.py:228-341)
def renormalize_C1_up(C1, T4, P):
    return renormalize_corner_P(C1.transpose(), T4.permute((3, 1, 2), (0,)), P).transpose()


def renormalize_T1(Pt, T1, A, P):
    nT = renormalize_T(Pt, T1.permute((1, 2, 3), (0,)), A.permute((0, 1, 4, 5), (2, 3)), P)
    return nT.permute((3,), (1, 2, 0))


def renormalize_C2_up(C2, T2, Pt):
    return renormalize_corner_Pt(C2, T2.permute((1, 2, 3), (0,)), Pt)


def renormalize_C2_right(C2, T1, P):
    return renormalize_corner_P(C2.transpose(), T1.permute((3, 1, 2), (0,)), P).transpose()


def renormalize_T2(Pt, T2, A, P):
    nT = renormalize_T(Pt, T2.permute((2, 3, 0), (1,)), A.permute((0, 1, 5, 2), (3, 4)), P)
    return nT.permute((0,), (3, 1, 2))


def renormalize_C3_right(C3, T3, Pt):
    return renormalize_corner_Pt(C3.transpose(), T3.permute((3, 0, 1), (2,)), Pt).transpose()


def renormalize_C3_down(C3, T2, P):
    return renormalize_corner_P(C3, T2.permute((0, 2, 3), (1,)), P)


def renormalize_T3(Pt, T3, A, P):
    nT = renormalize_T(Pt, T3.permute((0, 1, 2), (3,)), A.permute((0, 1, 2, 3), (4, 5)), P)
    return nT.permute((1, 2, 0), (3,))


def renormalize_C4_down(C4, T4, Pt):
    return renormalize_corner_Pt(C4, T4.permute((0, 1, 2), (3,)), Pt)


def renormalize_C4_left(C4, T3, P):
    return renormalize_corner_P(C4.transpose(), T3.permute((2, 0, 1), (3,)), P).transpose()


def renormalize_T4(Pt, T4, A, P):
    nT = renormalize_T(Pt, T4.permute((1, 2, 3), (0,)), A.permute((0, 1, 3, 4), (5, 2)), P)
    return nT.permute((3,), (1, 2, 0))


def renormalize_C1_left(C1, T1, Pt):
    return renormalize_corner_Pt(C1, T1.permute((0, 1, 2), (3,)), Pt)
