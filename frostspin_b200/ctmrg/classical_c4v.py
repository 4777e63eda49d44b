"""C4v-symmetric classical CTMRG on the square lattice (single layer).

Mirrors examples/ising_classical_ctmrg.py:115-304 (iterate_ctm, env_1site,
env_2sites) of the reference: the corner is kept as its eigenvalue spectrum s
(a DiagonalTensor) and the edge as T (chi, D, chi).  Works for any abelian
device SymmetricTensor; the Ising site tensors are built in the Z2 basis
exactly as the reference example does (:44-64, :362-384).
"""

import numpy as np
import scipy.linalg as lg
import torch

from ..symmetric_tensor import DiagonalTensor, U1SymmetricTensor


def iterate_c4v(s, T, a, a2, chi_target):
    """One C4v CTMRG iteration (examples/ising_classical_ctmrg.py:115-204)."""
    Tp = T.permute((0, 1), (2,))
    matC = Tp * s
    matC = matC @ T
    matC = matC.permute((1, 2), (0, 3))
    matC = a2 @ matC
    matC = matC.permute((0, 2), (1, 3))
    news, U = matC.truncated_eigh(chi_target)
    news /= news.norm_device()
    newT = U.permute((1,), (0, 2))
    newT = Tp @ newT
    newT = newT.permute((1, 2), (0, 3))
    newT = a @ newT
    newT = newT.permute((0, 2), (1, 3))
    newT = U.dagger() @ newT
    newT /= newT.norm_device()
    return news, newT


def iterate_c4v_many(runs):
    """One iteration of many independent C4v runs advanced in lock step:
    runs is a list of (s, T, a, a2, chi_target); returns [(s, T)].  Each run
    does exactly what iterate_c4v does (examples/ising_classical_ctmrg.py
    :115-204), but every step issues its sector GEMMs of all runs as one
    grouped launch and its permutes of all runs as one multi-buffer launch
    (linalg.shared_launches), and the corner eigendecompositions of all runs
    are batched by block size."""
    from .. import linalg
    from ..symmetric_tensor.symmetric_tensor import SymmetricTensor

    def each(fn, *lists):
        with linalg.shared_launches():
            return [fn(*xs) for xs in zip(*lists, strict=True)]

    ss = [r[0] for r in runs]
    Ts = [r[1] for r in runs]
    As = [r[2] for r in runs]
    A2s = [r[3] for r in runs]
    chis = [r[4] for r in runs]
    Tp = each(lambda T: T.permute((0, 1), (2,)), Ts)
    mat = [t * s for t, s in zip(Tp, ss, strict=True)]
    mat = each(lambda m, T: m @ T, mat, Ts)
    mat = each(lambda m: m.permute((1, 2), (0, 3)), mat)
    mat = each(lambda a2, m: a2 @ m, A2s, mat)
    mat = each(lambda m: m.permute((0, 2), (1, 3)), mat)
    eig = SymmetricTensor.truncated_eigh_many(mat, chis)
    news = [s for s, _ in eig]
    Us = [u for _, u in eig]
    for s in news:
        s /= s.norm_device()
    nT = each(lambda U: U.permute((1,), (0, 2)), Us)
    nT = each(lambda tp, t: tp @ t, Tp, nT)
    nT = each(lambda t: t.permute((1, 2), (0, 3)), nT)
    nT = each(lambda a, t: a @ t, As, nT)
    nT = each(lambda t: t.permute((0, 2), (1, 3)), nT)
    nT = each(lambda U, t: U.dagger() @ t, Us, nT)
    for t in nT:
        t /= t.norm_device()
    return list(zip(news, nT, strict=True))


def env_1site(s, T):
    """examples/ising_classical_ctmrg.py:207-251."""
    Tp = T.permute((0, 1), (2,))
    corner = Tp * s
    half = corner @ corner.permute((0,), (1, 2))
    left = half.permute((1, 2), (0, 3))
    right = half.permute((3, 0), (1, 2))
    full = left @ right
    return full.permute((0, 3), (2, 1))


def env_2sites(s, T):
    """examples/ising_classical_ctmrg.py:254-304."""
    Tp = T.permute((0, 1), (2,))
    env = Tp * s
    env = env @ env.permute((0,), (1, 2))
    env = Tp @ env.permute((0,), (1, 2, 3))
    left = env.permute((1, 2, 3), (0, 4))
    right = env.permute((4, 0), (1, 2, 3))
    return left @ right


def ising_site_tensors(beta):
    """Z2-basis Ising tensors (a, a2) plus dense a0 and the magnetisation
    operator in the same basis (examples/ising_classical_ctmrg.py:44-64,
    :362-384)."""
    d = 2
    h = -2 * np.eye(2) + 1
    sq_bw = lg.sqrtm(np.exp(-beta * h)).real
    delta = np.zeros((d,) * 4)
    delta[0, 0, 0, 0] = delta[1, 1, 1, 1] = 1
    a0 = np.einsum("abcd,ai,bj,ck,dl->ijkl", delta, sq_bw, sq_bw, sq_bw, sq_bw)
    mop = delta.copy()
    mop[1, 1, 1, 1] = -1
    mop = np.einsum("abcd,ai,bj,ck,dl->ijkl", mop, sq_bw, sq_bw, sq_bw, sq_bw)
    K = np.array([[-1.0, 1.0], [1.0, 1.0]]) / np.sqrt(2)
    a0d = np.einsum("abcd,ai,bj,ck,dl->ijkl", a0, K, K, K, K)
    mopd = np.einsum("abcd,ai,bj,ck,dl->ijkl", mop, K, K, K, K)
    rep = np.array([-128, 0], dtype=np.int8)
    siga = np.array([False, False, True, True])
    a = U1SymmetricTensor.from_array(a0d, (rep, rep), (rep, rep), signature=siga)
    siga2 = np.array([False, True, True, True])
    a2 = U1SymmetricTensor(a.row_reps, a.col_reps, a.blocks, a.block_irreps, siga2)
    return a, a2, a0d, mopd


def ising_initial_environment(chi, rng):
    """Seeded Z2 corner spectrum and symmetric edge tensor
    (examples/ising_classical_ctmrg.py:386-412)."""
    d0o = d0e = chi // 2
    s_odd = rng.normal(size=(d0o,))
    s_odd = s_odd[np.abs(s_odd).argsort()[::-1]] / lg.norm(s_odd)
    s_even = rng.normal(size=(d0e,))
    s_even = s_even[np.abs(s_even).argsort()[::-1]] / lg.norm(s_even)
    corner = np.array([-128] * d0o + [0] * d0e, dtype=np.int8)
    s = DiagonalTensor(
        (s_odd, s_even), corner, np.array([-128, 0], dtype=np.int8), [1, 1], "U1"
    )
    rep = np.array([-128, 0], dtype=np.int8)
    sigT = np.array([False, False, True])
    T = U1SymmetricTensor.random((corner,), (rep, corner), signature=sigT, rng=rng)
    temp = U1SymmetricTensor((corner,), (rep, corner), T.blocks, T.block_irreps, [1, 0, 0])
    T = T + temp.permute((2,), (1, 0))
    T /= T.norm()
    return s, T


def energy_per_bond(s, T, a0d, mopd):
    """-<s_i s_j> on one bond from the two-site environment; the reference
    example prints the per-site energy, 2 bonds (:344-350)."""
    env2 = env_2sites(s, T).toarray()
    nr = np.einsum("abcdef,bgdc,afeg->", env2, a0d, a0d)
    sdsr = np.einsum("abcdef,bgdc,afeg->", env2, mopd, mopd)
    return -sdsr / nr


def edge_transfer_spectrum(T, nvals=4):
    """Leading eigenvalues (by modulus, largest first) of the edge transfer
    operator of the C4v environment: M[(l1, l2), (r1, r2)] = sum_p T[l1, p, r1]
    T[l2, p, r2], the chi^2 x chi^2 operator of two edge tensors contracted
    over the physical leg.  Formed with the device block operations (one
    grouped GEMM and one permute); its sectors are diagonalised on the device.
    The corner representation must be self-conjugate (Z2), so that the row
    pairs (l1, l2) and column pairs (r1, r2) of a sector are the same states in
    the same order."""
    Tr = T.permute((0, 2), (1,))
    M = (Tr @ Tr.dagger()).permute((0, 2), (1, 3))
    vals = []
    for b in M.blocks:
        if b.shape[0] != b.shape[1]:
            raise ValueError("edge transfer sector is not square: corner not self-conjugate")
        if b.shape[0]:
            vals.append(torch.linalg.eigvals(b.contiguous()))
    lam = torch.cat(vals).cpu().numpy()
    return lam[np.argsort(-np.abs(lam), kind="stable")][:nvals]


def correlation_length(T):
    """xi = -1 / ln|lambda_2 / lambda_1| of the edge transfer operator
    (edge_transfer_spectrum), in lattice spacings."""
    lam = edge_transfer_spectrum(T, 2)
    return -1.0 / np.log(abs(lam[1]) / abs(lam[0]))
