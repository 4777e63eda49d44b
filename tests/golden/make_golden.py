#!/usr/bin/env python
"""Generate golden fixtures from the reference frostspin implementation.

Run where the reference tree is available (read-only), naming it:

    FROSTSPIN_REFERENCE=<path of the reference tree> python -O tests/golden/make_golden.py

It imports frostspin 1.0.0 from that tree, builds seeded inputs, runs the
reference's own operations and stores inputs and outputs as .npz files next to
this script.  The fixtures are what pins the CPU oracle (oracle/) and, through
it and directly, the device path.  Nothing at test time reads the reference.
"""

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("FROSTSPIN_REFERENCE")
if not REF:
    sys.exit("set FROSTSPIN_REFERENCE to the path of the reference (frostspin 1.0.0) tree")
if REF not in sys.path:
    sys.path.insert(0, REF)

from frostspin import DiagonalTensor, U1SymmetricTensor  # noqa: E402
from frostspin.misc_tools.svd_tools import find_block_cuts  # noqa: E402


def pack_tensor(prefix, t, data):
    """Store a reference SymmetricTensor with its own get_data_dic format."""
    d = t.get_data_dic(prefix=prefix)
    for k, v in d.items():
        data[k] = np.asarray(v)


def pack_diag(prefix, s, data):
    for k, v in s.get_data_dic(prefix=prefix).items():
        data[k] = np.asarray(v)


def save(name, data):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **data)
    print("wrote", path, os.path.getsize(path), "bytes")


def case_u1_reference_test():
    """Shapes and signature of the reference's tests/test_u1_tensor.py:46-56."""
    rng = np.random.default_rng(42)
    c1 = np.array([-2, 0, 2], dtype=np.int8)
    c2 = np.array([-3, -1, 1, 3], dtype=np.int8)
    c3 = np.array([-2, -2, 0, 0, 0, 2, 2], dtype=np.int8)
    c4 = np.array([-2, -1, 0, 1, 2], dtype=np.int8)
    c5 = np.array([-3, -1, 0, 2], dtype=np.int8)
    sig = np.array([1, 0, 0, 1, 1], dtype=bool)
    t = U1SymmetricTensor.random((c1, c2), (c3, c4, c5), signature=sig, rng=rng)
    data = {}
    pack_tensor("in", t, data)
    perms = [
        ((3, 0, 2), (1, 4)),
        ((3,), (1, 0, 4, 2)),
        ((2, 3, 4), (0, 1)),
        ((4, 1), (0, 3, 2)),
        ((0, 1, 2, 3), (4,)),
    ]
    for i, (ra, ca) in enumerate(perms):
        p = t.permute(ra, ca)
        pack_tensor(f"perm{i}", p, data)
        data[f"perm{i}_axes"] = np.array(ra + ca)
        data[f"perm{i}_nrr"] = np.array(len(ra))
        data[f"perm{i}_dense"] = p.toarray()
    pack_tensor("transpose", t.transpose(), data)
    pack_tensor("dagger", t.dagger(), data)
    data["dense"] = t.toarray()
    data["norm"] = np.array(t.norm())
    data["full_contract_dagger"] = np.array(t.full_contract(t.dagger()))
    # matmul: t (2 rows | 3 cols) @ t.dagger() (3 rows | 2 cols)
    m = t @ t.dagger()
    pack_tensor("matmul", m, data)
    data["matmul_trace"] = np.array(m.trace())
    # svd reconstruction and truncated svd spectra
    u, s, v = t.svd()
    pack_diag("svd_s", s, data)
    ut, st, vt = t.truncated_svd(6)
    pack_diag("tsvd_s", st, data)
    pack_tensor("tsvd_usv", (ut * st) @ vt, data)
    save("u1_reference_test", data)


def z2_rep(pattern):
    return np.array([-128 if c == "o" else 0 for c in pattern], dtype=np.int8)


def case_z2_rank6():
    """Z2 tensors with unsorted (interleaved) representations, rank 6."""
    rng = np.random.default_rng(7)
    reps = [z2_rep("eoeeo"), z2_rep("oe"), z2_rep("eeoo"), z2_rep("oeo"),
            z2_rep("e"), z2_rep("oeeo")]
    sig = np.array([0, 1, 1, 0, 1, 0], dtype=bool)
    t = U1SymmetricTensor.random(tuple(reps[:3]), tuple(reps[3:]), signature=sig,
                                 rng=rng)
    data = {}
    pack_tensor("in", t, data)
    perms = [
        ((0, 2, 4), (1, 3, 5)),
        ((5, 1), (2, 0, 4, 3)),
        ((3, 4, 5, 0, 1), (2,)),
        ((2,), (5, 4, 3, 1, 0)),
        ((1, 0, 3, 2), (5, 4)),
    ]
    for i, (ra, ca) in enumerate(perms):
        p = t.permute(ra, ca)
        pack_tensor(f"perm{i}", p, data)
        data[f"perm{i}_axes"] = np.array(ra + ca)
        data[f"perm{i}_nrr"] = np.array(len(ra))
    save("z2_rank6", data)


def microbench_rep(total, qmax):
    """Charges -qmax..qmax with degeneracy ~ exp(-q^2/8), largest-remainder
    rounding to `total`, sorted by charge."""
    q = np.arange(-qmax, qmax + 1)
    w = np.exp(-(q**2) / 8.0)
    raw = w / w.sum() * total
    deg = np.floor(raw).astype(int)
    rem = total - deg.sum()
    order = np.argsort(-(raw - deg), kind="stable")
    deg[order[:rem]] += 1
    return np.repeat(q, deg).astype(np.int8), deg


def normal_tensor(cls, row_reps, col_reps, sig, rng):
    irreps, shapes = cls.get_block_sizes(row_reps, col_reps, sig)
    blocks = [rng.standard_normal(tuple(sh)) for sh in shapes]
    return cls(row_reps, col_reps, blocks, irreps, sig)


def case_u1_microbench_small():
    """The U(1) microbench structure at reduced leg size (permute (0,2),(1,3)
    then matmul against a tensor of the same structure)."""
    rep, deg = microbench_rep(24, 4)
    rng = np.random.default_rng(2024)
    sig1 = np.array([False, False, True, True])
    t1 = normal_tensor(U1SymmetricTensor, (rep, rep), (rep, rep), sig1, rng)
    p = t1.permute((0, 2), (1, 3))
    sig2 = np.array([True, False, False, True])
    t2 = normal_tensor(U1SymmetricTensor, (rep, rep), (rep, rep), sig2, rng)
    m = p @ t2
    data = {"degen": deg}
    pack_tensor("t1", t1, data)
    pack_tensor("t2", t2, data)
    pack_tensor("perm", p, data)
    pack_tensor("matmul", m, data)
    save("u1_microbench_small", data)
    # full-size degeneracies of the benchmark legs (256 states, charges -4..4)
    _, deg256 = microbench_rep(256, 4)
    np.save(os.path.join(HERE, "u1_microbench_degen256.npy"), deg256)


def case_find_block_cuts():
    rng = np.random.default_rng(11)
    data = {}
    cases = []
    for c in range(12):
        nb = int(rng.integers(1, 7))
        blocks = []
        for _ in range(nb):
            n = int(rng.integers(1, 30))
            v = np.ascontiguousarray(np.sort(rng.random(n) ** 3)[::-1])
            # plant quasi-degenerate multiplets
            if n > 3:
                v[1] = v[0] * (1 - 1e-6)
                v[3] = v[2]
            blocks.append(v)
        if c % 3 == 0 and nb > 1:
            blocks[1] = blocks[0].copy()
        dims = rng.integers(1, 5, size=nb)
        cut = int(rng.integers(1, 60))
        degen = [1.0, 0.9999, 0.99][c % 3]
        rtol = [None, 1e-3, 0.0][c % 3]
        res = find_block_cuts(blocks, cut, dims=dims, rtol=rtol, degen_ratio=degen)
        for i, b in enumerate(blocks):
            data[f"c{c}_b{i}"] = b
        data[f"c{c}_nb"] = np.array(nb)
        data[f"c{c}_dims"] = dims
        data[f"c{c}_cut"] = np.array(cut)
        data[f"c{c}_degen"] = np.array(degen)
        data[f"c{c}_rtol"] = np.array(np.nan if rtol is None else rtol)
        data[f"c{c}_out"] = np.asarray(res)
        cases.append(c)
    data["ncases"] = np.array(len(cases))
    save("find_block_cuts", data)


def ising_reference_run(beta, chi, n_iter, seed, snapshots):
    """examples/ising_classical_ctmrg.py Z2 part, restated with reference calls."""
    import scipy.linalg as lg

    D = 2
    h = -2 * np.eye(2) + 1
    sq_bw = lg.sqrtm(np.exp(-beta * h)).real
    delta = np.zeros((D,) * 4)
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
    a2 = U1SymmetricTensor((rep, rep), (rep, rep), a.blocks, a.block_irreps, siga2)

    rng = np.random.default_rng(seed)
    d0o = d0e = chi // 2
    s_odd = rng.normal(size=(d0o,))
    s_odd = s_odd[np.abs(s_odd).argsort()[::-1]] / lg.norm(s_odd)
    s_even = rng.normal(size=(d0e,))
    s_even = s_even[np.abs(s_even).argsort()[::-1]] / lg.norm(s_even)
    corner = np.array([-128] * d0o + [0] * d0e, dtype=np.int8)
    s = DiagonalTensor((s_odd, s_even), corner, np.array([-128, 0], dtype=np.int8),
                       [1, 1], "U1")
    sigT = np.array([False, False, True])
    T = U1SymmetricTensor.random((corner,), (rep, corner), signature=sigT, rng=rng)
    temp = U1SymmetricTensor((corner,), (rep, corner), T.blocks, T.block_irreps,
                             [1, 0, 0])
    T = T + temp.permute((2,), (1, 0))
    T /= T.norm()

    def iterate(s, T):
        Tp = T.permute((0, 1), (2,))
        matC = Tp * s
        matC = matC @ T
        matC = matC.permute((1, 2), (0, 3))
        matC = a2 @ matC
        matC = matC.permute((0, 2), (1, 3))
        news, U = matC.truncated_eigh(chi)
        news /= news.norm()
        newT = U.permute((1,), (0, 2))
        newT = Tp @ newT
        newT = newT.permute((1, 2), (0, 3))
        newT = a @ newT
        newT = newT.permute((0, 2), (1, 3))
        newT = U.dagger() @ newT
        newT /= newT.norm()
        return news, newT

    def energy(s, T):
        Tp = T.permute((0, 1), (2,))
        env = Tp * s
        env = env @ env.permute((0,), (1, 2))
        env = Tp @ env.permute((0,), (1, 2, 3))
        left = env.permute((1, 2, 3), (0, 4))
        right = env.permute((4, 0), (1, 2, 3))
        env2 = (left @ right).toarray()
        nr = np.einsum("abcdef,bgdc,afeg->", env2, a0d, a0d)
        sdsr = np.einsum("abcdef,bgdc,afeg->", env2, mopd, mopd)
        return -sdsr / nr

    data = {"beta": np.array(beta), "chi": np.array(chi), "seed": np.array(seed)}
    pack_diag("s0", s, data)
    pack_tensor("T0", T, data)
    for it in range(1, n_iter + 1):
        s, T = iterate(s, T)
        if it in snapshots:
            pack_diag(f"s{it}", s, data)
            pack_tensor(f"T{it}", T, data)
            data[f"energy{it}"] = np.array(energy(s, T))
    return data


def case_ising():
    data = ising_reference_run(0.44, 8, 10, 42, {1, 2, 3, 10})
    save("ising_chi8", data)
    data = ising_reference_run(0.44, 32, 100, 42, {1, 5, 100})
    save("ising_chi32", data)


def case_ctmrg_u1():
    """SequentialCTMRG on the random U(1) AB/BA network of the reference's
    tests/test_ctmrg.py:57-80 (distinct representation on every bond)."""
    from frostspin.ctmrg import SequentialCTMRG

    rng = np.random.default_rng(42)
    rp = np.array([1, -1], dtype=np.int8)
    ra = np.array([1, -1, 2], dtype=np.int8)
    ru = np.array([1, 1, -1, 0, 2, -2], dtype=np.int8)
    rr = np.array([2, 0, 1, -1, 0, 1, -1], dtype=np.int8)
    rd = np.array([1, 1, -1, -2], dtype=np.int8)
    rl = np.array([1, -2, 1, 0, 0], dtype=np.int8)
    sA = np.array([False, False, True, True, True, True])
    sB = np.array([False, False, False, False, False, False])
    reps_A = (rp, ra, ru, rr, rd, rl)
    reps_B = (rp, ra, rd, rl, ru, rr)
    A = U1SymmetricTensor.random(reps_A[:2], reps_A[2:], rng=rng, signature=sA)
    B = U1SymmetricTensor.random(reps_B[:2], reps_B[2:], rng=rng, signature=sB)
    data = {}
    pack_tensor("A", A, data)
    pack_tensor("B", B, data)
    ctm = SequentialCTMRG.from_elementary_tensors("AB\nBA", (A, B), 20)
    for it in range(4):
        if it:
            ctm.iterate()
        for (x, y) in ctm.site_coords:
            data[f"it{it}_rdm1x2_{x}{y}"] = ctm.compute_rdm1x2(x, y).toarray()
            data[f"it{it}_rdm2x1_{x}{y}"] = ctm.compute_rdm2x1(x, y).toarray()
        data[f"it{it}_chi"] = np.array(ctm.chi_values)
        data[f"it{it}_logZ"] = np.array(ctm.compute_PEPS_norm_log())
    save("ctmrg_u1_random", data)


SDS_22 = np.array(
    [[0.25, 0.0, 0.0, 0.0], [0.0, -0.25, 0.5, 0.0], [0.0, 0.5, -0.25, 0.0],
     [0.0, 0.0, 0.0, 0.25]]
)


def case_simple_update_u1():
    """Heisenberg spin-1/2 on the square lattice, U(1) symmetric simple update
    (examples/heisenberg_simple_update.py:67-82 with D=6), then CTMRG on the
    resulting tensors."""
    from frostspin.ctmrg import SequentialCTMRG
    from frostspin.simple_update import SimpleUpdate

    reps = (np.array([1, -1], dtype=np.int8),) * 2
    h = U1SymmetricTensor.from_array(SDS_22.reshape(2, 2, 2, 2), reps, reps)
    su = SimpleUpdate.square_lattice_first_neighbor(h, 6, 0.01, rcutoff=1e-10,
                                                    degen_ratio=0.9999)
    data = {"D": np.array(6), "tau": np.array(0.01)}
    pack_tensor("h", h, data)
    for k, beta in enumerate((0.2, 0.4)):
        su.evolve(0.2)
        data[f"b{k}_beta"] = np.array(su.beta)
        data[f"b{k}_logZ"] = np.array(su.logZ)
        for i, w in enumerate(su.get_weights()):
            data[f"b{k}_w{i}"] = w
        for i, r in enumerate(su.get_bond_representations()):
            data[f"b{k}_rep{i}"] = r
    tensors = su.get_tensors()
    ctm = SequentialCTMRG.from_elementary_tensors("AB\nBA", tensors, 16, cutoff=1e-10,
                                                  degen_ratio=0.9999)
    for it in range(3):
        ctm.iterate()
    for (x, y) in ctm.site_coords:
        data[f"rdm1x2_{x}{y}"] = ctm.compute_rdm1x2(x, y).toarray()
        data[f"rdm2x1_{x}{y}"] = ctm.compute_rdm2x1(x, y).toarray()
    data["logZ_ctm"] = np.array(ctm.compute_PEPS_norm_log())
    save("simple_update_u1", data)


def case_simple_update_su2():
    """The same Heisenberg simple update with SU(2) symmetry (D=8 states),
    then SU(2) SequentialCTMRG on the resulting tensors."""
    from frostspin import SU2SymmetricTensor
    from frostspin.ctmrg import SequentialCTMRG
    from frostspin.simple_update import SimpleUpdate

    r = np.array([[1], [2]])
    h = SU2SymmetricTensor.from_array(SDS_22.reshape(2, 2, 2, 2), (r, r), (r, r))
    su = SimpleUpdate.square_lattice_first_neighbor(h, 8, 0.01, rcutoff=1e-10,
                                                    degen_ratio=0.9999)
    data = {"D": np.array(8), "tau": np.array(0.01)}
    pack_tensor("h", h, data)
    for k in range(2):
        su.evolve(0.2)
        data[f"b{k}_beta"] = np.array(su.beta)
        data[f"b{k}_logZ"] = np.array(su.logZ)
        for i, w in enumerate(su.get_weights()):
            data[f"b{k}_w{i}"] = w
        for i, rep in enumerate(su.get_bond_representations()):
            data[f"b{k}_rep{i}"] = rep
    tensors = su.get_tensors()
    for i, t in enumerate(tensors):
        pack_tensor(f"A{i}", t, data)
    ctm = SequentialCTMRG.from_elementary_tensors("AB\nBA", tensors, 20, cutoff=1e-10,
                                                  degen_ratio=0.9999)
    for it in range(3):
        ctm.iterate()
        data[f"it{it}_chi"] = np.array(ctm.chi_values)
    for (x, y) in ctm.site_coords:
        data[f"rdm1x2_{x}{y}"] = ctm.compute_rdm1x2(x, y).toarray()
        data[f"rdm2x1_{x}{y}"] = ctm.compute_rdm2x1(x, y).toarray()
    data["logZ_ctm"] = np.array(ctm.compute_PEPS_norm_log())
    save("simple_update_su2", data)


def case_simultaneous_ctmrg():
    """SimultaneousCTMRG (simultaneous_ctmrg.py:14-132) of the reference on
    two existing fixtures' site tensors: the random U(1) AB/BA network and the
    SU(2) simple-update tensors; chi = 20, 3 iterations; chi values, rdms and
    the PEPS norm after each."""
    from frostspin import SU2SymmetricTensor
    from frostspin.ctmrg import SimultaneousCTMRG

    data = {}
    for tag, cls, fix, names in (("u1", U1SymmetricTensor, "ctmrg_u1_random", ("A", "B")),
                                 ("su2", SU2SymmetricTensor, "simple_update_su2", ("A0", "A1"))):
        d = np.load(os.path.join(HERE, fix + ".npz"))
        tensors = [cls.load_from_dic(d, prefix=p) for p in names]
        ctm = SimultaneousCTMRG.from_elementary_tensors("AB\nBA", tensors, 20, cutoff=1e-10,
                                                        degen_ratio=0.9999)
        for it in range(3):
            ctm.iterate()
            data[f"{tag}_it{it}_chi"] = np.array(ctm.chi_values)
            for (x, y) in ctm.site_coords:
                data[f"{tag}_it{it}_rdm1x2_{x}{y}"] = ctm.compute_rdm1x2(x, y).toarray()
                data[f"{tag}_it{it}_rdm2x1_{x}{y}"] = ctm.compute_rdm2x1(x, y).toarray()
            data[f"{tag}_it{it}_logZ"] = np.array(ctm.compute_PEPS_norm_log())
    save("simultaneous_ctmrg", data)


def case_ctmrg_variants():
    """Second-neighbour observables (abstract_ctmrg.py:438-518, rdm.py:190-269)
    of the reference's SequentialCTMRG on the SU(2) simple-update tensors, and
    SymmetrizedCTMRG (symmetrized_ctmrg.py:19-274) on the input of the
    reference's tests/test_symmetrized_ctm.py (random SU(2) site tensor, seed
    42, B = rotated dagger of A, chi = 50): chi values, rdms and PEPS norm
    after each of 3 iterations, then the second-neighbour rdms."""
    from frostspin import SU2SymmetricTensor
    from frostspin.ctmrg import SequentialCTMRG, SymmetrizedCTMRG

    data = {}
    d = np.load(os.path.join(HERE, "simple_update_su2.npz"))
    tensors = [SU2SymmetricTensor.load_from_dic(d, prefix=p) for p in ("A0", "A1")]
    ctm = SequentialCTMRG.from_elementary_tensors("AB\nBA", tensors, 20, cutoff=1e-10,
                                                  degen_ratio=0.9999)
    for _ in range(3):
        ctm.iterate()
    for i, r in enumerate(ctm.compute_rdm1x1_cell()):
        data[f"seq_rdm1x1_{i}"] = r.toarray()
    dr, ur = ctm.compute_rdm_2nd_neighbor_cell()
    for i, (a, b) in enumerate(zip(dr, ur, strict=True)):
        data[f"seq_rdm_dr_{i}"] = a.toarray()
        data[f"seq_rdm_ur_{i}"] = b.toarray()

    rng = np.random.default_rng(42)
    r2 = np.array([[1], [2]])
    rDu = np.array([[2, 3], [1, 3]])
    rDr = np.array([[3, 3], [1, 3]])
    rDd = np.array([[1, 3], [1, 3]])
    rDl = np.array([[4, 3], [1, 3]])
    A = SU2SymmetricTensor.random((r2, r2), (rDu, rDr, rDd, rDl), rng=rng)
    A /= A.norm()
    pack_tensor("symA", A, data)
    B = A.dagger().permute((4, 5), (2, 3, 0, 1))
    ctm = SymmetrizedCTMRG.from_elementary_tensors("AB\nBA", [A, B], 50)
    data["sym_it-1_logZ"] = np.array(ctm.compute_PEPS_norm_log())
    for it in range(3):
        ctm.iterate()
        data[f"sym_it{it}_chi"] = np.array(ctm.chi_values)
        for (x, y) in ctm.site_coords:
            data[f"sym_it{it}_rdm1x2_{x}{y}"] = ctm.compute_rdm1x2(x, y).toarray()
            data[f"sym_it{it}_rdm2x1_{x}{y}"] = ctm.compute_rdm2x1(x, y).toarray()
        data[f"sym_it{it}_logZ"] = np.array(ctm.compute_PEPS_norm_log())
    (dr0, dr1), (ur0, ur1) = ctm.compute_rdm_2nd_neighbor_cell()
    data["sym_rdm_dr"] = dr0.toarray()
    data["sym_rdm_ur"] = ur0.toarray()
    save("ctmrg_variants", data)


def _plain(v):
    """Nested lists / tuples of numpy scalars -> JSON-able Python values."""
    if isinstance(v, (list, tuple)):
        return [_plain(x) for x in v]
    if v is None:
        return None
    return v.item() if hasattr(v, "item") else v


def case_su_schedules():
    """Update schedules of the reference's simple update (get_update_data,
    simple_update.py:68-184) for the first-neighbour square lattice and the
    three second-neighbour models of su_models.py, with scalar stand-ins for
    the Hamiltonians (the schedule only multiplies them by 2)."""
    from frostspin.simple_update.simple_update import get_update_data
    from frostspin.simple_update.su_models import j1_j2_models

    data = {}
    cases = {"first": ([[0, 1, 2, 3], [2, 3, 0, 1]],
                       np.array([[b, b, 0, 0, 1, -1] for b in range(4)]), [1.0])}
    tbi2 = [[0, 1, 2, 3], [4, 3, 5, 1], [2, 6, 0, 7], [5, 7, 4, 6]]
    for name, table in j1_j2_models.items():
        cases[name] = (tbi2, table, [1.0, 0.5])
    for name, (tbi, table, hams) in cases.items():
        out = get_update_data(tbi, table, hams)
        keys = ("bond1", "bond2", "gate", "left", "right", "middle", "lperm", "rperm",
                "mperm", "hamiltonians", "initial_swap", "final_swap")
        for k, v in zip(keys, out, strict=True):
            data[f"{name}_{k}"] = np.array(json.dumps(_plain(v)))
        data[f"{name}_table"] = np.asarray(table)
    save("su_schedules", data)


def case_simple_update_j1j2():
    """U(1) J1-J2 simple update of the reference (square_lattice_second_neighbor,
    simple_update.py:366-407; J2 = 0.5, D = 4, tau = 0.01) for each model, two
    evolve steps: weights, logZ and bond representations."""
    from frostspin.simple_update import SimpleUpdate

    reps = (np.array([1, -1], dtype=np.int8),) * 2
    h1 = U1SymmetricTensor.from_array(SDS_22.reshape(2, 2, 2, 2), reps, reps)
    data = {}
    pack_tensor("h1", h1, data)
    for model in ("J1-J2", "checkerboard", "Shastry-Sutherland"):
        su = SimpleUpdate.square_lattice_second_neighbor(h1, 0.5 * h1, 4, 0.01, model=model,
                                                         rcutoff=1e-10, degen_ratio=0.9999)
        for k in range(2):
            su.evolve(0.04)
            data[f"{model}_b{k}_beta"] = np.array(su.beta)
            data[f"{model}_b{k}_logZ"] = np.array(su.logZ)
            for i, w in enumerate(su.get_weights()):
                data[f"{model}_b{k}_w{i}"] = w
            for i, r in enumerate(su.get_bond_representations()):
                data[f"{model}_b{k}_rep{i}"] = r
    save("simple_update_j1j2", data)


def case_symmetrized_simple_update():
    """SymmetrizedSimpleUpdate (symmetrized_simple_update.py:10-271) of the
    reference on the input of its tests/test_symmetrized_ctm.py (S.S in the
    rotated basis, signature (0, 1, 1, 0), D = 7), tau = 0.01, two evolve
    steps of 0.1: beta, logZ, bond representations and weights."""
    from frostspin import SU2SymmetricTensor
    from frostspin.simple_update import SymmetrizedSimpleUpdate

    r2 = su2_rep([1], [2])
    arrb = np.array([[-0.25, 0.0, 0.0, -0.5], [0.0, 0.25, 0.0, 0.0],
                     [0.0, 0.0, 0.25, 0.0], [-0.5, 0.0, 0.0, -0.25]]).reshape(2, 2, 2, 2)
    h = SU2SymmetricTensor.from_array(arrb, (r2, r2), (r2, r2), [0, 1, 1, 0])
    data = {}
    pack_tensor("h", h, data)
    su = SymmetrizedSimpleUpdate.from_infinite_temperature(7, 0.01, [h])
    for k in range(2):
        su.evolve(0.1)
        data[f"b{k}_beta"] = np.array(su.beta)
        data[f"b{k}_logZ"] = np.array(su.logZ)
        for i, w in enumerate(su.get_weights()):
            data[f"b{k}_w{i}"] = w
        for i, r in enumerate(su.get_bond_representations()):
            data[f"b{k}_rep{i}"] = r
    save("symmetrized_simple_update", data)


def case_su2_d24_beta2():
    """Site tensors of the SU(2) CTMRG benchmark: the reference's SU(2) simple
    update of the Heisenberg model, D=24, tau=0.01, evolved to beta=2."""
    from frostspin import SU2SymmetricTensor
    from frostspin.simple_update import SimpleUpdate

    r = np.array([[1], [2]])
    h = SU2SymmetricTensor.from_array(SDS_22.reshape(2, 2, 2, 2), (r, r), (r, r))
    su = SimpleUpdate.square_lattice_first_neighbor(h, 24, 0.01, rcutoff=1e-10,
                                                    degen_ratio=0.9999)
    su.evolve(2.0)
    data = {"beta": np.array(su.beta), "logZ": np.array(su.logZ), "Dmax": np.array(su.Dmax)}
    for i, w in enumerate(su.get_weights()):
        data[f"w{i}"] = w
    for i, rep in enumerate(su.get_bond_representations()):
        data[f"rep{i}"] = rep
    for i, t in enumerate(su.get_tensors()):
        pack_tensor(f"A{i}", t, data)
    save("su2_d24_beta2", data)


def _load_ref_tensor(cls, d, prefix):
    return cls.load_from_dic(d, prefix=prefix)


def case_corr_length():
    """Transfer spectra and correlation lengths (abstract_ctmrg.py:519-579,
    observables.py:4-154) after 3 CTMRG iterations at chi=20, on the SU(2)
    simple-update tensors of simple_update_su2.npz and on the random U(1)
    tensors of ctmrg_u1_random.npz."""
    from frostspin import SU2SymmetricTensor
    from frostspin.ctmrg import SequentialCTMRG

    data = {}
    for tag, cls, fix, names in (("su2", SU2SymmetricTensor, "simple_update_su2", ("A0", "A1")),
                                 ("u1", U1SymmetricTensor, "ctmrg_u1_random", ("A", "B"))):
        d = np.load(os.path.join(HERE, fix + ".npz"))
        tensors = [_load_ref_tensor(cls, d, n) for n in names]
        ctm = SequentialCTMRG.from_elementary_tensors("AB\nBA", tensors, 20, cutoff=1e-10,
                                                      degen_ratio=0.9999)
        for _ in range(3):
            ctm.iterate()
        for k in range(2):
            data[f"{tag}_spec_h{k}"] = ctm.compute_transfer_spectrum_h(k, 4)
            data[f"{tag}_spec_v{k}"] = ctm.compute_transfer_spectrum_v(k, 4)
            data[f"{tag}_xi_h{k}"] = np.array(ctm.compute_corr_length_h(k))
            data[f"{tag}_xi_v{k}"] = np.array(ctm.compute_corr_length_v(k))
        data[f"{tag}_chi"] = np.array(ctm.chi_values)
    save("corr_length", data)


def case_ctmrg_su2_d24():
    """SU(2) SequentialCTMRG from the reference's D=24 simple-update tensors
    (su2_d24_beta2.npz) at chi=24, 2 iterations: chi values, rdms, energy."""
    from frostspin import SU2SymmetricTensor
    from frostspin.ctmrg import SequentialCTMRG

    import tempfile

    from frostspin.groups.su2_clebsch_gordan import save_su2_cg

    # the reference's shipped CG table stops at irrep dimension 10; these
    # corners need larger irreps, so the reference's own generator writes a
    # table up to 18 first (a transient file, deleted afterwards)
    with tempfile.TemporaryDirectory(dir=HERE) as tmp:
        cg_file = os.path.join(tmp, "cg18.npz")
        save_su2_cg(cg_file, 18)
        SU2SymmetricTensor.reload_clebsch_gordan(cg_file)
    d = np.load(os.path.join(HERE, "su2_d24_beta2.npz"))
    tensors = [SU2SymmetricTensor.load_from_dic(d, prefix=p) for p in ("A0", "A1")]
    ctm = SequentialCTMRG.from_elementary_tensors("AB\nBA", tensors, 24, cutoff=1e-10,
                                                  degen_ratio=0.9999)
    data = {}
    for it in range(2):
        ctm.iterate()
        data[f"it{it}_chi"] = np.array(ctm.chi_values)
    h = SDS_22.reshape(2, 2, 2, 2)
    es = []
    for (x, y) in ctm.site_coords:
        r12 = ctm.compute_rdm1x2(x, y).toarray()
        r21 = ctm.compute_rdm2x1(x, y).toarray()
        data[f"rdm1x2_{x}{y}"] = r12
        data[f"rdm2x1_{x}{y}"] = r21
        es += [np.einsum("ijkl,klij->", r12, h), np.einsum("ijkl,klij->", r21, h)]
    data["energy"] = np.array(np.mean(es))
    save("ctmrg_su2_d24", data)


def case_heisenberg_d12_beta2():
    """Site tensors of the CTMRG benchmark: the reference's U(1) simple update of
    the Heisenberg model, D=12, tau=0.01, evolved to beta=2 (get_tensors)."""
    from frostspin.simple_update import SimpleUpdate

    reps = (np.array([1, -1], dtype=np.int8),) * 2
    h = U1SymmetricTensor.from_array(SDS_22.reshape(2, 2, 2, 2), reps, reps)
    su = SimpleUpdate.square_lattice_first_neighbor(h, 12, 0.01, rcutoff=1e-10,
                                                    degen_ratio=0.9999)
    su.evolve(2.0)
    data = {"beta": np.array(su.beta), "logZ": np.array(su.logZ)}
    for i, w in enumerate(su.get_weights()):
        data[f"w{i}"] = w
    for i, t in enumerate(su.get_tensors()):
        pack_tensor(f"A{i}", t, data)
    save("heisenberg_d12_beta2", data)


def su2_rep(degen, irreps):
    return np.array([degen, irreps], dtype=int)


def _su2_permute_cases(t, perms, data, prefix):
    for i, (ra, ca) in enumerate(perms):
        p = t.permute(ra, ca)
        pack_tensor(f"{prefix}perm{i}", p, data)
        data[f"{prefix}perm{i}_axes"] = np.array(ra + ca)
        data[f"{prefix}perm{i}_nrr"] = np.array(len(ra))
        data[f"{prefix}perm{i}_dense"] = p.toarray()


def case_su2():
    """SU(2) fixtures.  Part 1 repeats the known-answer inputs of the
    reference's tests/test_su2_tensor.py (S.S of two spins 1/2, the
    external-degeneracy tensor, the missing-block tensor); part 2 is random
    tensors with several irreps and degeneracies per leg, permuted in many ways,
    plus transpose, dagger, matmul, norm and truncated SVD spectra."""
    from frostspin import SU2SymmetricTensor

    data = {}
    r = su2_rep([1], [2])
    sds = SDS_22.reshape(2, 2, 2, 2)
    st = SU2SymmetricTensor.from_array(sds, (r, r), (r, r))
    pack_tensor("sds", st, data)
    data["sds_dense"] = sds
    _su2_permute_cases(st, [((0, 1, 2), (3,)), ((3, 0, 2), (1,)), ((1, 3), (2, 0))],
                       data, "sds_")
    arrb = np.array([[-0.25, 0.0, 0.0, -0.5], [0.0, 0.25, 0.0, 0.0],
                     [0.0, 0.0, 0.25, 0.0], [-0.5, 0.0, 0.0, -0.25]]).reshape(2, 2, 2, 2)
    stb = SU2SymmetricTensor.from_array(arrb, (r, r), (r, r), signature=[0, 1, 1, 0])
    pack_tensor("sdsb", stb, data)
    data["sdsb_dense"] = arrb
    _su2_permute_cases(stb, [((0, 1, 2), (3,)), ((3, 0, 2), (1,))], data, "sdsb_")

    r1 = su2_rep([1], [1])
    r12 = su2_rep([1, 2, 1], [1, 3, 5])
    arr = np.eye(12).reshape(1, 12, 12, 1)
    st3 = SU2SymmetricTensor.from_array(arr, (r1,), (r12, r12, r1), signature=[0, 0, 1, 1])
    pack_tensor("ext", st3, data)
    data["ext_dense"] = arr
    _su2_permute_cases(st3, [((0, 1), (2, 3)), ((2, 0), (3, 1))], data, "ext_")

    rng = np.random.default_rng(7)
    r3 = su2_rep([1], [3])
    t = SU2SymmetricTensor.random((r3, r3, r3), (r3,), rng=rng)
    t = t @ t.dagger()
    pack_tensor("miss", t, data)
    _su2_permute_cases(t, [((3, 2, 1), (0, 5, 4)), ((0,), (1, 2, 3, 4, 5))], data, "miss_")

    rng = np.random.default_rng(11)
    ra = su2_rep([2, 1], [1, 3])
    rb = su2_rep([1, 2], [2, 4])
    rc = su2_rep([1, 1, 1], [1, 2, 3])
    rd = su2_rep([2], [2])
    re = su2_rep([1, 1], [1, 3])
    sig = np.array([0, 1, 0, 1, 1], dtype=bool)
    t = SU2SymmetricTensor.random((ra, rb), (rc, rd, re), signature=sig, rng=rng)
    pack_tensor("r5", t, data)
    data["r5_dense"] = t.toarray()
    perms = [
        ((3, 0, 2), (1, 4)),
        ((3,), (1, 0, 4, 2)),
        ((2, 3, 4), (0, 1)),
        ((4, 1), (0, 3, 2)),
        ((0, 1, 2, 3), (4,)),
        ((1, 4, 0), (3, 2)),
    ]
    _su2_permute_cases(t, perms, data, "r5_")
    pack_tensor("r5_transpose", t.transpose(), data)
    pack_tensor("r5_dagger", t.dagger(), data)
    data["r5_norm"] = np.array(t.norm())
    m = t @ t.dagger()
    pack_tensor("r5_matmul", m, data)
    data["r5_matmul_trace"] = np.array(m.trace())
    _, s, _ = m.truncated_svd(7)
    pack_diag("r5_tsvd_s", s, data)

    rng = np.random.default_rng(13)
    rp = su2_rep([1], [2])
    rv = su2_rep([1, 2, 1], [1, 2, 3])
    sig6 = np.array([0, 0, 1, 1, 0, 1], dtype=bool)
    t6 = SU2SymmetricTensor.random((rp, rp, rv), (rv, rv, rv), signature=sig6, rng=rng)
    pack_tensor("r6", t6, data)
    _su2_permute_cases(t6, [((0, 2, 4), (1, 3, 5)), ((5, 1), (0, 4, 3, 2)),
                            ((2, 3, 0, 5, 1), (4,))], data, "r6_")
    save("su2", data)


def _o2_pack_all(name, t, perms, data):
    """An O(2) tensor with its dense form, its U(1) cast, a list of permutes
    (each with its dense form and U(1) cast) and its transpose."""
    pack_tensor(name, t, data)
    data[name + "_dense"] = t.toarray()
    pack_tensor(name + "_u1", t.toU1(), data)
    for i, (ra, ca) in enumerate(perms):
        p = t.permute(ra, ca)
        pre = f"{name}_perm{i}"
        pack_tensor(pre, p, data)
        pack_tensor(pre + "_u1", p.toU1(), data)
        data[pre + "_axes"] = np.array(ra + ca)
        data[pre + "_nrr"] = np.array(len(ra))
        data[pre + "_dense"] = p.toarray()
    tt = t.transpose()
    pack_tensor(name + "_transpose", tt, data)
    data[name + "_transpose_dense"] = tt.toarray()


def case_o2():
    """O(2) fixtures.  The inputs of the reference's tests/test_o2_tensor.py
    (representations r1..r7, seed 42, the pathological tensors with the 0odd,
    0even or both blocks removed, only doublets, only odd or only even fixed
    points in the columns), plus a random tensor with a mixed signature, each
    permuted in several ways, transposed and cast to U(1)."""
    from frostspin import O2SymmetricTensor

    data = {}
    rng = np.random.default_rng(42)
    r1 = np.array([[1, 1, 1, 1], [-1, 0, 1, 2]])
    r2 = np.array([[2, 1, 1, 1], [-1, 0, 1, 2]])
    r3 = np.array([[1, 2, 1, 1], [-1, 0, 1, 2]])
    r4 = np.array([[1, 1, 1, 1], [-1, 0, 2, 3]])
    r5 = np.array([[2, 1, 1, 1], [-1, 0, 2, 3]])
    perms = [((2, 1, 4), (0, 3)), ((0, 1, 3), (2, 4)), ((4,), (3, 2, 1, 0)),
             ((3, 0, 4, 1), (2,))]
    t = O2SymmetricTensor.random((r1, r2, r3), (r4, r5), rng=rng)
    t /= t.norm()
    _o2_pack_all("base", t, perms, data)
    data["base_norm"] = np.array(t.norm())
    pack_tensor("base_dagger", t.dagger(), data)
    m = t @ t.dagger()
    pack_tensor("base_matmul", m, data)

    z = t.copy()
    z.blocks[0][:] = 0
    no_odd = O2SymmetricTensor(z.row_reps, z.col_reps, z.blocks[1:], z.block_irreps[1:],
                               z.signature)
    _o2_pack_all("noodd", no_odd, perms[:2], data)
    z = t.copy()
    no_even = O2SymmetricTensor(z.row_reps, z.col_reps, z.blocks[:1] + z.blocks[2:],
                                (-1, *z.block_irreps[2:]), z.signature)
    _o2_pack_all("noeven", no_even, perms[:2], data)
    z = t.copy()
    no_zero = O2SymmetricTensor(z.row_reps, z.col_reps, z.blocks[2:], z.block_irreps[2:],
                                z.signature)
    _o2_pack_all("nozero", no_zero, perms[:2], data)
    z = t.copy()
    only_zero = O2SymmetricTensor(z.row_reps, z.col_reps, z.blocks[:2], z.block_irreps[:2],
                                  z.signature)
    _o2_pack_all("onlyzero", only_zero, perms[:2], data)

    for name, r6, r7 in (
        ("doublets", np.array([[1, 1, 1], [2, 3, 4]]), np.array([[2, 1], [2, 3]])),
        ("oddfix", np.array([[4], [-1]]), np.array([[5], [-1]])),
        ("evenfix", np.array([[4], [0]]), np.array([[5], [0]])),
    ):
        t2 = O2SymmetricTensor.random((r1, r2, r6), (r3, r7), rng=rng)
        t2 /= t2.norm()
        _o2_pack_all(name, t2, [((0, 1, 3), (2, 4)), ((4, 2), (1, 0, 3))], data)

    rng = np.random.default_rng(5)
    sig = np.array([0, 1, 1, 0], dtype=bool)
    ra = np.array([[1, 2, 1], [-1, 0, 1]])
    rb = np.array([[1, 1, 2], [0, 1, 2]])
    t4 = O2SymmetricTensor.random((ra, rb), (rb, ra), signature=sig, rng=rng)
    _o2_pack_all("sig", t4, [((0, 2), (1, 3)), ((3,), (0, 1, 2)), ((1, 2, 3), (0,))], data)

    # SU(2) -> O(2) casts (su2_symmetric_tensor.py:249-318): integer and
    # half-integer spins up to spin 5/2, whose sign convention differs
    from frostspin import SU2SymmetricTensor

    rng = np.random.default_rng(9)
    for name, rows, cols, sig in (
        ("su2cast_int", (su2_rep([1, 2], [1, 3]), su2_rep([1, 1], [3, 5])),
         (su2_rep([2, 1], [1, 3]), su2_rep([1], [5])), [0, 1, 1, 0]),
        ("su2cast_half", (su2_rep([1, 1], [2, 4]), su2_rep([2], [2])),
         (su2_rep([1, 1], [2, 4]), su2_rep([1, 1], [2, 6])), [0, 0, 1, 1]),
        ("su2cast_mixed", (su2_rep([1, 1, 1], [2, 4, 6]),),
         (su2_rep([1, 1], [3, 7]), su2_rep([1, 1], [2, 4])), [1, 0, 0]),
    ):
        ts = SU2SymmetricTensor.random(rows, cols, signature=np.array(sig, dtype=bool), rng=rng)
        pack_tensor(name + "_su2", ts, data)
        pack_tensor(name, ts.toO2(), data)
    save("o2", data)


def case_checkpoints():
    """Checkpoint interchange: files written by the reference's own
    save_to_file (SequentialCTMRG, abstract_ctmrg.py:194-216 with
    ctm_environment.py:262-276; SimpleUpdate, abstract_simple_update.py:149-187)
    copied as fixtures, plus what the reference computes after reloading them
    with its own load_from_file and continuing."""
    import shutil
    import tempfile

    from frostspin.ctmrg import SequentialCTMRG
    from frostspin.simple_update import SimpleUpdate

    tmp = tempfile.mkdtemp()
    expect = {}
    d = np.load(os.path.join(HERE, "ctmrg_u1_random.npz"))
    tensors = [U1SymmetricTensor.load_from_dic(d, prefix=p) for p in ("A", "B")]
    ctm = SequentialCTMRG.from_elementary_tensors("AB\nBA", tensors, 20, cutoff=1e-10,
                                                  degen_ratio=0.9999)
    for _ in range(2):
        ctm.iterate()
    f = os.path.join(tmp, "ctm.npz")
    ctm.save_to_file(f)
    shutil.copy(f, os.path.join(HERE, "ckpt_ctmrg_u1.npz"))
    ctm2 = SequentialCTMRG.load_from_file(f)
    ctm2.iterate()
    expect["ctm_chi"] = np.array(ctm2.chi_values)
    for (x, y) in ctm2.site_coords:
        expect[f"ctm_rdm1x2_{x}{y}"] = ctm2.compute_rdm1x2(x, y).toarray()
        expect[f"ctm_rdm2x1_{x}{y}"] = ctm2.compute_rdm2x1(x, y).toarray()
    expect["ctm_logZ"] = np.array(ctm2.compute_PEPS_norm_log())

    reps = (np.array([1, -1], dtype=np.int8),) * 2
    h = U1SymmetricTensor.from_array(SDS_22.reshape(2, 2, 2, 2), reps, reps)
    su = SimpleUpdate.square_lattice_first_neighbor(h, 6, 0.01, rcutoff=1e-10,
                                                    degen_ratio=0.9999)
    su.evolve(0.2)
    f = os.path.join(tmp, "su.npz")
    su.save_to_file(f)
    shutil.copy(f, os.path.join(HERE, "ckpt_su_u1.npz"))
    su2 = SimpleUpdate.load_from_file(f)
    su2.evolve(0.2)
    expect["su_beta"] = np.array(su2.beta)
    expect["su_logZ"] = np.array(su2.logZ)
    for i, w in enumerate(su2.get_weights()):
        expect[f"su_w{i}"] = w
    for i, r in enumerate(su2.get_bond_representations()):
        expect[f"su_rep{i}"] = r
    save("ckpt_expect", expect)
    shutil.rmtree(tmp)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        for name in sys.argv[1:]:
            globals()["case_" + name]()
        sys.exit(0)
    case_u1_reference_test()
    case_z2_rank6()
    case_u1_microbench_small()
    case_find_block_cuts()
    case_ising()
    case_ctmrg_u1()
    case_simple_update_u1()
