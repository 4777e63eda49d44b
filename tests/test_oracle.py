"""Pin the CPU oracle against outputs of the reference implementation
(fixtures written by tests/golden/make_golden.py)."""

import numpy as np
import pytest

from oracle import frostspin_oracle as fo
from tests.helpers import (
    assert_blocks_close,
    assert_blocks_equal,
    assert_same_structure,
    diag_from_dic,
    load,
    oracle_from_dic,
)


@pytest.mark.parametrize("name", ["u1_reference_test", "z2_rank6"])
def test_oracle_permute_bit_exact(name):
    d = load(name)
    t = oracle_from_dic(d, "in")
    i = 0
    while f"perm{i}_axes" in d:
        axes = tuple(int(a) for a in d[f"perm{i}_axes"])
        nrr = int(d[f"perm{i}_nrr"])
        ref = oracle_from_dic(d, f"perm{i}")
        got = fo.permute(t, axes[:nrr], axes[nrr:])
        assert_same_structure(got, ref)
        assert_blocks_equal(got, ref)
        i += 1
    assert i >= 5


def test_oracle_dense_roundtrip_and_reductions():
    d = load("u1_reference_test")
    t = oracle_from_dic(d, "in")
    assert np.array_equal(fo.toarray(t), d["dense"])
    back = fo.from_array(d["dense"], t.row_reps, t.col_reps, t.signature)
    assert_blocks_equal(back, t)
    assert abs(fo.norm(t) - float(d["norm"])) <= 1e-14 * float(d["norm"])
    fc = fo.full_contract(t, fo.dagger(t))
    assert abs(fc - float(d["full_contract_dagger"])) <= 1e-13 * abs(fc)
    i = 0
    while f"perm{i}_axes" in d:
        axes = tuple(int(a) for a in d[f"perm{i}_axes"])
        assert np.array_equal(fo.toarray(oracle_from_dic(d, f"perm{i}")),
                              d["dense"].transpose(axes))
        i += 1


def test_oracle_transpose_dagger_matmul():
    d = load("u1_reference_test")
    t = oracle_from_dic(d, "in")
    tr = fo.transpose(t)
    ref = oracle_from_dic(d, "transpose")
    assert_same_structure(tr, ref)
    assert_blocks_equal(tr, ref)
    dg = fo.dagger(t)
    ref = oracle_from_dic(d, "dagger")
    assert_same_structure(dg, ref)
    assert_blocks_equal(dg, ref)
    m = fo.matmul(t, dg)
    ref = oracle_from_dic(d, "matmul")
    assert_same_structure(m, ref)
    assert_blocks_close(m, ref, 1e-14)
    assert abs(fo.trace(m) - float(d["matmul_trace"])) <= 1e-13 * abs(fo.trace(m))


def test_oracle_truncated_svd_spectrum():
    d = load("u1_reference_test")
    t = oracle_from_dic(d, "in")
    _, s_blocks, s_irr, _ = fo.truncated_svd(t, 6)
    ref_blocks, ref_irr = diag_from_dic(d, "tsvd_s")
    assert np.array_equal(s_irr, ref_irr)
    for a, b in zip(s_blocks, ref_blocks, strict=True):
        np.testing.assert_allclose(a, b, rtol=1e-13, atol=1e-15)


def test_oracle_microbench_small():
    d = load("u1_microbench_small")
    t1 = oracle_from_dic(d, "t1")
    t2 = oracle_from_dic(d, "t2")
    p = fo.permute(t1, (0, 2), (1, 3))
    ref = oracle_from_dic(d, "perm")
    assert_same_structure(p, ref)
    assert_blocks_equal(p, ref)
    m = fo.matmul(p, t2)
    ref = oracle_from_dic(d, "matmul")
    assert_same_structure(m, ref)
    assert_blocks_close(m, ref, 1e-13)


def test_oracle_find_block_cuts():
    d = load("find_block_cuts")
    for c in range(int(d["ncases"])):
        nb = int(d[f"c{c}_nb"])
        blocks = [d[f"c{c}_b{i}"] for i in range(nb)]
        rtol = float(d[f"c{c}_rtol"])
        res = fo.find_block_cuts(
            blocks, int(d[f"c{c}_cut"]), dims=d[f"c{c}_dims"],
            rtol=None if np.isnan(rtol) else rtol, degen_ratio=float(d[f"c{c}_degen"]),
        )
        assert np.array_equal(res, d[f"c{c}_out"]), c


def test_oracle_ising_iterations_chi8():
    d = load("ising_chi8")
    a, a2, a0d, mopd = fo.ising_tensors(float(d["beta"]))
    s_blocks, s_irr = diag_from_dic(d, "s0")
    T = oracle_from_dic(d, "T0")
    chi = int(d["chi"])
    for it in range(1, 11):
        s_blocks, s_irr, T = fo.ising_c4v_iteration(s_blocks, s_irr, T, a, a2, chi)
        if f"s{it}_block_irreps" in d:
            ref_blocks, ref_irr = diag_from_dic(d, f"s{it}")
            assert np.array_equal(s_irr, ref_irr)
            for x, y in zip(s_blocks, ref_blocks, strict=True):
                np.testing.assert_allclose(x, y, rtol=1e-10, atol=1e-13)
            e = fo.ising_energy_per_bond(s_blocks, s_irr, T, a0d, mopd)
            assert abs(e - float(d[f"energy{it}"])) < 1e-10


def test_oracle_ising_energy_chi32():
    d = load("ising_chi32")
    a, a2, a0d, mopd = fo.ising_tensors(float(d["beta"]))
    s_blocks, s_irr = diag_from_dic(d, "s0")
    T = oracle_from_dic(d, "T0")
    for _ in range(5):
        s_blocks, s_irr, T = fo.ising_c4v_iteration(s_blocks, s_irr, T, a, a2, 32)
    e = fo.ising_energy_per_bond(s_blocks, s_irr, T, a0d, mopd)
    assert abs(e - float(d["energy5"])) < 1e-9


def test_oracle_ctmrg_matches_reference_run():
    from oracle import ctmrg_oracle as co

    d = load("ctmrg_u1_random")
    A = oracle_from_dic(d, "A")
    B = oracle_from_dic(d, "B")
    ctm = co.SequentialCTMRG(A, B, 20)
    for it in range(3):
        if it:
            ctm.iterate()
        tol = 1e-12 if it == 0 else 1e-9
        for x, y in ctm.coords:
            r12 = co.ctm_rdm1x2(ctm, x, y)
            r21 = co.ctm_rdm2x1(ctm, x, y)
            ref12 = d[f"it{it}_rdm1x2_{x}{y}"]
            ref21 = d[f"it{it}_rdm2x1_{x}{y}"]
            assert np.abs(r12 - ref12).max() < tol * max(1.0, np.abs(ref12).max())
            assert np.abs(r21 - ref21).max() < tol * max(1.0, np.abs(ref21).max())


def test_oracle_ising_correlation_length_of_reference_tensors():
    """The oracle's C4v correlation length on the reference's own edge tensors
    (beta = 0.44, chi = 32): it grows along the run (critical slowing near
    beta_c = 0.4407) and the leading transfer eigenvalue is simple."""
    from tests.helpers import load, oracle_from_dic

    d = load("ising_chi32")
    xis = [fo.ising_correlation_length(oracle_from_dic(d, f"T{it}"))[0] for it in (1, 5, 100)]
    assert xis[0] < xis[1] < xis[2]
    assert 50 < xis[2] < 200
    lam = fo.ising_correlation_length(oracle_from_dic(d, "T100"))[1]
    assert abs(lam[0]) > abs(lam[1])
